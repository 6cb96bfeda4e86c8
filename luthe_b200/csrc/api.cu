// C ABI of the engine: context, key upload, batched KS+PBS, NTT, linear DOps,
// CUDA-graph replay and the blind-rotation autotuner.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdarg.h>
#include <algorithm>
#include <atomic>
#include <ctype.h>
#include <string>
#include <vector>
#include "../../include/luthe.h"
#include "kernels.cuh"
#include "ctx.h"

using namespace luthe;

thread_local char g_err[512] = "";

int fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

extern "C" const char *luthe_last_error(void) { return g_err; }

extern "C" void luthe_params_default(luthe_params *p)
{
    p->lwe_dim = 804;
    p->glwe_dim = 1;
    p->poly_size = 2048;
    p->pbs_base_log = 23;
    p->pbs_level = 1;
    p->ks_base_log = 3;
    p->ks_level = 6;
    p->ks_width = 21;
    p->msg_width = 2;
    p->carry_width = 2;
}

static int check_params(const luthe_params *p)
{
    if (!p) return fail(LUTHE_E_PARAM, "null params");
    if (p->glwe_dim != 1 || p->poly_size != (uint32_t)N || !pbs_supported(p->pbs_base_log) || p->pbs_level != 1 ||
        !ks_supported(p->ks_base_log, p->ks_level) || p->ks_width != (uint32_t)KS_W)
        return fail(LUTHE_E_PARAM,
                    "unsupported parameter set (engine is built for k=1 N=2048, PBS 2^23 or 2^22 x 1, "
                    "KS 3x6, 3x5, 2x8 or 2x7 mod 2^21)");
    if (p->lwe_dim == 0 || p->lwe_dim > 4096) return fail(LUTHE_E_PARAM, "lwe_dim %u out of range", p->lwe_dim);
    if (p->msg_width + p->carry_width + 1 > 32) return fail(LUTHE_E_PARAM, "message width too large");
    return LUTHE_OK;
}

int dalloc(luthe_ctx *c, void **ptr, size_t bytes)
{
    if (c->used + bytes > c->budget)
        return fail(LUTHE_E_BUDGET, "HBM budget exceeded: %llu + %zu > %llu bytes", (unsigned long long)c->used,
                    bytes, (unsigned long long)c->budget);
    CUDA_TRY(cudaMalloc(ptr, bytes));
    c->used += bytes;
    return LUTHE_OK;
}
void dfree(luthe_ctx *c, void *ptr, size_t bytes)
{
    if (ptr) {
        cudaFree(ptr);
        c->used -= bytes;
    }
}

void drop_graphs(luthe_ctx *c)
{
    for (auto &g : c->graphs) cudaGraphExecDestroy(g.exec);
    c->graphs.clear();
}

int tuning_autoload(luthe_ctx *c);

extern "C" int luthe_ctx_create(const luthe_params *p, int device, uint64_t budget, luthe_ctx **out)
{
    if (!out) return fail(LUTHE_E_PARAM, "null out");
    *out = nullptr;
    int r = check_params(p);
    if (r) return r;
    CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(LUTHE_E_CUDA, "device %d is sm_%d%d; this build targets sm_100a", device,
                                      prop.major, prop.minor);
    luthe_ctx *c = new luthe_ctx();
    c->p = *p;
    c->device = device;
    c->nsm = prop.multiProcessorCount;
    c->budget = budget ? budget : 80ull * 1000 * 1000 * 1000;
    std::vector<uint64_t> tw(4096);
    build_twiddles(tw.data());
    if ((r = dalloc(c, (void **)&c->d_tw, 4096 * 8)) || (r = dalloc(c, (void **)&c->d_err, 4))) {
        luthe_ctx_destroy(c);
        return r;
    }
    cudaError_t e = cudaMemcpy(c->d_tw, tw.data(), 4096 * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, 4);
    if (e == cudaSuccess) e = br_set_attributes(BrConfig{1, 1}, p->lwe_dim);
    if (e == cudaSuccess) e = br_set_attributes(BrConfig{2, 1}, p->lwe_dim);
    if (e == cudaSuccess) {
        // diagnostics: LUTHE_SLAB_WAIT_POLLS bounds each BSK-slab wait (0: run out at once)
        const char *polls = getenv("LUTHE_SLAB_WAIT_POLLS");
        e = set_slab_wait_polls(polls ? strtoull(polls, nullptr, 10) : (1ull << 26));
    }
    if (e != cudaSuccess) {
        luthe_ctx_destroy(c);
        return fail(LUTHE_E_CUDA, "context init: %s", cudaGetErrorString(e));
    }
    if ((r = tuning_autoload(c))) {
        luthe_ctx_destroy(c);
        return r;
    }
    *out = c;
    return LUTHE_OK;
}

extern "C" void luthe_ctx_destroy(luthe_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    drop_graphs(c);
    const size_t n = c->p.lwe_dim;
    dfree(c, c->d_tw, 4096 * 8);
    dfree(c, c->d_err, 4);
    dfree(c, c->d_bsk, n * SLAB_BYTES);
    dfree(c, c->d_ksk, (size_t)N * c->p.ks_level / 4 * KS_PLANES * c->xpad * 4);
    dfree(c, c->d_ks_part, (size_t)KS_BM * c->xpad * 4);
    dfree(c, c->d_luts, (size_t)c->nlut * 2 * N * 8);
    dfree(c, c->d_lwe2N, c->cap * (n + 1) * 4);
    dfree(c, c->d_hin, c->hcap * (N + 1) * 8);
    dfree(c, c->d_hout, c->hcap * (N + 1) * 8);
    dfree(c, c->d_hids, c->hcap * 4);
    if (c->ev_main) cudaEventDestroy(c->ev_main);
    if (c->ev_in) cudaEventDestroy(c->ev_in);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    delete c;
}

extern "C" uint64_t luthe_device_bytes(const luthe_ctx *c) { return c ? c->used : 0; }

extern "C" int luthe_upload_bsk(luthe_ctx *c, const uint64_t *h)
{
    if (!c || !h) return fail(LUTHE_E_PARAM, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t n = c->p.lwe_dim, words = n * 4 * N;
    for (size_t i = 0; i < words; i++)
        if (h[i] >= 0xFFFFFFFF00000001ull) return fail(LUTHE_E_PARAM, "BSK word %zu is not reduced mod p", i);
    int r;
    if (!c->d_bsk && (r = dalloc(c, (void **)&c->d_bsk, n * SLAB_BYTES))) return r;
    uint64_t *d_std = nullptr;
    if ((r = dalloc(c, (void **)&d_std, words * 8))) return r;
    cudaError_t e = cudaMemcpy(d_std, h, words * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_bsk_prepare(d_std, c->d_bsk, c->d_tw, (uint32_t)n, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    dfree(c, d_std, words * 8);
    if (e != cudaSuccess) return fail(LUTHE_E_CUDA, "BSK upload: %s", cudaGetErrorString(e));
    return LUTHE_OK;
}

extern "C" int luthe_upload_bsk_eval(luthe_ctx *c, const uint64_t *h)
{
    if (!c || !h) return fail(LUTHE_E_PARAM, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t n = c->p.lwe_dim, words = n * 4 * N;
    for (size_t i = 0; i < words; i++)
        if (h[i] >= 0xFFFFFFFF00000001ull) return fail(LUTHE_E_PARAM, "BSK word %zu is not reduced mod p", i);
    // slab[i][p][row*2+col][t] = N^-1 * BSK_i[row][col](psi^(2k+1)), k = eval_index(t, p):
    // the layout bsk_prepare_kernel writes from the standard domain
    const uint64_t n_inv = 0xffdfffff00200001ull;  // 2048^-1 mod p
    std::vector<uint64_t> slab(words);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++)
        for (int pp = 0; pp < 8; pp++)
            for (int q = 0; q < 4; q++)
                for (int t = 0; t < 256; t++) {
                    const int k = (t & 31) + 32 * (t >> 5) + 256 * (((pp & 1) << 2) | (pp & 2) | ((pp >> 2) & 1));
                    const unsigned __int128 x = (unsigned __int128)h[((size_t)i * 4 + q) * N + k] * n_inv;
                    slab[(((size_t)i * 8 + pp) * 4 + q) * 256 + t] = (uint64_t)(x % 0xFFFFFFFF00000001ull);
                }
    int r;
    if (!c->d_bsk && (r = dalloc(c, (void **)&c->d_bsk, n * SLAB_BYTES))) return r;
    CUDA_TRY(cudaMemcpy(c->d_bsk, slab.data(), words * 8, cudaMemcpyHostToDevice));
    return LUTHE_OK;
}

extern "C" int luthe_set_tie_rule(luthe_ctx *c, int rule)
{
    if (!c) return fail(LUTHE_E_PARAM, "null ctx");
    if (rule != LUTHE_TIE_RTL && rule != LUTHE_TIE_GENERATOR) return fail(LUTHE_E_PARAM, "unknown tie rule %d", rule);
    if ((uint32_t)rule != c->tie_rule) {
        CUDA_TRY(cudaSetDevice(c->device));
        drop_graphs(c);  // captured launches carry the old rule
        c->tie_rule = (uint32_t)rule;
    }
    return LUTHE_OK;
}

extern "C" int luthe_upload_ksk(luthe_ctx *c, const uint32_t *h)
{
    if (!c || !h) return fail(LUTHE_E_PARAM, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t n = c->p.lwe_dim, K = (size_t)N * c->p.ks_level;
    const uint32_t xpad = (uint32_t)(((n + 1) + KS_BN - 1) / KS_BN * KS_BN);
    // device layout [K/4][3][xpad] for the group g = k/4 of four rows: word 0
    // the low bytes of rows 4g..4g+3, words 1 and 2 their upper 13 bits as
    // 16-bit halves (rows 4g, 4g+1 and 4g+2, 4g+3)
    const size_t words = K / 4 * KS_PLANES * xpad;
    std::vector<uint32_t> t(words, 0);
    const uint32_t M = (1u << KS_W) - 1;
    for (size_t x = 0; x <= n; x++)
        for (size_t k = 0; k < K; k++) {
            const uint32_t v = h[x * K + k] & M, r = (uint32_t)(k % 4);
            const size_t g = (k / 4) * KS_PLANES;
            t[g * xpad + x] |= (v & 0xFFu) << (8 * r);
            t[(g + 1 + r / 2) * xpad + x] |= (v >> 8) << (16 * (r % 2));
        }
    int r;
    if (!c->d_ksk) {
        if ((r = dalloc(c, (void **)&c->d_ksk, words * 4))) return r;
        c->xpad = xpad;
        if ((r = dalloc(c, (void **)&c->d_ks_part, (size_t)KS_BM * xpad * 4))) return r;
        CUDA_TRY(cudaMemset(c->d_ks_part, 0, (size_t)KS_BM * xpad * 4));
    }
    CUDA_TRY(cudaMemcpy(c->d_ksk, t.data(), words * 4, cudaMemcpyHostToDevice));
    return LUTHE_OK;
}

extern "C" int luthe_upload_luts(luthe_ctx *c, const uint64_t *h, uint32_t count)
{
    if (!c || !h || count == 0) return fail(LUTHE_E_PARAM, "bad LUT arguments");
    CUDA_TRY(cudaSetDevice(c->device));
    drop_graphs(c);
    dfree(c, c->d_luts, (size_t)c->nlut * 2 * N * 8);
    c->d_luts = nullptr;
    c->nlut = 0;
    int r;
    if ((r = dalloc(c, (void **)&c->d_luts, (size_t)count * 2 * N * 8))) return r;
    c->nlut = count;
    CUDA_TRY(cudaMemcpy(c->d_luts, h, (size_t)count * 2 * N * 8, cudaMemcpyHostToDevice));
    return LUTHE_OK;
}

int ensure_scratch(luthe_ctx *c, size_t count)
{
    if (count <= c->cap) return LUTHE_OK;
    drop_graphs(c);
    const size_t n1 = c->p.lwe_dim + 1;
    dfree(c, c->d_lwe2N, c->cap * n1 * 4);
    c->d_lwe2N = nullptr;
    c->cap = 0;
    int r = dalloc(c, (void **)&c->d_lwe2N, count * n1 * 4);
    if (r) return r;
    c->cap = count;
    return LUTHE_OK;
}

extern "C" int luthe_reserve(luthe_ctx *c, size_t max_count)
{
    if (!c) return fail(LUTHE_E_PARAM, "null ctx");
    CUDA_TRY(cudaSetDevice(c->device));
    return ensure_scratch(c, max_count);
}

int need_keys(luthe_ctx *c)
{
    if (!c) return fail(LUTHE_E_PARAM, "null ctx");
    if (!c->d_bsk || !c->d_ksk) return fail(LUTHE_E_STATE, "keys not uploaded");
    if (!c->d_luts) return fail(LUTHE_E_STATE, "LUTs not uploaded");
    return LUTHE_OK;
}

static int enqueue_ks_pbs(luthe_ctx *c, const uint64_t *d_in, const uint32_t *d_ids, uint64_t *d_out, size_t count,
                          cudaStream_t s)
{
    const uint32_t n = c->p.lwe_dim;
    CUDA_TRY(launch_keyswitch(d_in, c->d_ksk, nullptr, c->d_lwe2N, count, n, c->xpad, s, nullptr, c->p.ks_base_log,
                              c->p.ks_level, c->tie_rule, c->d_ks_part));
    CUDA_TRY(launch_blind_rotate(c->br, c->nsm, c->d_lwe2N, c->d_luts, d_ids, c->nlut, c->d_bsk, c->d_tw, d_out,
                                 count, n, c->d_err, s, nullptr, 1, c->p.pbs_base_log, c->tie_rule));
    return LUTHE_OK;
}

extern "C" int luthe_ks_pbs(luthe_ctx *c, const uint64_t *d_in, const uint32_t *d_ids, uint64_t *d_out,
                            size_t count, void *stream)
{
    int r = need_keys(c);
    if (r) return r;
    if (count == 0) return LUTHE_OK;
    if (!d_in || !d_ids || !d_out) return fail(LUTHE_E_PARAM, "null buffer");
    CUDA_TRY(cudaSetDevice(c->device));
    if ((r = ensure_scratch(c, count))) return r;
    return enqueue_ks_pbs(c, d_in, d_ids, d_out, count, (cudaStream_t)stream);
}

extern "C" int luthe_ks_pbs_ml(luthe_ctx *c, const uint64_t *d_in, const uint32_t *d_ids, uint64_t *d_out,
                               size_t count, uint32_t mlk, void *stream)
{
    int r = need_keys(c);
    if (r) return r;
    if (mlk != 1 && mlk != 2 && mlk != 4 && mlk != 8) return fail(LUTHE_E_PARAM, "many-LUT factor %u not in {1,2,4,8}", mlk);
    if (count == 0) return LUTHE_OK;
    if (!d_in || !d_ids || !d_out) return fail(LUTHE_E_PARAM, "null buffer");
    CUDA_TRY(cudaSetDevice(c->device));
    if ((r = ensure_scratch(c, count))) return r;
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t n = c->p.lwe_dim;
    CUDA_TRY(launch_keyswitch(d_in, c->d_ksk, nullptr, c->d_lwe2N, count, n, c->xpad, s, nullptr, c->p.ks_base_log,
                              c->p.ks_level, c->tie_rule, c->d_ks_part));
    CUDA_TRY(launch_blind_rotate(c->br, c->nsm, c->d_lwe2N, c->d_luts, d_ids, c->nlut, c->d_bsk, c->d_tw, d_out, count,
                                 n, c->d_err, s, nullptr, mlk, c->p.pbs_base_log, c->tie_rule));
    return LUTHE_OK;
}

extern "C" int luthe_ks_pbs_graph(luthe_ctx *c, const uint64_t *d_in, const uint32_t *d_ids, uint64_t *d_out,
                                  size_t count, void *stream)
{
    int r = need_keys(c);
    if (r) return r;
    if (count == 0) return LUTHE_OK;
    if (!d_in || !d_ids || !d_out) return fail(LUTHE_E_PARAM, "null buffer");
    CUDA_TRY(cudaSetDevice(c->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (!s) return fail(LUTHE_E_PARAM, "graph capture needs a non-default stream");
    if ((r = ensure_scratch(c, count))) return r;
    for (auto &g : c->graphs)
        if (g.in == d_in && g.ids == d_ids && g.out == d_out && g.count == count && g.stream == s) {
            CUDA_TRY(cudaGraphLaunch(g.exec, s));
            return LUTHE_OK;
        }
    cudaGraph_t graph;
    CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    r = enqueue_ks_pbs(c, d_in, d_ids, d_out, count, s);
    cudaError_t e = cudaStreamEndCapture(s, &graph);
    if (r) return r;
    if (e != cudaSuccess) return fail(LUTHE_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
    cudaGraphExec_t exec;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(LUTHE_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    if (c->graphs.size() >= 8) {
        cudaGraphExecDestroy(c->graphs.front().exec);
        c->graphs.erase(c->graphs.begin());
    }
    c->graphs.push_back(GraphEntry{d_in, d_ids, d_out, count, s, exec});
    CUDA_TRY(cudaGraphLaunch(exec, s));
    return LUTHE_OK;
}

// The host-buffer path's copies and launches: the inputs in two chunks on the
// context's copy stream under the key switch, the full waves' outputs back on
// it while a tail launch runs.  The caller drains both streams.
static int enqueue_host_ks_pbs(luthe_ctx *c, const uint64_t *h_in, const uint32_t *h_ids, uint64_t *h_out,
                               size_t count)
{
    cudaStream_t s = 0;
    const uint32_t n = c->p.lwe_dim;
    const size_t row = (size_t)(N + 1);
    CUDA_TRY(cudaMemcpyAsync(c->d_hids, h_ids, count * 4, cudaMemcpyHostToDevice, s));
    // inputs in two chunks on the copy stream, each chunk's key switch as soon
    // as it has landed: a quarter first, whose copy is the only one not hidden
    // behind compute, then the rest, whose key switch still fills the GPU
    const size_t first = count >= 1024 ? (count / 4 + KS_BM - 1) / KS_BM * KS_BM : count;
    for (int k = 0; k < 2; k++) {
        const size_t off = k ? first : 0, m = (k ? count : first) - off;
        if (m == 0) continue;
        CUDA_TRY(cudaMemcpyAsync(c->d_hin + off * row, h_in + off * row, m * row * 8, cudaMemcpyHostToDevice,
                                 c->copy_stream));
        CUDA_TRY(cudaEventRecord(c->ev_in, c->copy_stream));
        CUDA_TRY(cudaStreamWaitEvent(s, c->ev_in, 0));
        CUDA_TRY(launch_keyswitch(c->d_hin + off * row, c->d_ksk, nullptr, c->d_lwe2N + off * (size_t)(n + 1), m,
                                  n, c->xpad, s, nullptr, c->p.ks_base_log, c->p.ks_level, c->tie_rule,
                                  c->d_ks_part));
    }
    size_t full = count;
    CUDA_TRY(launch_blind_rotate(c->br, c->nsm, c->d_lwe2N, c->d_luts, c->d_hids, c->nlut, c->d_bsk, c->d_tw,
                                 c->d_hout, count, n, c->d_err, s, nullptr, 1, c->p.pbs_base_log, c->tie_rule,
                                 c->ev_main, &full));
    size_t early = 0;  // outputs read back on the copy stream while the tail launch runs
    if (full < count) {
        // the full waves' outputs are final before the tail launch: their
        // read-back overlaps the tail on the copy stream
        early = full;
        CUDA_TRY(cudaStreamWaitEvent(c->copy_stream, c->ev_main, 0));
        CUDA_TRY(cudaMemcpyAsync(h_out, c->d_hout, early * row * 8, cudaMemcpyDeviceToHost, c->copy_stream));
    }
    CUDA_TRY(cudaMemcpyAsync(h_out + early * row, c->d_hout + early * row, (count - early) * row * 8,
                             cudaMemcpyDeviceToHost, s));
    return LUTHE_OK;
}

extern "C" int luthe_ks_pbs_host(luthe_ctx *c, const uint64_t *h_in, const uint32_t *h_ids, uint64_t *h_out,
                                 size_t count)
{
    int r = need_keys(c);
    if (r) return r;
    if (count == 0) return LUTHE_OK;
    if (!h_in || !h_ids || !h_out) return fail(LUTHE_E_PARAM, "null buffer");
    CUDA_TRY(cudaSetDevice(c->device));
    for (size_t i = 0; i < count; i++)
        if (h_ids[i] >= c->nlut) return fail(LUTHE_E_PARAM, "LUT id %u at %zu out of range", h_ids[i], i);
    if (count > c->hcap) {
        drop_graphs(c);
        dfree(c, c->d_hin, c->hcap * (N + 1) * 8);
        dfree(c, c->d_hout, c->hcap * (N + 1) * 8);
        dfree(c, c->d_hids, c->hcap * 4);
        c->d_hin = c->d_hout = nullptr;
        c->d_hids = nullptr;
        c->hcap = 0;
        if ((r = dalloc(c, (void **)&c->d_hin, count * (N + 1) * 8)) ||
            (r = dalloc(c, (void **)&c->d_hout, count * (N + 1) * 8)) ||
            (r = dalloc(c, (void **)&c->d_hids, count * 4)))
            return r;
        c->hcap = count;
    }
    if ((r = ensure_scratch(c, count))) return r;
    if (!c->copy_stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&c->ev_main, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming));
    }
    r = enqueue_host_ks_pbs(c, h_in, h_ids, h_out, count);
    // both streams are drained before returning, on an error too: no copy
    // may still write into the caller's buffer afterwards
    const cudaError_t e0 = cudaStreamSynchronize(0), e1 = cudaStreamSynchronize(c->copy_stream);
    if (r) return r;
    if (e0 != cudaSuccess || e1 != cudaSuccess)
        return fail(LUTHE_E_CUDA, "stream synchronize: %s", cudaGetErrorString(e0 != cudaSuccess ? e0 : e1));
    return luthe_check_device_error(c);
}

extern "C" int luthe_keyswitch(luthe_ctx *c, const uint64_t *d_in, uint32_t *d_out21, uint32_t *d_out2N,
                               size_t count, void *stream)
{
    if (!c) return fail(LUTHE_E_PARAM, "null ctx");
    if (!c->d_ksk) return fail(LUTHE_E_STATE, "KSK not uploaded");
    if (count == 0) return LUTHE_OK;
    if (!d_in || !d_out2N) return fail(LUTHE_E_PARAM, "null buffer");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(launch_keyswitch(d_in, c->d_ksk, d_out21, d_out2N, count, c->p.lwe_dim, c->xpad,
                              (cudaStream_t)stream, nullptr, c->p.ks_base_log, c->p.ks_level, c->tie_rule,
                              c->d_ks_part));
    return LUTHE_OK;
}

extern "C" int luthe_blind_rotate(luthe_ctx *c, const uint32_t *d_lwe2N, const uint32_t *d_ids, uint64_t *d_out,
                                  size_t count, void *stream)
{
    int r = need_keys(c);
    if (r) return r;
    if (count == 0) return LUTHE_OK;
    if (!d_lwe2N || !d_ids || !d_out) return fail(LUTHE_E_PARAM, "null buffer");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(launch_blind_rotate(c->br, c->nsm, d_lwe2N, c->d_luts, d_ids, c->nlut, c->d_bsk, c->d_tw, d_out, count,
                                 c->p.lwe_dim, c->d_err, (cudaStream_t)stream, nullptr, 1, c->p.pbs_base_log, c->tie_rule));
    return LUTHE_OK;
}

extern "C" int luthe_ntt_fwd(luthe_ctx *c, const uint64_t *d_in, uint64_t *d_out, size_t count, void *stream)
{
    if (!c || (count && (!d_in || !d_out))) return fail(LUTHE_E_PARAM, "bad argument");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(launch_ntt_fwd(d_in, d_out, c->d_tw, count, (cudaStream_t)stream));
    return LUTHE_OK;
}
extern "C" int luthe_ntt_inv(luthe_ctx *c, const uint64_t *d_in, uint64_t *d_out, size_t count, void *stream)
{
    if (!c || (count && (!d_in || !d_out))) return fail(LUTHE_E_PARAM, "bad argument");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(launch_ntt_inv(d_in, d_out, c->d_tw, count, (cudaStream_t)stream));
    return LUTHE_OK;
}
extern "C" int luthe_ntt_mul(luthe_ctx *c, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out, size_t count,
                             void *stream)
{
    if (!c || (count && (!d_a || !d_b || !d_out))) return fail(LUTHE_E_PARAM, "bad argument");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(launch_ntt_mul(d_a, d_b, d_out, c->d_tw, count, (cudaStream_t)stream));
    return LUTHE_OK;
}

extern "C" int luthe_lwe_op(luthe_ctx *c, int op, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out,
                            uint64_t imm, size_t count, void *stream)
{
    if (!c) return fail(LUTHE_E_PARAM, "null ctx");
    if (op < LUTHE_OP_ADD || op > LUTHE_OP_MULS) return fail(LUTHE_E_PARAM, "unknown linear op %d", op);
    const bool two = op == LUTHE_OP_ADD || op == LUTHE_OP_SUB || op == LUTHE_OP_MAC;
    if (count && (!d_a || !d_out || (two && !d_b))) return fail(LUTHE_E_PARAM, "null buffer");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(launch_lwe_op(op, d_a, d_b, d_out, imm, count, (uint32_t)(c->p.glwe_dim * c->p.poly_size),
                           (cudaStream_t)stream));
    return LUTHE_OK;
}

extern "C" int luthe_set_br_config(luthe_ctx *c, int g, int per_sm)
{
    if (!c) return fail(LUTHE_E_PARAM, "null ctx");
    if (g < 1 || g > 2 || per_sm < 1) return fail(LUTHE_E_PARAM, "bad BR config %d/%d", g, per_sm);
    BrConfig cfg{g, per_sm};
    CUDA_TRY(cudaSetDevice(c->device));
    size_t smem = br_smem_bytes(cfg, c->p.lwe_dim);
    int max_smem = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device));
    int blocks = (int)(max_smem / (smem + 1024));
    if (blocks < per_sm) return fail(LUTHE_E_PARAM, "BR config %d/%d needs %zu B shared memory per CTA", g, per_sm,
                                     smem);
    drop_graphs(c);
    c->br = cfg;
    return LUTHE_OK;
}

extern "C" int luthe_check_device_error(luthe_ctx *c)
{
    if (!c) return fail(LUTHE_E_PARAM, "null ctx");
    uint32_t e = 0;
    CUDA_TRY(cudaMemcpy(&e, c->d_err, 4, cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(c->d_err, 0, 4);
        if (e & DEVERR_DRAIN)
            return fail(LUTHE_E_TIMEOUT,
                        "blind rotation: a bounded wait ran out and a BSK copy still in flight did not finish "
                        "landing in shared memory; the device state is unsafe: destroy this context and "
                        "end the process before further use of the device");
        if (e & DEVERR_TIMEOUT)
            return fail(LUTHE_E_TIMEOUT, "blind rotation: bounded wait for a BSK slab ran out%s",
                        (e & DEVERR_LUT_ID) ? " (and a LUT id was out of range)" : "");
        return fail(LUTHE_E_PARAM, "blind rotation: a LUT id was >= the uploaded LUT count (%u)", c->nlut);
    }
    return LUTHE_OK;
}

// ------------------------------------------------------------ autotuner
//
// The blind rotation's launch shape is chosen per batch size (kernels.cu,
// launch_blind_rotate): ciphertexts per CTA (G), and the batch sizes up to
// which a batch runs one ciphertext per 2-SM cluster (pair_max) or one per
// CTA (split_max), and up to which a partial last wave runs as its own launch
// of those forms (tail_max).  The autotuner times every form around each
// decision point on this device and keeps the fastest; the choice can be
// saved as JSON and loaded by later contexts (the counterpart of the HPU's
// batch configuration, pep_sequencer.sv:573-620 and docs/hpu_parameters.md).

namespace {

struct Timer {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    Timer() { cudaEventCreate(&e0); cudaEventCreate(&e1); }
    ~Timer() { cudaEventDestroy(e0); cudaEventDestroy(e1); }
};

// median of three timed launches after one untimed launch, in ms; < 0 on error
float time_br(luthe_ctx *c, const BrConfig &cfg, const uint32_t *d_l, const uint32_t *d_ids, uint64_t *d_o, size_t B,
              Timer &t)
{
    const uint32_t n = c->p.lwe_dim;
    float ms[3];
    for (int r = -1; r < 3; r++) {
        if (r >= 0) cudaEventRecord(t.e0, 0);
        cudaError_t e = launch_blind_rotate(cfg, c->nsm, d_l, c->d_luts, d_ids, c->nlut, c->d_bsk, c->d_tw, d_o, B, n,
                                            c->d_err, 0, nullptr, 1, c->p.pbs_base_log, c->tie_rule);
        if (e != cudaSuccess) return -1.f;
        if (r >= 0) {
            cudaEventRecord(t.e1, 0);
            if (cudaEventSynchronize(t.e1) != cudaSuccess) return -1.f;
            cudaEventElapsedTime(&ms[r], t.e0, t.e1);
        }
    }
    if (ms[0] > ms[1]) std::swap(ms[0], ms[1]);
    if (ms[1] > ms[2]) std::swap(ms[1], ms[2]);
    if (ms[0] > ms[1]) std::swap(ms[0], ms[1]);
    return ms[1];
}

std::string tuning_key(const luthe_ctx *c)
{
    cudaDeviceProp prop;
    std::string name = cudaGetDeviceProperties(&prop, c->device) == cudaSuccess ? prop.name : "unknown";
    for (auto &ch : name)
        if (!isalnum((unsigned char)ch)) ch = '_';
    char buf[160];
    snprintf(buf, sizeof buf, "%s_sm%d_n%u_ks%ux%u_pbs%u", name.c_str(), c->nsm, c->p.lwe_dim, c->p.ks_base_log,
             c->p.ks_level, c->p.pbs_base_log);
    return buf;
}

std::string tuning_json(const luthe_ctx *c)
{
    char buf[512];
    snprintf(buf, sizeof buf,
             "{\"format\":\"luthe-tuning-1\",\"key\":\"%s\",\"cts_per_cta\":%d,\"ctas_per_sm\":%d,"
             "\"pair_max\":%d,\"split_max\":%d,\"tail_max\":%d}",
             tuning_key(c).c_str(), c->br.cts_per_cta, c->br.ctas_per_sm, c->br.pair_max, c->br.split_max,
             c->br.tail_max);
    return buf;
}

// integer value of "key": in a flat JSON object written by tuning_json
bool json_int(const std::string &js, const char *key, int *out)
{
    const std::string k = std::string("\"") + key + "\":";
    size_t at = js.find(k);
    if (at == std::string::npos) return false;
    char *end = nullptr;
    long v = strtol(js.c_str() + at + k.size(), &end, 10);
    if (end == js.c_str() + at + k.size()) return false;
    *out = (int)v;
    return true;
}

std::string tuning_dir_path(const luthe_ctx *c)
{
    const char *dir = getenv("LUTHE_TUNING_DIR");
    if (!dir || !*dir) return "";
    return std::string(dir) + "/luthe_tune_" + tuning_key(c) + ".json";
}

}  // namespace

extern "C" int luthe_tuning_load(luthe_ctx *c, const char *path)
{
    if (!c || !path) return fail(LUTHE_E_PARAM, "null argument");
    FILE *f = fopen(path, "r");
    if (!f) return fail(LUTHE_E_PARAM, "tuning file %s: cannot open", path);
    std::string js;
    char buf[1024];
    size_t got;
    while ((got = fread(buf, 1, sizeof buf, f)) > 0) js.append(buf, got);
    fclose(f);
    if (js.find("\"format\":\"luthe-tuning-1\"") == std::string::npos)
        return fail(LUTHE_E_PARAM, "tuning file %s: not a luthe-tuning-1 record", path);
    const std::string key = "\"key\":\"" + tuning_key(c) + "\"";
    if (js.find(key) == std::string::npos)
        return fail(LUTHE_E_PARAM, "tuning file %s was made for another device or parameter set (want %s)", path,
                    tuning_key(c).c_str());
    BrConfig b = c->br;
    if (!json_int(js, "cts_per_cta", &b.cts_per_cta) || !json_int(js, "ctas_per_sm", &b.ctas_per_sm) ||
        !json_int(js, "pair_max", &b.pair_max) || !json_int(js, "split_max", &b.split_max) ||
        !json_int(js, "tail_max", &b.tail_max))
        return fail(LUTHE_E_PARAM, "tuning file %s: missing fields", path);
    if (b.cts_per_cta < 1 || b.cts_per_cta > 2 || b.ctas_per_sm != 1)
        return fail(LUTHE_E_PARAM, "tuning file %s: unsupported launch shape %d/%d", path, b.cts_per_cta, b.ctas_per_sm);
    CUDA_TRY(cudaSetDevice(c->device));
    drop_graphs(c);
    c->br = b;
    return LUTHE_OK;
}

extern "C" int luthe_tuning_save(luthe_ctx *c, const char *path)
{
    if (!c || !path) return fail(LUTHE_E_PARAM, "null argument");
    FILE *f = fopen(path, "w");
    if (!f) return fail(LUTHE_E_PARAM, "tuning file %s: cannot write", path);
    const std::string js = tuning_json(c) + "\n";
    const bool ok = fwrite(js.data(), 1, js.size(), f) == js.size();
    if (fclose(f) != 0 || !ok) return fail(LUTHE_E_PARAM, "tuning file %s: write failed", path);
    return LUTHE_OK;
}

int tuning_autoload(luthe_ctx *c)
{
    const std::string path = tuning_dir_path(c);
    if (path.empty()) return LUTHE_OK;
    FILE *f = fopen(path.c_str(), "r");
    if (!f) return LUTHE_OK;  // nothing tuned yet for this device and parameter set
    fclose(f);
    return luthe_tuning_load(c, path.c_str());
}

extern "C" int luthe_autotune(luthe_ctx *c, size_t sample, char *json, size_t cap)
{
    int r = need_keys(c);
    if (r) return r;
    CUDA_TRY(cudaSetDevice(c->device));
    const int nsm = c->nsm;
    if (sample == 0) sample = (size_t)nsm * 8;  // four two-per-CTA waves
    const size_t maxB = std::max(sample, (size_t)nsm * 2 + (size_t)nsm * 3 / 2);
    const uint32_t n = c->p.lwe_dim;
    uint32_t *d_l = nullptr, *d_ids = nullptr;
    uint64_t *d_o = nullptr;
    if ((r = dalloc(c, (void **)&d_l, maxB * (n + 1) * 4))) return r;
    if ((r = dalloc(c, (void **)&d_ids, maxB * 4)) || (r = dalloc(c, (void **)&d_o, maxB * (N + 1) * 8))) {
        dfree(c, d_l, maxB * (n + 1) * 4);
        dfree(c, d_ids, maxB * 4);
        return r;
    }
    auto release = [&]() {
        dfree(c, d_l, maxB * (n + 1) * 4);
        dfree(c, d_ids, maxB * 4);
        dfree(c, d_o, maxB * (N + 1) * 8);
    };
    // deterministic pseudo-random mod-switched inputs
    std::vector<uint32_t> hl(maxB * (n + 1));
    uint64_t st = 0x9E3779B97F4A7C15ull;
    for (auto &v : hl) {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        v = (uint32_t)(st & (TWO_N - 1));
    }
    cudaError_t ce = cudaMemcpy(d_l, hl.data(), hl.size() * 4, cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemset(d_ids, 0, maxB * 4);
    if (ce != cudaSuccess) {
        release();
        return fail(LUTHE_E_CUDA, "autotune: %s", cudaGetErrorString(ce));
    }
    Timer tm;
    std::string rec = "{\"sample\":" + std::to_string(sample) + ",\"trials\":[";
    bool first = true, failed = false;
    auto trial = [&](const char *what, size_t B, const BrConfig &cfg) -> float {
        float ms = time_br(c, cfg, d_l, d_ids, d_o, B, tm);
        if (ms < 0) failed = true;
        char buf[200];
        snprintf(buf, sizeof buf, "%s{\"form\":\"%s\",\"B\":%zu,\"ms\":%.4f}", first ? "" : ",", what, B, ms);
        rec += buf;
        first = false;
        return ms;
    };
    const int BIG = 1 << 30;
    BrConfig best = c->br;
    // 1. ciphertexts per CTA on full waves
    {
        BrConfig g1{1, 1, 0, 0, 0}, g2{2, 1, 0, 0, 0};
        const float t1 = trial("G1", sample, g1), t2 = trial("G2", sample, g2);
        best.cts_per_cta = (t1 >= 0 && t1 < t2) ? 1 : 2;
        best.ctas_per_sm = 1;
    }
    if (best.cts_per_cta == 2 && !failed) {
        // 2. small batches: 2-SM clusters, one per CTA, or a two-per-CTA launch
        int pair_max = 0, split_max = 0;
        for (int k = 1; k <= 12; k++) {
            const size_t B = (size_t)nsm * k / 8;
            if (B == 0) continue;
            const float tp = trial("pair", B, BrConfig{2, 1, BIG, BIG, 0});
            const float ts = trial("split", B, BrConfig{2, 1, 0, BIG, 0});
            const float tw = trial("wave", B, BrConfig{2, 1, 0, 0, 0});
            if (tp >= 0 && tp <= ts && tp <= tw) pair_max = (int)B;
            if (std::min(tp, ts) >= 0 && std::min(tp, ts) < tw) split_max = (int)B;
        }
        // 3. a partial last wave: its own small launch, or part of the wave launch
        int tail_max = 0;
        for (int k = 1; k <= 8; k++) {
            const size_t t = (size_t)nsm * k / 4, B = (size_t)2 * nsm + t;
            if (t == 0 || t >= (size_t)2 * nsm || B > maxB) continue;
            const float ta = trial("wave+tail", B, BrConfig{2, 1, pair_max, split_max, BIG});
            const float tb = trial("waves", B, BrConfig{2, 1, pair_max, split_max, 0});
            if (ta >= 0 && ta < tb) tail_max = (int)t;
        }
        best.pair_max = pair_max;
        best.split_max = std::max(split_max, pair_max);
        best.tail_max = tail_max;
    }
    release();
    if (failed) return fail(LUTHE_E_CUDA, "autotune: a trial launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    drop_graphs(c);
    c->br = best;
    rec += "],\"chosen\":" + tuning_json(c);
    const std::string path = tuning_dir_path(c);
    if (!path.empty() && (r = luthe_tuning_save(c, path.c_str()))) return r;
    rec += ",\"saved_to\":\"" + path + "\"}";
    if (json && cap) {
        strncpy(json, rec.c_str(), cap - 1);
        json[cap - 1] = 0;
    }
    return luthe_check_device_error(c);
}

// ------------------------------------------------------------------------
// KS+PBS without any device allocation.
//
// Some callers cannot call cudaMalloc while they run: code inside a memory
// arena or allocator hook (a cudaMalloc there re-enters the allocator), code
// running under a budget that forbids new device memory once it is set up, or
// a host framework that owns all device memory and hands out only the buffers
// it allocated.  For them, the key-switched intermediate (count x (n+1) u32)
// lives in the fixed array below instead of the context's growable scratch.
//
// The array is 4 MiB and exists on every GPU that loads this library, for the
// life of the process.  Every call shares it and it keeps the last call's
// contents; the key switch overwrites every word the blind rotation then reads,
// so nothing needs clearing between calls.  Calls that overlap on the GPU
// (several streams, or several contexts on one device) race on it.
static constexpr size_t NOALLOC_SCRATCH_WORDS = 1u << 20;
static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_SCRATCH_WORDS];

// In host code g_noalloc_scratch names a host-side stand-in, not device memory:
// the kernels get the device address, looked up once per device with that
// device current.  The per-device address is published with release/acquire
// ordering, so host threads making their first calls at the same time (on one
// device or on several) either see the full address or look it up again; a
// repeated lookup returns the same address.
static std::atomic<uint32_t *> g_noalloc_addr[64];

extern "C" int luthe_ks_pbs_noalloc(luthe_ctx *c, const uint64_t *d_in, const uint32_t *d_ids, uint64_t *d_out,
                                    size_t count, void *stream)
{
    int r = need_keys(c);
    if (r) return r;
    if (count == 0) return LUTHE_OK;
    if (!d_in || !d_ids || !d_out) return fail(LUTHE_E_PARAM, "null buffer");
    const size_t n1 = (size_t)c->p.lwe_dim + 1;
    if (count > NOALLOC_SCRATCH_WORDS / n1)
        return fail(LUTHE_E_PARAM, "luthe_ks_pbs_noalloc: %zu ciphertexts exceed the fixed scratch (at most %zu at n=%u)",
                    count, NOALLOC_SCRATCH_WORDS / n1, c->p.lwe_dim);
    if (c->device < 0 || c->device >= 64) return fail(LUTHE_E_PARAM, "device index %d out of range", c->device);
    CUDA_TRY(cudaSetDevice(c->device));
    uint32_t *scratch = g_noalloc_addr[c->device].load(std::memory_order_acquire);
    if (!scratch) {
        void *addr = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&addr, g_noalloc_scratch));
        if (!addr) return fail(LUTHE_E_CUDA, "luthe_ks_pbs_noalloc: no device address for the fixed scratch");
        scratch = (uint32_t *)addr;
        g_noalloc_addr[c->device].store(scratch, std::memory_order_release);
    }
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t n = c->p.lwe_dim;
    CUDA_TRY(launch_keyswitch(d_in, c->d_ksk, nullptr, scratch, count, n, c->xpad, s, nullptr, c->p.ks_base_log, c->p.ks_level, c->tie_rule));
    CUDA_TRY(launch_blind_rotate(c->br, c->nsm, scratch, c->d_luts, d_ids, c->nlut, c->d_bsk, c->d_tw, d_out, count, n,
                                 c->d_err, s, nullptr, 1, c->p.pbs_base_log, c->tie_rule));
    return LUTHE_OK;
}
