// CPU harness of the serving loop (test infrastructure only): the real
// scheduler of luthe_b200/csrc/serve.cu over a plaintext model of the device.
// A pool slot's first word holds the clear payload; the ALU batch applies the
// DOp arithmetic mod 32 (padding bit included); a "PBS" applies the LUT of the
// request's gid to the payload, many-LUT outputs to consecutive slots.
#include <stdarg.h>
#include <stdio.h>
#include "../../luthe_b200/csrc/serve.cu"

thread_local char g_err[512] = "";
int fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}
int dalloc(luthe_ctx *c, void **p, size_t bytes)
{
    if (c->used + bytes > c->budget) return fail(LUTHE_E_BUDGET, "budget");
    *p = calloc(1, bytes);
    c->used += bytes;
    return *p ? LUTHE_OK : LUTHE_E_BUDGET;
}
void dfree(luthe_ctx *c, void *p, size_t bytes)
{
    if (p) {
        free(p);
        c->used -= bytes;
    }
}
void drop_graphs(luthe_ctx *) {}
int ensure_scratch(luthe_ctx *, size_t) { return LUTHE_OK; }
int need_keys(luthe_ctx *c) { return c->d_luts ? LUTHE_OK : fail(LUTHE_E_STATE, "no LUTs"); }

namespace luthe {
static uint32_t g_w = 2049;
cudaError_t launch_alu_batch(const AluOp *ops, uint64_t *pool, uint32_t nops, uint32_t, cudaStream_t)
{
    for (uint32_t i = 0; i < nops; i++) {
        const AluOp &o = ops[i];
        const uint64_t a = pool[(size_t)o.a * g_w], b = pool[(size_t)o.b * g_w];
        uint64_t v;
        switch (o.op) {
        case LWE_ADD: v = a + b; break;
        case LWE_SUB: v = a - b; break;
        case LWE_MAC: v = a * o.imm + b; break;
        case LWE_ADDS: v = a + o.imm; break;
        case LWE_SUBS: v = a - o.imm; break;
        case LWE_SSUB: v = o.imm - a; break;
        case LWE_MULS: v = a * o.imm; break;
        default: v = a; break;
        }
        pool[(size_t)o.dst * g_w] = v & 31;
    }
    return cudaSuccess;
}
cudaError_t launch_keyswitch(const uint64_t *in, const uint32_t *, uint32_t *, uint32_t *out2N, size_t B, uint32_t n,
                             uint32_t, cudaStream_t, const uint32_t *src_idx, uint32_t, uint32_t, uint32_t, uint32_t *)
{
    for (size_t c = 0; c < B; c++) out2N[c * (n + 1)] = (uint32_t)in[(size_t)(src_idx ? src_idx[c] : c) * g_w];
    return cudaSuccess;
}
// launches seen: batch size and the cluster-pair cut-off the scheduler passed
static std::vector<std::pair<size_t, int>> g_launch_log;
cudaError_t launch_blind_rotate(const BrConfig &cfg, int, const uint32_t *l2n, const uint64_t *luts, const uint32_t *ids,
                                uint32_t, const uint64_t *, const uint64_t *, uint64_t *out, size_t B, uint32_t n,
                                uint32_t *, cudaStream_t, const uint32_t *dst_idx, uint32_t mlk, uint32_t, uint32_t,
                                cudaEvent_t, size_t *)
{
    g_launch_log.push_back({B, cfg.pair_max});
    for (size_t c = 0; c < B; c++) {
        const uint32_t x = l2n[c * (n + 1)];
        if (x >= 16 / mlk) return cudaErrorInvalidValue;  // payload out of the LUT's range
        for (uint32_t m = 0; m < mlk; m++)
            out[(size_t)(dst_idx[c] + m) * g_w] = luts[(size_t)ids[c] * 16 + m * (16 / mlk) + x];
    }
    return cudaSuccess;
}
}  // namespace luthe

extern "C" luthe_ctx *harness_ctx(uint32_t n, const uint64_t *tables, uint32_t nlut, uint64_t budget)
{
    luthe_ctx *c = new luthe_ctx();
    c->p.lwe_dim = n;
    c->p.poly_size = 2048;
    c->xpad = 896;
    c->budget = budget;
    c->nlut = nlut;
    c->d_err = (uint32_t *)calloc(1, 4);
    c->d_luts = (uint64_t *)malloc((size_t)nlut * 16 * 8);
    memcpy(c->d_luts, tables, (size_t)nlut * 16 * 8);
    return c;
}
extern "C" void harness_set_event_lag(int polls) { g_fake_event_lag = polls; }
extern "C" void harness_set_nsm(luthe_ctx *c, int nsm) { c->nsm = nsm; }
// copies up to cap logged launches (batch size, pair cut-off), clears the log,
// returns how many there were
extern "C" int harness_launch_log(int64_t *batch, int *pair_max, int cap)
{
    const int n = (int)luthe::g_launch_log.size();
    for (int i = 0; i < n && i < cap; i++) {
        batch[i] = (int64_t)luthe::g_launch_log[i].first;
        pair_max[i] = luthe::g_launch_log[i].second;
    }
    luthe::g_launch_log.clear();
    return n;
}

extern "C" void harness_ctx_free(luthe_ctx *c)
{
    free(c->d_err);
    free(c->d_luts);
    delete c;
}
