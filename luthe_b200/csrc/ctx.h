// Internal: the context shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>
#include "../../include/luthe.h"
#include "kernels.cuh"

struct GraphEntry {
    const void *in, *ids;
    void *out;
    size_t count;
    cudaStream_t stream;
    cudaGraphExec_t exec;
};

struct luthe_ctx {
    luthe_params p;
    int device = 0;
    int nsm = 148;
    uint64_t budget = 0, used = 0;
    uint64_t *d_tw = nullptr;     // [2][8][256]
    uint64_t *d_bsk = nullptr;    // [n][8][2][2][256]
    uint32_t *d_ksk = nullptr;    // [kN*L/4][KS_PLANES][xpad]: 4 K-rows per group (low bytes, upper halves)
    uint32_t xpad = 0;
    uint32_t *d_ks_part = nullptr;  // [KS_BM][xpad] split-K partial sums of small key switches (kept zero)
    uint64_t *d_luts = nullptr;   // [nlut][2][N]
    uint32_t nlut = 0;
    uint32_t *d_err = nullptr;
    // scratch
    uint32_t *d_lwe2N = nullptr;  // [cap][n+1]
    size_t cap = 0;
    // host-path staging
    uint64_t *d_hin = nullptr, *d_hout = nullptr;
    uint32_t *d_hids = nullptr;
    size_t hcap = 0;
    cudaStream_t copy_stream = nullptr;  // host path: read-back of the full waves while the tail runs
    cudaEvent_t ev_main = nullptr;       // recorded after the full waves' launch
    cudaEvent_t ev_in = nullptr;         // host path: a chunk of inputs has landed
    luthe::BrConfig br{2, 1};
    uint32_t tie_rule = luthe::TIE_RTL;  // decomposition tie rule (luthe_set_tie_rule)
    std::vector<GraphEntry> graphs;
};

extern thread_local char g_err[512];
int fail(int code, const char *fmt, ...);
int dalloc(luthe_ctx *c, void **ptr, size_t bytes);
void dfree(luthe_ctx *c, void *ptr, size_t bytes);
void drop_graphs(luthe_ctx *c);
int ensure_scratch(luthe_ctx *c, size_t count);
int need_keys(luthe_ctx *c);

#define CUDA_TRY(expr)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (expr);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(LUTHE_E_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_),    \
                        __FILE__, __LINE__);                                              \
    } while (0)
