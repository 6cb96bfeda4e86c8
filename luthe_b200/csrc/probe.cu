// Integer-pipe peak probes: the roofline denominators of the integer-bound
// kernels (no vendor figure exists for them).
//  - 32-bit IMAD: independent multiply-add chains, 16 per thread.
//  - Goldilocks multiply: independent gl::mul chains, 8 per thread.
#include <cuda_runtime.h>
#include "../../include/luthe.h"
#include "gl.cuh"

namespace {

constexpr int ITERS = 1024;

__global__ void __launch_bounds__(256) imad_probe(u32 *out, u32 seed)
{
    u32 a[16];
#pragma unroll
    for (int i = 0; i < 16; i++) a[i] = seed + threadIdx.x * 17u + i;
    const u32 m = seed | 1u, c = seed * 3u + 1u;
#pragma unroll 4
    for (int it = 0; it < ITERS; it++)
#pragma unroll
        for (int i = 0; i < 16; i++) a[i] = a[i] * m + c;
    u32 r = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) r ^= a[i];
    if (r == 0x12345678u) out[0] = r;  // keeps the chains live
}

__global__ void __launch_bounds__(256) glmul_probe(u64 *out, u64 seed)
{
    u64 a[8];
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = seed + threadIdx.x * 977ull + i;
    const u64 m = seed | 0x1234567890ull;
#pragma unroll 2
    for (int it = 0; it < ITERS; it++)
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] = gl::mul(a[i], m);
    u64 r = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) r ^= a[i];
    if (r == 0x123456789ull) out[0] = r;
}

template <typename K, typename T>
float time_probe(K kernel, T *buf, T seed, int blocks)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    kernel<<<blocks, 256>>>(buf, seed);
    float best = 1e30f;
    for (int round = 0; round < 3; round++) {  // best of three rounds of five launches
        cudaEventRecord(e0);
        for (int r = 0; r < 5; r++) kernel<<<blocks, 256>>>(buf, seed + r);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best / 5;
}

}  // namespace

extern "C" int luthe_measure_int_peak(int device, double *imad_per_s, double *glmul_per_s)
{
    if (cudaSetDevice(device) != cudaSuccess) return LUTHE_E_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8;
    void *buf = nullptr;
    if (cudaMalloc(&buf, 64) != cudaSuccess) return LUTHE_E_CUDA;
    float t1 = time_probe(imad_probe, (u32 *)buf, 12345u, blocks);
    float t2 = time_probe(glmul_probe, (u64 *)buf, (u64)0x9E3779B97F4A7C15ull, blocks);
    cudaError_t e = cudaGetLastError();
    cudaFree(buf);
    if (e != cudaSuccess) return LUTHE_E_CUDA;
    const double threads = (double)blocks * 256;
    if (imad_per_s) *imad_per_s = threads * ITERS * 16 / (t1 * 1e-3);
    if (glmul_per_s) *glmul_per_s = threads * ITERS * 8 / (t2 * 1e-3);
    return LUTHE_OK;
}
