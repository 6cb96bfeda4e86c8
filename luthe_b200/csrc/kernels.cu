// sm_100a kernels of the KS+PBS engine: BSK preparation, standalone NTTs,
// the LWE key switch, the persistent blind rotation and the linear DOps.
#include <cooperative_groups.h>

#include "kernels.cuh"
#include "ntt.cuh"

namespace luthe {

using ntt::TPG;
using ntt::POLY_WORDS;

// ------------------------------------------------------------------ twiddles

static uint64_t h_mulmod(uint64_t a, uint64_t b)
{
    unsigned __int128 x = (unsigned __int128)a * b;
    return (uint64_t)(x % gl::P);
}
static uint64_t h_pow(uint64_t a, uint64_t e)
{
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = h_mulmod(r, a);
        a = h_mulmod(a, a);
        e >>= 1;
    }
    return r;
}
// psi: primitive 4096-th root of unity with psi^64 = 8
static const uint64_t PSI_4096 = 0x984ec5194d005735ull;

void build_twiddles(uint64_t *tw)
{
    for (int s = 0; s < 8; s++)
        for (int t = 0; t < TPG; t++) {
            int k1 = ntt::a2_k1(t, s), j2 = t & 63;
            uint64_t e = (uint64_t)(j2 * (2 * k1 + 1)) % TWO_N;
            tw[s * TPG + t] = h_pow(PSI_4096, e);
            tw[2048 + s * TPG + t] = h_pow(PSI_4096, (TWO_N - e) % TWO_N);
        }
}

static const uint64_t N_INV = 0xffdfffff00200001ull;  // 2048^-1 mod p

// ------------------------------------------------------------ BSK prepare
//
// One CTA per blind-rotation step i: the four standard-domain polynomials
// BSK_i[row][col] (values < p) go through the forward NTT and are scaled by
// N^-1 (the INTT's 1/N is folded here), then stored in the evaluation layout
// of the BR kernel: slab[i][p][row][col][t], 64 KiB per step, so that a step's
// slab is one contiguous bulk copy.
__global__ void __launch_bounds__(256) bsk_prepare_kernel(const u64 *__restrict__ std_p, u64 *__restrict__ slab,
                                                           const u64 *__restrict__ tw)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    u64 *buf = reinterpret_cast<u64 *>(smem_raw);
    const int t = threadIdx.x;
    const size_t i = blockIdx.x;
    u64 x[4][8];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int e = 0; e < 8; e++) x[q][e] = std_p[(i * 4 + q) * N + ntt::coef_index(t, e)];
    ntt::forward<4>(x, buf, tw, t, 1);
#pragma unroll
    for (int p = 0; p < 8; p++)
#pragma unroll
        for (int q = 0; q < 4; q++) slab[((i * 8 + p) * 4 + q) * TPG + t] = gl::canon(gl::mul(x[q][p], N_INV));
}

cudaError_t launch_bsk_prepare(const uint64_t *d_std_p, uint64_t *d_slab, const uint64_t *d_tw, uint32_t n,
                               cudaStream_t s)
{
    size_t smem = 4 * POLY_WORDS * 8;
    cudaError_t e = cudaFuncSetAttribute(bsk_prepare_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    bsk_prepare_kernel<<<n, TPG, smem, s>>>(d_std_p, d_slab, d_tw);
    return cudaGetLastError();
}

// ------------------------------------------------------------ standalone NTT
//
// G polynomials (or pairs) per CTA, 256 threads each; the twiddle tables are
// staged once per CTA in shared memory.

template <int G>
__device__ __forceinline__ void load_tw(u64 *tws, const u64 *__restrict__ tw, int words)
{
    for (int i = threadIdx.x; i < words; i += G * TPG) tws[i] = tw[i];
}

// forward: coefficient order in, evaluation order k out (A_k = A(psi^{2k+1}))
template <int G>
__global__ void __launch_bounds__(G * 256) ntt_fwd_kernel(const u64 *__restrict__ in, u64 *__restrict__ out,
                                                           const u64 *__restrict__ tw, size_t count)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    u64 *tws = reinterpret_cast<u64 *>(smem_raw);
    u64 *buf = tws + 2048 + (threadIdx.x >> 8) * POLY_WORDS;
    load_tw<G>(tws, tw, 2048);
    __syncthreads();
    const int t = threadIdx.x & 255, bar = 1 + (threadIdx.x >> 8);
    for (size_t poly = (size_t)blockIdx.x * G + (threadIdx.x >> 8); poly < ((count + G - 1) / G) * G;
         poly += (size_t)gridDim.x * G) {
        const size_t src = poly < count ? poly : count - 1;
        u64 x[1][8];
#pragma unroll
        for (int e = 0; e < 8; e++) x[0][e] = in[src * N + ntt::coef_index(t, e)];
        ntt::forward<1>(x, buf, tws, t, bar);
        if (poly < count) {
#pragma unroll
            for (int p = 0; p < 8; p++) out[poly * N + ntt::eval_index(t, p)] = gl::canon(x[0][p]);
        }
        ntt::group_sync(bar);
    }
}

// inverse: evaluation order in, coefficient order out, with the 1/N factor
template <int G>
__global__ void __launch_bounds__(G * 256) ntt_inv_kernel(const u64 *__restrict__ in, u64 *__restrict__ out,
                                                           const u64 *__restrict__ tw, size_t count)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    u64 *tws = reinterpret_cast<u64 *>(smem_raw);
    u64 *buf = tws + 2048 + (threadIdx.x >> 8) * POLY_WORDS;
    load_tw<G>(tws, tw + 2048, 2048);
    __syncthreads();
    const int t = threadIdx.x & 255, bar = 1 + (threadIdx.x >> 8);
    for (size_t poly = (size_t)blockIdx.x * G + (threadIdx.x >> 8); poly < ((count + G - 1) / G) * G;
         poly += (size_t)gridDim.x * G) {
        const size_t src = poly < count ? poly : count - 1;
        u64 x[1][8];
#pragma unroll
        for (int p = 0; p < 8; p++) x[0][p] = gl::div2k(in[src * N + ntt::eval_index(t, p)], 11);  // x N^-1 = x 2^-11
        ntt::inverse<1>(x, buf, tws, t, bar);
        if (poly < count) {
#pragma unroll
            for (int e = 0; e < 8; e++) out[poly * N + ntt::coef_index(t, e)] = gl::canon(x[0][e]);
        }
        ntt::group_sync(bar);
    }
}

// negacyclic product of pairs: INTT(NTT(a) * NTT(b))
template <int G>
__global__ void __launch_bounds__(G * 256, 2) ntt_mul_kernel(const u64 *__restrict__ a, const u64 *__restrict__ b,
                                                           u64 *__restrict__ out, const u64 *__restrict__ tw,
                                                           size_t count)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    u64 *tws = reinterpret_cast<u64 *>(smem_raw);
    u64 *buf = tws + 4096 + (threadIdx.x >> 8) * 2 * POLY_WORDS;
    load_tw<G>(tws, tw, 4096);
    __syncthreads();
    const int t = threadIdx.x & 255, bar = 1 + (threadIdx.x >> 8);
    for (size_t pr = (size_t)blockIdx.x * G + (threadIdx.x >> 8); pr < ((count + G - 1) / G) * G;
         pr += (size_t)gridDim.x * G) {
        const size_t src = pr < count ? pr : count - 1;
        u64 x[2][8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            x[0][e] = a[src * N + ntt::coef_index(t, e)];
            x[1][e] = b[src * N + ntt::coef_index(t, e)];
        }
        ntt::forward<2>(x, buf, tws, t, bar);
        u64 r[1][8];
#pragma unroll
        for (int p = 0; p < 8; p++) r[0][p] = gl::div2k(gl::mul(x[0][p], x[1][p]), 11);  // N^-1 = 2^-11: one exact division
        ntt::group_sync(bar);
        ntt::inverse<1>(r, buf, tws + 2048, t, bar);
        if (pr < count) {
#pragma unroll
            for (int e = 0; e < 8; e++) out[pr * N + ntt::coef_index(t, e)] = gl::canon(r[0][e]);
        }
        ntt::group_sync(bar);
    }
}

static int num_sms()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

template <typename K>
static cudaError_t launch_grid(K kernel, int G, size_t smem, size_t units, const void *const *args,
                               cudaStream_t s)
{
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, G * TPG, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    size_t want = (units + G - 1) / G;
    size_t grid = (size_t)per_sm * num_sms();
    if (grid > want) grid = want;
    if (grid == 0) grid = 1;
    return cudaLaunchKernel((const void *)kernel, dim3((unsigned)grid), dim3(G * TPG), (void **)args, smem, s);
}

cudaError_t launch_ntt_fwd(const uint64_t *d_in, uint64_t *d_out, const uint64_t *d_tw, size_t count,
                           cudaStream_t s)
{
    if (count == 0) return cudaSuccess;
    constexpr int G = 2;
    const void *args[] = {&d_in, &d_out, &d_tw, &count};
    return launch_grid(ntt_fwd_kernel<G>, G, (2048 + G * POLY_WORDS) * 8, count, args, s);
}
cudaError_t launch_ntt_inv(const uint64_t *d_in, uint64_t *d_out, const uint64_t *d_tw, size_t count,
                           cudaStream_t s)
{
    if (count == 0) return cudaSuccess;
    constexpr int G = 2;
    const void *args[] = {&d_in, &d_out, &d_tw, &count};
    return launch_grid(ntt_inv_kernel<G>, G, (2048 + G * POLY_WORDS) * 8, count, args, s);
}
cudaError_t launch_ntt_mul(const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out, const uint64_t *d_tw,
                           size_t count, cudaStream_t s)
{
    if (count == 0) return cudaSuccess;
    constexpr int G = 2;
    const void *args[] = {&d_a, &d_b, &d_out, &d_tw, &count};
    return launch_grid(ntt_mul_kernel<G>, G, (4096 + G * 2 * POLY_WORDS) * 8, count, args, s);
}

// ---------------------------------------------------------------- key switch
//
// out21[c][x] = [x==n] b21 - sum_{y,z} d_{c,y,z} KSK[y][z][x]   (mod 2^21)
// out2N[c][x] = round(out21 / 2^9) mod 2N
// (pep_ks_blram_format.sv:158-172,240-243, pep_ks_mult_node.sv:95-104,
//  pep_ks_out_process.sv:276-280,336-341).  A SIMT integer GEMM: M = ciphertexts,
// N = output coefficients, K = (y, z) pairs.  The digits (in [-4, 4]) are made
// on the fly from the 64-bit mask coefficients; 32-bit wrap-around keeps the
// low 21 bits exact.  On upload the KSK is transposed to K-rows k = y*L+z and
// split by groups of four rows g: word [g][0][x] holds the low bytes of rows
// 4g..4g+3, words [g][1][x] and [g][2][x] their upper 13 bits as 16-bit
// halves (rows 4g, 4g+1 and 4g+2, 4g+3).  One dp4a multiplies the four low
// bytes by four packed digits (signed bytes) and two dp2a the upper parts:
// three instructions replace four 32-bit multiply-adds, with two
// accumulators per output.  Templated
// on the decomposition (base 2^BL, L levels) of the reference's parameter sets.
// GEN = false: the RTL's tie rule; GEN = true: the rule of the reference's
// test-vector generator (TFHE-rs), which takes the digit above the top one as
// 0, so that a top digit equal to B/2 stays positive.  Both give the same
// value mod 2^(BL*L); they differ only in that top digit.
template <int BL, int L, bool GEN>
__device__ __forceinline__ void ks_decomp(u64 v, int *d)
{
    // closest_rep = top BL*L bits + round bit; tie rule of
    // balanced_decomp_unfix_sign_round_bit.py:42-101 / decomp_parallel.sv:73-75,142-150
    constexpr int TOT = BL * L;
    constexpr u32 MASK = (1u << BL) - 1, HALF = 1u << (BL - 1);
    u32 rb = (u32)(v >> (63 - TOT)) & 1u;
    u32 c = (u32)(v >> (64 - TOT)) + rb;  // 0 .. 2^TOT
    u32 last_sign = GEN ? 0u : (((c >> (TOT - 1)) & 1u) && ((c & ((1u << (TOT - 1)) - 1)) || rb));
    u32 carry = 0;
#pragma unroll
    for (int i = 0; i < L; i++) {
        u32 raw = (c >> (BL * i)) & MASK;
        u32 nxt = (i + 1 < L) ? ((c >> (BL * (i + 1))) & MASK) : (last_sign ? MASK : 0u);
        u32 tv = raw + carry;
        bool negd = (tv >> BL) || ((tv & HALF) && ((tv & (HALF - 1)) || (nxt & HALF)));
        d[i] = negd ? (int)tv - (1 << BL) : (int)tv;
        carry = negd ? 1u : 0u;
    }
}

// acc + sum over the 4 bytes of (unsigned byte of k) * (signed byte of d)
__device__ __forceinline__ int dp4a_us(u32 k, u32 d, int acc)
{
    int r;
    asm("dp4a.u32.s32 %0, %1, %2, %3;" : "=r"(r) : "r"(k), "r"(d), "r"(acc));
    return r;
}
// acc + (unsigned halves of k) . (signed bytes 0, 1 of d)   [HI: bytes 2, 3]
template <bool HI>
__device__ __forceinline__ int dp2a_us(u32 k, u32 d, int acc)
{
    int r;
    if constexpr (HI) asm("dp2a.hi.u32.s32 %0, %1, %2, %3;" : "=r"(r) : "r"(k), "r"(d), "r"(acc));
    else asm("dp2a.lo.u32.s32 %0, %1, %2, %3;" : "=r"(r) : "r"(k), "r"(d), "r"(acc));
    return r;
}

// three CTAs per SM (80 registers, no spills with two accumulators per
// output): the multiply pipe needs the warps to hide the dp4a/dp2a latency
template <int BL, int L, bool GEN>
__global__ void __launch_bounds__(256, 3) ks_kernel(const u64 *__restrict__ in, const u32 *__restrict__ src_idx,
                                                  const u32 *__restrict__ ksk_t, u32 *__restrict__ out21,
                                                  u32 *__restrict__ out2N, u32 B, u32 n, u32 xpad,
                                                  u32 *__restrict__ part)
{
    constexpr int KR = KS_KC * L;   // K rows of one chunk (a multiple of 4)
    constexpr int KG = KR / 4;      // 4-row groups of one chunk
    __shared__ __align__(16) unsigned char dsm[KS_BM][KR];     // digits, one signed byte each, [ct][k]
    __shared__ __align__(16) u32 ksm[KG][KS_PLANES][KS_BN];    // KSK bytes, 4 rows per word, [group][plane][x]
    const int tid = threadIdx.x;
    const int ty = tid >> 5, tx = tid & 31;  // 8 x 4 cts, 32 x 4 outputs
    const u32 c0 = blockIdx.y * KS_BM, x0 = blockIdx.x * KS_BN;
    // KSK = lo + hi 2^8 (lo its low byte, hi its upper 13 bits): one
    // accumulator for the low bytes (dp4a over four rows), one for the upper
    // parts (dp2a over two rows, twice)
    int acc_lo[4][4], acc_hi[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc_lo[i][j] = acc_hi[i][j] = 0;

    const int dct = tid >> 3, dy = tid & 7;  // decomposition role: 32 cts x 8 coefs
    const u32 dct_c = min(c0 + dct, B - 1);
    const size_t dct_g = src_idx ? src_idx[dct_c] : dct_c;  // row of the input array
    // split-K (gridDim.z > 1, small batches): this CTA sums its slice of the
    // mask coefficients and adds the partial sums into `part`
    const u32 span = (u32)N / gridDim.z, y_lo = blockIdx.z * span;
    for (u32 y0 = y_lo; y0 < y_lo + span; y0 += KS_KC) {
        {
            int d[L];
            ks_decomp<BL, L, GEN>(in[(size_t)dct_g * (N + 1) + y0 + dy], d);
#pragma unroll
            for (int z = 0; z < L; z++) dsm[dct][dy * L + z] = (unsigned char)(signed char)d[z];
        }
        // the chunk's KSK rows y0 L .. y0 L + KR - 1 are groups y0 L / 4 ..
        const uint4 *src = reinterpret_cast<const uint4 *>(ksk_t + (size_t)(y0 * L / 4) * KS_PLANES * xpad + x0);
        for (int idx = tid; idx < KG * KS_PLANES * (KS_BN / 4); idx += 256) {
            const int row = idx / (KS_BN / 4), xv = idx % (KS_BN / 4);  // row = group * planes + plane
            reinterpret_cast<uint4 *>(&ksm[0][0][0] + row * KS_BN)[xv] = src[(size_t)row * (xpad / 4) + xv];
        }
        __syncthreads();
#pragma unroll 4
        for (int g = 0; g < KG; g++) {
            u32 dv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) dv[i] = *reinterpret_cast<const u32 *>(&dsm[ty * 4 + i][4 * g]);
            const uint4 k0 = reinterpret_cast<const uint4 *>(&ksm[g][0][0])[tx];  // low bytes, rows 0-3
            const uint4 k1 = reinterpret_cast<const uint4 *>(&ksm[g][1][0])[tx];  // upper parts, rows 0, 1
            const uint4 k2 = reinterpret_cast<const uint4 *>(&ksm[g][2][0])[tx];  // upper parts, rows 2, 3
            const u32 w0[4] = {k0.x, k0.y, k0.z, k0.w}, w1[4] = {k1.x, k1.y, k1.z, k1.w},
                      w2[4] = {k2.x, k2.y, k2.z, k2.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    acc_lo[i][j] = dp4a_us(w0[j], dv[i], acc_lo[i][j]);
                    acc_hi[i][j] = dp2a_us<false>(w1[j], dv[i], acc_hi[i][j]);
                    acc_hi[i][j] = dp2a_us<true>(w2[j], dv[i], acc_hi[i][j]);
                }
        }
        __syncthreads();
    }
    u32 sum[4][4];  // sum_{k} d_k KSK_k mod 2^32 (exact mod 2^21)
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) sum[i][j] = (u32)acc_lo[i][j] + ((u32)acc_hi[i][j] << 8);
    if (part) {
        // 32-bit wrap-around sums are exact mod 2^21 in any order
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const u32 c = c0 + ty * 4 + i;
            if (c >= B) continue;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const u32 x = x0 + tx * 4 + j;
                if (x <= n) atomicAdd(&part[(size_t)c * xpad + x], sum[i][j]);
            }
        }
        return;
    }
    const u32 M = (1u << KS_W) - 1;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        u32 c = c0 + ty * 4 + i;
        if (c >= B) continue;
        u64 b = in[(size_t)(src_idx ? src_idx[c] : c) * (N + 1) + N];
        u32 b21 = (u32)(((b >> (64 - KS_W)) + ((b >> (63 - KS_W)) & 1ull)) & M);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            u32 x = x0 + tx * 4 + j;
            if (x > n) continue;
            u32 v = (((x == n) ? b21 : 0u) - sum[i][j]) & M;
            if (out21) out21[(size_t)c * (n + 1) + x] = v;
            out2N[(size_t)c * (n + 1) + x] = ((v >> 9) + ((v >> 8) & 1u)) & (TWO_N - 1);
        }
    }
}

bool ks_supported(uint32_t bl, uint32_t L)
{
    return (bl == 3 && (L == 6 || L == 5)) || (bl == 2 && (L == 8 || L == 7));
}

// The split-K form's epilogue: out = [x == n] b21 - sum (mod 2^21) and its 2N
// switch, as ks_kernel's own epilogue; the partial sums are cleared behind
// it, so `part` is zero again for the next call.
__global__ void __launch_bounds__(256) ks_finish(const u64 *__restrict__ in, const u32 *__restrict__ src_idx,
                                                  u32 *__restrict__ part, u32 *__restrict__ out21,
                                                  u32 *__restrict__ out2N, u32 B, u32 n, u32 xpad)
{
    const u32 M = (1u << KS_W) - 1;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < B * (n + 1); i += gridDim.x * blockDim.x) {
        const u32 c = i / (n + 1), x = i % (n + 1);
        u32 *pp = &part[(size_t)c * xpad + x];
        u32 v = (0u - *pp) & M;
        *pp = 0;
        if (x == n) {
            const u64 b = in[(size_t)(src_idx ? src_idx[c] : c) * (N + 1) + N];
            v = (v + (u32)((b >> (64 - KS_W)) + ((b >> (63 - KS_W)) & 1ull))) & M;
        }
        if (out21) out21[(size_t)c * (n + 1) + x] = v;
        out2N[(size_t)c * (n + 1) + x] = ((v >> 9) + ((v >> 8) & 1u)) & (TWO_N - 1);
    }
}

template <bool GEN>
static cudaError_t launch_keyswitch_rule(const uint64_t *d_in, const uint32_t *d_ksk_t, uint32_t *d_out21,
                                         uint32_t *d_out2N, u32 B, uint32_t n, uint32_t xpad, cudaStream_t s,
                                         const uint32_t *d_src_idx, uint32_t bl, uint32_t L, uint32_t *d_part)
{
    // one ciphertext tile: split the mask coefficients over KS_SPLIT CTAs per
    // output tile (a tile walks all 256 coefficient chunks in sequence otherwise)
    const bool split = d_part && B <= (u32)KS_BM;
    dim3 grid(xpad / KS_BN, (B + KS_BM - 1) / KS_BM, split ? KS_SPLIT : 1);
    u32 *part = split ? d_part : nullptr;
    if (bl == 3 && L == 6) ks_kernel<3, 6, GEN><<<grid, 256, 0, s>>>(d_in, d_src_idx, d_ksk_t, d_out21, d_out2N, B, n, xpad, part);
    else if (bl == 3 && L == 5) ks_kernel<3, 5, GEN><<<grid, 256, 0, s>>>(d_in, d_src_idx, d_ksk_t, d_out21, d_out2N, B, n, xpad, part);
    else if (bl == 2 && L == 8) ks_kernel<2, 8, GEN><<<grid, 256, 0, s>>>(d_in, d_src_idx, d_ksk_t, d_out21, d_out2N, B, n, xpad, part);
    else if (bl == 2 && L == 7) ks_kernel<2, 7, GEN><<<grid, 256, 0, s>>>(d_in, d_src_idx, d_ksk_t, d_out21, d_out2N, B, n, xpad, part);
    else return cudaErrorInvalidValue;
    if (split) {
        const u32 total = B * (n + 1);
        ks_finish<<<(total + 255) / 256, 256, 0, s>>>(d_in, d_src_idx, d_part, d_out21, d_out2N, B, n, xpad);
    }
    return cudaGetLastError();
}

cudaError_t launch_keyswitch(const uint64_t *d_in, const uint32_t *d_ksk_t, uint32_t *d_out21, uint32_t *d_out2N,
                             size_t B, uint32_t n, uint32_t xpad, cudaStream_t s, const uint32_t *d_src_idx,
                             uint32_t bl, uint32_t L, uint32_t tie_rule, uint32_t *d_part)
{
    if (B == 0) return cudaSuccess;
    if (tie_rule == TIE_GENERATOR)
        return launch_keyswitch_rule<true>(d_in, d_ksk_t, d_out21, d_out2N, (u32)B, n, xpad, s, d_src_idx, bl, L,
                                           d_part);
    if (tie_rule != TIE_RTL) return cudaErrorInvalidValue;
    return launch_keyswitch_rule<false>(d_in, d_ksk_t, d_out21, d_out2N, (u32)B, n, xpad, s, d_src_idx, bl, L,
                                        d_part);
}

// ---------------------------------------------------------- blind rotation
//
// Persistent kernel: each CTA owns G ciphertexts at a time (256 threads each)
// and runs all n steps for them; per step one 64 KiB BSK slab is fetched by a
// bulk asynchronous copy into shared memory and read by every ciphertext of
// the CTA.  The accumulator lives in registers (8 coefficients x 2 polys per
// thread); shared memory carries the rotation gather and the NTT exchanges.
// Step i (pe_pbs hot loop, feed_rot.sv:305-307, feed_final.sv:324,
// decomp_balseq_core.sv:135-150, ntt_core_gf64, pp_core, mod_switch_to_2powerN,
// acc_core.sv:8-12):
//   diff_t = X^{a_i} ACC_t - ACC_t      (t = mask, body)
//   d_t    = decomp_{2^23,1}(diff_t)    in Z_p
//   R_col  = INTT( sum_row NTT(d_row) * BSK_i[row][col] )
//   ACC_col += modsw_{p->2^64}(R_col)
// then the sample extract of X^{-b} ACC (sxt_core.sv:8-14).

// Bound on the polls of one BSK-slab wait (set per device by the host, see
// set_slab_wait_polls) and on the final wait for copies still in flight.
constexpr unsigned long long SLAB_WAIT_POLLS_DEFAULT = 1ull << 26;
constexpr unsigned long long DRAIN_POLLS = 1ull << 26;
__device__ unsigned long long g_slab_wait_polls = SLAB_WAIT_POLLS_DEFAULT;

cudaError_t set_slab_wait_polls(unsigned long long polls)
{
    return cudaMemcpyToSymbol(g_slab_wait_polls, &polls, sizeof polls);
}

__device__ __forceinline__ u32 smem_addr(const void *p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(u64 *mbar, u32 count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(u64 *mbar, u32 bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar)), "r"(bytes)
                 : "memory");
}
// BSK slabs are re-read by every CTA at every step of every wave: they are
// fetched with an L2 evict-last policy so that the output BLWEs streaming
// through L2 do not push them out between waves.
__device__ __forceinline__ u64 bsk_l2_policy()
{
    u64 pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, u32 bytes, u64 *mbar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(mbar)), "l"(bsk_l2_policy())
        : "memory");
}
// bounded wait on the given phase parity; returns false after `polls` polls
__device__ __forceinline__ bool mbar_wait(u64 *mbar, u32 parity, unsigned long long polls)
{
    u32 a = smem_addr(mbar);
    for (unsigned long long it = 0; it < polls; it++) {
        u32 done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// named-barrier OR-reduction over one 256-thread ciphertext group
__device__ __forceinline__ bool group_sync_or(int bar_id, bool pred)
{
    u32 r;
    asm volatile("{\n\t.reg .pred p, q;\n\t"
                 "setp.ne.u32 p, %1, 0;\n\t"
                 "barrier.cta.red.or.pred q, %2, %3, p;\n\t"
                 "selp.u32 %0, 1, 0, q;\n\t}"
                 : "=r"(r)
                 : "r"((u32)pred), "r"(bar_id), "r"(TPG)
                 : "memory");
    return r != 0;
}

// Output BLWEs are written once and not read again by this launch: a
// streaming (evict-first) store keeps them from pushing the BSK, which every
// CTA re-reads at every step, out of L2.
__device__ __forceinline__ void st_stream(u64 *p, u64 v) { __stcs(reinterpret_cast<unsigned long long *>(p), v); }

__device__ __forceinline__ void issue_slab(u64 *slab, const u64 *src, u64 *mbar)
{
    mbar_expect_tx(mbar, (u32)SLAB_BYTES);
#pragma unroll
    for (int c = 0; c < 4; c++) bulk_g2s(slab + c * (SLAB_WORDS / 4), src + c * (SLAB_WORDS / 4), SLAB_BYTES / 4, mbar);
}

template <int G, int BW>
__global__ void __launch_bounds__(G * 256, 1)
    br_kernel(const u32 *__restrict__ lwe2N, const u64 *__restrict__ luts, const u32 *__restrict__ lut_id, u32 nlut,
              const u64 *__restrict__ bsk, const u64 *__restrict__ tw, u64 *__restrict__ out, u32 B, u32 n,
              u32 *__restrict__ err, const u32 *__restrict__ dst_idx, u32 mlk,
              u32 tie_rule)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    u64 *slab = reinterpret_cast<u64 *>(smem_raw);
    u64 *tws = slab + SLAB_WORDS;
    u64 *bufs = tws + 4096;
    u64 *mbar = bufs + G * 4 * POLY_WORDS;
    u32 *slab_done = reinterpret_cast<u32 *>(mbar + 1);  // groups that finished the current slab
    u32 *failed = slab_done + 1;
    u32 *last_parity = failed + 1;  // phase parity of the last slab issued
    const unsigned long long polls = g_slab_wait_polls;
    const u64 tie_rtl = tie_rule == TIE_RTL ? 1ull : 0ull;
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255, bar = 1 + g;
    // two staging buffers per ciphertext group (fixed roles, see the step below)
    u64 *bp = bufs + g * 4 * POLY_WORDS, *bq = bp + 2 * POLY_WORDS;

    for (int i = threadIdx.x; i < 4096; i += G * TPG) tws[i] = tw[i];
    if (threadIdx.x == 0) {
        mbar_init(mbar, 1);
        *failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    u32 phase = 0;
    const u32 ngroups = (B + G - 1) / G;
    for (u32 grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
        const u32 cidx = grp * G + g;
        const bool active = cidx < B;
        const u32 ct = active ? cidx : B - 1;
        const u32 *my_lwe = lwe2N + (size_t)ct * (n + 1);  // read in place; every thread of the group loads the same word
        u32 lid = lut_id[ct];
        if (lid >= nlut) {  // device-resident ids cannot be checked by the host: flag it, stay in bounds
            if (t == 0) atomicOr(err, DEVERR_LUT_ID);
            lid = 0;
        }
        const u64 *lut = luts + (size_t)lid * 2 * N;
        // ACC: registers (coefficient layout, 16 coefficients per thread), copied
        // to the thread's own slots of bp at the start of every step
        u64 acc[2][8];
#pragma unroll
        for (int q = 0; q < 2; q++)
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const int j = ntt::coef_index(t, e);
                acc[q][e] = lut[q * N + j];
                bp[q * POLY_WORDS + j] = acc[q][e];
            }
        if (threadIdx.x == 0) {
            *slab_done = 0;
            *last_parity = phase;
            issue_slab(slab, bsk, mbar);
        }
        __syncthreads();

        // The G groups run their steps independently (so one group's NTT overlaps
        // another's BSK multiply); they share only the slab, which the last group
        // to finish a step's multiply refills.  A group that times out on the slab
        // stops; the others then time out too (no refill comes) and all meet at
        // the block barrier after the loop.
        //
        // One step, buffer by buffer (every write follows the barrier after the
        // last read of what it overwrites; "own" slots are read and written only
        // by the thread that owns them):
        //   ACC (bp, own) --barrier--> rotate+decompose+A1 -> bq --> A2 -> bp
        //   --> C1 -> bq --> C2 -> bp (own) ; BSK MAC bp (own) -> bp (own)
        //   --barrier--> C2^-1 -> bq --> C1^-1 -> bp --> A2^-1 -> bq --> A1^-1
        //   -> bp (own) ; accumulate into ACC, ACC -> bp (own)
        // (the own slots of thread t are t + 256 e in both the coefficient and
        // the evaluation layout)
        // Passes run one polynomial at a time (rolled loops): one copy of each
        // pass's code keeps the step inside the instruction cache.
        bool ok = true;
        u32 a_next = my_lwe[0];
        for (u32 i = 0; i < n; i++) {
            const u32 a = a_next;
            a_next = my_lwe[i + 1];  // i + 1 <= n: the body word at the end
            ntt::group_sync(bar);
            // feed: diff = X^a ACC - ACC, decomposed into Z_p, then A1
#pragma unroll 1
            for (int q = 0; q < 2; q++) {
                const u64 *accq = bp + q * POLY_WORDS;
                u64 y[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const u32 j = ntt::coef_index(t, e);
                    const u32 src = (j + TWO_N - a) & (TWO_N - 1);
                    u64 v = accq[src & (N - 1)];
                    if (src >= (u32)N) v = 0ull - v;
                    y[e] = gl::decomp_to_p<BW>(v - accq[j], tie_rtl);
                }
                ntt::a1_fwd(y, bq + q * POLY_WORDS, t);
            }
            ntt::group_sync(bar);
            ntt::a2_fwd<2>(bq, bp, tws, t);
            ntt::group_sync(bar);
            ntt::c1_fwd<2>(bp, bq, t);
            ntt::group_sync(bar);
#pragma unroll 1
            for (int q = 0; q < 2; q++) {
                u64 y[8];
                ntt::c2_fwd(bq + q * POLY_WORDS, y, t);
#pragma unroll
                for (int p = 0; p < 8; p++) bp[q * POLY_WORDS + p * TPG + t] = y[p];  // own slots
            }
            // BSK multiply-accumulate in the evaluation domain
            ok = mbar_wait(mbar, phase, polls);
            phase ^= 1;
#pragma unroll
            for (int p = 0; p < 8; p++) {
                const u64 *sb = slab + p * 4 * TPG + t;
                const u64 b00 = sb[0], b01 = sb[TPG], b10 = sb[2 * TPG], b11 = sb[3 * TPG];
                const u64 x0 = bp[p * TPG + t], x1 = bp[POLY_WORDS + p * TPG + t];
                bp[p * TPG + t] = gl::mul_add2(x0, b00, x1, b10);
                bp[POLY_WORDS + p * TPG + t] = gl::mul_add2(x0, b01, x1, b11);
            }
            if (group_sync_or(bar, !ok)) {
                ok = false;
                break;
            }
            if (t == 0) {
                __threadfence_block();
                const u32 done = atomicAdd(slab_done, 1u) + 1;
                if (done == (u32)G * (i + 1) && i + 1 < n) {
                    // every group has read slab i: reuse the buffer for slab i+1
                    __threadfence_block();
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    *last_parity = phase;
                    issue_slab(slab, bsk + (size_t)(i + 1) * SLAB_WORDS, mbar);
                }
            }
#pragma unroll 1
            for (int q = 0; q < 2; q++) {
                u64 y[8];
#pragma unroll
                for (int p = 0; p < 8; p++) y[p] = bp[q * POLY_WORDS + p * TPG + t];
                ntt::c2_inv(y, bq + q * POLY_WORDS, t);
            }
            ntt::group_sync(bar);
            ntt::c1_inv<2>(bq, bp, t);
            ntt::group_sync(bar);
            ntt::a2_inv<2>(bp, bq, tws + 2048, t);
            ntt::group_sync(bar);
#pragma unroll 1
            for (int q = 0; q < 2; q++) {
                u64 y[8];
                ntt::a1_inv(bq + q * POLY_WORDS, y, t);
#pragma unroll
                for (int e = 0; e < 8; e++) bp[q * POLY_WORDS + ntt::coef_index(t, e)] = y[e];  // own slots
            }
            // p -> 2^64 switch, accumulate, and ACC to the own slots for the next step
#pragma unroll
            for (int q = 0; q < 2; q++)
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    u64 *slot = bp + q * POLY_WORDS + ntt::coef_index(t, e);
                    acc[q][e] += gl::modsw_p_to_q(gl::canon(*slot));
                    *slot = acc[q][e];
                }
        }

        // sample extract of coefficient 0 of X^{-b} ACC.  Many-LUT (mlk = 2, 4, 8
        // functions packed in one LUT, docs/dop.md:113-121): output m extracts
        // coefficient m*N/mlk, i.e. coefficient 0 of X^{-(b + m N/mlk)} ACC,
        // into consecutive output rows.
        ntt::group_sync(bar);  // ACC (bp) complete
        if (!ok) {
            if (t == 0) {
                atomicExch(failed, 1u);
                atomicOr(err, DEVERR_TIMEOUT);
            }
        } else if (active) {
            const size_t row0 = dst_idx ? dst_idx[cidx] : (size_t)cidx * mlk;
            const u32 body = my_lwe[n];
            for (u32 m = 0; m < mlk; m++) {
                const u32 b = (body + m * (N / mlk)) & (TWO_N - 1);
                u64 *o = out + (row0 + m) * (N + 1);
#pragma unroll
                for (int r = 0; r < 8; r++) {
                    const u32 oi = t + 256 * r;
                    const u32 j = oi == 0 ? 0 : N - oi;
                    const u32 src = (j + b) & (TWO_N - 1);
                    u64 v = bp[src & (N - 1)];
                    if (src >= (u32)N) v = 0ull - v;
                    st_stream(o + oi, oi == 0 ? v : 0ull - v);
                }
                if (t == 0) {
                    u64 v = bp[POLY_WORDS + (b & (N - 1))];
                    st_stream(o + N, b >= (u32)N ? 0ull - v : v);
                }
            }
        }
        __syncthreads();
        if (*failed) {  // read by every thread after the barrier: uniform
            // the last slab issued may still be landing in this block's shared
            // memory: wait for it (bounded) before the block ends
            if (threadIdx.x == 0 && !mbar_wait(mbar, *last_parity, DRAIN_POLLS))
                atomicOr(err, DEVERR_DRAIN);  // a copy may still land in shared memory
            return;
        }
    }
}

// Latency form for batches of at most one ciphertext per SM: one ciphertext
// per CTA, its two GLWE polynomials split over the two 256-thread groups.
// Group g owns polynomial g of the accumulator and runs the feed, the forward
// transform of digit polynomial g, the product for output column g and the
// inverse transform of column g; the groups meet only around the BSK
// multiply, which needs both forward transforms (block barriers).  Each group
// does half of a step's work, but one SM's integer throughput still bounds a
// lone ciphertext: measured about 10 % faster than one ciphertext per group.
// The two-SM form below halves the work per SM.
template <int BW>
__global__ void __launch_bounds__(512, 1)
    br_kernel_split(const u32 *__restrict__ lwe2N, const u64 *__restrict__ luts, const u32 *__restrict__ lut_id,
                    u32 nlut, const u64 *__restrict__ bsk, const u64 *__restrict__ tw, u64 *__restrict__ out, u32 B,
                    u32 n, u32 *__restrict__ err, const u32 *__restrict__ dst_idx, u32 mlk,
              u32 tie_rule)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    u64 *slab = reinterpret_cast<u64 *>(smem_raw);
    u64 *tws = slab + SLAB_WORDS;
    u64 *bufs = tws + 4096;  // [group][2 buffers][POLY_WORDS]
    u64 *mbar = bufs + 4 * POLY_WORDS;
    u32 *last_parity = reinterpret_cast<u32 *>(mbar + 1);  // phase parity of the last slab issued
    const unsigned long long polls = g_slab_wait_polls;
    const u64 tie_rtl = tie_rule == TIE_RTL ? 1ull : 0ull;
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255, bar = 1 + g;
    u64 *bp = bufs + g * 2 * POLY_WORDS, *bq = bp + POLY_WORDS;  // this group's polynomial
    const u64 *bp0 = bufs, *bp1 = bufs + 2 * POLY_WORDS;          // both groups' bp (MAC operands, extract)

    for (int i = threadIdx.x; i < 4096; i += 512) tws[i] = tw[i];
    if (threadIdx.x == 0) {
        mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    u32 phase = 0;
    for (u32 ct = blockIdx.x; ct < B; ct += gridDim.x) {
        const u32 *my_lwe = lwe2N + (size_t)ct * (n + 1);
        u32 lid = lut_id[ct];
        if (lid >= nlut) {
            if (threadIdx.x == 0) atomicOr(err, DEVERR_LUT_ID);
            lid = 0;
        }
        const u64 *lut = luts + ((size_t)lid * 2 + g) * N;  // polynomial g of the LUT
        u64 acc[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int j = ntt::coef_index(t, e);
            acc[e] = lut[j];
            bp[j] = acc[e];
        }
        if (threadIdx.x == 0) {
            *last_parity = phase;
            issue_slab(slab, bsk, mbar);
        }
        __syncthreads();

        // Buffers of group g as in br_kernel (bp: ACC own slots, A2, C2 own
        // slots, C1^-1; bq: A1, C1, C2^-1, A2^-1); the other group reads this
        // group's bp own slots only between the two block barriers of the MAC.
        bool ok = true;
        u32 a_next = my_lwe[0];
        for (u32 i = 0; i < n; i++) {
            const u32 a = a_next;
            a_next = my_lwe[i + 1];
            ntt::group_sync(bar);
            {
                u64 y[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const u32 j = ntt::coef_index(t, e);
                    const u32 src = (j + TWO_N - a) & (TWO_N - 1);
                    u64 v = bp[src & (N - 1)];
                    if (src >= (u32)N) v = 0ull - v;
                    y[e] = gl::decomp_to_p<BW>(v - bp[j], tie_rtl);
                }
                ntt::a1_fwd(y, bq, t);
            }
            ntt::group_sync(bar);
            ntt::a2_fwd<1>(bq, bp, tws, t);
            ntt::group_sync(bar);
            ntt::c1_fwd<1>(bp, bq, t);
            ntt::group_sync(bar);
            {
                u64 y[8];
                ntt::c2_fwd(bq, y, t);
#pragma unroll
                for (int p = 0; p < 8; p++) bp[p * TPG + t] = y[p];  // own slots
            }
            ok = mbar_wait(mbar, phase, polls);
            phase ^= 1;
            if (__syncthreads_or(!ok)) {  // both transforms written; uniform over the block
                ok = false;
                break;
            }
            u64 r[8];
#pragma unroll
            for (int p = 0; p < 8; p++) {
                const u64 *sb = slab + p * 4 * TPG + t;  // [row][col]: column g of rows 0 and 1
                r[p] = gl::mul_add2(bp0[p * TPG + t], sb[g * TPG], bp1[p * TPG + t], sb[(2 + g) * TPG]);
            }
            __syncthreads();  // every read of the slab and of the other group's bp is done
            if (threadIdx.x == 0 && i + 1 < n) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                *last_parity = phase;
                issue_slab(slab, bsk + (size_t)(i + 1) * SLAB_WORDS, mbar);
            }
            ntt::c2_inv(r, bq, t);
            ntt::group_sync(bar);
            ntt::c1_inv<1>(bq, bp, t);
            ntt::group_sync(bar);
            ntt::a2_inv<1>(bp, bq, tws + 2048, t);
            ntt::group_sync(bar);
            {
                u64 y[8];
                ntt::a1_inv(bq, y, t);
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int j = ntt::coef_index(t, e);
                    acc[e] += gl::modsw_p_to_q(gl::canon(y[e]));
                    bp[j] = acc[e];
                }
            }
        }
        __syncthreads();  // both accumulator polynomials complete
        if (!ok) {        // the block agreed on the timeout above
            if (threadIdx.x == 0) {
                atomicOr(err, DEVERR_TIMEOUT);
                if (!mbar_wait(mbar, *last_parity, DRAIN_POLLS))  // a slab still landing here
                    atomicOr(err, DEVERR_DRAIN);
            }
            return;
        }
        // sample extract (as in br_kernel): mask from polynomial 0, body from 1
        const size_t row0 = dst_idx ? dst_idx[ct] : (size_t)ct * mlk;
        const u32 body = my_lwe[n];
        for (u32 m = 0; m < mlk; m++) {
            const u32 b = (body + m * (N / mlk)) & (TWO_N - 1);
            u64 *o = out + (row0 + m) * (N + 1);
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const u32 oi = threadIdx.x + 512 * r;
                const u32 j = oi == 0 ? 0 : N - oi;
                const u32 src = (j + b) & (TWO_N - 1);
                u64 v = bp0[src & (N - 1)];
                if (src >= (u32)N) v = 0ull - v;
                st_stream(o + oi, oi == 0 ? v : 0ull - v);
            }
            if (threadIdx.x == 0) {
                u64 v = bp1[b & (N - 1)];
                st_stream(o + N, b >= (u32)N ? 0ull - v : v);
            }
        }
        __syncthreads();
    }
}

static size_t br_split_smem_bytes() { return (size_t)(SLAB_WORDS + 4096 + 4 * POLY_WORDS + 2) * 8; }

// Half of a step's BSK slab: column col of both rows, hs[(p*2 + row)*TPG + t]
// = slab[(p*4 + row*2 + col)*TPG + t] -- sixteen 2 KiB bulk copies.
// Called by the 32 lanes of warp 0: lane 0 arms the mbarrier with the byte
// count, then lanes 0-15 each start one of the 16 pieces of column `col`
// (2 KiB each), so that no single thread issues sixteen copies in a row
// while the rest of the CTA waits at the next barrier.  Each issuing lane
// first orders its earlier shared-memory accesses before the async copies.
__device__ __forceinline__ void issue_half_slab_warp(u64 *hs, const u64 *src, u32 col, u64 *mbar, int lane)
{
    if (lane == 0) mbar_expect_tx(mbar, (u32)(SLAB_BYTES / 2));
    __syncwarp();
    if (lane < 16) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const int p = lane >> 1, row = lane & 1;
        bulk_g2s(hs + (p * 2 + row) * TPG, src + (p * 4 + row * 2 + col) * TPG, TPG * 8, mbar);
    }
}

// More than half an SM's shared memory, so that the two CTAs of a pair never
// share an SM.
constexpr size_t PAIR_SMEM_BYTES = 132 * 1024;

// Lowest-latency form, for batches of at most one ciphertext per two SMs: a
// cluster of two CTAs (256 threads each, one per SM) per ciphertext, CTA r
// owning polynomial r -- the split form above with the two groups on two
// SMs.  Each CTA streams only its half of the slab (column r); for the BSK
// multiply each CTA stores its forward transform into a receive buffer in the
// other CTA's shared memory as it computes it (remote stores do not stall the
// writer), and reads only local shared memory after the cluster barrier.
// The receive buffers and the status flags alternate by step parity, so a
// buffer is written again only two steps later, after the next step's
// cluster barrier has ordered this step's reads: one cluster barrier a step.
// A slab timeout is agreed by the pair through those status flags, written
// into both CTAs' shared memory before the step's cluster barrier, so both
// leave the step loop at the same point and every cluster barrier is reached
// by both.
template <int BW>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(256, 1)
    br_kernel_pair(const u32 *__restrict__ lwe2N, const u64 *__restrict__ luts, const u32 *__restrict__ lut_id,
                   u32 nlut, const u64 *__restrict__ bsk, const u64 *__restrict__ tw, u64 *__restrict__ out, u32 B,
                   u32 n, u32 *__restrict__ err, const u32 *__restrict__ dst_idx, u32 mlk,
              u32 tie_rule)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const u32 r = cluster.block_rank();
    extern __shared__ __align__(128) unsigned char smem_raw[];
    u64 *hs = reinterpret_cast<u64 *>(smem_raw);  // half slab, SLAB_WORDS / 2
    u64 *tws = hs + SLAB_WORDS / 2;
    u64 *bp = tws + 4096, *bq = bp + POLY_WORDS;
    u64 *mbar = bq + POLY_WORDS;
    u32 *flags = reinterpret_cast<u32 *>(mbar + 1);  // [step parity][rank]: step status of rank 0 and rank 1
    u32 *last_parity = flags + 4;                     // phase parity of the last half slab issued
    u64 *rx = mbar + 4;  // [step parity][2048]: the other CTA's forward transform, own-slot layout
    const unsigned long long polls = g_slab_wait_polls;
    const u64 tie_rtl = tie_rule == TIE_RTL ? 1ull : 0ull;
    const int t = threadIdx.x;
    u64 *peer_rx = cluster.map_shared_rank(rx, r ^ 1u);
    u32 *peer_flags = cluster.map_shared_rank(flags, r ^ 1u);
    u32 step = 0;  // steps run by this CTA, over all its ciphertexts: the parity of rx and flags

    for (int i = t; i < 4096; i += TPG) tws[i] = tw[i];
    if (t == 0) {
        mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    cluster.sync();  // both CTAs' shared memory is set up before any remote access

    u32 phase = 0;
    bool ok = true;
    const u32 npairs = gridDim.x / 2;
    for (u32 ct = blockIdx.x / 2; ct < B && ok; ct += npairs) {
        const u32 *my_lwe = lwe2N + (size_t)ct * (n + 1);
        u32 lid = lut_id[ct];
        if (lid >= nlut) {
            if (t == 0 && r == 0) atomicOr(err, DEVERR_LUT_ID);
            lid = 0;
        }
        const u64 *lut = luts + ((size_t)lid * 2 + r) * N;
        u64 acc[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int j = ntt::coef_index(t, e);
            acc[e] = lut[j];
            bp[j] = acc[e];
        }
        if (t < 32) {  // warp 0; the last reads of hs were before this ciphertext's barriers
            if (t == 0) *last_parity = phase;
            issue_half_slab_warp(hs, bsk, r, mbar, t);
        }

        u32 a_next = my_lwe[0];
        for (u32 i = 0; i < n; i++) {
            const u32 a = a_next;
            a_next = my_lwe[i + 1];
            __syncthreads();
            {
                u64 y[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const u32 j = ntt::coef_index(t, e);
                    const u32 src = (j + TWO_N - a) & (TWO_N - 1);
                    u64 v = bp[src & (N - 1)];
                    if (src >= (u32)N) v = 0ull - v;
                    y[e] = gl::decomp_to_p<BW>(v - bp[j], tie_rtl);
                }
                ntt::a1_fwd(y, bq, t);
            }
            __syncthreads();
            ntt::a2_fwd<1>(bq, bp, tws, t);
            __syncthreads();
            ntt::c1_fwd<1>(bp, bq, t);
            __syncthreads();
            {
                u64 y[8];
                ntt::c2_fwd(bq, y, t);
#pragma unroll
                for (int p = 0; p < 8; p++) {
                    bp[p * TPG + t] = y[p];                           // own slots
                    peer_rx[(step & 1) * N + p * TPG + t] = y[p];  // the other CTA's receive buffer
                }
            }
            const bool cta_ok = !__syncthreads_or(!mbar_wait(mbar, phase, polls));
            phase ^= 1;
            u32 *fl = flags + 2 * (step & 1);
            if (t == 0) {
                fl[r] = cta_ok;
                peer_flags[2 * (step & 1) + r] = cta_ok;
            }
            cluster.sync();  // both transforms (rx) and both status flags are visible
            if (!(fl[0] && fl[1])) {
                ok = false;  // same decision in both CTAs
                break;
            }
            const u64 *rxs = rx + (step & 1) * N;
            const u64 *x0src = r == 0 ? bp : rxs, *x1src = r == 0 ? rxs : bp;
            step++;
            u64 rr[8];
#pragma unroll
            for (int p = 0; p < 8; p++)
                rr[p] = gl::mul_add2(x0src[p * TPG + t], hs[(p * 2) * TPG + t], x1src[p * TPG + t],
                                     hs[(p * 2 + 1) * TPG + t]);
            __syncthreads();  // every read of the half slab is done
            if (t < 32 && i + 1 < n) {  // warp 0
                if (t == 0) *last_parity = phase;
                issue_half_slab_warp(hs, bsk + (size_t)(i + 1) * SLAB_WORDS, r, mbar, t);
            }
            ntt::c2_inv(rr, bq, t);
            __syncthreads();
            ntt::c1_inv<1>(bq, bp, t);
            __syncthreads();
            ntt::a2_inv<1>(bp, bq, tws + 2048, t);
            __syncthreads();
            {
                u64 y[8];
                ntt::a1_inv(bq, y, t);
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int j = ntt::coef_index(t, e);
                    acc[e] += gl::modsw_p_to_q(gl::canon(y[e]));
                    bp[j] = acc[e];
                }
            }
        }
        __syncthreads();
        if (!ok) break;
        // sample extract: rank 0 writes the mask (polynomial 0), rank 1 the body
        const size_t row0 = dst_idx ? dst_idx[ct] : (size_t)ct * mlk;
        const u32 body = my_lwe[n];
        for (u32 m = 0; m < mlk; m++) {
            const u32 b = (body + m * (N / mlk)) & (TWO_N - 1);
            u64 *o = out + (row0 + m) * (N + 1);
            if (r == 0) {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const u32 oi = t + TPG * k;
                    const u32 j = oi == 0 ? 0 : N - oi;
                    const u32 src = (j + b) & (TWO_N - 1);
                    u64 v = bp[src & (N - 1)];
                    if (src >= (u32)N) v = 0ull - v;
                    st_stream(o + oi, oi == 0 ? v : 0ull - v);
                }
            } else if (t == 0) {
                u64 v = bp[b & (N - 1)];
                st_stream(o + N, b >= (u32)N ? 0ull - v : v);
            }
        }
        __syncthreads();
    }
    if (!ok && t == 0) {
        if (r == 0) atomicOr(err, DEVERR_TIMEOUT);
        if (!mbar_wait(mbar, *last_parity, DRAIN_POLLS))  // a half slab still landing here
            atomicOr(err, DEVERR_DRAIN);
    }
    cluster.sync();  // no CTA leaves while the other may still address its shared memory
}

size_t br_smem_bytes(const BrConfig &cfg, uint32_t n)
{
    const int G = cfg.cts_per_cta;
    (void)n;
    return (size_t)(SLAB_WORDS + 4096 + G * 4 * POLY_WORDS + 3) * 8;
}

template <int G, int BW>
static cudaError_t br_attr(size_t smem)
{
    return cudaFuncSetAttribute(br_kernel<G, BW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

bool pbs_supported(uint32_t bw) { return bw == 23 || bw == 22; }

cudaError_t br_set_attributes(const BrConfig &cfg, uint32_t n)
{
    size_t smem = br_smem_bytes(cfg, n);
    cudaError_t e = cudaFuncSetAttribute(br_kernel_split<23>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)br_split_smem_bytes());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(br_kernel_split<22>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)br_split_smem_bytes());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(br_kernel_pair<23>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)PAIR_SMEM_BYTES);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(br_kernel_pair<22>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)PAIR_SMEM_BYTES);
    if (e != cudaSuccess) return e;
    switch (cfg.cts_per_cta) {
    case 1: e = br_attr<1, 23>(smem); return e != cudaSuccess ? e : br_attr<1, 22>(smem);
    case 2: e = br_attr<2, 23>(smem); return e != cudaSuccess ? e : br_attr<2, 22>(smem);
    default: return cudaErrorInvalidValue;
    }
}

// One blind-rotation launch.  G: ciphertexts per CTA (1 or 2, br_kernel);
// 0: one ciphertext per CTA split over its two groups (br_kernel_split);
// -1: one ciphertext per cluster of two CTAs (br_kernel_pair).
static cudaError_t launch_br_once(int G, int ctas_per_sm, int nsm, const uint32_t *d_lwe2N, const uint64_t *d_luts,
                                  const uint32_t *d_lut_id, uint32_t nlut, const uint64_t *d_bsk,
                                  const uint64_t *d_tw, uint64_t *d_out, size_t B, uint32_t n, uint32_t *d_err,
                                  cudaStream_t s, const uint32_t *d_dst_idx, uint32_t mlk, uint32_t pbs_bw,
                                  uint32_t tie_rule)
{
    if (G == -1) {  // lowest-latency form: a cluster of two CTAs (two SMs) per ciphertext
        size_t pairs = B < (size_t)(nsm / 2) ? B : (size_t)(nsm / 2);
        u32 Bu = (u32)B;
        void *args[] = {(void *)&d_lwe2N, (void *)&d_luts, (void *)&d_lut_id, (void *)&nlut, (void *)&d_bsk,
                        (void *)&d_tw,    (void *)&d_out,  (void *)&Bu,       (void *)&n,    (void *)&d_err,
                        (void *)&d_dst_idx, (void *)&mlk, (void *)&tie_rule};
        const void *k = pbs_bw == 22 ? (const void *)br_kernel_pair<22> : (const void *)br_kernel_pair<23>;
        return cudaLaunchKernel(k, dim3((unsigned)(2 * pairs)), dim3(TPG), args, PAIR_SMEM_BYTES, s);
    }
    if (G == 0) {  // latency form: one ciphertext per CTA, polynomials split over the groups
        size_t grid = B < (size_t)nsm ? B : (size_t)nsm;
        u32 Bu = (u32)B;
        void *args[] = {(void *)&d_lwe2N, (void *)&d_luts, (void *)&d_lut_id, (void *)&nlut, (void *)&d_bsk,
                        (void *)&d_tw,    (void *)&d_out,  (void *)&Bu,       (void *)&n,    (void *)&d_err,
                        (void *)&d_dst_idx, (void *)&mlk, (void *)&tie_rule};
        const void *k = pbs_bw == 22 ? (const void *)br_kernel_split<22> : (const void *)br_kernel_split<23>;
        return cudaLaunchKernel(k, dim3((unsigned)grid), dim3(512), args, br_split_smem_bytes(), s);
    }
    size_t groups = (B + G - 1) / G;
    size_t grid = (size_t)nsm * ctas_per_sm;
    if (grid > groups) grid = groups;
    size_t smem = br_smem_bytes(BrConfig{G, ctas_per_sm}, n);
    u32 Bu = (u32)B;
    void *args[] = {(void *)&d_lwe2N, (void *)&d_luts, (void *)&d_lut_id, (void *)&nlut, (void *)&d_bsk,
                    (void *)&d_tw,    (void *)&d_out,  (void *)&Bu,       (void *)&n,    (void *)&d_err,
                    (void *)&d_dst_idx, (void *)&mlk, (void *)&tie_rule};
    const void *k;
    if (G == 1) k = pbs_bw == 22 ? (const void *)br_kernel<1, 22> : (const void *)br_kernel<1, 23>;
    else if (G == 2) k = pbs_bw == 22 ? (const void *)br_kernel<2, 22> : (const void *)br_kernel<2, 23>;
    else return cudaErrorInvalidValue;
    return cudaLaunchKernel(k, dim3((unsigned)grid), dim3(256 * G), args, smem, s);
}

cudaError_t launch_blind_rotate(const BrConfig &cfg, int nsm, const uint32_t *d_lwe2N, const uint64_t *d_luts,
                                const uint32_t *d_lut_id, uint32_t nlut, const uint64_t *d_bsk, const uint64_t *d_tw,
                                uint64_t *d_out, size_t B, uint32_t n, uint32_t *d_err, cudaStream_t s,
                                const uint32_t *d_dst_idx, uint32_t mlk, uint32_t pbs_bw, uint32_t tie_rule,
                                cudaEvent_t main_done, size_t *main_count)
{
    // main_count (optional) receives the number of leading ciphertexts whose
    // outputs are final once main_done (optional) fires on s: the full waves
    // when a tail launch follows them (the event is then recorded between the
    // two launches), else the whole batch (no event is recorded).
    if (main_count) *main_count = B;
    if (B == 0) return cudaSuccess;
    if (mlk != 1 && mlk != 2 && mlk != 4 && mlk != 8) return cudaErrorInvalidValue;
    if (!pbs_supported(pbs_bw)) return cudaErrorInvalidValue;
    if (tie_rule != TIE_RTL && tie_rule != TIE_GENERATOR) return cudaErrorInvalidValue;
    const int G = cfg.cts_per_cta, cps = cfg.ctas_per_sm;
    const size_t wave = (size_t)nsm * cps * G;
    const size_t pair_max = cfg.pair_max >= 0 ? (size_t)cfg.pair_max : (size_t)(nsm / 2);
    const size_t split_max = cfg.split_max >= 0 ? (size_t)cfg.split_max : (size_t)nsm;
    const size_t tail_max = cfg.tail_max >= 0 ? (size_t)cfg.tail_max : (size_t)nsm;
    // A batch that fits one ciphertext per SM runs in the latency form (one
    // ciphertext per CTA, its polynomials split over the two groups): with
    // G = 2 ciphertexts per CTA half the SMs would idle.
    // At most one ciphertext per two SMs: the two-SM form, lower latency still.
    // (Both forms are persistent over their ciphertexts, so any cut-off is correct.)
    auto small_form = [&](size_t count) { return count <= pair_max ? -1 : 0; };
    if (G > 1 && B <= split_max)
        return launch_br_once(small_form(B), 1, nsm, d_lwe2N, d_luts, d_lut_id, nlut, d_bsk, d_tw, d_out, B, n,
                              d_err, s, d_dst_idx, mlk, pbs_bw, tie_rule);
    // A partial last wave of at most one ciphertext per SM runs as its own
    // latency-form launch after the full waves instead of a full G-per-CTA wave.
    const size_t tail = B % wave;
    if (G > 1 && B > wave && tail > 0 && tail <= tail_max) {
        const size_t full = B - tail;
        cudaError_t e = launch_br_once(G, cps, nsm, d_lwe2N, d_luts, d_lut_id, nlut, d_bsk, d_tw, d_out, full, n,
                                       d_err, s, d_dst_idx, mlk, pbs_bw, tie_rule);
        if (e != cudaSuccess) return e;
        if (main_done && (e = cudaEventRecord(main_done, s)) != cudaSuccess) return e;
        if (main_count) *main_count = full;
        uint64_t *out_tail = d_dst_idx ? d_out : d_out + full * mlk * (size_t)(N + 1);
        return launch_br_once(small_form(tail), 1, nsm, d_lwe2N + full * (size_t)(n + 1), d_luts, d_lut_id + full,
                              nlut, d_bsk, d_tw, out_tail, tail, n, d_err, s, d_dst_idx ? d_dst_idx + full : nullptr,
                              mlk, pbs_bw, tie_rule);
    }
    return launch_br_once(G, cps, nsm, d_lwe2N, d_luts, d_lut_id, nlut, d_bsk, d_tw, d_out, B, n, d_err, s,
                          d_dst_idx, mlk, pbs_bw, tie_rule);
}

// ---------------------------------------------------------- linear DOps
//
// pea_alu_core.sv:59-61,124-161: per coefficient, with the message constant
// placed at the body only (imm << (64 - 5), 1 padding + 2 msg + 2 carry bits):
//   ADD a+b, SUB a-b, MAC a*m+b, ADDS a+c, SUBS a-c, SSUB c-a, MULS a*m.
__global__ void lwe_op_kernel(int op, const u64 *__restrict__ a, const u64 *__restrict__ b, u64 *__restrict__ o,
                              u64 imm, size_t total, u32 dim)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const bool body = (i % (dim + 1)) == dim;
        const u64 cst = body ? (imm << 59) : 0ull;
        u64 v;
        switch (op) {
        case LWE_ADD: v = a[i] + b[i]; break;
        case LWE_SUB: v = a[i] - b[i]; break;
        case LWE_MAC: v = a[i] * imm + b[i]; break;
        case LWE_ADDS: v = a[i] + cst; break;
        case LWE_SUBS: v = a[i] - cst; break;
        case LWE_SSUB: v = cst - a[i]; break;
        default: v = a[i] * imm; break;
        }
        o[i] = v;
    }
}

// A batch of linear DOps (and register copies) over a pool of BLWE slots:
// op i writes slot dst[i] from slots a[i], b[i] and the immediate imm[i]
// (the serving loop issues every ready ALU DOp of every request in one launch).
__global__ void alu_batch_kernel(const AluOp *__restrict__ ops, u64 *__restrict__ pool, u32 nops, u32 dim)
{
    const size_t w = dim + 1, total = (size_t)nops * w;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const AluOp o = ops[i / w];
        const size_t c = i % w;
        const bool body = c == dim;
        const u64 cst = body ? (o.imm << 59) : 0ull;
        const u64 a = pool[(size_t)o.a * w + c];
        const u64 b = (o.op == LWE_ADD || o.op == LWE_SUB || o.op == LWE_MAC) ? pool[(size_t)o.b * w + c] : 0ull;
        u64 v;
        switch (o.op) {
        case LWE_ADD: v = a + b; break;
        case LWE_SUB: v = a - b; break;
        case LWE_MAC: v = a * o.imm + b; break;
        case LWE_ADDS: v = a + cst; break;
        case LWE_SUBS: v = a - cst; break;
        case LWE_SSUB: v = cst - a; break;
        case LWE_MULS: v = a * o.imm; break;
        default: v = a; break;  // copy
        }
        pool[(size_t)o.dst * w + c] = v;
    }
}

cudaError_t launch_alu_batch(const AluOp *d_ops, uint64_t *d_pool, uint32_t nops, uint32_t dim, cudaStream_t s)
{
    if (nops == 0) return cudaSuccess;
    size_t total = (size_t)nops * (dim + 1);
    size_t blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    alu_batch_kernel<<<(unsigned)blocks, 256, 0, s>>>(d_ops, d_pool, nops, dim);
    return cudaGetLastError();
}

cudaError_t launch_lwe_op(int op, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out, uint64_t imm,
                          size_t count, uint32_t dim, cudaStream_t s)
{
    size_t total = count * (size_t)(dim + 1);
    if (total == 0) return cudaSuccess;
    size_t blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    lwe_op_kernel<<<(unsigned)blocks, 256, 0, s>>>(op, d_a, d_b, d_out, imm, total, dim);
    return cudaGetLastError();
}

}  // namespace luthe
