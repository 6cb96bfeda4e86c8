// Negacyclic NTT / INTT of N = 2048 over Goldilocks, one polynomial group per
// 256 threads, 8 coefficients per thread and polynomial, staged through a
// per-group shared-memory buffer.
//
// The transform computes A_k = sum_j a_j psi^{j(2k+1)} (psi a primitive 4096-th
// root with psi^64 = 8), the same evaluation map as the reference's negacyclic
// model sw/ntt/ntt_gf64.sage:367-445 (output order aside).  It is split as
// 2048 = 32 x 64 with j = 64 j1 + j2, k = k1 + 32 k2:
//   A  (32-point negacyclic, psi_32 = 8) over j1, itself 8 x 4:
//      A1: 8-point negacyclic CT over j1b (psi_8 = 2^12), twiddle 2^{3 j1a (2 k1b + 1)}
//      A2: 4-point cyclic over j1a (omega_4 = 2^48)
//   B  twiddle psi^{j2 (2 k1 + 1)}          <- the only general multiplies
//   C  (64-point cyclic, omega_64 = 8) over j2, itself 8 x 8:
//      C1: 8-point cyclic over j2b (omega_8 = 2^24), twiddle 2^{3 j2a k2b}
//      C2: 8-point cyclic over j2a
// A and C use shifts only (powers of two are roots of unity mod p), which is
// the Goldilocks property the reference's ntt_core_gf64 exploits with its
// radix cuts and power-of-2 twiddles (ntt_gf64.sage:35-50,104-127).
//
// Thread roles (t in [0,256) within the group):
//   A1: j1a = t>>6, j2 = t&63   holds j1b = 0..7     (coefficient layout)
//   A2: kp  = t>>6, j2 = t&63   holds k1b in {kp, kp+4} x k1a
//   C1: j2a = t>>5, k1 = t&31   holds j2b / k2b
//   C2: k2b = t>>5, k1 = t&31   holds k2a  (evaluation layout)
// so every runtime twiddle exponent (j1a, j2a) is warp-uniform.  Shared-memory
// layouts are chosen so that each warp touches consecutive 8-byte words (the
// 32 x 65 padded layout removes the 32-way conflict of the k1-strided access).
//
// The inverse runs the passes backwards with inverted twiddles and no 1/N:
// callers fold N^{-1} into the operand they multiply with (the BSK).
#pragma once
#include "gl.cuh"

namespace ntt {

constexpr int N = 2048;
constexpr int TPG = 256;             // threads per polynomial group
constexpr int POLY_WORDS = 32 * 65;  // per-polynomial staging words (padded layout)

__host__ __device__ constexpr int brv3(int p) { return ((p & 1) << 2) | (p & 2) | ((p >> 2) & 1); }
__host__ __device__ constexpr int brv2(int p) { return ((p & 1) << 1) | ((p >> 1) & 1); }

__device__ __forceinline__ void group_sync(int bar_id)
{
    asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(TPG) : "memory");
}

// ------------------------------------------------------------- small kernels

// 8-point negacyclic CT, psi = 2^12: natural in, position p holds k = brv3(p)
__device__ __forceinline__ void ct8_neg(u64 *x)
{
    gl::ct_bf<48>(x[0], x[4]);
    gl::ct_bf<48>(x[1], x[5]);
    gl::ct_bf<48>(x[2], x[6]);
    gl::ct_bf<48>(x[3], x[7]);
    gl::ct_bf<24>(x[0], x[2]);
    gl::ct_bf<24>(x[1], x[3]);
    gl::ct_bf<72>(x[4], x[6]);
    gl::ct_bf<72>(x[5], x[7]);
    gl::ct_bf<12>(x[0], x[1]);
    gl::ct_bf<60>(x[2], x[3]);
    gl::ct_bf<36>(x[4], x[5]);
    gl::ct_bf<84>(x[6], x[7]);
}
// exact inverse of ct8_neg up to a factor 8
__device__ __forceinline__ void gs8_neg_inv(u64 *x)
{
    gl::gs_bf<-12>(x[0], x[1]);
    gl::gs_bf<-60>(x[2], x[3]);
    gl::gs_bf<-36>(x[4], x[5]);
    gl::gs_bf<-84>(x[6], x[7]);
    gl::gs_bf<-24>(x[0], x[2]);
    gl::gs_bf<-24>(x[1], x[3]);
    gl::gs_bf<-72>(x[4], x[6]);
    gl::gs_bf<-72>(x[5], x[7]);
    gl::gs_bf<-48>(x[0], x[4]);
    gl::gs_bf<-48>(x[1], x[5]);
    gl::gs_bf<-48>(x[2], x[6]);
    gl::gs_bf<-48>(x[3], x[7]);
}
// 8-point cyclic DIF, omega = 2^24: natural in, position p holds k = brv3(p)
__device__ __forceinline__ void dif8(u64 *x)
{
    gl::gs_bf<0>(x[0], x[4]);
    gl::gs_bf<24>(x[1], x[5]);
    gl::gs_bf<48>(x[2], x[6]);
    gl::gs_bf<72>(x[3], x[7]);
    gl::gs_bf<0>(x[0], x[2]);
    gl::gs_bf<48>(x[1], x[3]);
    gl::gs_bf<0>(x[4], x[6]);
    gl::gs_bf<48>(x[5], x[7]);
    gl::gs_bf<0>(x[0], x[1]);
    gl::gs_bf<0>(x[2], x[3]);
    gl::gs_bf<0>(x[4], x[5]);
    gl::gs_bf<0>(x[6], x[7]);
}
// exact inverse of dif8 up to a factor 8 (position-p input, natural output)
__device__ __forceinline__ void dit8_inv(u64 *x)
{
    gl::ct_bf<0>(x[0], x[1]);
    gl::ct_bf<0>(x[2], x[3]);
    gl::ct_bf<0>(x[4], x[5]);
    gl::ct_bf<0>(x[6], x[7]);
    gl::ct_bf<0>(x[0], x[2]);
    gl::ct_bf<-48>(x[1], x[3]);
    gl::ct_bf<0>(x[4], x[6]);
    gl::ct_bf<-48>(x[5], x[7]);
    gl::ct_bf<0>(x[0], x[4]);
    gl::ct_bf<-24>(x[1], x[5]);
    gl::ct_bf<-48>(x[2], x[6]);
    gl::ct_bf<-72>(x[3], x[7]);
}
// 4-point cyclic DIF, omega = 2^48 (position p holds k = brv2(p))
__device__ __forceinline__ void dif4(u64 *x)
{
    gl::gs_bf<0>(x[0], x[2]);
    gl::gs_bf<48>(x[1], x[3]);
    gl::gs_bf<0>(x[0], x[1]);
    gl::gs_bf<0>(x[2], x[3]);
}
__device__ __forceinline__ void dit4_inv(u64 *x)
{
    gl::ct_bf<0>(x[0], x[1]);
    gl::ct_bf<0>(x[2], x[3]);
    gl::ct_bf<0>(x[0], x[2]);
    gl::ct_bf<-48>(x[1], x[3]);
}

// -------------------------------------------------- warp-uniform shift twiddles

template <int J1A, int SIGN>
__device__ __forceinline__ void tw_a1(u64 *y)
{
    y[0] = gl::shl<SIGN * 3 * J1A * (2 * brv3(0) + 1)>(y[0]);
    y[1] = gl::shl<SIGN * 3 * J1A * (2 * brv3(1) + 1)>(y[1]);
    y[2] = gl::shl<SIGN * 3 * J1A * (2 * brv3(2) + 1)>(y[2]);
    y[3] = gl::shl<SIGN * 3 * J1A * (2 * brv3(3) + 1)>(y[3]);
    y[4] = gl::shl<SIGN * 3 * J1A * (2 * brv3(4) + 1)>(y[4]);
    y[5] = gl::shl<SIGN * 3 * J1A * (2 * brv3(5) + 1)>(y[5]);
    y[6] = gl::shl<SIGN * 3 * J1A * (2 * brv3(6) + 1)>(y[6]);
    y[7] = gl::shl<SIGN * 3 * J1A * (2 * brv3(7) + 1)>(y[7]);
}
// 2^e mod p for e in [0, 192), built at compile time: the runtime pass
// twiddles below are one multiply by a constant-cache word (the exponent is
// warp-uniform, so every lane reads the same word).  A branch-free multiply
// is shorter code than a shift with its range cases, and half of its work
// runs on the multiply pipe instead of the saturated integer ALU.
struct Pow2Table {
    u64 v[192];
};
__host__ __device__ constexpr Pow2Table make_pow2_table()
{
    Pow2Table t{};
    u64 x = 1;
    for (int e = 0; e < 192; e++) {
        t.v[e] = x;
        const bool top = (x >> 63) != 0;
        u64 y = x << 1;
        if (top || y >= gl::P) y -= gl::P;  // 2x < 2p: one subtraction (mod 2^64)
        x = y;
    }
    return t;
}
static __constant__ Pow2Table c_pow2 = make_pow2_table();

// Runtime forms: one copy of the twiddle code for every warp-uniform j1a / j2a
// (the templated forms above, one per value, overflow the instruction cache).
template <int SIGN>
__device__ __forceinline__ void tw_a1_rt(u64 *y, int j1a)
{
    if (j1a == 0) return;
#pragma unroll
    for (int p = 0; p < 8; p++) {
        const u32 e = 3u * j1a * (2 * brv3(p) + 1);  // < 192
        y[p] = gl::mul(y[p], c_pow2.v[SIGN > 0 ? e : (192u - e) % 192u]);
    }
}
template <int J2A, int SIGN>
__device__ __forceinline__ void tw_c1(u64 *y)
{
    y[0] = gl::shl<SIGN * 3 * J2A * brv3(0)>(y[0]);
    y[1] = gl::shl<SIGN * 3 * J2A * brv3(1)>(y[1]);
    y[2] = gl::shl<SIGN * 3 * J2A * brv3(2)>(y[2]);
    y[3] = gl::shl<SIGN * 3 * J2A * brv3(3)>(y[3]);
    y[4] = gl::shl<SIGN * 3 * J2A * brv3(4)>(y[4]);
    y[5] = gl::shl<SIGN * 3 * J2A * brv3(5)>(y[5]);
    y[6] = gl::shl<SIGN * 3 * J2A * brv3(6)>(y[6]);
    y[7] = gl::shl<SIGN * 3 * J2A * brv3(7)>(y[7]);
}
template <int SIGN>
__device__ __forceinline__ void tw_c1_rt(u64 *y, int j2a)
{
    if (j2a == 0) return;
#pragma unroll
    for (int p = 1; p < 8; p++) {  // p = 0 has k2b = 0: twiddle 1
        const u32 e = 3u * j2a * brv3(p);  // < 192
        y[p] = gl::mul(y[p], c_pow2.v[SIGN > 0 ? e : (192u - e) % 192u]);
    }
}

// ----------------------------------------------------------- twiddle tables

// Twiddle table layout: tw[(c*4 + p) * 256 + t] for the A2 role of thread t
// (kp = t>>6, j2 = t&63): k1 = kp + 4c + 8 brv2(p), value psi^{+-j2(2 k1 + 1)}.
__host__ __device__ inline int a2_k1(int t, int slot) { return (t >> 6) + 4 * (slot >> 2) + 8 * brv2(slot & 3); }

// ------------------------------------------------------------------ passes

// Forward transform of NP polynomials held as x[q][j1b] in the coefficient
// layout (thread t holds a[64 j1a + 256 j1b + j2]).  On return x[q][p] holds
// A_k for k = k1 + 32 k2b + 256 brv3(p), (k2b, k1) = (t>>5, t&31).
// `buf` holds NP * POLY_WORDS words.  The caller places a barrier before the
// call if `buf` was just read, and another before the next write to `buf`.
template <int NP>
__device__ __forceinline__ void forward(u64 (&x)[NP][8], u64 *buf, const u64 *tw_fwd, int t, int bar_id)
{
    // A1
    {
        const int j1a = t >> 6, j2 = t & 63;
#pragma unroll
        for (int q = 0; q < NP; q++) {
            ct8_neg(x[q]);
            tw_a1_rt<1>(x[q], j1a);
            u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int p = 0; p < 8; p++) b[(j1a * 8 + brv3(p)) * 64 + j2] = x[q][p];
        }
    }
    group_sync(bar_id);
    // A2 + B
    {
        const int kp = t >> 6, j2 = t & 63;
#pragma unroll
        for (int q = 0; q < NP; q++) {
            const u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int c = 0; c < 2; c++)
#pragma unroll
                for (int j1a = 0; j1a < 4; j1a++) x[q][c * 4 + j1a] = b[(j1a * 8 + kp + 4 * c) * 64 + j2];
        }
        group_sync(bar_id);
#pragma unroll
        for (int q = 0; q < NP; q++) {
            dif4(x[q]);
            dif4(x[q] + 4);
            u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int s = 0; s < 8; s++) {
                u64 v = gl::mul(x[q][s], tw_fwd[s * TPG + t]);
                b[(kp + 4 * (s >> 2) + 8 * brv2(s & 3)) * 65 + j2] = v;
            }
        }
    }
    group_sync(bar_id);
    // C1
    {
        const int j2a = t >> 5, k1 = t & 31;
#pragma unroll
        for (int q = 0; q < NP; q++) {
            const u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int j2b = 0; j2b < 8; j2b++) x[q][j2b] = b[k1 * 65 + j2a + 8 * j2b];
        }
        group_sync(bar_id);
#pragma unroll
        for (int q = 0; q < NP; q++) {
            dif8(x[q]);
            tw_c1_rt<1>(x[q], j2a);
            u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int p = 0; p < 8; p++) b[(j2a * 8 + brv3(p)) * 32 + k1] = x[q][p];
        }
    }
    group_sync(bar_id);
    // C2
    {
        const int k2b = t >> 5, k1 = t & 31;
#pragma unroll
        for (int q = 0; q < NP; q++) {
            const u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int j2a = 0; j2a < 8; j2a++) x[q][j2a] = b[(j2a * 8 + k2b) * 32 + k1];
            dif8(x[q]);
        }
    }
}

// Inverse (no 1/N): x[q][p] in the evaluation layout -> x[q][j1b] in the
// coefficient layout, scaled by N.  The caller must have placed a barrier
// after the last read of `buf` (the C2 read in forward) before calling, and
// must place one before the next write to `buf`.
template <int NP>
__device__ __forceinline__ void inverse(u64 (&x)[NP][8], u64 *buf, const u64 *tw_inv, int t, int bar_id)
{
    // C2^-1
    {
        const int k2b = t >> 5, k1 = t & 31;
#pragma unroll
        for (int q = 0; q < NP; q++) {
            dit8_inv(x[q]);
            u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int j2a = 0; j2a < 8; j2a++) b[(j2a * 8 + k2b) * 32 + k1] = x[q][j2a];
        }
    }
    group_sync(bar_id);
    // C1^-1
    {
        const int j2a = t >> 5, k1 = t & 31;
#pragma unroll
        for (int q = 0; q < NP; q++) {
            const u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int p = 0; p < 8; p++) x[q][p] = b[(j2a * 8 + brv3(p)) * 32 + k1];
        }
        group_sync(bar_id);
#pragma unroll
        for (int q = 0; q < NP; q++) {
            tw_c1_rt<-1>(x[q], j2a);
            dit8_inv(x[q]);
            u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int j2b = 0; j2b < 8; j2b++) b[k1 * 65 + j2a + 8 * j2b] = x[q][j2b];
        }
    }
    group_sync(bar_id);
    // B^-1 + A2^-1
    {
        const int kp = t >> 6, j2 = t & 63;
#pragma unroll
        for (int q = 0; q < NP; q++) {
            const u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int s = 0; s < 8; s++)
                x[q][s] = gl::mul(b[(kp + 4 * (s >> 2) + 8 * brv2(s & 3)) * 65 + j2], tw_inv[s * TPG + t]);
        }
        group_sync(bar_id);
#pragma unroll
        for (int q = 0; q < NP; q++) {
            dit4_inv(x[q]);
            dit4_inv(x[q] + 4);
            u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int c = 0; c < 2; c++)
#pragma unroll
                for (int j1a = 0; j1a < 4; j1a++) b[(j1a * 8 + kp + 4 * c) * 64 + j2] = x[q][c * 4 + j1a];
        }
    }
    group_sync(bar_id);
    // A1^-1
    {
        const int j1a = t >> 6, j2 = t & 63;
#pragma unroll
        for (int q = 0; q < NP; q++) {
            const u64 *b = buf + q * POLY_WORDS;
#pragma unroll
            for (int p = 0; p < 8; p++) x[q][p] = b[(j1a * 8 + brv3(p)) * 64 + j2];
            tw_a1_rt<-1>(x[q], j1a);
            gs8_neg_inv(x[q]);
        }
    }
}

// Single-pass building blocks for callers that run a transform one polynomial
// at a time (a rolled loop: one copy of the pass code for every polynomial,
// which keeps a whole blind-rotation step inside the instruction cache).  Each
// reads one staging buffer and writes another; barriers are the caller's.
// Layouts as in forward/inverse above.

// A1 of one polynomial held in registers (coefficient layout) -> dst
__device__ __forceinline__ void a1_fwd(u64 *y, u64 *dst, int t)
{
    const int j1a = t >> 6, j2 = t & 63;
    ct8_neg(y);
    tw_a1_rt<1>(y, j1a);
#pragma unroll
    for (int p = 0; p < 8; p++) dst[(j1a * 8 + brv3(p)) * 64 + j2] = y[p];
}
// A2 + B of NP polynomials: src (A1 layout) -> dst (padded k1 layout)
template <int NP>
__device__ __forceinline__ void a2_fwd(const u64 *src, u64 *dst, const u64 *tw_fwd, int t)
{
    const int kp = t >> 6, j2 = t & 63;
#pragma unroll 1
    for (int q = 0; q < NP; q++) {
        const u64 *b = src + q * POLY_WORDS;
        u64 y[8];
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
            for (int j1a = 0; j1a < 4; j1a++) y[c * 4 + j1a] = b[(j1a * 8 + kp + 4 * c) * 64 + j2];
        dif4(y);
        dif4(y + 4);
        u64 *o = dst + q * POLY_WORDS;
#pragma unroll
        for (int s = 0; s < 8; s++) o[(kp + 4 * (s >> 2) + 8 * brv2(s & 3)) * 65 + j2] = gl::mul(y[s], tw_fwd[s * TPG + t]);
    }
}
// C1 of NP polynomials: src (padded k1 layout) -> dst (C1 layout)
template <int NP>
__device__ __forceinline__ void c1_fwd(const u64 *src, u64 *dst, int t)
{
    const int j2a = t >> 5, k1 = t & 31;
#pragma unroll 1
    for (int q = 0; q < NP; q++) {
        const u64 *b = src + q * POLY_WORDS;
        u64 y[8];
#pragma unroll
        for (int j2b = 0; j2b < 8; j2b++) y[j2b] = b[k1 * 65 + j2a + 8 * j2b];
        dif8(y);
        tw_c1_rt<1>(y, j2a);
        u64 *o = dst + q * POLY_WORDS;
#pragma unroll
        for (int p = 0; p < 8; p++) o[(j2a * 8 + brv3(p)) * 32 + k1] = y[p];
    }
}
// C2 of one polynomial: src (C1 layout) -> y, evaluation layout
__device__ __forceinline__ void c2_fwd(const u64 *src, u64 *y, int t)
{
    const int k2b = t >> 5, k1 = t & 31;
#pragma unroll
    for (int j2a = 0; j2a < 8; j2a++) y[j2a] = src[(j2a * 8 + k2b) * 32 + k1];
    dif8(y);
}
// C2^-1 of one polynomial held in registers (evaluation layout) -> dst
__device__ __forceinline__ void c2_inv(u64 *y, u64 *dst, int t)
{
    const int k2b = t >> 5, k1 = t & 31;
    dit8_inv(y);
#pragma unroll
    for (int j2a = 0; j2a < 8; j2a++) dst[(j2a * 8 + k2b) * 32 + k1] = y[j2a];
}
// C1^-1 of NP polynomials: src (C1 layout) -> dst (padded k1 layout)
template <int NP>
__device__ __forceinline__ void c1_inv(const u64 *src, u64 *dst, int t)
{
    const int j2a = t >> 5, k1 = t & 31;
#pragma unroll 1
    for (int q = 0; q < NP; q++) {
        const u64 *b = src + q * POLY_WORDS;
        u64 y[8];
#pragma unroll
        for (int p = 0; p < 8; p++) y[p] = b[(j2a * 8 + brv3(p)) * 32 + k1];
        tw_c1_rt<-1>(y, j2a);
        dit8_inv(y);
        u64 *o = dst + q * POLY_WORDS;
#pragma unroll
        for (int j2b = 0; j2b < 8; j2b++) o[k1 * 65 + j2a + 8 * j2b] = y[j2b];
    }
}
// B^-1 + A2^-1 of NP polynomials: src (padded k1 layout) -> dst (A1 layout)
template <int NP>
__device__ __forceinline__ void a2_inv(const u64 *src, u64 *dst, const u64 *tw_inv, int t)
{
    const int kp = t >> 6, j2 = t & 63;
#pragma unroll 1
    for (int q = 0; q < NP; q++) {
        const u64 *b = src + q * POLY_WORDS;
        u64 y[8];
#pragma unroll
        for (int s = 0; s < 8; s++)
            y[s] = gl::mul(b[(kp + 4 * (s >> 2) + 8 * brv2(s & 3)) * 65 + j2], tw_inv[s * TPG + t]);
        dit4_inv(y);
        dit4_inv(y + 4);
        u64 *o = dst + q * POLY_WORDS;
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
            for (int j1a = 0; j1a < 4; j1a++) o[(j1a * 8 + kp + 4 * c) * 64 + j2] = y[c * 4 + j1a];
    }
}
// A1^-1 of one polynomial: src (A1 layout) -> y, coefficient layout (times N)
__device__ __forceinline__ void a1_inv(const u64 *src, u64 *y, int t)
{
    const int j1a = t >> 6, j2 = t & 63;
#pragma unroll
    for (int p = 0; p < 8; p++) y[p] = src[(j1a * 8 + brv3(p)) * 64 + j2];
    tw_a1_rt<-1>(y, j1a);
    gs8_neg_inv(y);
}

// Coefficient index held by thread t in slot e of the coefficient layout.
__host__ __device__ inline int coef_index(int t, int e) { return 64 * (t >> 6) + 256 * e + (t & 63); }
// Evaluation index k held by thread t in slot p of the evaluation layout.
__host__ __device__ inline int eval_index(int t, int p) { return (t & 31) + 32 * (t >> 5) + 256 * brv3(p); }

}  // namespace ntt
