// Goldilocks field arithmetic, p = 2^64 - 2^32 + 1, on the integer pipes.
//
// Values travel in "lazy" form: any u64 congruent to the residue (so in
// [0, 2^64), possibly >= p).  add/sub/mul accept lazy inputs and return lazy
// outputs; canon() brings a value to [0, p).  The reduction uses
// 2^64 = 2^32 - 1 and 2^96 = -1 (mod p), the Solinas form that the reference
// models in sw/solinas/solinas.py:218-319 and sw/ntt/ntt_gf64.sage:31-50.
// Multiplication by 2^s is a shift plus that reduction: powers of two are the
// 192-th roots of unity of this field (8 is a primitive 64-th root), which is
// what makes the radix-32/radix-64 sub-transforms of the NTT multiply-free.
#pragma once
#include <stdint.h>

typedef uint64_t u64;
typedef uint32_t u32;

namespace gl {

constexpr u64 P = 0xFFFFFFFF00000001ull;
constexpr u64 EPS = 0xFFFFFFFFull;  // 2^64 mod p

// a + b: a 64-bit add whose carry (2^64 == EPS) is folded back at most twice;
// written with explicit carry chains, which the compiler does not find from C.
__device__ __forceinline__ u64 add(u64 a, u64 b)
{
    u64 r;
    asm("{\n\t.reg .u32 c;\n\t.reg .u64 m;\n\t"
        "add.cc.u64 %0, %1, %2;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "neg.s32 c, c;\n\t"
        "cvt.u64.u32 m, c;\n\t"
        "add.cc.u64 %0, %0, m;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "neg.s32 c, c;\n\t"
        "cvt.u64.u32 m, c;\n\t"
        "add.u64 %0, %0, m;\n\t}"
        : "=l"(r)
        : "l"(a), "l"(b));
    return r;
}

// a - b: a borrow (-2^64 == -EPS) is folded back at most twice.
__device__ __forceinline__ u64 sub(u64 a, u64 b)
{
    u64 r;
    asm("{\n\t.reg .u32 c;\n\t.reg .u64 m;\n\t"
        "sub.cc.u64 %0, %1, %2;\n\t"
        "subc.u32 c, 0, 0;\n\t"
        "cvt.u64.u32 m, c;\n\t"
        "sub.cc.u64 %0, %0, m;\n\t"
        "subc.u32 c, 0, 0;\n\t"
        "cvt.u64.u32 m, c;\n\t"
        "sub.u64 %0, %0, m;\n\t}"
        : "=l"(r)
        : "l"(a), "l"(b));
    return r;
}

// lo + hi * 2^64  ->  lazy residue:  lo - h1 + h0 (2^32 - 1), hi = h1:h0
// (h1 2^96 == -h1, h0 2^64 == h0 (2^32 - 1)); the h0 product goes to IMAD.
__device__ __forceinline__ u64 reduce128(u64 lo, u64 hi)
{
    u64 r;
    asm("{\n\t.reg .u32 c;\n\t.reg .u64 m, u, h;\n\t"
        "cvt.u64.u32 h, %3;\n\t"
        "sub.cc.u64 %0, %1, h;\n\t"
        "subc.u32 c, 0, 0;\n\t"
        "cvt.u64.u32 m, c;\n\t"
        "sub.u64 %0, %0, m;\n\t"
        "mul.wide.u32 u, %2, 0xFFFFFFFF;\n\t"
        "add.cc.u64 %0, %0, u;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "neg.s32 c, c;\n\t"
        "cvt.u64.u32 m, c;\n\t"
        "add.u64 %0, %0, m;\n\t}"
        : "=l"(r)
        : "l"(lo), "r"((u32)hi), "r"((u32)(hi >> 32)));
    return r;
}

// lo + h0 * 2^64 with h0 < 2^32: lo + h0 (2^32 - 1)
__device__ __forceinline__ u64 reduce96(u64 lo, u32 h0)
{
    u64 r;
    asm("{\n\t.reg .u32 c;\n\t.reg .u64 m, u;\n\t"
        "mul.wide.u32 u, %2, 0xFFFFFFFF;\n\t"
        "add.cc.u64 %0, %1, u;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "neg.s32 c, c;\n\t"
        "cvt.u64.u32 m, c;\n\t"
        "add.u64 %0, %0, m;\n\t}"
        : "=l"(r)
        : "l"(lo), "r"(h0));
    return r;
}

__device__ __forceinline__ u64 mul(u64 a, u64 b) { return reduce128(a * b, __umul64hi(a, b)); }

__device__ __forceinline__ u64 canon(u64 a) { return a >= P ? a - P : a; }

__device__ __forceinline__ u64 neg(u64 a) { return sub(0ull, a); }

__host__ __device__ constexpr int mod192(int s) { return ((s % 192) + 192) % 192; }

// x * 2^S for a compile-time S (any sign; 2^192 == 1).
template <int S>
__device__ __forceinline__ u64 shl(u64 x)
{
    constexpr int s = mod192(S);
    if constexpr (s == 0) {
        return x;
    } else if constexpr (s >= 96) {
        return neg(shl<s - 96>(x));  // 2^96 == -1
    } else if constexpr (s <= 32) {
        return reduce96(x << s, (u32)(x >> (64 - s)));
    } else {
        return shl<32>(shl<s - 32>(x));  // two 96-bit folds beat one 128-bit fold
    }
}

// x * 2^s for a runtime s in [0, 192) that is uniform across the warp: one
// copy of the code serves every exponent (the pass twiddles), the branches
// never diverge.
__device__ __forceinline__ u64 shl_rt(u64 x, u32 s)
{
    const bool negate = s >= 96;
    if (negate) s -= 96;
    if (s > 32) {
        const u32 s1 = s > 64 ? 32 : s - 32;  // first fold: s1 in [1, 32]
        x = reduce96(x << s1, (u32)(x >> (64 - s1)));
        s -= s1;
        if (s > 32) {
            x = reduce96(x << 32, (u32)(x >> 32));
            s -= 32;
        }
    }
    if (s) x = reduce96(x << s, (u32)(x >> (64 - s)));
    return negate ? neg(x) : x;
}

// a*b + c*d with one reduction: the two 128-bit products are summed first;
// a carry out of bit 128 is worth 2^128 == -2^32 (mod p).
__device__ __forceinline__ u64 mul_add2(u64 a, u64 b, u64 c, u64 d)
{
    u64 lo, hi;
    u32 c2;
    const u64 l1 = a * b, h1 = __umul64hi(a, b), l2 = c * d, h2 = __umul64hi(c, d);
    asm("add.cc.u64 %0, %3, %4;\n\t"
        "addc.cc.u64 %1, %5, %6;\n\t"
        "addc.u32 %2, 0, 0;"
        : "=l"(lo), "=l"(hi), "=r"(c2)
        : "l"(l1), "l"(l2), "l"(h1), "l"(h2));
    return sub(reduce128(lo, hi), (u64)c2 << 32);
}

// Cooley-Tukey butterfly: (u, v) <- (u + v 2^S, u - v 2^S)
template <int S>
__device__ __forceinline__ void ct_bf(u64 &u, u64 &v)
{
    constexpr int s = mod192(S);
    if constexpr (s >= 96) {
        u64 t = shl<s - 96>(v);
        u64 a = sub(u, t);
        v = add(u, t);
        u = a;
    } else {
        u64 t = shl<s>(v);
        u64 a = add(u, t);
        v = sub(u, t);
        u = a;
    }
}

// Gentleman-Sande butterfly: (u, v) <- (u + v, (u - v) 2^S)
template <int S>
__device__ __forceinline__ void gs_bf(u64 &u, u64 &v)
{
    constexpr int s = mod192(S);
    if constexpr (s >= 96) {
        u64 a = add(u, v);
        v = shl<s - 96>(sub(v, u));
        u = a;
    } else {
        u64 a = add(u, v);
        v = shl<s>(sub(u, v));
        u = a;
    }
}

// p -> 2^64 modulus switch of a canonical residue a:
//   z = ((a * CST) >> 96) + bit95(a * CST),  CST = floor(2^160 / p) = 2^96 + 2^64 - 2
// (hw/common_lib/.../mod_switch_to_2powerN.sv:62-64,132-134 with
//  MOD_Q_W = 64, PRECISION_W = 96).
__device__ __forceinline__ u64 modsw_p_to_q(u64 a)
{
    const u64 cst_lo = 0xFFFFFFFFFFFFFFFEull;  // CST mod 2^64; CST >> 64 = 2^32
    u64 ph = __umul64hi(a, cst_lo);
    u64 m = ph + (a << 32);
    u64 top = (a >> 32) + (m < ph ? 1ull : 0ull);
    return (top << 32) + (m >> 32) + ((m >> 31) & 1ull);
}

// Balanced decomposition, base 2^23, one level, of a 64-bit torus value,
// embedded in Z_p (decomp_balseq_core.sv:135-150; the rounding and tie rule of
// sw/decomposer/balanced_decomp_unfix_sign_round_bit.py:42-101 with bw=23, L=1).
template <int BW>
__device__ __forceinline__ u64 decomp_to_p(u64 v)
{
    constexpr u64 B = 1ull << BW, HALF = B >> 1;
    u64 rb = (v >> (63 - BW)) & 1ull;
    u64 c = (v >> (64 - BW)) + rb;      // 0 .. 2^BW
    u64 t = c & (B - 1);
    // with one level the digit above is last_sign * (B-1), last_sign = rb at a tie
    bool negd = (t > HALF) || (t == HALF && rb);
    // negative digit t - 2^BW embeds as p - (2^BW - t)
    return negd ? (P - (B - t)) : t;
}
__device__ __forceinline__ u64 decomp23_to_p(u64 v) { return decomp_to_p<23>(v); }

}  // namespace gl
