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

// a * b as 128 bits (hi:lo): the four 32 x 32 partial products and their
// carries as one multiply-add chain (mad.lo/madc.hi with carry flags), which
// keeps the whole product on the multiply pipe.
__device__ __forceinline__ void mul_wide(u64 a, u64 b, u64 &lo, u64 &hi)
{
    asm("{\n\t.reg .u32 a0, a1, b0, b1, r0, r1, r2, r3;\n\t"
        "mov.b64 {a0, a1}, %2;\n\t"
        "mov.b64 {b0, b1}, %3;\n\t"
        "mul.lo.u32 r0, a0, b0;\n\t"
        "mul.hi.u32 r1, a0, b0;\n\t"
        "mad.lo.cc.u32 r1, a0, b1, r1;\n\t"
        "madc.hi.u32 r2, a0, b1, 0;\n\t"
        "mad.lo.cc.u32 r1, a1, b0, r1;\n\t"
        "madc.hi.cc.u32 r2, a1, b0, r2;\n\t"
        "madc.hi.u32 r3, a1, b1, 0;\n\t"
        "mad.lo.cc.u32 r2, a1, b1, r2;\n\t"
        "addc.u32 r3, r3, 0;\n\t"
        "mov.b64 %0, {r0, r1};\n\t"
        "mov.b64 %1, {r2, r3};\n\t}"
        : "=l"(lo), "=l"(hi)
        : "l"(a), "l"(b));
}

__device__ __forceinline__ u64 mul(u64 a, u64 b)
{
    u64 lo, hi;
    mul_wide(a, b, lo, hi);
    return reduce128(lo, hi);
}

__device__ __forceinline__ u64 canon(u64 a) { return a >= P ? a - P : a; }

__device__ __forceinline__ u64 neg(u64 a) { return sub(0ull, a); }

__host__ __device__ constexpr int mod192(int s) { return ((s % 192) + 192) % 192; }

// x * 2^-k for 0 < k < 32 and any x < 2^64: (x + m p) / 2^k with
// m = -x mod 2^k.  p = 1 (mod 2^32) makes x + m p divisible by 2^k, and the
// quotient is below 2^64 (it is below p + 2^(32-k)), so one exact division
// replaces the three folds that x * 2^(96-k) would take.
__device__ __forceinline__ u64 div2k(u64 x, u32 k)
{
    const u32 m = (0u - (u32)x) & ((1u << k) - 1u);
    u64 r;
    asm("{\n\t.reg .u32 t0, t1, c, top, r0, r1;\n\t"
        "mov.b64 {t0, t1}, %1;\n\t"
        "add.cc.u32 t0, t0, %2;\n\t"   // x + m
        "addc.cc.u32 t1, t1, 0;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "sub.cc.u32 t1, t1, %2;\n\t"   // - m 2^32
        "subc.u32 top, %2, 0;\n\t"     // + m 2^64, less the borrow
        "add.u32 top, top, c;\n\t"
        "shf.r.wrap.b32 r0, t0, t1, %3;\n\t"
        "shf.r.wrap.b32 r1, t1, top, %3;\n\t"
        "mov.b64 %0, {r0, r1};\n\t}"
        : "=l"(r)
        : "l"(x), "r"(m), "r"(k));
    return r;
}

// x * 2^S for a compile-time S (any sign; 2^192 == 1) is (-1)^shl_neg(S) *
// shl_abs<S>(x): with s = S mod 96, shifts up to 32 are one 96-bit fold, up
// to 64 two, and above 64 the division x 2^s = -x / 2^(96-s).  Butterflies
// absorb the sign by swapping their add and subtract.
__host__ __device__ constexpr bool shl_neg(int S)
{
    return (mod192(S) >= 96) != (mod192(S) % 96 > 64);
}
template <int S>
__device__ __forceinline__ u64 shl_abs(u64 x)
{
    constexpr int s = mod192(S) % 96;
    if constexpr (s == 0) {
        return x;
    } else if constexpr (s <= 32) {
        return reduce96(x << s, (u32)(x >> (64 - s)));
    } else if constexpr (s > 64) {
        return div2k(x, 96 - s);
    } else {
        return shl_abs<32>(shl_abs<s - 32>(x));  // two 96-bit folds beat one 128-bit fold
    }
}
template <int S>
__device__ __forceinline__ u64 shl(u64 x)
{
    if constexpr (shl_neg(S)) return neg(shl_abs<S>(x));
    else return shl_abs<S>(x);
}

// x * 2^s for a runtime s in [0, 192) that is uniform across the warp: one
// copy of the code serves every exponent (the pass twiddles), the branches
// never diverge.
__device__ __forceinline__ u64 shl_rt(u64 x, u32 s)
{
    bool negate = s >= 96;
    if (negate) s -= 96;
    if (s > 64) {
        x = div2k(x, 96 - s);  // x 2^s = -x / 2^(96-s)
        negate = !negate;
    } else {
        if (s > 32) {
            x = reduce96(x << 32, (u32)(x >> 32));
            s -= 32;
        }
        if (s) x = reduce96(x << s, (u32)(x >> (64 - s)));
    }
    return negate ? neg(x) : x;
}

// a*b + c*d with one reduction: the two 128-bit products are summed first;
// a carry out of bit 128 is worth 2^128 == -2^32 (mod p).
__device__ __forceinline__ u64 mul_add2(u64 a, u64 b, u64 c, u64 d)
{
    u64 lo, hi, l1, h1, l2, h2;
    u32 c2;
    mul_wide(a, b, l1, h1);
    mul_wide(c, d, l2, h2);
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
    const u64 t = shl_abs<S>(v);
    if constexpr (shl_neg(S)) {
        const u64 a = sub(u, t);
        v = add(u, t);
        u = a;
    } else {
        const u64 a = add(u, t);
        v = sub(u, t);
        u = a;
    }
}

// Gentleman-Sande butterfly: (u, v) <- (u + v, (u - v) 2^S)
template <int S>
__device__ __forceinline__ void gs_bf(u64 &u, u64 &v)
{
    const u64 a = add(u, v);
    v = shl_abs<S>(shl_neg(S) ? sub(v, u) : sub(u, v));
    u = a;
}

// p -> 2^64 modulus switch of a canonical residue a:
//   z = ((a * CST) >> 96) + bit95(a * CST),  CST = floor(2^160 / p) = 2^96 + 2^64 - 2
// (hw/common_lib/.../mod_switch_to_2powerN.sv:62-64,132-134 with
//  MOD_Q_W = 64, PRECISION_W = 96).  a * CST = a 2^96 + (a 2^64 - 2a), and the
// 64-bit word above 2^64 of a 2^64 - 2a is hx = a - [a > 0] - [a > 2^63], so
// z = a + round(hx / 2^32) mod 2^64 -- no multiply.
__device__ __forceinline__ u64 modsw_p_to_q(u64 a)
{
    const u64 hx = a - (a != 0 ? 1ull : 0ull) - (a > 0x8000000000000000ull ? 1ull : 0ull);
    return a + ((hx + 0x80000000ull) >> 32);
}

// Balanced decomposition, base 2^23, one level, of a 64-bit torus value,
// embedded in Z_p (decomp_balseq_core.sv:135-150; the rounding and tie rule of
// sw/decomposer/balanced_decomp_unfix_sign_round_bit.py:42-101 with bw=23, L=1).
// tie_rtl = 1 selects the RTL's rule at a tie (t = B/2: negative when the
// rounding bit is set), tie_rtl = 0 the reference generator's (TFHE-rs: the
// digit above is 0, so the digit stays +B/2).
template <int BW>
__device__ __forceinline__ u64 decomp_to_p(u64 v, u64 tie_rtl = 1)
{
    constexpr u64 B = 1ull << BW, HALF = B >> 1;
    u64 rb = (v >> (63 - BW)) & 1ull;
    u64 c = (v >> (64 - BW)) + rb;      // 0 .. 2^BW
    u64 t = c & (B - 1);
    // with one level the digit above is last_sign * (B-1), last_sign = rb at a tie
    bool negd = (t > HALF) || (t == HALF && (rb & tie_rtl));
    // negative digit t - 2^BW embeds as p - (2^BW - t)
    return negd ? (P - (B - t)) : t;
}
__device__ __forceinline__ u64 decomp23_to_p(u64 v) { return decomp_to_p<23>(v); }

}  // namespace gl
