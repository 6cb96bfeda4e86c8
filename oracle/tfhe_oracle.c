/*
 * tfhe_oracle.c -- CPU restatement of the HPU KS+PBS datapath.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine in
 * luthe_b200/csrc: the parity tests, the smoke check and the CPU-baseline leg
 * of bench.py call it; the engine never links it and never falls back to it.
 *
 * Every stage restates the reference's algorithm (paths are relative to the
 * reference project root, xiurui-pan/LUTHE):
 *   - balanced decomposition, "unfixed sign + rounding bit":
 *       sw/decomposer/balanced_decomp_unfix_sign_round_bit.py:42-101 (hw_decompose),
 *       hw/module/decomposer/module/decomp_parallel/rtl/decomp_parallel.sv:73-75,107,142-150
 *   - key switch (body rounding 2^64 -> 2^21, MAC mod 2^21, 2^21 -> 2N switch):
 *       hw/module/pep_key_switch/module/pep_ks_blwe_ram/rtl/pep_ks_blram_format.sv:158-172,240-243
 *       hw/module/pep_key_switch/module/pep_ks_mult/rtl/pep_ks_mult_node.sv:95-104,150-153
 *       hw/module/pep_key_switch/module/pep_ks_out_process/rtl/pep_ks_out_process.sv:276-280,336-341
 *   - monomial multiply X^e * P mod X^N+1:
 *       sw/monomial_mult/monomial_mult.py:156-176 (monomial_mult_definition)
 *   - Goldilocks reduction 2^64 = 2^32-1, 2^96 = -1:
 *       sw/solinas/solinas.py:218-319 (compute_modulo)
 *   - negacyclic NTT / INTT over p = 2^64-2^32+1 (the product it computes):
 *       sw/ntt/ntt_gf64.sage:273-314,319-362,515-578
 *   - BSK multiply-accumulate in the NTT domain:
 *       hw/module/number_theoretic_transform/module/ntt_core_gf64/module/
 *         ntt_core_gf64_post_process/rtl/ntt_core_gf64_pp_core.sv (header)
 *   - modulus switch p -> 2^64, CST = floor(2^160/p), round on bit 95:
 *       hw/common_lib/mod_arithmetic/module/mod_switch/module/mod_switch_to_2powerN/
 *         rtl/mod_switch_to_2powerN.sv:9-20,62-64,132-134
 *   - blind rotation loop (rotate-sub, decompose, ext. product, accumulate):
 *       hw/module/pep_mono_mult_acc/.../feed/rtl/pep_mmacc_splitc_feed_rot.sv:305-323,
 *       feed_final.sv:260,324, acc/rtl/pep_mmacc_splitc_acc_core.sv:8-12
 *   - sample extract with the final rotation by the KS body:
 *       hw/module/pep_mono_mult_acc/.../sxt/rtl/pep_mmacc_splitc_sxt_core.sv:8-14
 *
 * The NTT here is a plain iterative radix-2 negacyclic transform, written
 * independently of the GPU's 32x64 decomposition: the two agree because both
 * compute the exact negacyclic product mod p.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;
#define GL_P 0xFFFFFFFF00000001ull
#define GL_EPS 0xFFFFFFFFull /* 2^64 mod p */

/* primitive 4096-th root of unity with psi^64 = 8 */
#define GL_PSI_4096 0x984ec5194d005735ull

/* ---------------------------------------------------------------- Goldilocks */

/* The carry and borrow corrections below are written as masks rather than
 * branches: the conditions are data-dependent coin flips, and branch-free code
 * runs several times faster on the host.  The arithmetic is unchanged. */
static inline uint64_t mask_if(int c) { return (uint64_t)0 - (uint64_t)(c != 0); }

uint64_t or_gl_reduce128(uint64_t lo, uint64_t hi)
{
    /* x = lo + 2^64 (h0 + 2^32 h1) = lo - h1 + h0 (2^32 - 1)  (mod p) */
    uint64_t h0 = hi & 0xFFFFFFFFull, h1 = hi >> 32;
    uint64_t t = lo - h1;
    t -= mask_if(lo < h1) & GL_EPS;       /* borrow: -2^64 = -(2^32-1) */
    uint64_t u = (h0 << 32) - h0;         /* h0 (2^32-1) < 2^64 */
    uint64_t r = t + u;
    r += mask_if(r < t) & GL_EPS;         /* carry: +2^64 = +(2^32-1) */
    r -= mask_if(r >= GL_P) & GL_P;
    return r;
}

static inline uint64_t gl_mul(uint64_t a, uint64_t b)
{
    u128 x = (u128)a * b;
    return or_gl_reduce128((uint64_t)x, (uint64_t)(x >> 64));
}
/* a, b < p */
static inline uint64_t gl_add(uint64_t a, uint64_t b)
{
    uint64_t s = a + b;
    s += mask_if(s < a) & GL_EPS;
    s -= mask_if(s >= GL_P) & GL_P;
    return s;
}
static inline uint64_t gl_sub(uint64_t a, uint64_t b)
{
    uint64_t d = a - b;
    d -= mask_if(a < b) & GL_EPS;
    d -= mask_if(d >= GL_P) & GL_P;
    return d;
}
static uint64_t gl_pow(uint64_t a, uint64_t e)
{
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = gl_mul(r, a);
        a = gl_mul(a, a);
        e >>= 1;
    }
    return r;
}
uint64_t or_gl_mul(uint64_t a, uint64_t b) { return gl_mul(a % GL_P, b % GL_P); }
uint64_t or_gl_inv(uint64_t a) { return gl_pow(a % GL_P, GL_P - 2); }

/* ------------------------------------------------------------- decomposition */

/*
 * Balanced decomposition of a 64-bit value into `level` signed digits of
 * `base_log` bits, LSB digit first, following hw_decompose
 * (balanced_decomp_unfix_sign_round_bit.py:42-101):
 *   closest_rep = (v >> (64 - bw*L)) + round_bit
 *   last_sign   = msb(closest_rep) && (lower bits != 0 || round_bit)
 *   digit i carries when it is > B/2, or == B/2 and the next raw digit's
 *   half bit is set (the digit above the top one is last_sign * (B-1)).
 * This is also the RTL's rule (decomp_parallel.sv:73-75,107,142-150).
 * gtv_top_tie != 0 selects the rule of the reference's test-vector generator
 * (gtv, built on TFHE-rs) instead: the digit above the top one is taken as 0,
 * so a top digit equal to B/2 stays positive.  Both give the same value mod
 * 2^(bw*L); they differ only in that top digit.
 */
void or_decompose2(uint64_t v, int bw, int L, int gtv_top_tie, int32_t *digits)
{
    int tot = bw * L;
    uint64_t mask = (1ull << bw) - 1, half = 1ull << (bw - 1);
    uint64_t rb = (v >> (64 - tot - 1)) & 1;
    uint64_t c = (v >> (64 - tot)) + rb;             /* may reach 2^tot */
    uint64_t msb = 1ull << (tot - 1);
    int last_sign = (c & msb) && ((c & (msb - 1)) || rb);
    uint64_t raw[65];
    for (int i = 0; i < L; i++) raw[i] = (c >> (bw * i)) & mask;
    raw[L] = (last_sign && !gtv_top_tie) ? mask : 0;
    uint64_t carry = 0;
    for (int i = 0; i < L; i++) {
        uint64_t t = raw[i] + carry;               /* 0 .. 2^bw */
        int neg = (t >> bw) & 1;
        if (!neg && (t & half) && ((t & (half - 1)) || (raw[i + 1] & half))) neg = 1;
        if (neg) {
            carry = 1;
            digits[i] = (int32_t)((int64_t)t - (int64_t)(1ull << bw));
        } else {
            carry = 0;
            digits[i] = (int32_t)t;
        }
    }
}
void or_decompose(uint64_t v, int bw, int L, int32_t *digits) { or_decompose2(v, bw, L, 0, digits); }

/* ----------------------------------------------------------- modulus switch */

/* p -> 2^64: z = ((a*CST) >> 96) + bit95(a*CST), CST = floor(2^160/p)
 * = 2^96 + 2^64 - 2 (mod_switch_to_2powerN.sv:62-64,132-134). */
uint64_t or_modsw_p_to_q(uint64_t a)
{
    const uint64_t cst_lo = 0xFFFFFFFFFFFFFFFEull, cst_hi = 0x100000000ull;
    u128 p0 = (u128)a * cst_lo;
    u128 u = (p0 >> 64) + (u128)a * cst_hi;   /* (a*CST) >> 64, < 2^98 */
    return (uint64_t)(u >> 32) + (uint64_t)((u >> 31) & 1);
}

/* 2^64 -> p rounding of a standard-domain key coefficient (the inverse
 * direction of the switch above): round(x * p / 2^64). */
uint64_t or_modsw_q_to_p(uint64_t x)
{
    u128 t = (u128)x * GL_P + ((u128)1 << 63);
    return (uint64_t)(t >> 64);
}

/* --------------------------------------------------------- monomial multiply */

/* out = X^e * in mod (X^N + 1, 2^64), e in [0, 2N) (monomial_mult.py:156-176) */
void or_monomial(const uint64_t *in, uint32_t e, uint64_t *out, uint32_t N)
{
    e %= 2 * N;
    for (uint32_t j = 0; j < N; j++) {
        uint32_t src = (j + 2 * N - e) % (2 * N);  /* X^e moves coef src to j */
        uint64_t v = in[src % N];
        if (src >= N) v = (uint64_t)0 - v;
        out[j] = v;
    }
}

/* ----------------------------------------------------------------------- NTT */

typedef struct {
    uint32_t N, logN;
    uint64_t *tw;    /* psi^bitrev(i), i in [0,N) */
    uint64_t *itw;   /* psi^-bitrev(i) */
    uint64_t ninv;
} or_ntt_t;

static uint32_t bitrev(uint32_t x, uint32_t bits)
{
    uint32_t r = 0;
    for (uint32_t i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
    return r;
}

static void ntt_init(or_ntt_t *t, uint32_t N)
{
    t->N = N;
    t->logN = 0;
    while ((1u << t->logN) < N) t->logN++;
    uint64_t psi = gl_pow(GL_PSI_4096, 4096 / (2 * N));
    uint64_t ipsi = gl_pow(psi, GL_P - 2);
    t->tw = malloc(N * 8);
    t->itw = malloc(N * 8);
    for (uint32_t i = 0; i < N; i++) {
        t->tw[i] = gl_pow(psi, bitrev(i, t->logN));
        t->itw[i] = gl_pow(ipsi, bitrev(i, t->logN));
    }
    t->ninv = gl_pow(N, GL_P - 2);
}
static void ntt_free(or_ntt_t *t)
{
    free(t->tw);
    free(t->itw);
}

/* forward negacyclic NTT, natural order in, bit-reversed order out:
 * out[bitrev(k)] = sum_j a_j psi^{j(2k+1)} */
static void ntt_fwd(const or_ntt_t *t, uint64_t *a)
{
    uint32_t N = t->N;
    for (uint32_t m = 1, len = N / 2; m < N; m <<= 1, len >>= 1) {
        for (uint32_t i = 0; i < m; i++) {
            uint64_t w = t->tw[m + i];
            uint64_t *x = a + 2 * i * len;
            for (uint32_t j = 0; j < len; j++) {
                uint64_t u = x[j], v = gl_mul(x[j + len], w);
                x[j] = gl_add(u, v);
                x[j + len] = gl_sub(u, v);
            }
        }
    }
}
/* inverse of ntt_fwd including the 1/N factor */
static void ntt_inv(const or_ntt_t *t, uint64_t *a)
{
    uint32_t N = t->N;
    for (uint32_t m = N / 2, len = 1; m >= 1; m >>= 1, len <<= 1) {
        for (uint32_t i = 0; i < m; i++) {
            uint64_t w = t->itw[m + i];
            uint64_t *x = a + 2 * i * len;
            for (uint32_t j = 0; j < len; j++) {
                uint64_t u = x[j], v = x[j + len];
                x[j] = gl_add(u, v);
                x[j + len] = gl_mul(gl_sub(u, v), w);
            }
        }
    }
    for (uint32_t j = 0; j < N; j++) a[j] = gl_mul(a[j], t->ninv);
}

/* Evaluations A(psi^{2k+1}) in natural k order (N <= 2048). */
void or_ntt_eval(const uint64_t *in, uint64_t *out, uint32_t N)
{
    or_ntt_t t;
    ntt_init(&t, N);
    uint64_t *a = malloc(N * 8);
    for (uint32_t j = 0; j < N; j++) a[j] = in[j] % GL_P;
    ntt_fwd(&t, a);
    for (uint32_t k = 0; k < N; k++) out[k] = a[bitrev(k, t.logN)];
    free(a);
    ntt_free(&t);
}

/* Coefficients from evaluations: in[k] = A(psi^{2k+1}) in natural k order
 * (the inverse of or_ntt_eval, including 1/N). */
void or_ntt_inv_natural(const uint64_t *in, uint64_t *out, uint32_t N)
{
    or_ntt_t t;
    ntt_init(&t, N);
    for (uint32_t k = 0; k < N; k++) out[bitrev(k, t.logN)] = in[k] % GL_P;
    ntt_inv(&t, out);
    ntt_free(&t);
}

/* Negacyclic product mod (X^N+1, p) of `count` pairs, via NTT. */
void or_negacyclic_mul(const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t N, uint32_t count)
{
    or_ntt_t t;
    ntt_init(&t, N);
#pragma omp parallel
    {
        uint64_t *x = malloc(N * 8), *y = malloc(N * 8);
#pragma omp for schedule(static)
        for (long c = 0; c < (long)count; c++) {
            for (uint32_t j = 0; j < N; j++) {
                x[j] = a[c * N + j] % GL_P;
                y[j] = b[c * N + j] % GL_P;
            }
            ntt_fwd(&t, x);
            ntt_fwd(&t, y);
            for (uint32_t j = 0; j < N; j++) x[j] = gl_mul(x[j], y[j]);
            ntt_inv(&t, x);
            memcpy(out + c * N, x, N * 8);
        }
        free(x);
        free(y);
    }
    ntt_free(&t);
}

/* Schoolbook negacyclic product mod p (the convolution check of
 * ntt_gf64.sage:515-578, stated without an NTT). */
void or_negacyclic_mul_schoolbook(const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t N)
{
    for (uint32_t k = 0; k < N; k++) out[k] = 0;
    for (uint32_t i = 0; i < N; i++)
        for (uint32_t j = 0; j < N; j++) {
            uint64_t p = gl_mul(a[i] % GL_P, b[j] % GL_P);
            uint32_t k = i + j;
            if (k < N) out[k] = gl_add(out[k], p);
            else out[k - N] = gl_sub(out[k - N], p);
        }
}

/* ---------------------------------------------------------------- key switch */

/*
 * LWE key switch of one BLWE (mask kN u64 + body) to n+1 coefficients mod 2^ks_w.
 * ksk layout [x][y][z] (x in [0,n], body column x=n last; y in [0,kN); z level,
 * z=0 the LSB digit), the layout of the reference's ksk_hwo files.
 * out21[x] = [x==n] b21 - sum_{y,z} d_{y,z} ksk[x][y][z]  (mod 2^ks_w)
 * out2N[x] = (out21[x] >> (ks_w - logN - 1)) + round bit, mod 2N.
 */
void or_keyswitch2(const uint64_t *blwe, const uint32_t *ksk, uint32_t n, uint32_t kN,
                   uint32_t ks_bl, uint32_t ks_lc, uint32_t ks_w, uint32_t N, int gtv_top_tie,
                   uint32_t *out21, uint32_t *out2N)
{
    uint32_t M = (1u << ks_w) - 1;
    int32_t *d = malloc(sizeof(int32_t) * kN * ks_lc);
    /* the KS decomposer sees the top bl*L bits of the 64-bit coefficient
     * (pep_ks_blram_format.sv:158-172) */
    for (uint32_t y = 0; y < kN; y++) or_decompose2(blwe[y], ks_bl, ks_lc, gtv_top_tie, d + y * ks_lc);
    uint64_t b = blwe[kN];
    uint32_t b21 = (uint32_t)(((b >> (64 - ks_w)) + ((b >> (63 - ks_w)) & 1)) & M);
    uint32_t logN = 0;
    while ((1u << logN) < N) logN++;
    uint32_t sh = ks_w - (logN + 1);
    for (uint32_t x = 0; x <= n; x++) {
        uint32_t acc = (x == n) ? b21 : 0;
        const uint32_t *row = ksk + (size_t)x * kN * ks_lc;
        for (uint32_t i = 0; i < kN * ks_lc; i++) acc -= (uint32_t)d[i] * row[i];
        acc &= M;
        out21[x] = acc;
        out2N[x] = ((acc >> sh) + ((acc >> (sh - 1)) & 1)) & (2 * N - 1);
    }
    free(d);
}
void or_keyswitch(const uint64_t *blwe, const uint32_t *ksk, uint32_t n, uint32_t kN, uint32_t ks_bl,
                  uint32_t ks_lc, uint32_t ks_w, uint32_t N, uint32_t *out21, uint32_t *out2N)
{
    or_keyswitch2(blwe, ksk, n, kN, ks_bl, ks_lc, ks_w, N, 0, out21, out2N);
}

/* ------------------------------------------------------------------- the PBS */

typedef struct {
    uint32_t n, N;
    uint64_t *bsk_hat; /* [n][row][col][N] oracle-NTT domain (bitrev order) */
    or_ntt_t ntt;
} or_bsk_t;

/* Prepare the BSK: input in the standard domain over Z_p, layout
 * [i][row][col][N] (row = decomposed GLWE component, col = output component). */
void *or_bsk_prepare(const uint64_t *bsk_std_p, uint32_t n, uint32_t N)
{
    or_bsk_t *k = calloc(1, sizeof(*k));
    k->n = n;
    k->N = N;
    ntt_init(&k->ntt, N);
    k->bsk_hat = malloc((size_t)n * 4 * N * 8);
    memcpy(k->bsk_hat, bsk_std_p, (size_t)n * 4 * N * 8);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n * 4; i++) ntt_fwd(&k->ntt, k->bsk_hat + (size_t)i * N);
    return k;
}
/* Prepare the BSK from the evaluation domain: bsk_eval[i][row][col][k] =
 * BSK_i[row][col](psi^{2k+1}), natural k order (values < p). */
void *or_bsk_prepare_eval(const uint64_t *bsk_eval, uint32_t n, uint32_t N)
{
    or_bsk_t *k = calloc(1, sizeof(*k));
    k->n = n;
    k->N = N;
    ntt_init(&k->ntt, N);
    k->bsk_hat = malloc((size_t)n * 4 * N * 8);
    for (size_t q = 0; q < (size_t)n * 4; q++)
        for (uint32_t j = 0; j < N; j++) k->bsk_hat[q * N + bitrev(j, k->ntt.logN)] = bsk_eval[q * N + j] % GL_P;
    return k;
}
void or_bsk_free(void *h)
{
    or_bsk_t *k = h;
    ntt_free(&k->ntt);
    free(k->bsk_hat);
    free(k);
}

/* Tie rule of the decompositions of the full path (blind rotation, and the
 * key switch of or_ks_pbs_ml): 0 the RTL's, 1 the reference generator's; set
 * for the whole oracle.  See or_decompose2. */
static int or_tie_gen = 0;
void or_set_tie_rule(int gen) { or_tie_gen = gen; }

/* One blind rotation + sample extract.  lwe2N: n masks then the body, in [0,2N).
 * lut: GLWE (mask poly, body poly).  out: BLWE, N mask coefs then body. */
static void br_one(const or_bsk_t *k, const uint32_t *lwe2N, const uint64_t *lut,
                   uint32_t pbs_bl, uint64_t *out, uint64_t *work, uint32_t mlk)
{
    uint32_t N = k->N, n = k->n;
    uint64_t *acc = work, *rot = work + 2 * N, *dh = work + 4 * N, *rh = work + 6 * N;
    memcpy(acc, lut, 2 * N * 8);
    int32_t dig;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t a = lwe2N[i];
        /* feed: diff = X^a ACC - ACC */
        for (int t = 0; t < 2; t++) {
            or_monomial(acc + t * N, a, rot + t * N, N);
            for (uint32_t j = 0; j < N; j++) {
                uint64_t dv = rot[t * N + j] - acc[t * N + j];
                or_decompose2(dv, pbs_bl, 1, or_tie_gen, &dig);
                dh[t * N + j] = dig >= 0 ? (uint64_t)dig : GL_P - (uint64_t)(-(int64_t)dig);
            }
            ntt_fwd(&k->ntt, dh + t * N);
        }
        const uint64_t *bk = k->bsk_hat + (size_t)i * 4 * N;
        for (int col = 0; col < 2; col++) {
            for (uint32_t j = 0; j < N; j++) {
                uint64_t s = gl_mul(dh[j], bk[(0 * 2 + col) * N + j]);
                s = gl_add(s, gl_mul(dh[N + j], bk[(1 * 2 + col) * N + j]));
                rh[col * N + j] = s;
            }
            ntt_inv(&k->ntt, rh + col * N);
            for (uint32_t j = 0; j < N; j++) acc[col * N + j] += or_modsw_p_to_q(rh[col * N + j]);
        }
    }
    /* sample extract of coefficient 0 of X^{-b} ACC; many-LUT output m takes
     * coefficient m N/mlk instead (docs/dop.md:113-121) */
    for (uint32_t m = 0; m < mlk; m++) {
        uint32_t b = (lwe2N[n] + m * (N / mlk)) % (2 * N);
        uint64_t *o = out + (size_t)m * (N + 1);
        or_monomial(acc, 2 * N - b, rot, N);
        or_monomial(acc + N, 2 * N - b, rot + N, N);
        o[0] = rot[0];
        for (uint32_t j = 1; j < N; j++) o[j] = (uint64_t)0 - rot[N - j];
        o[N] = rot[N];
    }
}

/* Blind rotation of `B` already key-switched ciphertexts. */
void or_blind_rotate_ml(void *bsk, const uint32_t *lwe2N, const uint64_t *luts, const uint32_t *lut_id,
                        uint64_t *out, uint32_t B, uint32_t pbs_bl, uint32_t mlk)
{
    or_bsk_t *k = bsk;
    uint32_t N = k->N, n = k->n;
#pragma omp parallel
    {
        uint64_t *work = malloc(8 * N * 8);
#pragma omp for schedule(dynamic, 1)
        for (long c = 0; c < (long)B; c++)
            br_one(k, lwe2N + (size_t)c * (n + 1), luts + (size_t)lut_id[c] * 2 * N, pbs_bl,
                   out + (size_t)c * mlk * (N + 1), work, mlk);
        free(work);
    }
}
void or_blind_rotate(void *bsk, const uint32_t *lwe2N, const uint64_t *luts, const uint32_t *lut_id,
                     uint64_t *out, uint32_t B, uint32_t pbs_bl)
{
    or_blind_rotate_ml(bsk, lwe2N, luts, lut_id, out, B, pbs_bl, 1);
}

/* Full KS+PBS of B ciphertexts (the PBS DOp: docs/dop.md:101-111). */
void or_ks_pbs_ml(void *bsk, const uint32_t *ksk, const uint64_t *blwe_in, const uint64_t *luts,
                  const uint32_t *lut_id, uint64_t *blwe_out, uint32_t B, uint32_t ks_bl, uint32_t ks_lc,
                  uint32_t ks_w, uint32_t pbs_bl, uint32_t mlk)
{
    or_bsk_t *k = bsk;
    uint32_t N = k->N, n = k->n;
    uint32_t *l2n = malloc(sizeof(uint32_t) * (size_t)B * (n + 1));
#pragma omp parallel
    {
        uint32_t *o21 = malloc(4 * (n + 1));
#pragma omp for schedule(static)
        for (long c = 0; c < (long)B; c++)
            or_keyswitch2(blwe_in + (size_t)c * (N + 1), ksk, n, N, ks_bl, ks_lc, ks_w, N, or_tie_gen, o21,
                          l2n + (size_t)c * (n + 1));
        free(o21);
    }
    or_blind_rotate_ml(bsk, l2n, luts, lut_id, blwe_out, B, pbs_bl, mlk);
    free(l2n);
}
void or_ks_pbs(void *bsk, const uint32_t *ksk, const uint64_t *blwe_in, const uint64_t *luts,
               const uint32_t *lut_id, uint64_t *blwe_out, uint32_t B, uint32_t ks_bl, uint32_t ks_lc,
               uint32_t ks_w, uint32_t pbs_bl)
{
    or_ks_pbs_ml(bsk, ksk, blwe_in, luts, lut_id, blwe_out, B, ks_bl, ks_lc, ks_w, pbs_bl, 1);
}

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void or_set_threads(int t)
{
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

/* ------------------------------------------------- keys, ciphertexts, LUTs */

/*
 * Seeded key material for the CPU reference timing and the CPU tests, so that
 * they need nothing from the engine library.  Every random word is a pure
 * function of (seed, stream, index) through the SplitMix64 finaliser:
 *   rnd(seed, stream, i) = mix(mix(seed ^ mix(stream * 0x100000001B3)) + i)
 * with the stream numbers below.  With the same seed the results equal
 * luthe_keygen / luthe_encrypt (tests/test_oracle_keygen.py checks this).
 * Keys are binary; the KSK level z of mask coefficient y encrypts
 * S_y 2^(W - bl (L - z)) under the LWE key mod 2^W; the BSK is a GGSW of
 * each LWE key bit over Z_2^64 (gadget 2^(64 - pbs_bl), one level), each
 * coefficient rounded to Z_p by or_modsw_q_to_p.
 */
static uint64_t kg_mix(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static uint64_t kg_rnd(uint64_t seed, uint64_t stream, uint64_t idx)
{
    return kg_mix(kg_mix(seed ^ kg_mix(stream * 0x100000001B3ull)) + idx);
}
/* Box-Muller on two uniforms, rounded to the nearest integer */
static int64_t kg_gauss(uint64_t seed, uint64_t stream, uint64_t idx, double sigma)
{
    if (sigma <= 0) return 0;
    double u1 = ((kg_rnd(seed, stream, 2 * idx) >> 11) + 1) * (1.0 / 9007199254740993.0);
    double u2 = (kg_rnd(seed, stream, 2 * idx + 1) >> 11) * (1.0 / 9007199254740992.0);
    double g = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    return (int64_t)llround(g * sigma);
}
enum { KG_LWE_KEY = 1, KG_GLWE_KEY, KG_KSK_MASK, KG_KSK_NOISE, KG_BSK_MASK, KG_BSK_NOISE, KG_ENC_MASK, KG_ENC_NOISE };
#define KG_LWE_SIGMA 5.3943e-6   /* 2^-17.5 of the modulus */
#define KG_GLWE_SIGMA 4.4409e-16 /* 2^-51 of the modulus */

void or_keygen(uint32_t n, uint32_t N, uint32_t ks_bl, uint32_t ks_lc, uint32_t ks_w, uint32_t pbs_bl,
               uint64_t seed, uint32_t *lwe_key, uint32_t *glwe_key, uint32_t *ksk, uint64_t *bsk_std_p)
{
    for (uint32_t i = 0; i < n; i++) lwe_key[i] = kg_rnd(seed, KG_LWE_KEY, i) & 1;
    for (uint32_t j = 0; j < N; j++) glwe_key[j] = kg_rnd(seed, KG_GLWE_KEY, j) & 1;
    const uint32_t M = ks_w == 32 ? 0xFFFFFFFFu : ((1u << ks_w) - 1);
    const double ks_sigma = KG_LWE_SIGMA * ldexp(1.0, (int)ks_w);
#pragma omp parallel for schedule(static)
    for (long yz = 0; yz < (long)N * ks_lc; yz++) {
        const uint32_t y = (uint32_t)(yz / ks_lc), z = (uint32_t)(yz % ks_lc);
        uint32_t body = 0;
        for (uint32_t x = 0; x < n; x++) {
            uint32_t a = (uint32_t)kg_rnd(seed, KG_KSK_MASK, (uint64_t)yz * n + x) & M;
            ksk[((size_t)x * N + y) * ks_lc + z] = a;
            body += a * lwe_key[x];
        }
        body += (uint32_t)kg_gauss(seed, KG_KSK_NOISE, yz, ks_sigma);
        body += glwe_key[y] << (ks_w - ks_bl * (ks_lc - z));
        ksk[((size_t)n * N + y) * ks_lc + z] = body & M;
    }
    const double glwe_sigma = KG_GLWE_SIGMA * 18446744073709551616.0;
    const uint64_t g = 1ull << (64 - pbs_bl);
#pragma omp parallel
    {
        uint64_t *A = malloc(N * 8), *B = malloc(N * 8);
#pragma omp for schedule(dynamic, 4)
        for (long ir = 0; ir < (long)n * 2; ir++) {
            const uint32_t i = (uint32_t)(ir / 2), row = (uint32_t)(ir % 2);
            for (uint32_t c = 0; c < N; c++) {
                A[c] = kg_rnd(seed, KG_BSK_MASK, (uint64_t)ir * N + c);
                B[c] = (uint64_t)kg_gauss(seed, KG_BSK_NOISE, (uint64_t)ir * N + c, glwe_sigma);
            }
            for (uint32_t j = 0; j < N; j++) /* B += A * S mod (X^N + 1, 2^64) */
                if (glwe_key[j])
                    for (uint32_t c = 0; c < N; c++) {
                        uint32_t k = c + j;
                        if (k < N) B[k] += A[c];
                        else B[k - N] -= A[c];
                    }
            if (lwe_key[i]) {
                if (row == 0) A[0] += g;
                else B[0] += g;
            }
            uint64_t *dst = bsk_std_p + ((size_t)i * 2 + row) * 2 * N;
            for (uint32_t c = 0; c < N; c++) {
                dst[c] = or_modsw_q_to_p(A[c]);
                dst[N + c] = or_modsw_q_to_p(B[c]);
            }
        }
        free(A);
        free(B);
    }
}

/* BLWE encryptions (mask N coefficients, body) of msgs[c] << (64 - bits),
 * bits = 1 + msg + carry, under the GLWE key seen as an LWE key. */
void or_encrypt(uint32_t N, uint32_t bits, const uint32_t *S, const uint32_t *msgs, uint64_t count, uint64_t seed,
                uint64_t *blwe)
{
    const double sigma = KG_GLWE_SIGMA * 18446744073709551616.0;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < (long)count; c++) {
        uint64_t *ct = blwe + (size_t)c * (N + 1), b = 0;
        for (uint32_t j = 0; j < N; j++) {
            ct[j] = kg_rnd(seed, KG_ENC_MASK, (uint64_t)c * N + j);
            if (S[j]) b += ct[j];
        }
        b += (uint64_t)kg_gauss(seed, KG_ENC_NOISE, (uint64_t)c, sigma);
        ct[N] = b + ((uint64_t)msgs[c] << (64 - bits));
    }
}

void or_decrypt(uint32_t N, uint32_t bits, const uint32_t *S, const uint64_t *blwe, uint64_t count, uint32_t *msgs)
{
    for (size_t c = 0; c < count; c++) {
        const uint64_t *ct = blwe + c * (N + 1);
        uint64_t ph = ct[N];
        for (uint32_t j = 0; j < N; j++)
            if (S[j]) ph -= ct[j];
        msgs[c] = (uint32_t)(((ph + (1ull << (63 - bits))) >> (64 - bits)) & ((1ull << bits) - 1));
    }
}

/* Trivial LUT GLWE of table[0 .. 2^(bits-1)): box m of N / 2^(bits-1)
 * coefficients holds f(m) << (64 - bits), rotated by half a box, the entries
 * past X^N negated (negacyclic); the layout of the reference's LUT vectors. */
void or_lut_build(uint32_t N, uint32_t bits, const uint32_t *table, uint64_t *glwe)
{
    const uint32_t nm = 1u << (bits - 1), box = N / nm, half = box / 2;
    memset(glwe, 0, (size_t)N * 8);
    for (uint32_t j = 0; j < N; j++)
        glwe[N + j] = j < N - half ? (uint64_t)table[((j + half) / box) % nm] << (64 - bits)
                                   : (uint64_t)0 - ((uint64_t)table[0] << (64 - bits));
}
