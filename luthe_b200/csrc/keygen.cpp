// Host-side key generation, encryption, decryption and LUT construction.
//
// Every random value is a pure function of (seed, stream, index) through the
// SplitMix64 finaliser, so results do not depend on thread scheduling.  The
// GGSW of the BSK is generated over Z_{2^64} and each coefficient is then
// rounded to Z_p (x -> round(x p / 2^64)): the engine's blind rotation
// multiplies digits by the BSK mod p and switches the result back with
// round(r 2^64 / p) (mod_switch_to_2powerN.sv), so a BSK scaled by p/2^64
// makes the two switches cancel.
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <vector>
#include "../../include/luthe.h"

namespace {

const uint64_t P = 0xFFFFFFFF00000001ull;

inline uint64_t mix(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline uint64_t rnd(uint64_t seed, uint64_t stream, uint64_t idx)
{
    return mix(mix(seed ^ mix(stream * 0x100000001B3ull)) + idx);
}
// Gaussian of standard deviation sigma (Box-Muller on two uniforms), rounded
inline int64_t gauss(uint64_t seed, uint64_t stream, uint64_t idx, double sigma)
{
    if (sigma <= 0) return 0;
    double u1 = ((rnd(seed, stream, 2 * idx) >> 11) + 1) * (1.0 / 9007199254740993.0);
    double u2 = (rnd(seed, stream, 2 * idx + 1) >> 11) * (1.0 / 9007199254740992.0);
    double g = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    return (int64_t)llround(g * sigma);
}
inline uint64_t q_to_p(uint64_t x)
{
    unsigned __int128 t = (unsigned __int128)x * P + ((unsigned __int128)1 << 63);
    return (uint64_t)(t >> 64);
}

enum : uint64_t { S_LWE_KEY = 1, S_GLWE_KEY, S_KSK_MASK, S_KSK_NOISE, S_BSK_MASK, S_BSK_NOISE, S_ENC_MASK, S_ENC_NOISE };

// LWE sigma 2^-17.5 and GLWE sigma 2^-51 relative to the modulus
const double LWE_SIGMA_REL = 5.3943e-6;   // 2^-17.5
const double GLWE_SIGMA_REL = 4.4409e-16; // 2^-51

int check(const luthe_params *p)
{
    if (!p || p->glwe_dim != 1 || p->poly_size == 0 || (p->poly_size & (p->poly_size - 1)) || p->lwe_dim == 0 ||
        p->ks_width > 32 || p->ks_base_log * p->ks_level > p->ks_width)
        return LUTHE_E_PARAM;
    return LUTHE_OK;
}

}  // namespace

extern "C" int luthe_keygen(const luthe_params *p, uint64_t seed, uint32_t *lwe_key, uint32_t *glwe_key,
                            uint32_t *ksk, uint64_t *bsk)
{
    if (check(p) || !lwe_key || !glwe_key || !ksk || !bsk) return LUTHE_E_PARAM;
    const uint32_t n = p->lwe_dim, N = p->poly_size, L = p->ks_level, bl = p->ks_base_log, W = p->ks_width;
    for (uint32_t i = 0; i < n; i++) lwe_key[i] = rnd(seed, S_LWE_KEY, i) & 1;
    for (uint32_t j = 0; j < N; j++) glwe_key[j] = rnd(seed, S_GLWE_KEY, j) & 1;

    // KSK[x][y][z]: LWE_s( S_y * 2^(W - bl*(L-z)) ) mod 2^W: level z = L-1 is the
    // most significant digit, weight 2^(W-bl) (pep_ks_mult_node.sv operands)
    const uint32_t M = W == 32 ? 0xFFFFFFFFu : ((1u << W) - 1);
    const double ks_sigma = LWE_SIGMA_REL * ldexp(1.0, (int)W);
#pragma omp parallel for schedule(static)
    for (long yz = 0; yz < (long)N * L; yz++) {
        const uint32_t y = (uint32_t)(yz / L), z = (uint32_t)(yz % L);
        uint32_t body = 0;
        for (uint32_t x = 0; x < n; x++) {
            uint32_t a = (uint32_t)rnd(seed, S_KSK_MASK, (uint64_t)yz * n + x) & M;
            ksk[((size_t)x * N + y) * L + z] = a;
            body += a * lwe_key[x];
        }
        body += (uint32_t)gauss(seed, S_KSK_NOISE, yz, ks_sigma);
        body += glwe_key[y] << (W - bl * (L - z));
        ksk[((size_t)n * N + y) * L + z] = body & M;
    }

    // BSK[i][row][col][c]: GGSW_S(s_i) over Z_{2^64}, gadget 2^(64 - 23) (l = 1),
    // then each coefficient rounded to Z_p.
    const double glwe_sigma = GLWE_SIGMA_REL * 18446744073709551616.0;
    const uint64_t g = 1ull << (64 - p->pbs_base_log * p->pbs_level);
    std::vector<uint32_t> ones;
    for (uint32_t j = 0; j < N; j++)
        if (glwe_key[j]) ones.push_back(j);
#pragma omp parallel
    {
        std::vector<uint64_t> A(N), Bv(N);
#pragma omp for schedule(dynamic, 4)
        for (long ir = 0; ir < (long)n * 2; ir++) {
            const uint32_t i = (uint32_t)(ir / 2), row = (uint32_t)(ir % 2);
            for (uint32_t c = 0; c < N; c++) {
                A[c] = rnd(seed, S_BSK_MASK, (uint64_t)ir * N + c);
                Bv[c] = (uint64_t)gauss(seed, S_BSK_NOISE, (uint64_t)ir * N + c, glwe_sigma);
            }
            // B += A * S  mod (X^N + 1, 2^64)
            for (uint32_t j : ones)
                for (uint32_t c = 0; c < N; c++) {
                    uint32_t k = c + j;
                    if (k < N) Bv[k] += A[c];
                    else Bv[k - N] -= A[c];
                }
            if (lwe_key[i]) {
                if (row == 0) A[0] += g;
                else Bv[0] += g;
            }
            uint64_t *dst = bsk + ((size_t)i * 2 + row) * 2 * N;
            for (uint32_t c = 0; c < N; c++) {
                dst[c] = q_to_p(A[c]);
                dst[N + c] = q_to_p(Bv[c]);
            }
        }
    }
    return LUTHE_OK;
}

extern "C" int luthe_encrypt(const luthe_params *p, const uint32_t *S, const uint32_t *msgs, size_t count,
                             uint64_t seed, uint64_t *blwe)
{
    if (check(p) || !S || !msgs || !blwe) return LUTHE_E_PARAM;
    const uint32_t N = p->poly_size;
    const int shift = 64 - (int)(1 + p->msg_width + p->carry_width);
    const double sigma = GLWE_SIGMA_REL * 18446744073709551616.0;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < (long)count; c++) {
        uint64_t *ct = blwe + (size_t)c * (N + 1);
        uint64_t b = 0;
        for (uint32_t j = 0; j < N; j++) {
            ct[j] = rnd(seed, S_ENC_MASK, (uint64_t)c * N + j);
            if (S[j]) b += ct[j];
        }
        b += (uint64_t)gauss(seed, S_ENC_NOISE, (uint64_t)c, sigma);
        b += (uint64_t)msgs[c] << shift;
        ct[N] = b;
    }
    return LUTHE_OK;
}

extern "C" int luthe_decrypt(const luthe_params *p, const uint32_t *S, const uint64_t *blwe, size_t count,
                             uint32_t *msgs)
{
    if (check(p) || !S || !blwe || !msgs) return LUTHE_E_PARAM;
    const uint32_t N = p->poly_size;
    const int bits = 1 + (int)(p->msg_width + p->carry_width), shift = 64 - bits;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < (long)count; c++) {
        const uint64_t *ct = blwe + (size_t)c * (N + 1);
        uint64_t ph = ct[N];
        for (uint32_t j = 0; j < N; j++)
            if (S[j]) ph -= ct[j];
        uint64_t m = (ph + (1ull << (shift - 1))) >> shift;
        msgs[c] = (uint32_t)(m & ((1ull << bits) - 1));
    }
    return LUTHE_OK;
}

extern "C" int luthe_lut_build(const luthe_params *p, const uint32_t *table, uint64_t *glwe)
{
    if (check(p) || !table || !glwe) return LUTHE_E_PARAM;
    const uint32_t N = p->poly_size, nm = 1u << (p->msg_width + p->carry_width);
    const int shift = 64 - (int)(1 + p->msg_width + p->carry_width);
    if (N < nm) return LUTHE_E_PARAM;
    const uint32_t box = N / nm, half = box / 2;
    memset(glwe, 0, (size_t)N * 8);  // trivial GLWE: null mask
    uint64_t *body = glwe + N;
    // box m holds f(m); the whole table is rotated by half a box so that the
    // noise around each encoded value stays in its box; the entries that wrap
    // past X^N come back negated (negacyclic).  Matches the reference's LUT
    // test vectors (glwe_sd_rev, body coefficients in bit-reversed order).
    for (uint32_t j = 0; j < N; j++) {
        if (j < N - half) body[j] = (uint64_t)table[((j + half) / box) % nm] << shift;
        else body[j] = (uint64_t)0 - ((uint64_t)table[0] << shift);
    }
    return LUTHE_OK;
}
