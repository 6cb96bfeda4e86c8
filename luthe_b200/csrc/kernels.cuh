// Launch wrappers for the sm_100a kernels of the KS+PBS engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

namespace luthe {

constexpr int N = 2048;
constexpr int TWO_N = 4096;
constexpr int KS_L = 6;
constexpr int KS_BL = 3;
constexpr int KS_W = 21;
constexpr int KS_BN = 128;                    // key-switch output tile
constexpr int KS_BM = 32;                     // key-switch ciphertext tile
constexpr int KS_KC = 8;                      // BLWE mask coefficients per K chunk
constexpr int KS_PLANES = 3;                  // words per 4 KSK rows and output (device layout [K/4][3][xpad])
constexpr int KS_SPLIT = 16;                  // K slices of the split-K key switch (batches <= KS_BM)
constexpr int SLAB_WORDS = 8 * 4 * 256;       // one BR step of BSK: 2x2 polys of 2048
constexpr size_t SLAB_BYTES = SLAB_WORDS * 8; // 64 KiB

struct BrConfig {
    int cts_per_cta;    // ciphertexts sharing one BSK slab per CTA (G)
    int ctas_per_sm;    // resident CTAs per SM of the persistent grid
    // batch-size cut-offs of the launch forms (launch_blind_rotate); -1 keeps
    // the default named beside each.  The autotuner (luthe_autotune) sets them.
    int pair_max = -1;   // batches up to this run one ciphertext per 2-SM cluster (default SMs / 2)
    int split_max = -1;  // ... else up to this, one ciphertext per CTA (default SMs)
    int tail_max = -1;   // a partial last wave up to this runs as its own small launch (default SMs)
};

// device twiddle tables: [fwd 8x256][inv 8x256]
void build_twiddles(uint64_t *host_tw /* 4096 words */);

cudaError_t launch_bsk_prepare(const uint64_t *d_std_p, uint64_t *d_slab, const uint64_t *d_tw,
                               uint32_t n, cudaStream_t s);
cudaError_t launch_ntt_fwd(const uint64_t *d_in, uint64_t *d_out, const uint64_t *d_tw, size_t count,
                           cudaStream_t s);
cudaError_t launch_ntt_inv(const uint64_t *d_in, uint64_t *d_out, const uint64_t *d_tw, size_t count,
                           cudaStream_t s);
cudaError_t launch_ntt_mul(const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out, const uint64_t *d_tw,
                           size_t count, cudaStream_t s);
// Tie rule of the balanced decompositions for a top digit equal to B/2:
// the RTL's (decomp_parallel.sv) or the reference's test-vector generator's.
constexpr uint32_t TIE_RTL = 0, TIE_GENERATOR = 1;
cudaError_t launch_keyswitch(const uint64_t *d_in, const uint32_t *d_ksk_t, uint32_t *d_out21, uint32_t *d_out2N,
                             size_t B, uint32_t n, uint32_t xpad, cudaStream_t s,
                             const uint32_t *d_src_idx = nullptr, uint32_t bl = KS_BL, uint32_t L = KS_L,
                             uint32_t tie_rule = TIE_RTL, uint32_t *d_part = nullptr);
// d_part: KS_BM x xpad u32, all zero, for the split-K form of batches of at
// most KS_BM ciphertexts (left zero again); nullptr: the one-pass form only.
// Calls that overlap on the GPU must not share it.
bool ks_supported(uint32_t bl, uint32_t L);
bool pbs_supported(uint32_t bw);
// Bound on the polls of each BSK-slab wait of the blind rotation on the
// current device (default 2^26); 0 makes every wait run out at once.
cudaError_t set_slab_wait_polls(unsigned long long polls);
cudaError_t launch_blind_rotate(const BrConfig &cfg, int num_sms, const uint32_t *d_lwe2N, const uint64_t *d_luts,
                                const uint32_t *d_lut_id, uint32_t nlut, const uint64_t *d_bsk, const uint64_t *d_tw,
                                uint64_t *d_out, size_t B, uint32_t n, uint32_t *d_err, cudaStream_t s,
                                const uint32_t *d_dst_idx = nullptr, uint32_t mlk = 1, uint32_t pbs_bw = 23,
                                uint32_t tie_rule = TIE_RTL, cudaEvent_t main_done = nullptr,
                                size_t *main_count = nullptr);
size_t br_smem_bytes(const BrConfig &cfg, uint32_t n);
cudaError_t br_set_attributes(const BrConfig &cfg, uint32_t n);

enum LweOp : int { LWE_ADD = 0, LWE_SUB = 1, LWE_MAC = 2, LWE_ADDS = 3, LWE_SUBS = 4, LWE_SSUB = 5, LWE_MULS = 6 };
// one linear DOp or register copy (op = LWE_COPY) on slots of a BLWE pool
constexpr int LWE_COPY = 7;
// device error flag bits (luthe_check_device_error)
constexpr uint32_t DEVERR_TIMEOUT = 1u;  // a bounded wait for a BSK slab ran out
constexpr uint32_t DEVERR_LUT_ID = 2u;   // a LUT id >= the uploaded LUT count
constexpr uint32_t DEVERR_DRAIN = 4u;    // after a timeout, a slab copy in flight did not finish landing
struct AluOp {
    uint32_t op, dst, a, b;
    uint64_t imm;
};
cudaError_t launch_alu_batch(const AluOp *d_ops, uint64_t *d_pool, uint32_t nops, uint32_t dim, cudaStream_t s);

cudaError_t launch_lwe_op(int op, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out, uint64_t imm,
                          size_t count, uint32_t dim, cudaStream_t s);

}  // namespace luthe
