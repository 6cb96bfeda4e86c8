/*
 * luthe.h -- C ABI of the B200 KS+PBS engine.
 *
 * The engine is a drop-in for the HPU's PBS processing element (pe_pbs) and
 * its linear-DOp neighbour (pe_alu).  On the HPU these are driven by DOps
 * (docs/dop.md:82-165; binary form fw/ublaze/src/hpu_dop_fmt.h:43-140): a PBS
 * DOp "PBS Dst Src LUT" reads a BLWE (k*N+1 u64) from the register file,
 * key-switches it, blind-rotates a LUT GLWE selected by `gid`, sample-extracts
 * the result and writes it back.  Here a batch of such DOps is one call; the
 * register file is replaced by caller-owned device (or host) buffers.
 *
 * Conventions
 *  - All pointers named d_* are device pointers, h_* host pointers.  The caller
 *    owns every buffer passed in.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *  - Functions return LUTHE_OK or one of the LUTHE_E_* codes; the message of
 *    the last failure on the calling thread is in luthe_last_error().  Errors
 *    are reported, never hidden: there is no CPU fallback.
 *  - A context is not thread-safe; one thread owns it (the HPU firmware loop
 *    is single-threaded too: fw/ublaze/src/ucore_fw.c:68).  Its calls share
 *    the context's scratch (the key-switched intermediate, the split-K sums of
 *    small key switches): calls of one context on different streams must be
 *    ordered by the caller (events) or use separate contexts.
 *
 * Data formats (u64 torus values mod 2^64 unless stated)
 *  - BLWE: N mask coefficients in natural order, then the body
 *    (the order of the reference's input/output BLWE test vectors).
 *  - KSK:  u32 words mod 2^ks_width, index (x*(k*N) + y)*ks_level + z, x in
 *    [0, n] (the body column last), y the BLWE mask coefficient, z the level
 *    (z = 0 is the least significant digit, weight
 *    2^(ks_width - ks_base_log*(ks_level-z)))
 *    -- the order of the reference's ksk_hwo files with one channel.
 *  - BSK:  standard domain over Z_p, p = 2^64 - 2^32 + 1 (values < p), index
 *    ((i*2 + row)*2 + col)*N + c: GGSW of LWE-key bit i, row = decomposed GLWE
 *    component (0 mask, 1 body), col = output component.  The engine converts
 *    it to its own evaluation layout on upload (the HPU too receives its BSK
 *    pre-transformed from the host: hw/module/bsk/module/bsk_manager).
 *  - LUT:  trivial GLWE, mask polynomial then body polynomial, natural order.
 */
#ifndef LUTHE_H
#define LUTHE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LUTHE_OK 0
#define LUTHE_E_PARAM 1   /* bad argument or unsupported parameter set */
#define LUTHE_E_BUDGET 2  /* HBM admission budget exceeded */
#define LUTHE_E_TIMEOUT 3 /* a bounded device wait ran out */
#define LUTHE_E_CUDA 4    /* CUDA runtime error (no device, launch failure...) */
#define LUTHE_E_STATE 5   /* keys or LUTs not uploaded yet */

/* Crypto parameter set (hw/module/param/module/<set>/rtl/param_tfhe_definition_pkg.sv). */
typedef struct luthe_params {
    uint32_t lwe_dim;      /* n      (804) */
    uint32_t glwe_dim;     /* k      (1)   */
    uint32_t poly_size;    /* N      (2048) */
    uint32_t pbs_base_log; /* 23 */
    uint32_t pbs_level;    /* 1  */
    uint32_t ks_base_log;  /* 3  */
    uint32_t ks_level;     /* 6  */
    uint32_t ks_width;     /* 21: KS modulus 2^21 (MOD_KSK_W) */
    uint32_t msg_width;    /* 2  */
    uint32_t carry_width;  /* 2  */
} luthe_params;

typedef struct luthe_ctx luthe_ctx;

/* Linear DOps (docs/dop.md:82-100; pea_alu_core.sv:59-61,124-161). */
enum luthe_lwe_op {
    LUTHE_OP_ADD = 0,  /* dst = a + b            */
    LUTHE_OP_SUB = 1,  /* dst = a - b            */
    LUTHE_OP_MAC = 2,  /* dst = a * imm + b      */
    LUTHE_OP_ADDS = 3, /* dst = a + imm*Delta    */
    LUTHE_OP_SUBS = 4, /* dst = a - imm*Delta    */
    LUTHE_OP_SSUB = 5, /* dst = imm*Delta - a    */
    LUTHE_OP_MULS = 6  /* dst = a * imm          */
};

/* Fill `p` with the engine's parameter set (n=804, k=1, N=2048, PBS 23x1,
 * KS 3x6 mod 2^21, 2-bit message + 2-bit carry). */
void luthe_params_default(luthe_params *p);

const char *luthe_last_error(void);

/* Context: binds a CUDA device; `hbm_budget` caps the device bytes the context
 * may hold (0 = 80 GB).  Replaces the HPU bring-up the host backend performs
 * over PCIe (docs/hpu.md:42-54).  Creating a context also sets, for the whole
 * device, the bound on each blind-rotation wait for a BSK slab: 2^26 polls,
 * or the value of the environment variable LUTHE_SLAB_WAIT_POLLS (a
 * diagnostic; 0 makes every wait run out at once, which the tests use to
 * exercise the timeout path). */
int luthe_ctx_create(const luthe_params *p, int device, uint64_t hbm_budget, luthe_ctx **out);
void luthe_ctx_destroy(luthe_ctx *ctx);
uint64_t luthe_device_bytes(const luthe_ctx *ctx);

/* Key material (bsk_manager.sv / ksk_manager.sv: keys resident before BR). */
int luthe_upload_bsk(luthe_ctx *ctx, const uint64_t *h_bsk_std_p);
/* The BSK given in the evaluation domain, as the HPU receives it from its
 * host (hw/module/bsk/module/bsk_manager; the reference generator's
 * bsk_nd_hwo files, whose AXI order is hw/module/hpu/simu/scripts/
 * gen_stimuli.py:108-127): index ((i*2 + row)*2 + col)*N + k holds
 * BSK_i[row][col](psi^(2k+1)) mod p, k in natural order, psi the 2N-th root
 * of luthe_ntt_fwd.  luthe_b200.hpu_files.load_bsk turns a bsk_nd_hwo file
 * into this form. */
int luthe_upload_bsk_eval(luthe_ctx *ctx, const uint64_t *h_bsk_eval);
int luthe_upload_ksk(luthe_ctx *ctx, const uint32_t *h_ksk);
/* LUT memory, indexed by the PBS DOp's gid (dflt_cfg.toml:18-19 lut_mem). */
int luthe_upload_luts(luthe_ctx *ctx, const uint64_t *h_glwe, uint32_t count);

/* Tie rule of both balanced decompositions (key switch, blind rotation) for a
 * top digit equal to B/2.  LUTHE_TIE_RTL (the default) follows the RTL
 * (hw/module/decomposer/module/decomp_parallel/rtl/decomp_parallel.sv:73-75,
 * 142-150): the digit is -B/2 when the rounded value's lower bits or rounding
 * bit are set.  LUTHE_TIE_GENERATOR follows the reference's test-vector
 * generator (sw/bin/gtv, built on TFHE-rs): the digit stays +B/2.  Both
 * decompose to the same value; with the generator's rule and the generator's
 * keys, outputs equal the generator's output_blwe files word for word. */
#define LUTHE_TIE_RTL 0
#define LUTHE_TIE_GENERATOR 1
int luthe_set_tie_rule(luthe_ctx *ctx, int rule);

/* Pre-size the per-call scratch for batches up to `max_count` ciphertexts, so
 * later calls (and graph captures) allocate nothing. */
int luthe_reserve(luthe_ctx *ctx, size_t max_count);

/* Batched PBS DOp: KS + blind rotation + sample extract of `count` BLWEs with
 * per-ciphertext LUT ids (PBS Dst Src LUT, docs/dop.md:101-111).  Replaces one
 * pe_pbs batch (pe_pbs.sv:346-762) -- here every batch size in one launch. */
int luthe_ks_pbs(luthe_ctx *ctx, const uint64_t *d_in, const uint32_t *d_lut_id, uint64_t *d_out, size_t count,
                 void *stream);
/* Same through host buffers (copies in, computes, copies out, synchronises).
 * Pinned host memory gives the full PCIe/C2C bandwidth.  Batches of 1024 or
 * more are copied in as two chunks (a quarter, then the rest) on a stream of
 * the context, each chunk's key switch starting once it has landed; when the
 * batch ends in a partial
 * wave that runs as its own launch, the outputs of the full waves are copied
 * back on that stream while that launch runs. */
int luthe_ks_pbs_host(luthe_ctx *ctx, const uint64_t *h_in, const uint32_t *h_lut_id, uint64_t *h_out,
                      size_t count);
/* Many-LUT PBS (PBS_ML2/ML4/ML8, docs/dop.md:101-121): one blind rotation per
 * ciphertext, `mlk` outputs per ciphertext written to rows count_index*mlk+m.
 * The LUT packs the mlk functions in consecutive blocks of 2^(msg+carry)/mlk
 * boxes (luthe_lut_build of the concatenated tables); inputs must stay below
 * 2^(msg+carry)/mlk. */
int luthe_ks_pbs_ml(luthe_ctx *ctx, const uint64_t *d_in, const uint32_t *d_lut_id, uint64_t *d_out, size_t count,
                    uint32_t mlk, void *stream);
/* CUDA-graph form of luthe_ks_pbs: the first call for a given (pointers,
 * count, stream) captures the launches, later calls replay the graph. */
int luthe_ks_pbs_graph(luthe_ctx *ctx, const uint64_t *d_in, const uint32_t *d_lut_id, uint64_t *d_out,
                       size_t count, void *stream);

/* luthe_ks_pbs for callers that must not allocate device memory while they run
 * (allocator hooks and arenas, fixed-budget or framework-owned device memory).
 * No counterpart in the reference.  It allocates nothing: the key-switched
 * intermediate goes to a fixed 4 MiB array (2^20 u32) that every GPU loading
 * this library holds until exit, so count * (n+1) must be <= 2^20 (1302
 * ciphertexts at n = 804) or LUTHE_E_PARAM is returned.  The first call on a
 * device looks up that array's device address; make that first call before
 * any stream capture.  Calls share the array: calls that overlap on the GPU
 * race.  Keys and LUTs come from the context as for luthe_ks_pbs. */
int luthe_ks_pbs_noalloc(luthe_ctx *ctx, const uint64_t *d_in, const uint32_t *d_lut_id, uint64_t *d_out,
                         size_t count, void *stream);

/* Stages on their own (pep_key_switch; pe_pbs BR + SXT). */
int luthe_keyswitch(luthe_ctx *ctx, const uint64_t *d_in, uint32_t *d_out21, uint32_t *d_out2N, size_t count,
                    void *stream);
int luthe_blind_rotate(luthe_ctx *ctx, const uint32_t *d_lwe2N, const uint32_t *d_lut_id, uint64_t *d_out,
                       size_t count, void *stream);

/* Negacyclic NTT over Goldilocks, N = 2048 (ntt_core_gf64).  Forward output
 * index k holds A(psi^(2k+1)), psi = 0x984ec5194d005735 (psi^64 = 8); the
 * inverse includes 1/N.  luthe_ntt_mul computes INTT(NTT(a) * NTT(b)). */
int luthe_ntt_fwd(luthe_ctx *ctx, const uint64_t *d_in, uint64_t *d_out, size_t count, void *stream);
int luthe_ntt_inv(luthe_ctx *ctx, const uint64_t *d_in, uint64_t *d_out, size_t count, void *stream);
int luthe_ntt_mul(luthe_ctx *ctx, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out, size_t count,
                  void *stream);

/* Linear DOps on `count` BLWEs (pe_alu). */
int luthe_lwe_op(luthe_ctx *ctx, int op, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out, uint64_t imm,
                 size_t count, void *stream);

/* ---------------------------------------------------------- serving loop
 *
 * Continuous batching of DOp programs (the firmware's IOp -> DOp expansion,
 * fw/ublaze/src/ucore_fw.c:54-130, and the instruction scheduler,
 * hw/module/instruction_scheduler): a request is a DOp program (32-bit words
 * in the field layouts of fw/ublaze/src/hpu_dop_fmt.h:49-117) over its own
 * 128-register file, with n_src input blocks (LD Rx TS.slot) and n_dst output
 * blocks (ST TD.slot Rx).  Opcodes: ADD 0x01 SUB 0x02 MAC 0x05 ADDS 0x09
 * SUBS 0x0A SSUB 0x0B MULS 0x0C SYNC 0x10 LD 0x20 ST 0x21 PBS 0x30
 * PBS_ML2/4/8 0x31-0x33 (| 0x08: flush variant).  Each luthe_server_step
 * admits pending requests while the slot pool (carved from the context's HBM
 * budget) has room, issues every ready linear DOp of every request in one
 * launch, gathers the ready PBS DOps of every request (one many-LUT factor per
 * launch) into a KS+PBS launch on each idle PBS lane (own stream and
 * scratch, so batches overlap on the GPU), and retires finished requests.
 * Latency is measured from submit to retire. */
typedef struct luthe_server luthe_server;
int luthe_server_create(luthe_ctx *ctx, uint64_t pool_bytes, uint32_t max_pbs, luthe_server **out);
void luthe_server_destroy(luthe_server *srv);
int luthe_server_submit(luthe_server *srv, const uint32_t *dops, uint32_t n_dops, const uint64_t *h_src,
                        uint32_t n_src, uint32_t n_dst, uint64_t *id);
int luthe_server_step(luthe_server *srv, uint32_t *n_completed, uint32_t *n_active, uint32_t *n_pending);
/* Copy a finished request's output blocks out and release it; LUTHE_E_STATE
 * while it is not finished. */
int luthe_server_fetch(luthe_server *srv, uint64_t id, uint64_t *h_dst, double *latency_s, double *queue_s);
int luthe_server_counters(luthe_server *srv, uint64_t *rounds, uint64_t *pbs, uint64_t *alu, uint64_t *launches);
/* Batching window of the PBS lanes, after the HPU's batch policy (a batch
 * leaves when full or when the batch-in-progress timeout runs out,
 * hw/module/pe_pbs/module/pep_sequencer/rtl/pep_sequencer.sv:573-620): ready
 * PBS DOps are held back while some lane is busy, fewer than `fill` (0: two
 * per SM, one full wave) are ready and the oldest has waited less than
 * `window_us`.  window_us = 0 (the default) issues whatever is ready on any
 * idle lane. */
int luthe_server_set_batching(luthe_server *srv, uint32_t fill, uint32_t window_us);

/* Blind-rotation launch shape (the HPU's batch configuration: the BSK slice
 * shared per batch, hw/module/pe_pbs/module/pep_sequencer/rtl/
 * pep_sequencer.sv:573-620, docs/hpu_parameters.md): ciphertexts per CTA
 * sharing one BSK slab (1 or 2) and CTAs per SM of the persistent grid;
 * luthe_set_br_config resets the batch-size cut-offs below to their defaults.
 *
 * luthe_autotune times, on this device, (1) one and two ciphertexts per CTA
 * on `sample` ciphertexts (0: four waves), (2) for batches of 1/8 .. 3/2 of
 * the SM count, one ciphertext per 2-SM cluster, one per CTA, and the
 * two-per-CTA launch, and (3) for partial last waves of 1/4 .. 7/4 of the SM
 * count, a separate small launch against one launch for all; it keeps the
 * fastest shape and cut-offs and writes a JSON record of every trial and the
 * choice into `json` (may be NULL).  When the environment variable
 * LUTHE_TUNING_DIR names a directory, the choice is also saved there, one
 * file per device and parameter set, and luthe_ctx_create loads that file if
 * it exists.  luthe_tuning_save / luthe_tuning_load write and read the choice
 * at an explicit path; loading refuses a file made for another device model,
 * SM count or parameter set. */
int luthe_set_br_config(luthe_ctx *ctx, int cts_per_cta, int ctas_per_sm);
int luthe_autotune(luthe_ctx *ctx, size_t sample, char *json, size_t json_cap);
int luthe_tuning_save(luthe_ctx *ctx, const char *path);
int luthe_tuning_load(luthe_ctx *ctx, const char *path);

/* Device-side error flags raised by blind rotations since the last check
 * (sticky, cleared by this call; the stream must have been synchronised):
 * LUTHE_E_TIMEOUT when a bounded wait for a BSK slab ran out, LUTHE_E_PARAM
 * when a device-resident LUT id was >= the uploaded LUT count (that
 * ciphertext was rotated against LUT 0; its output is not meaningful).  A
 * timeout whose block could not confirm, within a second bound, that its last
 * slab copy had finished landing in shared memory is also LUTHE_E_TIMEOUT,
 * with a message saying that the device state is unsafe: destroy the context
 * and end the process before using the device again. */
int luthe_check_device_error(luthe_ctx *ctx);

/* Integer-pipe peaks of `device` measured by probe kernels: 32-bit IMAD per
 * second and Goldilocks 64x64 multiply-reduce per second (the denominators of
 * the integer roofline; no reference counterpart -- the HPU is an FPGA). */
int luthe_measure_int_peak(int device, double *imad_per_s, double *glmul_per_s);

/* ------------------------------------------------------------ host helpers */

/* Seeded key generation (binary keys, Gaussian noise: LWE sigma 2^-17.5,
 * GLWE sigma 2^-51, relative to the modulus).  Buffers:
 *   lwe_key[n], glwe_key[k*N], ksk[(n+1)*k*N*ks_level], bsk[n*4*N]. */
int luthe_keygen(const luthe_params *p, uint64_t seed, uint32_t *lwe_key, uint32_t *glwe_key, uint32_t *ksk,
                 uint64_t *bsk_std_p);
/* Encrypt `count` messages (message+carry bits, < 2^(msg+carry)) under the
 * GLWE key seen as an LWE key of dimension k*N. */
int luthe_encrypt(const luthe_params *p, const uint32_t *glwe_key, const uint32_t *msgs, size_t count,
                  uint64_t seed, uint64_t *blwe);
/* Decrypt `count` BLWEs: msgs[i] = round(phase / Delta) mod 2^(1+msg+carry). */
int luthe_decrypt(const luthe_params *p, const uint32_t *glwe_key, const uint64_t *blwe, size_t count,
                  uint32_t *msgs);
/* Build the trivial LUT GLWE for f given as table[2^(msg+carry)] (values
 * < 2^(msg+carry)); the box layout of the reference's LUT test vectors. */
int luthe_lut_build(const luthe_params *p, const uint32_t *table, uint64_t *glwe);

#ifdef __cplusplus
}
#endif
#endif /* LUTHE_H */
