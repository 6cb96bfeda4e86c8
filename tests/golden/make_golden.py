"""Generate the golden fixtures of tests/golden from the reference itself.

Run from the repository root with the path of the reference project checkout:

    python tests/golden/make_golden.py REF [--models-only]

Sources (all run, none copied):
  * sw/bin/gtv/v1.4.1/gtv        -- the reference's test-vector generator
                                    (keys, BLWE in/out, KS outputs, LUT GLWE, BSK)
  * sw/decomposer/balanced_decomp_unfix_sign_round_bit.py  (hw_decompose)
  * sw/monomial_mult/monomial_mult.py                      (definition)
  * sw/solinas/solinas.py                                  (compute_modulo)

gtv's text files are read by luthe_b200.hpu_files (format and layouts in its
docstring).  The arrays of the .npz fixtures keep the files' own coefficient
order (BLWE masks bit-reversed, KSK mask index in the same order); the
decoded LUT is stored in natural order.  For the runs marked keep_bsk the
generator's BSK file itself is kept, gzipped, beside the fixture
(gtv_raw_<name>/bsk_nd_hwo_0.dat.gz), with the NTT network parameters it was
written for in the fixture (ntt_psi, ntt_delta; radix 2).
"""
import contextlib
import io
import os
import random
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from luthe_b200.hpu_files import read_sections  # noqa: E402
P = 2**64 - 2**32 + 1


def bitrev(x, bits):
    return int(format(x, "0%db" % bits)[::-1], 2)


RAW_FILES = ["ksk_hwo_0.dat", "glwe_sd_rev.dat", "batch#0/input_blwe_sd_rev.dat",
             "batch#0/output_blwe_sd_rev.dat", "batch#0/inner_slwe.dat", "batch#0/inner_slwe_2N.dat"]


NTT_PSI, NTT_DELTA = 4, 3  # the generator's --psi / --ntt-delta for every run (radix 2)


def read_words(path, w):
    return {k: [int(x) for x in v] for k, v in read_sections(path, w).items()}


def run_gtv(ref, name, n, N, per_batch, seed, noise, timeout=120, ks_bl=3, ks_lc=6, pbs_bl=23, keep_raw=False,
            keep_bsk=False):
    gtv = os.path.join(ref, "sw/bin/gtv/v1.4.1/gtv")
    out = tempfile.mkdtemp(prefix="gtv_")
    lwe_sd, glwe_sd = noise
    # gtv searches for NTT roots unless given; pass the ones the reference's
    # simulation flow uses (run.sh:429-458): phi = psi^(2048/N), omega = phi^2
    phi = pow(0x984ec5194d005735, 2048 // N, P)
    cmd = [gtv, "--omega-ru-n", str(phi * phi % P), "--phi-ru-2n", str(phi), "--lwe-dim", str(n), "--glwe-dim", "1", "--poly-size", str(N), "--pbs-bl", str(pbs_bl), "--pbs-lc", "1",
           "--ks-bl", str(ks_bl), "--ks-lc", str(ks_lc), "--ct-w", "64", "--ks-w", "21", "--msg-w", "2", "--carry-w", "2",
           "--pbs-batch", "1", "--pbs-per-batch", str(per_batch), "--seed", str(seed), "--ntt-radix", "2",
           "--psi", str(NTT_PSI), "--ntt-delta", str(NTT_DELTA), "--lwe-std-dev", repr(lwe_sd), "--glwe-std-dev", repr(glwe_sd),
           "--ksk-pc", "1", "--bsk-pc", "1", "--ks-lbx", "1", "--ks-lby", "1", "--ks-lbz", "1",
           "--panic-on-failure", "--verbose", "-o", out]
    log = subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=timeout).stdout
    d = os.path.realpath(os.path.join(out, "latest"))
    key = [int(x) for x in re.search(r"LweSecretKey \{ data: \[([^\]]*)\]", log).group(1).split(",")]
    msgs = [int(m) for m in re.findall(r"Generate Pbs_\d+ -> msg::(\d+)", log)]
    ksk = read_words(os.path.join(d, "ksk_hwo_0.dat"), 32)[""]
    glwe = read_words(os.path.join(d, "glwe_sd_rev.dat"), 64)
    b = os.path.join(d, "batch#0")
    ins = read_words(os.path.join(b, "input_blwe_sd_rev.dat"), 64)
    outs = read_words(os.path.join(b, "output_blwe_sd_rev.dat"), 64)
    s21 = read_words(os.path.join(b, "inner_slwe.dat"), 32)
    s2n = read_words(os.path.join(b, "inner_slwe_2N.dat"), 32)
    lb = N.bit_length() - 1
    lut0 = glwe[sorted(glwe)[0]]
    lut_nat = [0] * (2 * N)
    for part in range(2):
        for j in range(N):
            lut_nat[part * N + bitrev(j, lb)] = lut0[part * N + j]
    names = sorted(ins, key=lambda s: int(s[4:]))
    fx = {
        "n": n, "N": N, "seed": seed, "lwe_std_dev": lwe_sd, "glwe_std_dev": glwe_sd,
        "ks_bl": ks_bl, "ks_lc": ks_lc, "pbs_bl": pbs_bl,
        "lwe_key": np.array(key, np.uint32),
        "msgs": np.array(msgs, np.uint32),
        "ksk": np.array(ksk, np.uint32),
        "blwe_in": np.array([ins[k] for k in names], np.uint64),
        "blwe_out": np.array([outs[k] for k in names], np.uint64),
        "inner_slwe": np.array([s21["SLwe" + k[4:]] for k in names], np.uint32),
        "inner_slwe_2N": np.array([s2n["SLwe2N" + k[4:]] for k in names], np.uint32),
        "lut_natural": np.array(lut_nat, np.uint64),
        "ntt_psi": NTT_PSI, "ntt_delta": NTT_DELTA,
    }
    np.savez_compressed(os.path.join(HERE, f"gtv_{name}.npz"), **fx)
    if keep_raw:  # the text files themselves, for the file importer's tests
        import shutil
        raw = os.path.join(HERE, f"gtv_raw_{name}")
        os.makedirs(raw, exist_ok=True)
        for f in RAW_FILES:
            shutil.copy(os.path.join(d, f), os.path.join(raw, f.replace("batch#0/", "")))
    if keep_bsk:  # the generator's BSK file, for the importer and the full-PBS pins
        import gzip
        raw = os.path.join(HERE, f"gtv_raw_{name}")
        os.makedirs(raw, exist_ok=True)
        with open(os.path.join(d, "bsk_nd_hwo_0.dat"), "rb") as src, \
                gzip.GzipFile(os.path.join(raw, "bsk_nd_hwo_0.dat.gz"), "wb", mtime=0) as dst:
            dst.write(src.read())
    print(f"gtv_{name}: n={n} N={N} pbs={len(names)} msgs={msgs}")


def decomposer_vectors(ref):
    sys.path.insert(0, os.path.join(ref, "sw/decomposer"))
    with contextlib.redirect_stdout(io.StringIO()):  # the module self-checks on import
        import balanced_decomp_unfix_sign_round_bit as dec
    rng = random.Random(7)
    out = {}
    for bw, L in ((3, 6), (23, 1)):
        tot = bw * L
        vals = [0, 1, P, 2**64 - 1, 1 << 63, (1 << 63) - 1]
        # ties: an exact half at every digit, with and without the rounding bit
        for i in range(L):
            base = (1 << (64 - tot)) * ((1 << (bw * i)) * (1 << (bw - 1)))
            vals += [base % 2**64, (base + (1 << (63 - tot))) % 2**64, (base - 1) % 2**64]
        for top in range(min(1 << bw, 16)):
            vals.append(((top << (64 - min(bw, 4))) | (1 << (62 - tot))) % 2**64)
        vals += [rng.getrandbits(64) for _ in range(4000)]
        digs = []
        for v in vals:
            d = dec.hw_decompose(v, 2**bw, L, 2**64)  # (bw+1)-bit two's complement digits
            digs.append([x - (1 << (bw + 1)) if x >= (1 << bw) else x for x in d])
        out[f"v_{bw}x{L}"] = np.array(vals, np.uint64)
        out[f"d_{bw}x{L}"] = np.array(digs, np.int32)
    np.savez_compressed(os.path.join(HERE, "decomposer.npz"), **out)
    print("decomposer:", {k: v.shape for k, v in out.items()})


def monomial_vectors(ref):
    sys.path.insert(0, os.path.join(ref, "sw/monomial_mult"))
    with contextlib.redirect_stdout(io.StringIO()):
        import monomial_mult as mm
    rng = random.Random(11)
    out = {}
    for N, exps in ((64, [0, 1, 5, 63, 64, 65, 100, 127]), (2048, [0, 1, 2047, 2048, 3001, 4095])):
        mm.N = N  # the model reads the polynomial size from a module global
        polys, res = [], []
        for e in exps:
            poly = [rng.getrandbits(64) for _ in range(N)]
            polys.append(poly)
            res.append(mm.monomial_mult_definition(poly, e, 2**64))
        out[f"in_{N}"] = np.array(polys, np.uint64)
        out[f"e_{N}"] = np.array(exps, np.uint32)
        out[f"out_{N}"] = np.array(res, np.uint64)
    np.savez_compressed(os.path.join(HERE, "monomial.npz"), **out)
    print("monomial:", {k: v.shape for k, v in out.items()})


def solinas_vectors(ref):
    sys.path.insert(0, os.path.join(ref, "sw/solinas"))
    import solinas
    pos_max = 2 * 64 + 1
    exp_l = solinas.get_exponent(P)
    pos_d = solinas.get_position(exp_l, pos_max)
    solinas.exp_l = exp_l  # compute_modulo reads these module globals
    solinas.MOD_W = 64
    rng = random.Random(13)
    vals = [0, 1, P - 1, P, P + 1, 2**64 - 1, 2**64, 2**96, 2**96 - 1, (P - 1) ** 2, 2**128 - 1]
    vals += [rng.getrandbits(64) * rng.getrandbits(64) for _ in range(3000)]
    vals += [rng.randrange(P) * rng.randrange(P) for _ in range(3000)]
    red = [solinas.compute_modulo(v, P, pos_max, exp_l, pos_d) for v in vals]
    assert all(r == v % P for r, v in zip(red, vals))
    lo = np.array([v & (2**64 - 1) for v in vals], np.uint64)
    hi = np.array([v >> 64 for v in vals], np.uint64)
    np.savez_compressed(os.path.join(HERE, "solinas.npz"), lo=lo, hi=hi, red=np.array(red, np.uint64))
    print("solinas:", len(vals))


def modswitch_vectors():
    # RTL formula of mod_switch_to_2powerN.sv (MOD_Q_W=64, PRECISION_W=96):
    #   CST = floor(2^(64+96) / p);  z = (a*CST >> 96) + bit95(a*CST)
    # and the rounding it implements, round(a * 2^64 / p) (modsw_to_2powN.py:27-41).
    rng = random.Random(17)
    cst = (1 << 160) // P
    a = [0, 1, P - 1, P // 2, (P + 1) // 2, 2**63] + [rng.randrange(P) for _ in range(5000)]
    z, ideal = [], []
    for x in a:
        v = x * cst
        z.append(((v >> 96) + ((v >> 95) & 1)) % 2**64)
        ideal.append(((2 * x * 2**64 + P) // (2 * P)) % 2**64)
    np.savez_compressed(os.path.join(HERE, "modswitch.npz"), a=np.array(a, np.uint64), z=np.array(z, np.uint64),
                        ideal=np.array(ideal, np.uint64))
    print("modswitch: mismatches vs ideal rounding:", sum(p != q for p, q in zip(z, ideal)))


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if len(args) != 1:
        sys.exit("usage: python tests/golden/make_golden.py REF [--models-only]  (REF: the reference checkout)")
    ref = args[0]
    if "--models-only" not in sys.argv:
        run_gtv(ref, "n8_N64_noiseless", 8, 64, 4, 7, (0.0, 0.0), keep_raw=True, keep_bsk=True)
        run_gtv(ref, "n32_N256", 32, 256, 6, 11, (5.3943e-6, 4.4409e-16), keep_bsk=True)
        run_gtv(ref, "n32_N2048", 32, 2048, 3, 13, (5.3943e-6, 4.4409e-16), keep_bsk=True)
        # decompositions of the reference's other parameter sets
        run_gtv(ref, "n32_N256_ks2x8", 32, 256, 6, 17, (5.3943e-6, 4.4409e-16), ks_bl=2, ks_lc=8, keep_bsk=True)
        run_gtv(ref, "n32_N256_ks2x7", 32, 256, 6, 19, (5.3943e-6, 4.4409e-16), ks_bl=2, ks_lc=7, keep_bsk=True)
        run_gtv(ref, "n32_N256_ks3x5", 32, 256, 6, 23, (5.3943e-6, 4.4409e-16), ks_bl=3, ks_lc=5, keep_bsk=True)
        run_gtv(ref, "n32_N256_ks3x5_pbs22", 32, 256, 6, 29, (5.3943e-6, 4.4409e-16), ks_bl=3, ks_lc=5, pbs_bl=22,
                keep_bsk=True)
    decomposer_vectors(ref)
    monomial_vectors(ref)
    solinas_vectors(ref)
    modswitch_vectors()
