"""The full KS+PBS of the oracle against the reference generator's own outputs.

For each fixture made by tests/golden/make_golden.py from a run of the
reference's test-vector generator (sw/bin/gtv), the generator's KSK, its BSK
file (bsk_nd_hwo, read by luthe_b200.hpu_files.load_bsk), its LUT and its
input ciphertexts go through the oracle's key switch and blind rotation with
the generator's tie rule, and every word of every output BLWE must equal the
generator's output_blwe file.  The fixtures cover the reference's parameter
sets' decompositions (KS 3x6, 2x8, 2x7, 3x5; PBS 2^23 and 2^22) at N = 256
and the benchmark's KS 3x6 / PBS 2^23 at N = 2048.

The last test repeats the check at the benchmark's n = 804, N = 2048 with the
generator run live; it needs the reference checkout (the environment variable
LUTHE_REFERENCE_DIR) and is skipped without it."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from luthe_b200 import hpu_files as H

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = ["n32_N2048", "n32_N256", "n32_N256_ks2x8", "n32_N256_ks2x7", "n32_N256_ks3x5", "n32_N256_ks3x5_pbs22"]
P = 2**64 - 2**32 + 1


@pytest.fixture(autouse=True)
def _generator_tie_rule():
    oracle.set_tie_rule(True)
    yield
    oracle.set_tie_rule(False)


def _oracle_pbs(g, bsk_eval, tie_generator=True):
    n, N = int(g["n"]), int(g["N"])
    ks_bl, ks_lc, pbs_bl = int(g["ks_bl"]), int(g["ks_lc"]), int(g["pbs_bl"])
    ob = oracle.OracleBsk(bsk_eval.reshape(-1), n, N, eval_domain=True)
    l2ns = []
    for blwe in g["blwe_in"]:
        _, o2n = oracle.keyswitch(blwe, g["ksk"], n, N, ks_bl, ks_lc, gtv_top_tie=tie_generator)
        l2ns.append(o2n)
    out = ob.blind_rotate(np.stack(l2ns), g["lut_natural"][None, :], np.zeros(len(l2ns), np.uint32), pbs_bl)
    return out, np.stack(l2ns)


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_pbs_equals_generator_output(name):
    g = np.load(os.path.join(GOLD, f"gtv_{name}.npz"))
    n, N = int(g["n"]), int(g["N"])
    bsk = H.load_bsk(os.path.join(GOLD, f"gtv_raw_{name}", "bsk_nd_hwo_0.dat.gz"), n, N,
                     int(g["ntt_psi"]), int(g["ntt_delta"]))
    out, l2n = _oracle_pbs(g, bsk)
    assert np.array_equal(l2n % (2 * N), g["inner_slwe_2N"] % (2 * N))
    # the generator writes the output mask in bit-reversed order
    assert np.array_equal(H.blwe_natural_to_file(out), g["blwe_out"]), name


def test_bsk_file_is_a_glwe_key_encryption():
    """The decoded BSK of a noiseless run is, in the standard domain, GGSW
    rows (a, a*S + e) with |e| <= a few units (the rounding from 2^64 to p),
    plus the gadget 2^41 p / 2^64 on the diagonal for a key bit of 1; S is the
    GLWE key recovered from the generator's KSK and its printed LWE key, in
    polynomial (natural) order."""
    g = np.load(os.path.join(GOLD, "gtv_n8_N64_noiseless.npz"))
    n, N, L = int(g["n"]), int(g["N"]), int(g["ks_lc"])
    raw = os.path.join(GOLD, "gtv_raw_n8_N64_noiseless", "bsk_nd_hwo_0.dat.gz")
    bsk = H.load_bsk(raw, n, N, int(g["ntt_psi"]), int(g["ntt_delta"]))
    ksk = g["ksk"].astype(np.int64).reshape(n + 1, N, L)
    s = g["lwe_key"].astype(np.int64)
    ph = (ksk[n, :, L - 1] - (ksk[:n, :, L - 1] * s[:, None]).sum(0)) % (1 << 21)
    key_file = np.round(ph / 2**18).astype(np.int64) % 8
    S = key_file[H.bitrev_perm(N)].astype(np.uint64)  # file order -> polynomial order
    gadget = (2**41 * P + 2**63) >> 64
    for i in range(n):
        for row in range(2):
            a = oracle.ntt_inv_natural(bsk[i, row, 0])
            b = oracle.ntt_inv_natural(bsk[i, row, 1])
            aS = oracle.negacyclic_mul_schoolbook(a, S)
            e = [(int(x) - int(y)) % P for x, y in zip(b, aS)]
            if s[i] == 1 and row == 1:
                e[0] = (e[0] - gadget) % P
            if s[i] == 1 and row == 0:  # the mask row carries the gadget: b = (a - g) S + e
                e = [(x + gadget * int(v)) % P for x, v in zip(e, S)]
            ec = [x - P if x > P // 2 else x for x in e]
            assert max(abs(x) for x in ec) <= 16, (i, row, max(abs(x) for x in ec))


def test_point_order_rule_small_cases():
    # log2 N = 6, delta 3: the last cut of 3 stages is bit-reversed
    k = H.bsk_point_order(64, 4, 2, 3)
    assert [int(x) for x in k[:9]] == [0, 32, 16, 48, 8, 40, 24, 56, 1]
    # delta dividing log2 N: d = delta;  d = log2 N mod delta otherwise
    assert [int(x) for x in H.bsk_point_order(2048, 32, 2, 5)[:3]] == [0, 1024, 1]
    assert sorted(H.bsk_point_order(2048, 4, 2, 3).tolist()) == list(range(2048))
    with pytest.raises(ValueError):
        H.bsk_point_order(2048, 4, 4, 3)


def test_oracle_matches_generator_at_n804(tmp_path):
    ref = os.environ.get("LUTHE_REFERENCE_DIR")
    gtv = os.path.join(ref, "sw/bin/gtv/v1.4.1/gtv") if ref else None
    if not gtv or not os.path.exists(gtv):
        pytest.skip("LUTHE_REFERENCE_DIR does not point at the reference checkout")
    n, N, per, seed, psi, delta = 804, 2048, 4, 21, 32, 5
    phi = pow(0x984EC5194D005735, 2048 // N, P)
    out = tempfile.mkdtemp(dir=tmp_path)
    cmd = [gtv, "--omega-ru-n", str(phi * phi % P), "--phi-ru-2n", str(phi), "--lwe-dim", str(n), "--glwe-dim", "1",
           "--poly-size", str(N), "--pbs-bl", "23", "--pbs-lc", "1", "--ks-bl", "3", "--ks-lc", "6", "--ct-w", "64",
           "--ks-w", "21", "--msg-w", "2", "--carry-w", "2", "--pbs-batch", "1", "--pbs-per-batch", str(per),
           "--seed", str(seed), "--ntt-radix", "2", "--psi", str(psi), "--ntt-delta", str(delta),
           "--lwe-std-dev", "5.3943e-06", "--glwe-std-dev", "4.4409e-16", "--ksk-pc", "1", "--bsk-pc", "1",
           "--ks-lbx", "1", "--ks-lby", "1", "--ks-lbz", "1", "--panic-on-failure", "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, timeout=900)
    d = os.path.realpath(os.path.join(out, "latest"))
    b = os.path.join(d, "batch#0")
    lut = H.load_glwes(os.path.join(d, "glwe_sd_rev.dat"), N)[0]
    g = {"n": n, "N": N, "ks_bl": 3, "ks_lc": 6, "pbs_bl": 23, "lut_natural": lut,
         "ksk": H.load_ksk(os.path.join(d, "ksk_hwo_0.dat")),
         "blwe_in": H.load_blwes(os.path.join(b, "input_blwe_sd_rev.dat"), natural=False)}
    want = H.load_blwes(os.path.join(b, "output_blwe_sd_rev.dat"), natural=False)
    bsk = H.load_bsk(os.path.join(d, "bsk_nd_hwo_0.dat"), n, N, psi, delta)
    out_gen, _ = _oracle_pbs(g, bsk, tie_generator=True)
    assert np.array_equal(H.blwe_natural_to_file(out_gen), want)
