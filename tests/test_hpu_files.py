"""The HPU test-vector file importer against the reference generator's own
files (tests/golden/gtv_raw_n8_N64_noiseless, written by
tests/golden/make_golden.py beside the decoded fixture of the same run)."""
import os

import numpy as np

import luthe_b200 as L
from luthe_b200 import hpu_files as H

HERE = os.path.dirname(os.path.abspath(__file__))
RAW = os.path.join(HERE, "golden", "gtv_raw_n8_N64_noiseless")
G = np.load(os.path.join(HERE, "golden", "gtv_n8_N64_noiseless.npz"))


def test_files_decode_to_the_fixture_arrays():
    assert np.array_equal(H.load_ksk(os.path.join(RAW, "ksk_hwo_0.dat")), G["ksk"])
    # the fixture arrays keep the file's bit-reversed mask order
    assert np.array_equal(H.load_blwes(os.path.join(RAW, "input_blwe_sd_rev.dat"), natural=False), G["blwe_in"])
    assert np.array_equal(H.load_blwes(os.path.join(RAW, "output_blwe_sd_rev.dat"), natural=False), G["blwe_out"])
    nat = H.load_blwes(os.path.join(RAW, "input_blwe_sd_rev.dat"))
    N = int(G["N"])
    assert np.array_equal(nat[:, N], G["blwe_in"][:, N])
    assert np.array_equal(nat[:, H.bitrev_perm(N)], G["blwe_in"][:, :N])
    assert np.array_equal(H.load_slwes(os.path.join(RAW, "inner_slwe.dat")), G["inner_slwe"])
    assert np.array_equal(H.load_slwes(os.path.join(RAW, "inner_slwe_2N.dat")), G["inner_slwe_2N"])
    luts = H.load_glwes(os.path.join(RAW, "glwe_sd_rev.dat"), int(G["N"]))
    assert np.array_equal(luts[0], G["lut_natural"])


def test_imported_lut_is_the_engines_lut():
    p = L.default_params(poly_size=int(G["N"]), lwe_dim=int(G["n"]))
    luts = H.load_glwes(os.path.join(RAW, "glwe_sd_rev.dat"), int(G["N"]))
    assert np.array_equal(L.lut_build(p, np.arange(16, dtype=np.uint32)), luts[0])


def test_blwe_file_round_trip_is_byte_identical(tmp_path):
    src = os.path.join(RAW, "input_blwe_sd_rev.dat")
    for natural in (True, False):
        out = tmp_path / f"blwe_{natural}.dat"
        H.write_blwes(out, H.load_blwes(src, natural=natural), natural=natural)
        assert open(out).read().split() == open(src).read().split()


def test_ksk_natural_order_matches_natural_ciphertexts():
    """A key switch gives the same result with (file-order KSK, file-order
    BLWE) and with both converted to natural order."""
    import oracle
    n, N, L = int(G["n"]), int(G["N"]), int(G["ks_lc"])
    ksk_nat = H.load_ksk(os.path.join(RAW, "ksk_hwo_0.dat"), N=N, levels=L)
    nat = H.load_blwes(os.path.join(RAW, "input_blwe_sd_rev.dat"))
    for c in range(nat.shape[0]):
        a = oracle.keyswitch(G["blwe_in"][c], G["ksk"], n, N, 3, L, gtv_top_tie=True)
        b = oracle.keyswitch(nat[c], ksk_nat, n, N, 3, L, gtv_top_tie=True)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_bsk_loader_checks_its_input():
    raw = os.path.join(RAW, "bsk_nd_hwo_0.dat.gz")
    n, N = int(G["n"]), int(G["N"])
    b = H.load_bsk(raw, n, N, int(G["ntt_psi"]), int(G["ntt_delta"]))
    assert b.shape == (n, 2, 2, N) and int(b.max()) < 2**64 - 2**32 + 1
    try:
        H.load_bsk(raw, n + 1, N, 4, 3)
    except ValueError:
        pass
    else:
        raise AssertionError("a BSK of the wrong size was accepted")


def test_bsk_points_relabel_for_another_root():
    """A file written for another primitive 2N-th root phi = psi^u holds
    A(phi^(2k+1)) = A(psi^(2k'+1)): the importer's map sends k to k'."""
    P = 2**64 - 2**32 + 1
    for N in (64, 2048):
        psi = pow(H.PSI_4096, 2048 // N, P)
        for u in (1, 3, 2 * N - 1):
            phi = pow(psi, u, P)
            kmap = H._point_map(N, phi)
            assert sorted(kmap.tolist()) == list(range(N))
            for k in (0, 1, N // 2, N - 1):
                assert pow(phi, 2 * k + 1, P) == pow(psi, 2 * int(kmap[k]) + 1, P)
    try:
        H._point_map(64, 2)  # 2 is not a primitive 128-th root
    except ValueError:
        pass
    else:
        raise AssertionError("a wrong root was accepted")
