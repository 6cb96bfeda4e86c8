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
    assert np.array_equal(H.load_blwes(os.path.join(RAW, "input_blwe_sd_rev.dat")), G["blwe_in"])
    assert np.array_equal(H.load_blwes(os.path.join(RAW, "output_blwe_sd_rev.dat")), G["blwe_out"])
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
    out = tmp_path / "blwe.dat"
    H.write_blwes(out, H.load_blwes(src))
    assert open(out).read().split() == open(src).read().split()
