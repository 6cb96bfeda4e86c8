"""The GPU engine on the reference generator's own material (n = 32,
N = 2048, KS 3 x 6, PBS 2^23; tests/golden/gtv_n32_N2048.npz and the
generator's BSK file tests/golden/gtv_raw_n32_N2048/bsk_nd_hwo_0.dat.gz, made
by tests/golden/make_golden.py).

With the generator's tie rule (luthe_set_tie_rule(LUTHE_TIE_GENERATOR)) the
engine's key switch equals the generator's inner_slwe and inner_slwe_2N, and
its full KS+PBS -- keys imported from the generator's files, BSK through
luthe_upload_bsk_eval -- equals the generator's output_blwe word for word.
With the RTL's tie rule (the default) the engine equals the oracle in RTL
mode bit for bit, and differs from the generator only in the top KS digit of
a tie: the phase stays within 8 e per tie and the message is unchanged."""
import os

import numpy as np
import pytest

import luthe_b200 as L
import oracle
from conftest import from_dev, to_dev
from luthe_b200 import hpu_files as H

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _fixture():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return np.load(os.path.join(GOLD, "gtv_n32_N2048.npz"))


def _keyswitch(eng, blwe, n):
    count = blwe.shape[0]
    d21 = to_dev(np.zeros((count, n + 1), np.uint32))
    d2n = to_dev(np.zeros((count, n + 1), np.uint32))
    eng.keyswitch(to_dev(blwe), d21, d2n, count)
    return from_dev(d21, np.uint32), from_dev(d2n, np.uint32)


def test_gpu_keyswitch_generator_rule_equals_generator():
    g = _fixture()
    n, N = int(g["n"]), int(g["N"])
    with L.Engine(L.default_params(lwe_dim=n)) as eng:
        eng.upload_ksk(g["ksk"])
        eng.set_tie_rule(L.TIE_GENERATOR)
        g21, g2n = _keyswitch(eng, g["blwe_in"], n)
    assert np.array_equal(g21, g["inner_slwe"])
    # the generator prints the rounded 2N value unreduced (4096 where the RTL's 12 bits wrap to 0)
    assert np.array_equal(g2n, g["inner_slwe_2N"] % (2 * N))


def test_gpu_keyswitch_rtl_rule_on_generator_vectors():
    g = _fixture()
    n, N = int(g["n"]), int(g["N"])
    s = g["lwe_key"].astype(np.int64)
    with L.Engine(L.default_params(lwe_dim=n)) as eng:
        eng.upload_ksk(g["ksk"])
        g21, g2n = _keyswitch(eng, g["blwe_in"], n)
    for c in range(g["blwe_in"].shape[0]):
        blwe = g["blwe_in"][c]
        o21, o2n = oracle.keyswitch(blwe, g["ksk"], n, N)  # RTL tie rule
        assert np.array_equal(g21[c], o21) and np.array_equal(g2n[c], o2n), c
        ties = sum(oracle.decompose(int(v), 3, 6) != oracle.decompose(int(v), 3, 6, True) for v in blwe[:N])
        ref = g["inner_slwe"][c]
        ph_gpu = (int(g21[c][n]) - int((g21[c][:n].astype(np.int64) * s).sum())) % (1 << 21)
        ph_ref = (int(ref[n]) - int((ref[:n].astype(np.int64) * s).sum())) % (1 << 21)
        diff = (ph_gpu - ph_ref + (1 << 20)) % (1 << 21) - (1 << 20)
        assert abs(diff) <= 8 * 64 * max(ties, 1), (c, diff, ties)
        if ties == 0:
            assert np.array_equal(g21[c], ref)
            assert np.array_equal(g2n[c], g["inner_slwe_2N"][c] % (2 * N))
        # message of the switched ciphertext: 4-bit payload under 1 padding bit
        assert round(ph_gpu / 2**21 * 32) % 32 == int(g["msgs"][c]), c


def test_gpu_ks_pbs_equals_generator_output():
    g = _fixture()
    n, N = int(g["n"]), int(g["N"])
    bsk = H.load_bsk(os.path.join(GOLD, "gtv_raw_n32_N2048", "bsk_nd_hwo_0.dat.gz"), n, N,
                     int(g["ntt_psi"]), int(g["ntt_delta"]))
    blwe = g["blwe_in"]
    count = blwe.shape[0]
    with L.Engine(L.default_params(lwe_dim=n)) as eng:
        eng.set_tie_rule(L.TIE_GENERATOR)
        eng.upload_ksk(g["ksk"])  # mask index in the file's order, as the ciphertexts
        eng.upload_bsk_eval(bsk)
        eng.upload_luts(g["lut_natural"][None, :])
        d_out = to_dev(np.zeros_like(blwe))
        eng.ks_pbs(to_dev(blwe), to_dev(np.zeros(count, np.uint32)), d_out, count)
        eng.check_device_error()
        out = from_dev(d_out, np.uint64)
        # the same keys in the engine's natural order give the same outputs
        eng.upload_ksk(H.load_ksk_words_natural(g["ksk"], N, int(g["ks_lc"])))
        d_nat = to_dev(np.zeros_like(blwe))
        eng.ks_pbs(to_dev(H.blwe_file_to_natural(blwe)), to_dev(np.zeros(count, np.uint32)), d_nat, count)
        eng.check_device_error()
        out_nat = from_dev(d_nat, np.uint64)
    assert np.array_equal(H.blwe_natural_to_file(out), g["blwe_out"])  # every word, every ciphertext
    assert np.array_equal(out_nat, out)
