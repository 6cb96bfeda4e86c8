"""The reference's other HPU parameter sets on the GPU (KS 2x8, 2x7, 3x5 and
PBS base 2^22): key switch and full KS+PBS bit-exact against the CPU oracle
run with the same decomposition, and decrypting to the LUT's values."""
import numpy as np
import pytest

import luthe_b200 as L
import oracle
from conftest import from_dev, to_dev

pytestmark = pytest.mark.gpu
N = 2048
SETS = [s for s in L.PARAM_SETS if s != "default"]


@pytest.fixture(scope="module", params=SETS)
def setup(request):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p = L.param_set(request.param)
    keys = L.keygen(p, 4242 + p.lwe_dim + p.ks_level)
    eng = L.Engine(p)
    eng.upload_keys(keys)
    ob = oracle.OracleBsk(keys["bsk"], p.lwe_dim, N)
    yield request.param, p, keys, eng, ob
    eng.close()


def test_keyswitch_matches_oracle(setup):
    name, p, keys, eng, _ = setup
    n, count = p.lwe_dim, 40
    rng = np.random.default_rng(p.lwe_dim)
    blwe = rng.integers(0, 2**64, (count, N + 1), dtype=np.uint64)
    # ties and extremes of the top digits
    blwe[0, :6] = [0, 1 << 63, (1 << 64) - 1, 1 << (64 - p.ks_base_log * p.ks_level),
                   1 << (63 - p.ks_base_log * p.ks_level), (1 << 64) - (1 << (63 - p.ks_base_log * p.ks_level))]
    d21 = to_dev(np.zeros((count, n + 1), np.uint32))
    d2n = to_dev(np.zeros((count, n + 1), np.uint32))
    eng.keyswitch(to_dev(blwe), d21, d2n, count)
    g21, g2n = from_dev(d21, np.uint32), from_dev(d2n, np.uint32)
    for c in range(count):
        o21, o2n = oracle.keyswitch(blwe[c], keys["ksk"], n, N, ks_bl=p.ks_base_log, ks_lc=p.ks_level)
        assert np.array_equal(g21[c], o21), (name, c)
        assert np.array_equal(g2n[c], o2n), (name, c)


def test_ks_pbs_matches_oracle_and_decrypts(setup):
    name, p, keys, eng, ob = setup
    rng = np.random.default_rng(7 + p.lwe_dim)
    tables = [rng.integers(0, 16, 16).astype(np.uint32) for _ in range(2)]
    luts = np.stack([L.lut_build(p, t) for t in tables])
    msgs = rng.integers(0, 16, 12).astype(np.uint32)
    ids = (np.arange(12) % 2).astype(np.uint32)
    ct = L.encrypt(p, keys["glwe_key"], msgs, 99 + p.lwe_dim)
    eng.upload_luts(luts)
    d_out = to_dev(np.zeros((12, N + 1), np.uint64))
    eng.ks_pbs(to_dev(ct), to_dev(ids), d_out, 12)
    eng.check_device_error()
    got = from_dev(d_out, np.uint64)
    want = ob.ks_pbs(keys["ksk"], ct, luts, ids, ks_bl=p.ks_base_log, ks_lc=p.ks_level, pbs_bl=p.pbs_base_log)
    assert np.array_equal(got, want), name
    dec = L.decrypt(p, keys["glwe_key"], got)
    assert [int(x) for x in dec] == [int(tables[i][m]) for m, i in zip(msgs, ids)], name


def test_host_entry_point(setup):
    name, p, keys, eng, ob = setup
    table = np.arange(16, dtype=np.uint32)[::-1].copy()
    luts = L.lut_build(p, table)[None]
    msgs = np.arange(16, dtype=np.uint32)
    ct = L.encrypt(p, keys["glwe_key"], msgs, 5)
    eng.upload_luts(luts)
    out = eng.ks_pbs_host(ct, np.zeros(16, np.uint32))
    assert np.array_equal(out, ob.ks_pbs(keys["ksk"], ct, luts, np.zeros(16, np.uint32), ks_bl=p.ks_base_log,
                                         ks_lc=p.ks_level, pbs_bl=p.pbs_base_log)), name
    assert [int(x) for x in L.decrypt(p, keys["glwe_key"], out)] == [15 - m for m in range(16)]


def test_generator_tie_rule_matches_oracle(setup):
    """Each set's key switch (2x8, 2x7, 3x5 decompositions) and blind rotation
    (2^23 or 2^22) in the reference generator's tie rule, against the oracle
    in the same rule; the rule changes the top digits of most ciphertexts."""
    name, p, keys, eng, ob = setup
    rng = np.random.default_rng(31 + p.lwe_dim)
    table = rng.integers(0, 16, 16).astype(np.uint32)
    luts = L.lut_build(p, table)[None]
    count = 24
    msgs = rng.integers(0, 16, count).astype(np.uint32)
    ids = np.zeros(count, np.uint32)
    ct = L.encrypt(p, keys["glwe_key"], msgs, 77 + p.lwe_dim)
    eng.upload_luts(luts)
    d_rtl, d_gen = to_dev(np.zeros((count, N + 1), np.uint64)), to_dev(np.zeros((count, N + 1), np.uint64))
    eng.ks_pbs(to_dev(ct), to_dev(ids), d_rtl, count)
    eng.set_tie_rule(L.TIE_GENERATOR)
    try:
        eng.ks_pbs(to_dev(ct), to_dev(ids), d_gen, count)
        eng.check_device_error()
    finally:
        eng.set_tie_rule(L.TIE_RTL)
    got = from_dev(d_gen, np.uint64)
    oracle.set_tie_rule(True)
    try:
        want = ob.ks_pbs(keys["ksk"], ct, luts, ids, ks_bl=p.ks_base_log, ks_lc=p.ks_level, pbs_bl=p.pbs_base_log)
    finally:
        oracle.set_tie_rule(False)
    assert np.array_equal(got, want), name
    assert not np.array_equal(got, from_dev(d_rtl, np.uint64)), name
    assert [int(x) for x in L.decrypt(p, keys["glwe_key"], got)] == [int(table[m]) for m in msgs], name
