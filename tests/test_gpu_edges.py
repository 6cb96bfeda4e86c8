"""Edge cases of the KS+PBS entry points on the GPU: empty batches, extreme
ciphertext words, and the largest batch of the benchmark's configurations
(16,384 BLWEs, the key-switch configuration's count) in one call."""
import numpy as np
import pytest

import luthe_b200 as L
from conftest import from_dev, to_dev

pytestmark = pytest.mark.gpu
N = 2048
M64 = (1 << 64) - 1


def test_empty_batches_are_noops(engine, params):
    import torch
    s = torch.cuda.Stream()
    engine.ks_pbs(None, None, None, 0)
    engine.ks_pbs_ml(None, None, None, 0, 2)
    engine.ks_pbs_graph(None, None, None, 0, s)
    engine.keyswitch(None, None, None, 0)
    engine.blind_rotate(None, None, None, 0)
    out = engine.ks_pbs_host(np.zeros((0, N + 1), np.uint64), np.zeros(0, np.uint32))
    assert out.shape == (0, N + 1)
    torch.cuda.synchronize()
    engine.check_device_error()


def test_extreme_ciphertext_words(engine, params, keys, oracle_bsk):
    """Masks and bodies at the ends of the torus and at the decomposition's
    rounding and tie points, through the key switch and the blind rotation:
    every output word equal to the oracle's."""
    n = params.lwe_dim
    tot = params.ks_base_log * params.ks_level          # 18 bits kept by the key switch
    rows = []
    for v in (0, 1, M64, 1 << 63, (1 << 63) - 1, 1 << (64 - tot), 1 << (63 - tot),
              (1 << 64) - (1 << (63 - tot)), 0x5555555555555555, 0xAAAAAAAAAAAAAAAA):
        rows.append(np.full(N + 1, v, np.uint64))
    rng = np.random.default_rng(5)
    mixed = rng.choice(np.array([0, 1 << 63, M64, 1 << (63 - tot), 3 << (62 - tot)], np.uint64), (6, N + 1))
    ct = np.concatenate([np.stack(rows), mixed])
    # the rotation amount of the body at both ends and at a half turn
    ct[-3:, N] = np.array([0, 1 << 63, M64], np.uint64)
    count = ct.shape[0]
    luts = np.stack([L.lut_build(params, np.arange(16, dtype=np.uint32)),
                     L.lut_build(params, (np.arange(16, dtype=np.uint32) * 7) % 16)])
    ids = (np.arange(count) % 2).astype(np.uint32)
    engine.upload_luts(luts)
    d_out = to_dev(np.zeros_like(ct))
    engine.ks_pbs(to_dev(ct), to_dev(ids), d_out, count)
    engine.check_device_error()
    got = from_dev(d_out, np.uint64)
    want = oracle_bsk.ks_pbs(keys["ksk"], ct, luts, ids)
    assert np.array_equal(got, want), np.nonzero((got != want).any(1))[0]
    # the key-switched intermediate lies in [0, 2N) for every input word
    d21 = to_dev(np.zeros((count, n + 1), np.uint32))
    d2n = to_dev(np.zeros((count, n + 1), np.uint32))
    engine.keyswitch(to_dev(ct), d21, d2n, count)
    assert int(from_dev(d2n, np.uint32).max()) < 2 * N


def test_largest_batch_in_one_call(engine, params, keys, oracle_bsk):
    """16,384 BLWEs (268 MB in, 268 MB out) in one call, four LUTs: every
    output decrypts to its LUT entry; 40 rows spread over the waves, the last
    ones included, equal the oracle word for word."""
    count = 16384
    rng = np.random.default_rng(16384)
    tables = [rng.integers(0, 16, 16).astype(np.uint32) for _ in range(4)]
    luts = np.stack([L.lut_build(params, t) for t in tables])
    msgs = rng.integers(0, 16, count).astype(np.uint32)
    ids = rng.integers(0, 4, count).astype(np.uint32)
    ct = L.encrypt(params, keys["glwe_key"], msgs, 777)
    engine.upload_luts(luts)
    engine.set_br_config(2, 1)
    d_out = to_dev(np.zeros_like(ct))
    engine.ks_pbs(to_dev(ct), to_dev(ids), d_out, count)
    engine.check_device_error()
    got = from_dev(d_out, np.uint64)
    dec = L.decrypt(params, keys["glwe_key"], got)
    want_msg = np.array([tables[i][m] for i, m in zip(ids, msgs)], np.uint32)
    assert np.array_equal(np.asarray(dec, np.uint32), want_msg)
    sel = np.unique(np.r_[0:8, count - 8:count, rng.choice(count, 24, replace=False)])
    want = oracle_bsk.ks_pbs(keys["ksk"], ct[sel], luts, ids[sel])
    assert np.array_equal(got[sel], want)


@pytest.mark.parametrize("count", [303, 1191])
def test_host_entry_point_with_a_tail_launch(engine, params, keys, oracle_bsk, count):
    """Batches of full waves plus a tail (1 and 4 waves of 296 on 148 SMs, + 7)
    through luthe_ks_pbs_host, whose read-back of the full waves overlaps the
    tail launch (1191 also copies its inputs in two chunks under the key
    switch): equal to the device entry point and, on a sample, to the oracle,
    on two calls in a row."""
    rng = np.random.default_rng(count)
    tables = [rng.integers(0, 16, 16).astype(np.uint32) for _ in range(3)]
    luts = np.stack([L.lut_build(params, t) for t in tables])
    msgs = rng.integers(0, 16, count).astype(np.uint32)
    ids = rng.integers(0, 3, count).astype(np.uint32)
    ct = L.encrypt(params, keys["glwe_key"], msgs, count)
    engine.upload_luts(luts)
    engine.set_br_config(2, 1)
    d_out = to_dev(np.zeros_like(ct))
    engine.ks_pbs(to_dev(ct), to_dev(ids), d_out, count)
    engine.check_device_error()
    want_dev = from_dev(d_out, np.uint64)
    for _ in range(2):
        got = engine.ks_pbs_host(ct, ids)
        assert np.array_equal(got, want_dev)
    sel = np.r_[0:4, count - 12:count]
    assert np.array_equal(want_dev[sel], oracle_bsk.ks_pbs(keys["ksk"], ct[sel], luts, ids[sel]))
