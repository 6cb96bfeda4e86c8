"""luthe_ks_pbs_noalloc: the KS+PBS entry point for callers that cannot
allocate device memory while they run (allocator hooks, fixed device budgets,
framework-owned memory).  Its results must equal luthe_ks_pbs's bit for bit.

This file is collected last on purpose: it works alone in a fresh process and
after every other test."""
import numpy as np
import pytest

import luthe_b200 as L
from conftest import from_dev, to_dev

pytestmark = pytest.mark.gpu
N = 2048


def _batch(params, keys, count, seed):
    rng = np.random.default_rng(seed)
    msgs = rng.integers(0, 16, count).astype(np.uint32)
    ids = rng.integers(0, 2, count).astype(np.uint32)
    return L.encrypt(params, keys["glwe_key"], msgs, seed), ids


def _launch_form_counts():
    """Batch sizes that reach each blind-rotation launch form on this GPU:
    one ciphertext per two SMs, one per SM, a full two-per-CTA wave, and a
    full wave plus a tail that runs as its own launch (it reads the fixed
    scratch at an offset of one wave)."""
    import torch
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    return (nsm // 4, nsm // 2 + 26, 2 * nsm, 2 * nsm + 5)


def test_noalloc_matches_ks_pbs_twice(engine, params, keys):
    tables = [np.arange(16, dtype=np.uint32)[::-1].copy(), (np.arange(16, dtype=np.uint32) * 5) % 16]
    engine.upload_luts(np.stack([L.lut_build(params, t) for t in tables]))
    for call, count in enumerate((37, 9)):  # two calls in a row; the second reuses the scratch
        ct, ids = _batch(params, keys, count, 900 + call)
        d_in, d_ids = to_dev(ct), to_dev(ids)
        d_ref, d_new = to_dev(np.zeros_like(ct)), to_dev(np.zeros_like(ct))
        engine.ks_pbs(d_in, d_ids, d_ref, count)
        engine.ks_pbs_noalloc(d_in, d_ids, d_new, count)
        engine.check_device_error()
        ref, new = from_dev(d_ref, np.uint64), from_dev(d_new, np.uint64)
        assert np.array_equal(new, ref), f"call {call}"
        dec = L.decrypt(params, keys["glwe_key"], new)
        msgs = L.decrypt(params, keys["glwe_key"], ct)
        assert [int(x) for x in dec] == [int(tables[i][m]) for i, m in zip(ids, msgs)]


def test_noalloc_rejects_batches_beyond_its_scratch(engine, params):
    too_many = (1 << 20) // (params.lwe_dim + 1) + 1
    with pytest.raises(L.LutheError) as ei:
        engine.ks_pbs_noalloc(1 << 12, 1 << 12, 1 << 12, too_many)  # rejected before any launch
    assert ei.value.code == L.E_PARAM


def test_noalloc_every_launch_form(engine, params, keys):
    """Each launch form reads the fixed scratch in its own pattern; every
    output row must equal luthe_ks_pbs's, on calls made back to back."""
    tables = [np.arange(16, dtype=np.uint32)[::-1].copy(), (np.arange(16, dtype=np.uint32) * 7) % 16]
    engine.upload_luts(np.stack([L.lut_build(params, t) for t in tables]))
    for call, count in enumerate(_launch_form_counts()):
        ct, ids = _batch(params, keys, count, 950 + call)
        d_in, d_ids = to_dev(ct), to_dev(ids)
        d_ref, d_new = to_dev(np.zeros_like(ct)), to_dev(np.zeros_like(ct))
        engine.ks_pbs(d_in, d_ids, d_ref, count)
        engine.ks_pbs_noalloc(d_in, d_ids, d_new, count)
        engine.check_device_error()
        ref, new = from_dev(d_ref, np.uint64), from_dev(d_new, np.uint64)
        assert np.array_equal(new, ref), f"count {count}"
