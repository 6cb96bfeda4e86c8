"""The two BSK upload forms give the same engine: the standard-domain key
(luthe_upload_bsk, transformed on the GPU) and its evaluations at the
roots psi^(2k+1) (luthe_upload_bsk_eval, the form the HPU's host writes)
produce identical KS+PBS outputs."""
import numpy as np
import pytest

import luthe_b200 as L
import oracle
from conftest import from_dev, to_dev

pytestmark = pytest.mark.gpu


def test_eval_domain_upload_equals_standard_upload():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p = L.default_params(lwe_dim=40)
    keys = L.keygen(p, 404)
    N = p.poly_size
    std = keys["bsk"].reshape(-1, N)
    ev = np.stack([oracle.ntt_eval(poly) for poly in std]).reshape(-1)
    rng = np.random.default_rng(4)
    count = 37
    table = rng.integers(0, 16, 16).astype(np.uint32)
    luts = L.lut_build(p, table)[None, :]
    msgs = rng.integers(0, 16, count).astype(np.uint32)
    ct = L.encrypt(p, keys["glwe_key"], msgs, 41)
    ids = np.zeros(count, np.uint32)
    outs = []
    for upload in ("std", "eval"):
        with L.Engine(p) as eng:
            eng.upload_ksk(keys["ksk"])
            if upload == "std":
                eng.upload_bsk(keys["bsk"])
            else:
                eng.upload_bsk_eval(ev)
            eng.upload_luts(luts)
            d_out = to_dev(np.zeros_like(ct))
            eng.ks_pbs(to_dev(ct), to_dev(ids), d_out, count)
            eng.check_device_error()
            outs.append(from_dev(d_out, np.uint64))
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], oracle.OracleBsk(keys["bsk"], p.lwe_dim, N).ks_pbs(keys["ksk"], ct, luts, ids))
    assert [int(x) for x in L.decrypt(p, keys["glwe_key"], outs[1])] == [int(table[m]) for m in msgs]


def test_eval_domain_upload_rejects_unreduced_words():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p = L.default_params(lwe_dim=4)
    bad = np.full(4 * 4 * p.poly_size, 2**64 - 1, np.uint64)
    with L.Engine(p) as eng, pytest.raises(L.LutheError) as ei:
        eng.upload_bsk_eval(bad)
    assert ei.value.code == L.E_PARAM
