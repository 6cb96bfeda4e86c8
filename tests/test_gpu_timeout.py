"""The blind rotation's bounded wait for a BSK slab, made to run out on purpose.

A child process sets the wait bound to zero polls (LUTHE_SLAB_WAIT_POLLS=0, so
no other test sees it) and runs KS+PBS in every launch shape: the two-SM pair
form (1 ciphertext), the one-per-SM form (100) and the two-per-CTA form with a
pair-form tail (301).  Each must report LUTHE_E_TIMEOUT through
luthe_check_device_error, and the context must stay usable afterwards: an NTT
product on the same engine still matches the oracle.  No fault is involved:
the kernels give up, wait (bounded) for the slab copies already in flight,
and return."""
import os
import subprocess
import sys
import textwrap

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import sys
    sys.path.insert(0, ROOT)
    import numpy as np
    import torch
    import luthe_b200 as L
    import oracle

    p = L.default_params()
    keys = L.keygen(p, 5)
    eng = L.Engine(p)
    eng.upload_keys(keys)
    eng.upload_luts(L.lut_build(p, np.arange(16, dtype=np.uint32))[None])
    for count in (1, 100, 301):
        ct = L.encrypt(p, keys["glwe_key"], np.zeros(count, np.uint32), count)
        d_in = torch.from_numpy(ct.view(np.int64)).cuda()
        d_ids = torch.zeros(count, dtype=torch.int32, device="cuda")
        d_out = torch.zeros((count, p.poly_size + 1), dtype=torch.int64, device="cuda")
        eng.ks_pbs(d_in, d_ids, d_out, count)
        torch.cuda.synchronize()
        try:
            eng.check_device_error()
        except L.LutheError as e:
            assert e.code == L.E_TIMEOUT, e
        else:
            raise SystemExit(f"no timeout reported for {count} ciphertexts")
    eng.check_device_error()                       # the flag was cleared
    rng = np.random.default_rng(1)
    P = 0xFFFFFFFF00000001
    a = rng.integers(0, 2**63, (2, 2048), dtype=np.uint64) % np.uint64(P)
    b = rng.integers(0, 2**63, (2, 2048), dtype=np.uint64) % np.uint64(P)
    d_o = torch.zeros((2, 2048), dtype=torch.int64, device="cuda")
    eng.ntt_mul(torch.from_numpy(a.view(np.int64)).cuda(), torch.from_numpy(b.view(np.int64)).cuda(), d_o, 2)
    assert np.array_equal(d_o.cpu().numpy().view(np.uint64), oracle.negacyclic_mul(a, b))
    eng.close()
    print("ok")
""").replace("ROOT", repr(ROOT))


def test_slab_wait_running_out_is_reported_and_the_context_survives():
    env = dict(os.environ, LUTHE_SLAB_WAIT_POLLS="0")
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-2000:]
