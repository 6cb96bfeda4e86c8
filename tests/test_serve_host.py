"""Host logic of the serving loop on the CPU: the real scheduler of
luthe_b200/csrc/serve.cu compiled against a fake CUDA runtime with a plaintext
device model (tests/serve_harness).  Checks dependency handling, many-LUT
destinations, admission under a small pool, retirement and rejection of bad
programs -- everything but the cryptography, which the GPU tests cover."""
import ctypes
import os
import random
import subprocess

import numpy as np
import pytest

from luthe_b200 import iops as I

HERE = os.path.dirname(os.path.abspath(__file__))
W = 2049
vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64


@pytest.fixture(scope="module")
def H():
    subprocess.run([os.path.join(HERE, "serve_harness", "build.sh")], check=True)
    lib = ctypes.CDLL(os.path.join(HERE, "serve_harness", "libserve_harness.so"))
    lib.harness_ctx.restype = vp
    lib.harness_ctx.argtypes = [u32, vp, u32, u64]
    lib.harness_ctx_free.argtypes = [vp]
    lib.luthe_server_create.argtypes = [vp, u64, u32, ctypes.POINTER(vp)]
    lib.luthe_server_destroy.argtypes = [vp]
    lib.luthe_server_submit.argtypes = [vp, vp, u32, vp, u32, u32, ctypes.POINTER(u64)]
    lib.luthe_server_step.argtypes = [vp] + [ctypes.POINTER(u32)] * 3
    lib.luthe_server_fetch.argtypes = [vp, u64, vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.luthe_server_set_batching.argtypes = [vp, u32, u32]
    lib.luthe_server_counters.argtypes = [vp] + [ctypes.POINTER(u64)] * 4
    lib.harness_set_event_lag.argtypes = [ctypes.c_int]
    lib.harness_set_nsm.argtypes = [vp, ctypes.c_int]
    lib.harness_launch_log.argtypes = [vp, vp, ctypes.c_int]
    lib.harness_launch_log.restype = ctypes.c_int
    return lib


class PlainServer:
    def __init__(self, H, pool_slots):
        self.H = H
        tables = np.array(I.lut_tables(), np.uint64)
        self.ctx = H.harness_ctx(804, tables.ctypes.data, len(tables), 1 << 40)
        self.srv = vp()
        assert H.luthe_server_create(self.ctx, pool_slots * W * 8, 4096, ctypes.byref(self.srv)) == 0

    def close(self):
        self.H.luthe_server_destroy(self.srv)
        self.H.harness_ctx_free(self.ctx)

    def submit(self, prog, vals, ndst):
        src = np.zeros((len(vals), W), np.uint64)
        src[:, 0] = vals
        rid = u64()
        rc = self.H.luthe_server_submit(self.srv, prog.ctypes.data, prog.size, src.ctypes.data, len(vals), ndst,
                                        ctypes.byref(rid))
        return rc, rid.value

    def step(self):
        c, a, p = u32(), u32(), u32()
        assert self.H.luthe_server_step(self.srv, ctypes.byref(c), ctypes.byref(a), ctypes.byref(p)) == 0
        return c.value, a.value, p.value

    def fetch(self, rid, ndst):
        out = np.zeros((ndst, W), np.uint64)
        lat, q = ctypes.c_double(), ctypes.c_double()
        rc = self.H.luthe_server_fetch(self.srv, rid, out.ctypes.data, ctypes.byref(lat), ctypes.byref(q))
        return out[:, 0] if rc == 0 else None


def run_all(s, reqs):
    ids = []
    for prog, vals, nd in reqs:
        rc, rid = s.submit(prog, vals, nd)
        assert rc == 0
        ids.append(rid)
    outs, max_active = {}, 0
    for _ in range(10000):
        c, active, pending = s.step()
        max_active = max(max_active, active)
        for k, (rid, (_, _, nd)) in enumerate(zip(ids, reqs)):
            if k not in outs:
                got = s.fetch(rid, nd)
                if got is not None:
                    outs[k] = got
        if len(outs) == len(reqs):
            break
    return [outs[k] for k in range(len(reqs))], max_active


def test_mixed_requests_give_the_right_integers(H):
    s = PlainServer(H, 1 << 14)
    rng = random.Random(3)
    reqs, expect = [], []
    for r in range(60):
        a, b = rng.randrange(65536), rng.randrange(65536)
        kind = rng.choice("acm")
        if kind == "a":
            reqs.append((I.prog_add(), I.to_blocks(a) + I.to_blocks(b), 8))
            expect.append((a + b) % 65536)
        elif kind == "c":
            reqs.append((I.prog_cmp_gt(b), I.to_blocks(a), 1))
            expect.append(int(a > b))
        else:
            reqs.append((I.prog_mul(), I.to_blocks(a) + I.to_blocks(b), 8))
            expect.append((a * b) % 65536)
    outs, _ = run_all(s, reqs)
    s.close()
    for out, want, (_, _, nd) in zip(outs, expect, reqs):
        assert (I.from_blocks(out) if nd == 8 else int(out[0])) == want


def test_admission_is_bounded_by_the_pool(H):
    s = PlainServer(H, 310)                                 # an ADD request takes 152 slots
    reqs = [(I.prog_add(), I.to_blocks(i) + I.to_blocks(3 * i), 8) for i in range(7)]
    outs, max_active = run_all(s, reqs)
    s.close()
    assert max_active <= 2
    assert [I.from_blocks(o) for o in outs] == [4 * i for i in range(7)]


def test_sync_orders_the_program(H):
    s = PlainServer(H, 1024)
    p = I.Program(1, 1)
    p.ld(0, 0)
    p.words.append(0x10 << 26)                              # SYNC
    p.add(1, 0, 0)
    p.pbs(2, 1, "MsgOnly")
    p.st(0, 2)
    outs, _ = run_all(s, [(p.array(), [3], 1)])
    s.close()
    assert int(outs[0][0]) == (3 + 3) & 3


def test_bad_programs_are_rejected(H):
    s = PlainServer(H, 1024)
    rc, _ = s.submit(np.array([I.enc_pbs("PBS", 0, 1, 4000)], np.uint32), [], 1)
    assert rc != 0                                          # LUT id not uploaded
    rc, _ = s.submit(np.array([I.enc_mem("LD", 0, I.MEM_SRC, 5)], np.uint32), [1], 1)
    assert rc != 0                                          # source block out of range
    rc, _ = s.submit(np.array([I.enc_pbs("PBS_ML2", 3, 1, 0)], np.uint32), [], 1)
    assert rc != 0                                          # many-LUT destination not aligned
    s.close()


def _mixed(rng, n):
    reqs, expect = [], []
    for r in range(n):
        a, b = rng.randrange(65536), rng.randrange(65536)
        if r % 2:
            reqs.append((I.prog_add(), I.to_blocks(a) + I.to_blocks(b), 8))
            expect.append((a + b) % 65536)
        else:
            reqs.append((I.prog_mul(), I.to_blocks(a) + I.to_blocks(b), 8))
            expect.append((a * b) % 65536)
    return reqs, expect


def run_staggered(s, reqs):
    """Submit one request per scheduler step (arrivals spread over time)."""
    ids, outs = [], {}
    for _ in range(20000):
        if len(ids) < len(reqs):
            rc, rid = s.submit(*reqs[len(ids)])
            assert rc == 0
            ids.append(rid)
        s.step()
        for k, rid in enumerate(ids):
            if k not in outs:
                got = s.fetch(rid, reqs[k][2])
                if got is not None:
                    outs[k] = got
        if len(outs) == len(reqs):
            break
    return [outs[k] for k in range(len(reqs))]


def test_batching_window_holds_partial_batches_and_stays_correct(H):
    """With lanes busy across steps (events lag), a batching window makes the
    scheduler hold partial PBS batches: fewer, larger launches, same results."""
    launches = {}
    for window in (0, 10_000_000):
        H.harness_set_event_lag(3)
        try:
            s = PlainServer(H, 1 << 15)
            assert H.luthe_server_set_batching(s.srv, 64, window) == 0
            reqs, expect = _mixed(random.Random(11), 24)
            outs = run_staggered(s, reqs)
            cnt = [u64() for _ in range(4)]
            H.luthe_server_counters(s.srv, *[ctypes.byref(x) for x in cnt])
            launches[window] = cnt[0].value  # PBS rounds (one KS+PBS launch each)
            s.close()
        finally:
            H.harness_set_event_lag(0)
        assert [I.from_blocks(o) for o in outs] == expect
    assert launches[10_000_000] < launches[0]


def test_loaded_gpu_runs_small_batches_one_per_cta(H):
    """Cluster pairs take two SMs per ciphertext: a batch whose ciphertexts,
    with those of the busy lanes, would need more SMs than the device has runs
    one ciphertext per CTA (pair cut-off 0); an idle device keeps the default
    cut-off.  Lanes stay busy across steps (events lag), the device has 8 SMs
    (room for 4 pairs), and the results stay right."""
    H.harness_set_event_lag(3)
    try:
        s = PlainServer(H, 1 << 15)
        H.harness_set_nsm(s.ctx, 8)
        H.harness_launch_log(None, None, 0)
        reqs, expect = _mixed(random.Random(12), 24)
        outs = run_staggered(s, reqs)
        batch, pair_max = np.zeros(100000, np.int64), np.zeros(100000, np.int32)
        n = H.harness_launch_log(batch.ctypes.data, pair_max.ctypes.data, len(batch))
        s.close()
    finally:
        H.harness_set_event_lag(0)
    assert [I.from_blocks(o) for o in outs] == expect
    batch, pair_max = batch[:n], pair_max[:n]
    assert n > 0 and set(pair_max.tolist()) <= {-1, 0}
    assert np.all(pair_max[2 * batch > 8] == 0)             # alone too big for the pairs
    assert np.any((pair_max == 0) & (2 * batch <= 8))       # too big with the busy lanes' ciphertexts
    assert np.any(pair_max == -1)                           # room left: the default cut-off
