"""Many-LUT PBS and the serving loop on the GPU: bit-exact against the CPU
oracle, decrypting to the right integers, and identical alone and in a mix."""
import numpy as np
import pytest

import luthe_b200 as L
import oracle
from luthe_b200 import iops as I
from conftest import from_dev, to_dev

pytestmark = pytest.mark.gpu
N = 2048


@pytest.fixture(scope="module")
def iop_luts(params):
    return np.stack([L.lut_build(params, t) for t in I.lut_tables()])


def enc_blocks(params, keys, values, seed):
    blocks = [b for v in values for b in I.to_blocks(v)]
    return L.encrypt(params, keys["glwe_key"], np.array(blocks, np.uint32), seed)


def dec_blocks(params, keys, blwe):
    return [int(x) for x in L.decrypt(params, keys["glwe_key"], blwe)]


# 5 and 3 ciphertexts run in the two-SM form, 100 in the one-per-SM form;
# 301 = a full two-per-CTA wave plus a 5-ciphertext tail launch whose outputs
# start at row 296 * mlk
@pytest.mark.parametrize("mlk,count", [(2, 5), (4, 5), (8, 3), (4, 100), (2, 301)])
def test_many_lut_matches_oracle(engine, params, keys, oracle_bsk, mlk, count):
    rng = np.random.default_rng(100 + mlk + count)
    span = 16 // mlk
    fs = [rng.integers(0, 16, span).astype(np.uint32) for _ in range(mlk)]
    table = np.concatenate(fs)
    luts = L.lut_build(params, table)[None]
    msgs = rng.integers(0, span, count).astype(np.uint32)
    ct = L.encrypt(params, keys["glwe_key"], msgs, 300 + mlk)
    engine.upload_luts(luts)
    engine.set_br_config(2, 1)
    ids = np.zeros(count, np.uint32)
    d_out = to_dev(np.zeros((count * mlk, N + 1), np.uint64))
    engine.ks_pbs_ml(to_dev(ct), to_dev(ids), d_out, count, mlk)
    engine.check_device_error()
    got = from_dev(d_out, np.uint64)
    dec = dec_blocks(params, keys, got)
    assert dec == [int(fs[m][x]) for x in msgs for m in range(mlk)]
    check = np.arange(count) if count <= 8 else np.r_[0:3, 296:count] if count > 296 else np.r_[0:3, count - 3:count]
    rows = (check[:, None] * mlk + np.arange(mlk)).ravel()
    want = oracle_bsk.ks_pbs(keys["ksk"], ct[check], luts, ids[check], mlk=mlk)
    assert np.array_equal(got[rows], want)


def oracle_run(program, src, n_dst, keys, oracle_bsk, luts):
    """Execute a DOp program on ciphertexts with the CPU oracle."""
    from oracle import dops
    return dops.run(program, src, n_dst, keys["ksk"], oracle_bsk, luts)


def test_serving_add_cmp_mul_bit_exact_vs_oracle(engine, params, keys, oracle_bsk, iop_luts):
    engine.upload_luts(iop_luts)
    srv = L.Server(engine, pool_bytes=256 << 20)
    a, b, k = 0xBEEF, 0x1357, 0x4000
    reqs = [(I.prog_add(), enc_blocks(params, keys, [a, b], 11), 8),
            (I.prog_cmp_gt(k), enc_blocks(params, keys, [a], 12), 1),
            (I.prog_mul(), enc_blocks(params, keys, [a, b], 13), 8),
            (I.prog_add_prefix(), enc_blocks(params, keys, [a, b], 14), 8)]
    outs = srv.run(reqs)
    srv.close()
    assert I.from_blocks(dec_blocks(params, keys, outs[0])) == (a + b) % 65536
    assert dec_blocks(params, keys, outs[1]) == [int(a > k)]
    assert I.from_blocks(dec_blocks(params, keys, outs[2])) == (a * b) % 65536
    assert I.from_blocks(dec_blocks(params, keys, outs[3])) == (a + b) % 65536
    from oracle import dops
    want = dops.run_many(reqs, keys["ksk"], oracle_bsk, iop_luts)  # all three programs side by side
    for got, w in zip(outs, want):
        assert np.array_equal(got, w)


def test_serving_mix_equals_alone(engine, params, keys, iop_luts):
    engine.upload_luts(iop_luts)
    rng = np.random.default_rng(5)
    reqs, expect = [], []
    for r in range(9):
        a, b = int(rng.integers(65536)), int(rng.integers(65536))
        kind = r % 3
        if kind == 0:
            reqs.append((I.prog_add(), enc_blocks(params, keys, [a, b], 50 + r), 8))
            expect.append((a + b) % 65536)
        elif kind == 1:
            reqs.append((I.prog_cmp_gt(b), enc_blocks(params, keys, [a], 50 + r), 1))
            expect.append(int(a > b))
        else:
            reqs.append((I.prog_mul(), enc_blocks(params, keys, [a, b], 50 + r), 8))
            expect.append((a * b) % 65536)
    srv = L.Server(engine, pool_bytes=512 << 20)
    mixed = srv.run(reqs)
    alone = [srv.run([r])[0] for r in reqs[:3]]      # one of each kind on its own
    counters = srv.counters()
    srv.close()
    for got, want, (prog, _, nd) in zip(mixed, expect, reqs):
        dec = dec_blocks(params, keys, got)
        assert (I.from_blocks(dec) if nd == 8 else dec[0]) == want
    for m, s in zip(mixed[:3], alone):
        assert np.array_equal(m, s)
    assert counters["pbs"] == 3 * (8 + 15 + 101) + 8 + 15 + 101


def test_serving_admission_is_bounded_by_the_pool(engine, params, keys, iop_luts):
    engine.upload_luts(iop_luts)
    slot = (N + 1) * 8
    srv = L.Server(engine, pool_bytes=310 * slot)      # an ADD request takes 152 slots: room for 2
    reqs = [(I.prog_add(), enc_blocks(params, keys, [i, 2 * i], 70 + i), 8) for i in range(5)]
    ids = [srv.submit(*r) for r in reqs]
    done, max_active = 0, 0
    while done < len(ids):
        c, active, pending = srv.step()                 # active: requests holding pool slots
        max_active = max(max_active, active)
        done += c
    assert max_active <= 2
    for i, rid in enumerate(ids):
        out, lat, q = srv.fetch(rid, 8)
        assert I.from_blocks(dec_blocks(params, keys, out)) == 3 * i
    srv.close()


def test_serving_rejects_bad_programs(engine, iop_luts):
    engine.upload_luts(iop_luts)
    srv = L.Server(engine, pool_bytes=64 << 20)
    with pytest.raises(L.LutheError):
        srv.submit(np.array([I.enc_pbs("PBS", 0, 1, 4000)], np.uint32), np.zeros((0, N + 1), np.uint64), 1)
    with pytest.raises(L.LutheError):
        srv.submit(np.array([I.enc_mem("LD", 0, I.MEM_SRC, 5)], np.uint32), np.zeros((1, N + 1), np.uint64), 1)
    srv.close()


def test_serving_staggered_load_bit_exact_vs_oracle(engine, params, keys, oracle_bsk, iop_luts):
    """Requests submitted one per scheduler step, so PBS lanes overlap on the
    GPU and small batches meet busy SMs (the loop then runs them one
    ciphertext per CTA instead of in 2-SM pairs): every output of every
    request equals the oracle's run of the same programs, and decrypts."""
    engine.upload_luts(iop_luts)
    rng = np.random.default_rng(21)
    reqs, expect = [], []
    kinds = [0, 3, 2, 1] * 4  # ripple ADD, prefix ADD, MUL, compare
    for r, kind in enumerate(kinds):
        a, b = int(rng.integers(65536)), int(rng.integers(65536))
        if kind == 1:
            reqs.append((I.prog_cmp_gt(b), enc_blocks(params, keys, [a], 400 + r), 1))
            expect.append([int(a > b)])
        else:
            prog = {0: I.prog_add, 2: I.prog_mul, 3: I.prog_add_prefix}[kind]()
            reqs.append((prog, enc_blocks(params, keys, [a, b], 400 + r), 8))
            expect.append(I.to_blocks((a * b if kind == 2 else a + b) % 65536))
    srv = L.Server(engine, pool_bytes=512 << 20)
    ids, outs = [], {}
    for _ in range(200000):
        if len(ids) < len(reqs):
            ids.append(srv.submit(*reqs[len(ids)]))
        srv.step()
        for k, rid in enumerate(ids):
            if k not in outs:
                got = srv.fetch(rid, reqs[k][2])
                if got is not None:
                    outs[k] = got[0]
        if len(outs) == len(reqs):
            break
    srv.close()
    assert len(outs) == len(reqs)
    for k, want in enumerate(expect):
        dec = dec_blocks(params, keys, outs[k])
        assert (dec if reqs[k][2] == 1 else [d & 3 for d in dec]) == want, k
    from oracle import dops
    ref = dops.run_many(reqs, keys["ksk"], oracle_bsk, iop_luts)
    for k, w in enumerate(ref):
        assert np.array_equal(outs[k], w), k
