"""Bit-exact parity of the CUDA engine (through its C ABI) against the CPU oracle.

Every comparison is exact: the path is integer arithmetic mod p and mod 2^64.
"""
import numpy as np
import pytest

import luthe_b200 as L
import oracle
from conftest import from_dev, to_dev

pytestmark = pytest.mark.gpu
P = oracle.P
N = 2048


def rand_p(rng, shape):
    return rng.integers(0, P, shape, dtype=np.uint64)


@pytest.mark.parametrize("count", [1, 2, 5])
def test_ntt_fwd_matches_oracle(engine, count):
    rng = np.random.default_rng(10 + count)
    a = rand_p(rng, (count, N))
    d_in, d_out = to_dev(a), to_dev(np.zeros_like(a))
    engine.ntt_fwd(d_in, d_out, count)
    got = from_dev(d_out, np.uint64)
    for c in range(count):
        assert np.array_equal(got[c], oracle.ntt_eval(a[c]))


def test_ntt_edge_values(engine):
    a = np.zeros((4, N), np.uint64)
    a[1, 0] = 1                      # delta -> all ones
    a[2, :] = P - 1                  # all -1
    a[3, 5] = P - 1
    d_in, d_out = to_dev(a), to_dev(np.zeros_like(a))
    engine.ntt_fwd(d_in, d_out, 4)
    got = from_dev(d_out, np.uint64)
    for c in range(4):
        assert np.array_equal(got[c], oracle.ntt_eval(a[c]))
    assert np.all(got[1] == 1)


@pytest.mark.parametrize("count", [1, 3])
def test_ntt_inverse_roundtrip(engine, count):
    rng = np.random.default_rng(20 + count)
    a = rand_p(rng, (count, N))
    d_a, d_f, d_b = to_dev(a), to_dev(np.zeros_like(a)), to_dev(np.zeros_like(a))
    engine.ntt_fwd(d_a, d_f, count)
    engine.ntt_inv(d_f, d_b, count)
    assert np.array_equal(from_dev(d_b, np.uint64), a)


@pytest.mark.parametrize("count", [1, 7, 1001])  # 1001: more pairs than one wave of CTAs, odd count
def test_ntt_mul_matches_oracle(engine, count):
    rng = np.random.default_rng(30 + count)
    a, b = rand_p(rng, (count, N)), rand_p(rng, (count, N))
    d_o = to_dev(np.zeros_like(a))
    engine.ntt_mul(to_dev(a), to_dev(b), d_o, count)
    assert np.array_equal(from_dev(d_o, np.uint64), oracle.negacyclic_mul(a, b))


@pytest.mark.parametrize("count", [1, 33])
def test_keyswitch_matches_oracle(engine, params, keys, count):
    rng = np.random.default_rng(40 + count)
    n = params.lwe_dim
    blwe = rng.integers(0, 2**64, (count, N + 1), dtype=np.uint64)
    blwe[0, :8] = [0, 1 << 63, (1 << 64) - 1, 1 << 45, 3 << 44, (1 << 64) - (1 << 45), 0x8000200000000000, 7]
    d_in = to_dev(blwe)
    d21 = to_dev(np.zeros((count, n + 1), np.uint32))
    d2n = to_dev(np.zeros((count, n + 1), np.uint32))
    engine.keyswitch(d_in, d21, d2n, count)
    g21, g2n = from_dev(d21, np.uint32), from_dev(d2n, np.uint32)
    for c in range(count):
        o21, o2n = oracle.keyswitch(blwe[c], keys["ksk"], n, N)
        assert np.array_equal(g21[c], o21), c
        assert np.array_equal(g2n[c], o2n), c


def test_keyswitch_split_k_consecutive_calls(engine, params, keys):
    """Batches of at most 32 ciphertexts switch keys in the split-K form (the
    mask coefficients summed by 16 CTAs per output tile into a context buffer
    that the finishing kernel leaves zero); calls in a row, both forms and
    both tie rules, each equal to the oracle."""
    n = params.lwe_dim
    rng = np.random.default_rng(48)
    for rule in (L.TIE_RTL, L.TIE_GENERATOR):
        engine.set_tie_rule(rule)
        try:
            for count in (1, 5, 32, 33, 1):
                blwe = rng.integers(0, 2**64, (count, N + 1), dtype=np.uint64)
                d21 = to_dev(np.zeros((count, n + 1), np.uint32))
                d2n = to_dev(np.zeros((count, n + 1), np.uint32))
                engine.keyswitch(to_dev(blwe), d21, d2n, count)
                g21, g2n = from_dev(d21, np.uint32), from_dev(d2n, np.uint32)
                for c in range(count):
                    o21, o2n = oracle.keyswitch(blwe[c], keys["ksk"], n, N, gtv_top_tie=rule == L.TIE_GENERATOR)
                    assert np.array_equal(g21[c], o21) and np.array_equal(g2n[c], o2n), (rule, count, c)
        finally:
            engine.set_tie_rule(L.TIE_RTL)


@pytest.mark.parametrize("g", [1, 2])
def test_blind_rotate_matches_oracle(engine, params, oracle_bsk, g):
    rng = np.random.default_rng(50 + g)
    n, count = params.lwe_dim, 3
    lwe = rng.integers(0, 2 * N, (count, n + 1), dtype=np.uint32)
    lwe[1, :] = 0                                   # identity rotation
    lut = rng.integers(0, 2**64, (2, 2 * N), dtype=np.uint64)
    ids = np.array([0, 1, 1], np.uint32)
    engine.upload_luts(lut)
    engine.set_br_config(g, 1)
    d_out = to_dev(np.zeros((count, N + 1), np.uint64))
    engine.blind_rotate(to_dev(lwe), to_dev(ids), d_out, count)
    engine.check_device_error()
    got = from_dev(d_out, np.uint64)
    want = oracle_bsk.blind_rotate(lwe, lut, ids)
    for c in range(count):
        assert np.array_equal(got[c], want[c]), c


def _msgs_luts(params, rng, count, nlut):
    msgs = rng.integers(0, 16, count).astype(np.uint32)
    tables = [rng.integers(0, 16, 16).astype(np.uint32) for _ in range(nlut)]
    luts = np.stack([L.lut_build(params, t) for t in tables])
    return msgs, tables, luts


# On 148 SMs with two ciphertexts per CTA: 1 and 5 run one ciphertext per two
# SMs (cluster pairs); 100 one per SM (polynomials split over the CTA's
# groups); 301 = one full wave + a 5-ciphertext tail in cluster pairs; 450 =
# one full wave + a partial two-per-CTA wave of 154.  The oracle checks every
# ciphertext.
@pytest.mark.parametrize("count", [1, 5, 100, 301, 450])
def test_ks_pbs_bit_exact_and_decrypts(engine, params, keys, oracle_bsk, count):
    rng = np.random.default_rng(60 + count)
    msgs, tables, luts = _msgs_luts(params, rng, count, 3)
    ids = rng.integers(0, 3, count).astype(np.uint32)
    ct = L.encrypt(params, keys["glwe_key"], msgs, 1000 + count)
    engine.upload_luts(luts)
    engine.set_br_config(2, 1)
    d_out = to_dev(np.zeros_like(ct))
    engine.ks_pbs(to_dev(ct), to_dev(ids), d_out, count)
    engine.check_device_error()
    got = from_dev(d_out, np.uint64)
    dec = L.decrypt(params, keys["glwe_key"], got)
    assert [int(d) for d in dec] == [int(tables[i][m]) for i, m in zip(ids, msgs)]
    want = oracle_bsk.ks_pbs(keys["ksk"], ct, luts, ids)
    assert np.array_equal(got, want)


# The batch sizes of the benchmark's batched configuration (1, 17, 256, 1000,
# 4096 BLWEs, each batch with its own LUT), each as its own call, every
# ciphertext checked against the oracle.  On 148 SMs: 17 runs in cluster
# pairs, 256 as one partial two-per-CTA wave, 1000 as three waves and a
# 112-ciphertext tail of one per SM, 4096 as thirteen waves and a partial one.
def test_configured_batch_sizes_bit_exact(engine, params, keys, oracle_bsk):
    rng = np.random.default_rng(65)
    engine.set_br_config(2, 1)
    for count in (17, 256, 1000, 4096):
        msgs, tables, luts = _msgs_luts(params, rng, count, 1)
        ids = np.zeros(count, np.uint32)
        ct = L.encrypt(params, keys["glwe_key"], msgs, 2000 + count)
        engine.upload_luts(luts)
        d_out = to_dev(np.zeros_like(ct))
        engine.ks_pbs(to_dev(ct), to_dev(ids), d_out, count)
        engine.check_device_error()
        got = from_dev(d_out, np.uint64)
        want = oracle_bsk.ks_pbs(keys["ksk"], ct, luts, ids)
        assert np.array_equal(got, want), f"batch of {count}: rows {np.nonzero((got != want).any(1))[0][:8]}"


def test_generator_tie_rule_matches_oracle(engine, params, keys, oracle_bsk):
    """With the reference generator's tie rule (luthe_set_tie_rule) the engine
    equals the oracle in the same rule on every ciphertext, across a wave and
    a tail launch: about one bootstrap in three at n = 804 meets a tie in its
    blind rotation, and nearly every one in its key switch."""
    rng = np.random.default_rng(67)
    count = 301
    msgs, tables, luts = _msgs_luts(params, rng, count, 2)
    ids = rng.integers(0, 2, count).astype(np.uint32)
    ct = L.encrypt(params, keys["glwe_key"], msgs, 2301)
    engine.upload_luts(luts)
    engine.set_br_config(2, 1)
    d_in, d_ids = to_dev(ct), to_dev(ids)
    d_rtl, d_gen = to_dev(np.zeros_like(ct)), to_dev(np.zeros_like(ct))
    engine.ks_pbs(d_in, d_ids, d_rtl, count)
    engine.set_tie_rule(L.TIE_GENERATOR)
    try:
        engine.ks_pbs(d_in, d_ids, d_gen, count)
        engine.check_device_error()
    finally:
        engine.set_tie_rule(L.TIE_RTL)
    got = from_dev(d_gen, np.uint64)
    oracle.set_tie_rule(True)
    try:
        want = oracle_bsk.ks_pbs(keys["ksk"], ct, luts, ids)
    finally:
        oracle.set_tie_rule(False)
    assert np.array_equal(got, want)
    rtl = from_dev(d_rtl, np.uint64)
    assert (rtl != got).any(1).sum() > count // 2  # the rules differ in the ciphertexts
    dec = L.decrypt(params, keys["glwe_key"], got)
    assert [int(d) for d in dec] == [int(tables[i][m]) for i, m in zip(ids, msgs)]


def test_ks_pbs_host_and_graph(engine, params, keys, oracle_bsk):
    import torch
    rng = np.random.default_rng(70)
    count = 4
    msgs, tables, luts = _msgs_luts(params, rng, count, 2)
    ids = np.array([0, 1, 0, 1], np.uint32)
    ct = L.encrypt(params, keys["glwe_key"], msgs, 77)
    engine.upload_luts(luts)
    got_host = engine.ks_pbs_host(ct, ids)
    s = torch.cuda.Stream()
    d_in, d_ids, d_out = to_dev(ct), to_dev(ids), to_dev(np.zeros_like(ct))
    engine.reserve(count)
    for _ in range(2):  # capture, then replay
        engine.ks_pbs_graph(d_in, d_ids, d_out, count, s)
    s.synchronize()
    want = oracle_bsk.ks_pbs(keys["ksk"], ct, luts, ids)
    assert np.array_equal(got_host, want)
    assert np.array_equal(from_dev(d_out, np.uint64), want)


def test_lwe_ops_match_numpy(engine):
    rng = np.random.default_rng(80)
    count, dim = 3, N
    a = rng.integers(0, 2**64, (count, dim + 1), dtype=np.uint64)
    b = rng.integers(0, 2**64, (count, dim + 1), dtype=np.uint64)
    imm = 5
    cst = np.zeros(dim + 1, np.uint64)
    cst[dim] = np.uint64(imm) << np.uint64(59)
    with np.errstate(over="ignore"):
        want = {
            L.OP_ADD: a + b, L.OP_SUB: a - b, L.OP_MAC: a * np.uint64(imm) + b, L.OP_ADDS: a + cst,
            L.OP_SUBS: a - cst, L.OP_SSUB: cst - a, L.OP_MULS: a * np.uint64(imm),
        }
    d_a, d_b = to_dev(a), to_dev(b)
    for op, w in want.items():
        d_o = to_dev(np.zeros_like(a))
        engine.lwe_op(op, d_a, d_b, d_o, imm, count)
        assert np.array_equal(from_dev(d_o, np.uint64), w), op


def test_errors_are_reported(engine, params):
    with pytest.raises(L.LutheError):
        engine.set_br_config(3, 1)
    with pytest.raises(L.LutheError):
        engine.ks_pbs_host(np.zeros((1, N + 1), np.uint64), np.array([99], np.uint32))


def test_out_of_range_device_lut_id_is_flagged(engine, params, keys, oracle_bsk):
    # ids on the device cannot be checked by the host: the kernel flags them
    rng = np.random.default_rng(77)
    luts = np.stack([L.lut_build(params, rng.integers(0, 16, 16).astype(np.uint32)) for _ in range(2)])
    engine.upload_luts(luts)
    ct = L.encrypt(params, keys["glwe_key"], np.array([3, 5, 7], np.uint32), 9)
    ids = np.array([1, 9, 0], np.uint32)                  # 9 >= 2 uploaded LUTs
    d_out = to_dev(np.zeros((3, N + 1), np.uint64))
    engine.ks_pbs(to_dev(ct), to_dev(ids), d_out, 3)
    with pytest.raises(L.LutheError) as ei:
        engine.check_device_error()
    assert ei.value.code == L.E_PARAM
    engine.check_device_error()                           # the flag was cleared
    got = from_dev(d_out, np.uint64)
    ok = np.array([0, 2])                                 # the valid ids are unaffected
    want = oracle_bsk.ks_pbs(keys["ksk"], ct[ok], luts, ids[ok])
    assert np.array_equal(got[ok], want)


def test_graph_replay_of_wave_and_tail_equals_direct_launches(engine, params, keys):
    # 301 BLWEs: a two-per-CTA wave plus a tail launch, captured in one graph
    import torch
    rng = np.random.default_rng(90)
    msgs, tables, luts = _msgs_luts(params, rng, 301, 2)
    ids = rng.integers(0, 2, 301).astype(np.uint32)
    ct = L.encrypt(params, keys["glwe_key"], msgs, 91)
    engine.upload_luts(luts)
    engine.set_br_config(2, 1)
    d_in, d_ids = to_dev(ct), to_dev(ids)
    d_direct, d_graph = to_dev(np.zeros_like(ct)), to_dev(np.zeros_like(ct))
    engine.ks_pbs(d_in, d_ids, d_direct, 301)
    s = torch.cuda.Stream()
    for _ in range(2):  # capture, then replay
        engine.ks_pbs_graph(d_in, d_ids, d_graph, 301, s)
    s.synchronize()
    engine.check_device_error()
    assert np.array_equal(from_dev(d_graph, np.uint64), from_dev(d_direct, np.uint64))
    dec = L.decrypt(params, keys["glwe_key"], from_dev(d_graph, np.uint64))
    assert [int(d) for d in dec] == [int(tables[i][m]) for i, m in zip(ids, msgs)]
