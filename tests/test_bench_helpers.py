"""Host logic of bench.py on the CPU: the blind-rotation launch count it
reports (mirroring launch_blind_rotate's shapes), the DRAM-traffic lookup from
the committed ncu record, and the CPU baselines of the NTT-product and
key-switch configurations against the oracle."""
import numpy as np

import bench
import luthe_b200 as L
import oracle


def test_blind_rotation_launches_per_step():
    # 148 SMs, two ciphertexts per CTA: a wave is 296
    assert bench.br_launches_per_step(1, 148, 2) == 1        # one small-batch launch
    assert bench.br_launches_per_step(148, 148, 2) == 1
    assert bench.br_launches_per_step(296, 148, 2) == 1      # exactly one wave
    assert bench.br_launches_per_step(301, 148, 2) == 2      # wave + 5-ciphertext tail launch
    assert bench.br_launches_per_step(450, 148, 2) == 1      # tail of 154 > 148 stays in the wave launch
    assert bench.br_launches_per_step(5370, 148, 2) == 2     # the benchmark: 18 waves + 42
    assert bench.br_launches_per_step(5370, 148, 1) == 1     # one per CTA: never split


def test_traffic_lookup():
    rec = {"commit": "abc", "captures": [{"ciphertexts": 5370, "dram_bytes": 1.6e8}],
           "traffic_model": {"from": 296, "fixed_bytes": 5.3e7, "bytes_per_ciphertext": 1.7e4}}
    full, how = bench.read_traffic(5370, rec)
    assert full == 1.6e8 and "5370" in how and "abc" in how
    small, how = bench.read_traffic(296, rec)
    assert small == 5.3e7 + 1.7e4 * 296 and "scaled" in how
    assert bench.read_traffic(296, None) == (None, None)
    assert bench.br_launches_per_step(5370, 148, 2, tail_max=0) == 1  # tuned: the tail stays in the wave launch


def test_cpu_baselines_are_bit_checked():
    rng = np.random.default_rng(3)
    P = np.uint64(0xFFFFFFFF00000001)
    a = rng.integers(0, 2**63, (2, 2048), dtype=np.uint64) % P
    b = rng.integers(0, 2**63, (2, 2048), dtype=np.uint64) % P
    res = bench.cpu_ntt_product(a, b, oracle.negacyclic_mul(a, b))
    assert res["bit_exact_vs_gpu"] and res["1_thread"]["pairs_per_s"] > 0
    bad = oracle.negacyclic_mul(a, b)
    bad[0, 0] ^= np.uint64(1)
    assert not bench.cpu_ntt_product(a, b, bad)["bit_exact_vs_gpu"]
    p = L.default_params(lwe_dim=16)
    keys = L.keygen(p, 1)
    blwe = rng.integers(0, 2**64, (2, 2049), dtype=np.uint64)
    want = np.stack([oracle.keyswitch(x, keys["ksk"], 16, 2048)[0] for x in blwe])
    res = bench.cpu_keyswitch(blwe, want, keys["ksk"], p)
    assert res["bit_exact_vs_gpu"] and res["all_threads"]["ciphertexts_per_s"] > 0
