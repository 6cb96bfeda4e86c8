#!/usr/bin/env python3
"""Benchmark of the batched KS+PBS hot path (TFHE n=804, k=1, N=2048, PBS 23x1,
KS 3x6 mod 2^21, Goldilocks NTT) on B200.

One step = one KS+PBS launch over the uneven batches 1+17+256+1000+4096
(5370 BLWEs, each batch with its own random LUT), inputs resident in HBM.
Prints one JSON line (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's KS+PBS algorithm on the host cores: the
reference's own CPU path is a prebuilt generator binary that is not shipped with
this tree, so the CPU restatement of it (oracle/, same algorithm, all host
threads) stands in, on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BATCHES = [1, 17, 256, 1000, 4096]
METRIC = "KS+PBS bootstraps/s on 1 B200, batched vs plain, bit-exact; p50/p99 op latency"
UNIT = "bootstraps/s"
MODMUL_PER_BOOTSTRAP = 804 * 53248          # 4 NTT-class transforms + BSK MAC per BR step
IMAD_PER_MODMUL = 4                         # 64x64->128 product as 4 32-bit IMAD
KS_MAC_PER_BOOTSTRAP = 2048 * 6 * 805
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-sample", type=int, default=48, help="ciphertexts in the CPU-baseline sample")
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-loop measurement")
    ap.add_argument("--no-param-sets", action="store_true",
                    help="skip the KS+PBS measurement of the reference's other parameter sets")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shape (profiling runs: no tuning trials among the launches)")
    ap.add_argument("--ncu-case", nargs="?", const="pbs", choices=("pbs", "other", "plain"),
                    help="small profiling case, then exit: 'pbs' (default) KS+PBS of 296 BLWEs (one persistent "
                         "wave), twice; 'other' the NTT product of 4096 pairs and the key switch of 16384 BLWEs, once "
                         "each; 'plain' KS+PBS of one BLWE (the 2-SM latency form), twice")
    return ap.parse_args()


def workload(L, params, keys, seed):
    rng = np.random.default_rng(seed)
    tables, msgs, ids = [], [], []
    for b, size in enumerate(BATCHES):
        tables.append(rng.integers(0, 16, 16).astype(np.uint32))
        msgs.append(rng.integers(0, 16, size).astype(np.uint32))
        ids.append(np.full(size, b, np.uint32))
    msgs, ids = np.concatenate(msgs), np.concatenate(ids)
    luts = np.stack([L.lut_build(params, t) for t in tables])
    ct = L.encrypt(params, keys["glwe_key"], msgs, seed + 1)
    expect = np.array([tables[i][m] for i, m in zip(ids, msgs)], np.uint32)
    return ct, ids, luts, expect


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.proc, self.path = index, None, None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        loaded = [s for s in sm if s > 0.5 * (max(sm) if sm else 0)]
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def ncu_record():
    """The ncu figures of the blind-rotation kernel kept in
    profiles/br_kernel_ncu.json (written from an ncu capture; it names the
    commit and the command it was captured with), or None."""
    path = os.path.join(ROOT, "profiles", "br_kernel_ncu.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def read_traffic(B, rec):
    """DRAM bytes (read + write) of one blind-rotation launch over B
    ciphertexts from the ncu record: the capture of a launch of this size when
    there is one, else the one-wave capture scaled as the BSK read once per
    launch plus the per-ciphertext bytes.  Returns (bytes, how)."""
    if not rec:
        return None, None
    for cap in rec.get("captures", []):
        if cap.get("ciphertexts") == B and cap.get("dram_bytes"):
            return cap["dram_bytes"], f"ncu, a launch of {B} ciphertexts (commit {cap.get('commit', rec.get('commit'))})"
    scale = rec.get("traffic_model")
    if scale:
        return (scale["fixed_bytes"] + scale["bytes_per_ciphertext"] * B,
                f"ncu, scaled from the {scale.get('from')}-ciphertext capture (commit {rec.get('commit')})")
    return None, None


class _OracleHost:
    """The host helpers the workload needs, from the oracle's own C code (the
    same values as the engine library's for the same seed), so that the CPU
    reference arm loads nothing from the engine library."""

    def __init__(self, oracle):
        self.o = oracle

    def lut_build(self, params, table):
        return self.o.lut_build(params.poly_size, table)

    def encrypt(self, params, glwe_key, msgs, seed):
        return self.o.encrypt(glwe_key, msgs, seed)

    def decrypt(self, params, glwe_key, blwe):
        return self.o.decrypt(glwe_key, blwe)


class _Params:
    lwe_dim, poly_size = 804, 2048


def reference_arm(args):
    import oracle
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    L = _OracleHost(oracle)
    params = _Params()
    keys = oracle.keygen(params.lwe_dim, params.poly_size, args.seed)
    ct, ids, luts, expect = workload(L, params, keys, args.seed)
    ob = oracle.OracleBsk(keys["bsk"], params.lwe_dim, params.poly_size)
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    sample = max(1, min(args.cpu_sample, threads * 4))
    times = []
    for step in range(args.warmup + args.steps):
        sl = slice((step * sample) % (len(ct) - sample), (step * sample) % (len(ct) - sample) + sample)
        t0 = time.perf_counter()
        out = ob.ks_pbs(keys["ksk"], ct[sl], luts, ids[sl])
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
        assert np.array_equal(L.decrypt(params, keys["glwe_key"], out), expect[sl])
    v = sample / statistics.mean(times)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": config_dict(),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{sample} BLWEs of the workload per step (KS+PBS), oracle/ CPU restatement"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def rank_seed(seed, rank):
    """Per-rank workload seed: replicas process independent ciphertexts."""
    return seed + 1000003 * rank


def max_over_ranks(x, dist, device):
    """The slowest rank's value (timing is the max over ranks)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def serving(L, eng, params, keys, seed, n_req=400, rate=300.0, ob=None, check_per_kind=8, window_us=0, fill=0,
            programs="fewest_pbs"):
    """Serving loop under Poisson arrivals of 16-bit radix IOps (50 % ADD with
    carry propagation, 30 % scalar compare, 20 % multiply); every result is
    checked by decryption, and with `ob` (an oracle BSK) the first
    `check_per_kind` requests of each kind bit for bit against the oracle's
    run of the same DOp programs (not timed).  `programs` picks the ADD
    program (MUL has one form, 101 PBS in 8 levels): "fewest_pbs" (ADD 8 PBS
    in 8 levels), "low_depth" (ADD 24 PBS in 5 levels) or "adaptive" (per
    request at submission, by the number of requests in flight:
    iops.programs_for_load)."""
    from luthe_b200 import iops as I
    prog_add, prog_mul = {"fewest_pbs": (I.prog_add, I.prog_mul), "adaptive": (I.prog_add, I.prog_mul),
                          "low_depth": (I.prog_add_prefix, I.prog_mul)}[programs]
    eng.upload_luts(np.stack([L.lut_build(params, t) for t in I.lut_tables()]))
    rng = np.random.default_rng(seed)
    kinds = rng.choice(3, size=n_req, p=[0.5, 0.3, 0.2])
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    vals = rng.integers(0, 65536, (n_req, 2))
    blocks, reqs, expect = [], [], []
    for r in range(n_req):
        a, b = int(vals[r, 0]), int(vals[r, 1])
        if kinds[r] == 0:
            reqs.append([prog_add(), 16, 8])
            expect.append((a + b) % 65536)
            blocks += I.to_blocks(a) + I.to_blocks(b)
        elif kinds[r] == 1:
            reqs.append([I.prog_cmp_gt(b), 8, 1])
            expect.append(int(a > b))
            blocks += I.to_blocks(a)
        else:
            reqs.append([prog_mul(), 16, 8])
            expect.append((a * b) % 65536)
            blocks += I.to_blocks(a) + I.to_blocks(b)
    n_low_add = len(I.prog_add_prefix())
    ct = L.encrypt(params, keys["glwe_key"], np.array(blocks, np.uint32), seed + 7)
    off = 0
    for r in reqs:
        r[1], off = ct[off:off + r[1]], off + r[1]
    srv = L.Server(eng, pool_bytes=4 << 30, max_pbs=4096)
    srv.set_batching(fill, window_us)
    srv.run([tuple(reqs[0]), tuple(reqs[1])])          # warm-up
    base = srv.counters()
    ids, outs, lat = [None] * n_req, {}, {}
    t0 = time.perf_counter()
    sub = 0
    while len(outs) < n_req:
        now = time.perf_counter() - t0
        while sub < n_req and arrivals[sub] <= now:
            if programs == "adaptive" and kinds[sub] == 0:
                reqs[sub][0] = I.programs_for_load(sub - len(outs))[0]()
            ids[sub] = srv.submit(*reqs[sub])
            sub += 1
        if sub == len(outs):
            time.sleep(max(0.0, min(0.002, arrivals[sub] - now)))
            continue
        srv.step()
        for r in range(sub):
            if r not in outs:
                got = srv.fetch(ids[r], reqs[r][2])
                if got is not None:
                    outs[r], lat[r] = got[0], got[1]
    wall = time.perf_counter() - t0
    cnt = {k: v - base[k] for k, v in srv.counters().items()}
    srv.close()
    ok = 0
    for r in range(n_req):
        dec = [int(x) for x in L.decrypt(params, keys["glwe_key"], outs[r])]
        ok += (I.from_blocks(dec) if reqs[r][2] == 8 else dec[0]) == expect[r]
    ls = np.array([lat[r] for r in range(n_req)]) * 1e3
    exact = None
    if ob is not None:
        from oracle import dops
        sel = [r for kind in range(3) for r in np.nonzero(kinds == kind)[0][:check_per_kind]]
        luts = np.stack([L.lut_build(params, t) for t in I.lut_tables()])
        want = dops.run_many([tuple(reqs[r]) for r in sel], keys["ksk"], ob, luts)
        eq = sum(bool(np.array_equal(outs[r], w)) for r, w in zip(sel, want))
        exact = f"{eq}/{len(sel)} (first {check_per_kind} requests of each kind, MUL included)"
    return {"requests": n_req, "arrival_rate_per_s": rate, "mix": "50% add, 30% scalar cmp, 20% mul (16-bit radix)",
            "programs": programs,
            "low_depth_share": (sum(len(r[0]) == n_low_add for r in reqs) / max(1, int((kinds == 0).sum()))
                                if programs == "adaptive" else None),
            "batching_window_us": window_us, "batching_fill": fill or "one wave (2 per SM)",
            "bit_exact_vs_oracle": exact,
            "throughput_requests_per_s": n_req / wall, "pbs_per_s": cnt["pbs"] / wall,
            "latency_ms_p50": float(np.percentile(ls, 50)), "latency_ms_p99": float(np.percentile(ls, 99)),
            "rounds": cnt["rounds"], "pbs": cnt["pbs"], "alu_dops": cnt["alu"], "launches": cnt["launches"],
            "results_decrypt_correct": f"{ok}/{n_req}"}


def param_set_runs(L, seed, steps, flush, stream):
    """KS+PBS throughput of each of the reference's other parameter sets on the
    same 5370-BLWE workload (fresh keys per set), decryption checked."""
    import torch
    res = {}
    for name in L.PARAM_SETS:
        if name == "default":
            continue
        p = L.param_set(name)
        keys = L.keygen(p, seed)
        ct, ids, luts, expect = workload(L, p, keys, seed + 1)
        B = len(ct)
        eng = L.Engine(p)
        eng.upload_keys(keys)
        eng.upload_luts(luts)
        eng.reserve(B)
        d_in = torch.from_numpy(ct.view(np.int64)).cuda()
        d_ids = torch.from_numpy(ids.view(np.int32)).cuda()
        d_out = torch.empty_like(d_in)
        eng.ks_pbs(d_in, d_ids, d_out, B, stream)
        torch.cuda.synchronize()
        ms = []
        for k in range(steps):
            flush.fill_(k)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.ks_pbs(d_in, d_ids, d_out, B, stream)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        eng.check_device_error()
        ok = bool(np.array_equal(L.decrypt(p, keys["glwe_key"], d_out.cpu().numpy().view(np.uint64)), expect))
        res[name] = {"lwe_dim": p.lwe_dim, "ks": f"{p.ks_base_log}x{p.ks_level}", "pbs_base_log": p.pbs_base_log,
                     "bootstraps_per_s": B * len(ms) / (sum(ms) * 1e-3), "ms_per_step": statistics.mean(ms),
                     "verified_decrypt": ok}
        eng.close()
        del d_in, d_ids, d_out
    return res


def cpu_ntt_product(a, b, gpu_out):
    """Config 1 on the host: the oracle's radix-2 NTT product (C) of the first
    64 pairs, 1 thread and all threads; bit-checked against the GPU rows."""
    import oracle
    res = {"kind": "port", "sample": f"first {len(a)} pairs of the 4096"}
    for label, th in (("1_thread", 1), ("all_threads", os.cpu_count() or 1)):
        oracle.set_threads(th)
        t0 = time.perf_counter()
        out = oracle.negacyclic_mul(a, b)
        dt = time.perf_counter() - t0
        res[label] = {"pairs_per_s": len(a) / dt, "threads": th}
    res["bit_exact_vs_gpu"] = bool(np.array_equal(out, gpu_out))
    return res


def cpu_keyswitch(blwe, gpu_out21, ksk, params):
    """Config 3 on the host: the oracle's key switch (C) of the first 64
    ciphertexts, 1 thread and all threads (one ciphertext per thread)."""
    import concurrent.futures as cf
    import oracle
    n, N = params.lwe_dim, params.poly_size
    one = lambda c: oracle.keyswitch(blwe[c], ksk, n, N)[0]
    res = {"kind": "port", "sample": f"first {len(blwe)} ciphertexts of the 16384"}
    t0 = time.perf_counter()
    outs = [one(c) for c in range(len(blwe))]
    res["1_thread"] = {"ciphertexts_per_s": len(blwe) / (time.perf_counter() - t0), "threads": 1}
    th = os.cpu_count() or 1
    with cf.ThreadPoolExecutor(th) as ex:                 # the C call releases the GIL
        t0 = time.perf_counter()
        list(ex.map(one, range(len(blwe))))
        res["all_threads"] = {"ciphertexts_per_s": len(blwe) / (time.perf_counter() - t0), "threads": th}
    res["bit_exact_vs_gpu"] = bool(np.array_equal(np.stack(outs), gpu_out21))
    return res


def hbm_peak_gbs():
    """The HBM copy bandwidth measured on this pool (MEASURED_PEAKS.json, when
    the file is present), else the pool's earlier measurement, 6650 GB/s."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = json.load(f).get("hbm_gbs")
        if v:
            return float(v), "measured (MEASURED_PEAKS.json)"
    except (OSError, ValueError):
        pass
    return 6650.0, "fallback (earlier measurement on this pool)"


def br_launches_per_step(B, nsm, g, tail_max=None):
    """Blind-rotation launches of one KS+PBS call (luthe_b200/csrc/kernels.cu,
    launch_blind_rotate): one, or two when a partial last wave of at most
    tail_max ciphertexts (default: the SM count) is split off into its own
    launch."""
    wave = nsm * g
    tail = B % wave
    tail_max = nsm if tail_max is None or tail_max < 0 else tail_max
    return 2 if (g > 1 and B > wave and 0 < tail <= tail_max) else 1


def config_dict():
    return {
        "workload": "batched KS+PBS of uneven batches 1+17+256+1000+4096 = 5370 BLWEs in one call, "
                    "each batch its own random 4-bit LUT; TFHE n=804 k=1 N=2048 PBS 23x1 KS 3x6 mod 2^21, "
                    "NTT mod 2^64-2^32+1",
        "launch": "one CUDA graph per step (luthe_ks_pbs_graph): key switch + persistent blind rotation "
                  "(+ a tail launch when the last wave is partial)",
        "batches": BATCHES, "ciphertexts_per_step": sum(BATCHES),
        "l2": "flushed between timed steps (256 MiB device write); BSK 52.7 MB and KSK 44 MB are L2-resident "
              "by design inside a step",
        "parallelism": "replicas (one independent engine per GPU, no collective on the data path)",
    }


def ncu_case(B=296):
    """KS+PBS of B identity-LUT BLWEs twice (296: one persistent wave, the case
    the blind-rotation ncu summaries under profiles/ are captured on; 1: the
    plain path), checked by decryption."""
    import torch
    import luthe_b200 as L
    p = L.default_params()
    k = L.keygen(p, 3)
    with L.Engine(p) as e:
        e.upload_keys(k)
        e.upload_luts(L.lut_build(p, np.arange(16, dtype=np.uint32)))
        ct = L.encrypt(p, k["glwe_key"], np.arange(B, dtype=np.uint32) % 16, 5)
        d_in = torch.from_numpy(ct.view(np.int64)).cuda()
        d_out = torch.empty_like(d_in)
        ids = torch.zeros(B, dtype=torch.int32, device="cuda")
        for _ in range(2):
            e.ks_pbs(d_in, ids, d_out, B)
        torch.cuda.synchronize()
        e.check_device_error()
        dec = L.decrypt(p, k["glwe_key"], d_out.cpu().numpy().view(np.uint64))
    assert np.array_equal(dec, np.arange(B) % 16)
    print("ncu case ok")


def ncu_case_other():
    """Configurations 1 and 3 once each at their full sizes (201 MB and 268 MB
    of inputs): the NTT product of 4096 polynomial pairs and the key switch of
    16384 BLWEs of dimension 2048, checked against the oracle on 4 rows."""
    import torch
    import luthe_b200 as L
    import oracle
    p = L.default_params()
    k = L.keygen(p, 3)
    g = torch.Generator(device="cuda").manual_seed(11)
    with L.Engine(p) as e:
        e.upload_keys(k)
        pa = torch.randint(0, 2**62, (4096, 2048), dtype=torch.int64, device="cuda", generator=g)
        pb = torch.randint(0, 2**62, (4096, 2048), dtype=torch.int64, device="cuda", generator=g)
        po = torch.empty_like(pa)
        e.ntt_mul(pa, pb, po, 4096)
        ks_in = torch.randint(-2**62, 2**62, (16384, 2049), dtype=torch.int64, device="cuda", generator=g)
        o21 = torch.empty((16384, p.lwe_dim + 1), dtype=torch.int32, device="cuda")
        o2n = torch.empty_like(o21)
        e.keyswitch(ks_in, o21, o2n, 16384)
        torch.cuda.synchronize()
        e.check_device_error()
        a4, b4, o4 = (x[:4].cpu().numpy().view(np.uint64) for x in (pa, pb, po))
        assert np.array_equal(o4, oracle.negacyclic_mul(a4, b4))
        k4, r4 = ks_in[:4].cpu().numpy().view(np.uint64), o21[:4].cpu().numpy().view(np.uint32)
        for c in range(4):
            assert np.array_equal(r4[c], oracle.keyswitch(k4[c], k["ksk"], p.lwe_dim, p.poly_size)[0])
    print("ncu case other ok")


def main():
    args = parse()
    if args.ncu_case:
        if args.ncu_case == "other":
            return ncu_case_other()
        return ncu_case(1 if args.ncu_case == "plain" else 296)
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    import luthe_b200 as L

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    params = L.default_params()
    keys = L.keygen(params, args.seed)
    ct, ids, luts, expect = workload(L, params, keys, rank_seed(args.seed, rank))
    B = len(ct)
    eng = L.Engine(params, device=local)
    eng.upload_keys(keys)
    eng.upload_luts(luts)
    tune = {"chosen": None, "skipped": "--no-autotune"} if args.no_autotune else eng.autotune(0)
    eng.reserve(B)

    d_in = torch.from_numpy(ct.view(np.int64)).cuda()
    d_ids = torch.from_numpy(ids.view(np.int32)).cuda()
    d_out = torch.empty_like(d_in)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    # the step is replayed from a CUDA graph (luthe_ks_pbs_graph: captured on
    # the first call, a non-default stream); flush and events go on that stream
    gstream = torch.cuda.Stream()

    def step():
        eng.ks_pbs_graph(d_in, d_ids, d_out, B, gstream)

    torch.cuda.synchronize()
    for _ in range(args.warmup):
        with torch.cuda.stream(gstream):
            flush.fill_(1)
        step()
    torch.cuda.synchronize()
    eng.check_device_error()
    got = L.decrypt(params, keys["glwe_key"], d_out.cpu().numpy().view(np.uint64))
    verified = bool(np.array_equal(got, expect))

    # ---- timed region: K steps, L2 flushed between them (outside the events)
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    evs = []
    for k in range(args.steps):
        with torch.cuda.stream(gstream):
            flush.fill_(k)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(gstream)
        step()
        e1.record(gstream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    clk = clocks.stop()
    step_out = d_out.cpu().numpy().view(np.uint64).copy()  # the timed step's outputs, checked at the end
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(sum(step_ms), dist, "cuda")
    if dist:
        dist.barrier()
    ms_per_step = total_ms / args.steps
    value = world * B * args.steps / (total_ms * 1e-3)

    # ---- dominant kernel: the blind rotation alone, CUDA events on its stream
    d_l2n = torch.empty((B, params.lwe_dim + 1), dtype=torch.int32, device="cuda")
    eng.keyswitch(d_in, None, d_l2n, B, stream)
    br_ms = []
    for r in range(3):
        flush.fill_(r)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.blind_rotate(d_l2n, d_ids, d_out, B, stream)
        e1.record(stream)
        e1.synchronize()
        br_ms.append(e0.elapsed_time(e1))
    br_s = statistics.median(br_ms) * 1e-3
    imad_peak, glmul_peak = L.measure_int_peak(local)
    achieved_imad = B * MODMUL_PER_BOOTSTRAP * IMAD_PER_MODMUL / br_s
    ncu = ncu_record()
    traffic, traffic_how = read_traffic(B, ncu)

    # ---- plain path: one ciphertext per launch
    plain_ms = []
    one_in, one_id, one_out = d_in[:1], d_ids[:1], d_out[:1]
    for r in range(8):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.ks_pbs(one_in, one_id, one_out, 1, stream)
        e1.record(stream)
        e1.synchronize()
        if r >= 2:
            plain_ms.append(e0.elapsed_time(e1))

    # ---- end to end through the host-buffer API (pinned memory, copies timed)
    h_in = torch.from_numpy(ct.view(np.int64)).pin_memory()
    h_ids = torch.from_numpy(ids.view(np.int32)).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    hin, hid, hout = (h_in.numpy().view(np.uint64), h_ids.numpy().view(np.uint32), h_out.numpy().view(np.uint64))
    eng.ks_pbs_host(hin, hid, hout)  # warm the staging buffers
    e2e_ms = []
    for r in range(max(2, min(args.steps, 3))):
        flush.fill_(r)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        eng.ks_pbs_host(hin, hid, hout)
        e1.record(torch.cuda.default_stream())
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    e2e_verified = bool(np.array_equal(L.decrypt(params, keys["glwe_key"], hout), expect))
    e2e_val = world * B / (max_over_ranks(statistics.mean(e2e_ms), dist, "cuda") * 1e-3)

    # ---- the other configurations: standalone NTT product and key switch
    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        ts = []
        for r in range(reps):
            flush.fill_(r)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            fn()
            a1.record(stream)
            a1.synchronize()
            ts.append(a0.elapsed_time(a1))
        return statistics.median(ts)

    P = 0xFFFFFFFF00000001
    g = torch.Generator(device="cuda").manual_seed(args.seed)
    pa = torch.randint(0, 2**62, (4096, 2048), dtype=torch.int64, device="cuda", generator=g)
    pb = torch.randint(0, 2**62, (4096, 2048), dtype=torch.int64, device="cuda", generator=g)
    po = torch.empty_like(pa)
    ntt_ms = timed(lambda: eng.ntt_mul(pa, pb, po, 4096, stream))
    ntt_sample = (pa[:64].cpu().numpy().view(np.uint64), pb[:64].cpu().numpy().view(np.uint64),
                  po[:64].cpu().numpy().view(np.uint64))
    del pa, pb, po
    ks_in = torch.randint(-2**62, 2**62, (16384, 2049), dtype=torch.int64, device="cuda", generator=g)
    ks_o21 = torch.empty((16384, params.lwe_dim + 1), dtype=torch.int32, device="cuda")
    ks_o2n = torch.empty_like(ks_o21)
    ks_ms = timed(lambda: eng.keyswitch(ks_in, ks_o21, ks_o2n, 16384, stream))
    ks_sample = (ks_in[:64].cpu().numpy().view(np.uint64), ks_o21[:64].cpu().numpy().view(np.uint32))
    del ks_in, ks_o21, ks_o2n
    hbm_peak, hbm_src = hbm_peak_gbs()
    other = {
        "ntt_product_4096_pairs": {
            "ms": ntt_ms, "pairs_per_s": 4096 / (ntt_ms * 1e-3),
            "modmul_per_s": 4096 * 35840 / (ntt_ms * 1e-3),
            "hbm_gbs_algorithmic": 4096 * 3 * 2048 * 8 / (ntt_ms * 1e-3) / 1e9,
            "hbm_frac": 4096 * 3 * 2048 * 8 / (ntt_ms * 1e-3) / 1e9 / hbm_peak, "hbm_peak_gbs": hbm_peak,
            "hbm_peak_source": hbm_src,
            "imad_frac_of_measured_peak": 4096 * 35840 * IMAD_PER_MODMUL / (ntt_ms * 1e-3) / imad_peak,
            "note": "N=2048 pairs, uniform in [0,2^62); 3 transforms + product per pair"},
        "keyswitch_16384": {
            "ms": ks_ms, "ciphertexts_per_s": 16384 / (ks_ms * 1e-3),
            "mac_per_s": 16384 * KS_MAC_PER_BOOTSTRAP / (ks_ms * 1e-3),
            "imad_frac_of_measured_peak": 16384 * KS_MAC_PER_BOOTSTRAP / (ks_ms * 1e-3) / imad_peak,
            "note": "16384 BLWEs of dimension 2048 -> n=804, KSK 3x6 mod 2^21"},
    }

    # ---- the reference's other parameter sets (one GPU)
    psets = None
    if world == 1 and not args.no_param_sets:
        psets = param_set_runs(L, args.seed + 7, 3, flush, stream)

    # CPU restatements of configs 1 and 3 (the oracle, C; 1 thread and all
    # host threads) on bounded samples, checked against the GPU rows
    if rank == 0 and world == 1 and args.cpu_sample > 0:
        other["ntt_product_4096_pairs"]["cpu"] = cpu_ntt_product(*ntt_sample)
        other["keyswitch_16384"]["cpu"] = cpu_keyswitch(*ks_sample, keys["ksk"], params)

    # ---- serving loop (one GPU): Poisson arrivals of radix IOps
    # at 300 req/s offered (above the loop's capacity for this mix: the queue
    # grows) and at 150 req/s (inside it)
    serve = serve_light = serve_win = serve_light_win = serve_pfx = serve_light_pfx = serve_ad = serve_light_ad = None
    if world == 1 and not args.no_serving:
        import oracle
        serve_ob = oracle.OracleBsk(keys["bsk"], params.lwe_dim, params.poly_size) if args.cpu_sample > 0 else None
        serve = serving(L, eng, params, keys, args.seed + 99, ob=serve_ob)
        serve_light = serving(L, eng, params, keys, args.seed + 98, rate=150.0)
        # the same loads with a batching window: partial PBS batches wait up
        # to 3 ms for more work while another batch is on the GPU
        serve_win = serving(L, eng, params, keys, args.seed + 99, window_us=3000)
        serve_light_win = serving(L, eng, params, keys, args.seed + 98, rate=150.0, window_us=3000)
        # the same loads with the prefix ADD (5 PBS levels instead of 8, 24 PBS
        # instead of 8)
        serve_pfx = serving(L, eng, params, keys, args.seed + 99, ob=serve_ob, programs="low_depth")
        serve_light_pfx = serving(L, eng, params, keys, args.seed + 98, rate=150.0, programs="low_depth")
        # and with the programs chosen per request by the load at submission
        serve_ad = serving(L, eng, params, keys, args.seed + 99, ob=serve_ob, programs="adaptive")
        serve_light_ad = serving(L, eng, params, keys, args.seed + 98, rate=150.0, programs="adaptive")

    # ---- CPU baseline (rank 0, one GPU): the CPU restatement on all host cores
    cpu = None
    if rank == 0 and world == 1 and args.cpu_sample > 0:
        import oracle
        threads = os.cpu_count() or 1
        oracle.set_threads(threads)
        ob = oracle.OracleBsk(keys["bsk"], params.lwe_dim, params.poly_size)
        s = min(args.cpu_sample, B)
        t0 = time.perf_counter()
        out = ob.ks_pbs(keys["ksk"], ct[:s], luts, ids[:s])
        dt = time.perf_counter() - t0
        cpu = {"value": s / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"first {s} BLWEs of the workload, KS+PBS, {dt:.1f} s",
               "bit_exact_vs_gpu": bool(np.array_equal(out, step_out[:s]))}
        # every output of the timed step against the oracle (not timed)
        t0 = time.perf_counter()
        want = ob.ks_pbs(keys["ksk"], ct, luts, ids)
        eq = int((want == step_out).all(axis=1).sum())
        cpu["bit_exact_all"] = f"{eq}/{B}"
        cpu["bit_exact_all_s"] = round(time.perf_counter() - t0, 1)

    # our kernels inside the timed region: per step one key switch and one or
    # two blind-rotation launches
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    chosen = tune.get("chosen") or {}
    launches = args.steps * (1 + br_launches_per_step(B, nsm, chosen.get("cts_per_cta", 2), chosen.get("tail_max")))

    if rank == 0:
        q = lambda xs, p: float(np.percentile(xs, p))
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": config_dict(),
            "verified_decrypt": verified and e2e_verified,
            "latency_ms": {"batch_step_p50": q(step_ms, 50), "batch_step_p99": q(step_ms, 99),
                           "plain_p50": q(plain_ms, 50), "plain_p99": q(plain_ms, 99)},
            "plain_bootstraps_per_s": 1e3 / statistics.mean(plain_ms),
            "batched_over_plain": value / world / (1e3 / statistics.mean(plain_ms)),
            "roofline": {"bound": "int", "kernel": "br_kernel", "achieved": achieved_imad / 1e12,
                         "peak": imad_peak / 1e12, "unit": "TIMAD/s", "frac": achieved_imad / imad_peak,
                         "peak_source": "measured live (luthe_measure_int_peak, 32-bit IMAD probe)",
                         "work": f"{MODMUL_PER_BOOTSTRAP} modmul x {IMAD_PER_MODMUL} IMAD per bootstrap",
                         "traffic": traffic, "traffic_unit": f"DRAM bytes per launch ({traffic_how})",
                         "modmul_frac": B * MODMUL_PER_BOOTSTRAP / br_s / glmul_peak,
                         "glmul_peak_per_s": glmul_peak, "br_ms": br_s * 1e3,
                         "ncu": ncu and {k: ncu.get(k) for k in ("commit", "kernel", "command", "pipes", "l2",
                                                                   "warp_instructions_per_ciphertext_step")}},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(ct.nbytes + ids.nbytes),
                    "d2h_bytes_per_step": int(ct.nbytes), "ms_per_step": statistics.mean(e2e_ms)},
            "gpu_launches": launches,
            "clocks": clk,
            "autotune": tune,
            "serving": serve,
            "serving_150": serve_light,
            "serving_window_3ms": serve_win,
            "serving_150_window_3ms": serve_light_win,
            "serving_low_depth": serve_pfx,
            "serving_150_low_depth": serve_light_pfx,
            "serving_adaptive": serve_ad,
            "serving_150_adaptive": serve_light_ad,
            "other_configs": other,
            "param_sets": psets,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
