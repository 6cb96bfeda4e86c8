"""CPU execution of DOp programs -- TEST INFRASTRUCTURE ONLY (the checker of
the serving loop).

A program is a list of 32-bit DOp words in the field layouts of the
reference's firmware header (fw/ublaze/src/hpu_dop_fmt.h:49-117) with the
opcodes of docs/dop.md:82-165: ADD SUB MAC ADDS SUBS SSUB MULS (linear DOps,
pea_alu_core.sv:59-61,124-161: the message constant is placed at the body as
cst << (64 - 5)), SYNC, LD/ST (source and destination blocks of the request)
and PBS / PBS_ML2/4/8 (| 0x08 flush), whose key switch and blind rotation run
through the oracle.  run_many executes several programs side by side, level
by level: every PBS ready in any program joins one oracle batch.
"""
import numpy as np

CST_SHIFT = 59


def _fields(w):
    return w >> 26, w & 0x7F, (w >> 7) & 0x7F, (w >> 14) & 0x7F


class _Req:
    def __init__(self, program, src, n_dst):
        self.words = [int(w) for w in program]
        self.src = src
        self.dst = [None] * n_dst
        self.regs = {}
        self.pc = 0


def _linear(r, w):
    op, d, s0, s1 = _fields(w)
    regs = r.regs
    with np.errstate(over="ignore"):
        if op == 0x20:
            regs[d] = r.src[(w >> 10) & 0xFFFF].copy()
        elif op == 0x21:
            r.dst[(w >> 10) & 0xFFFF] = regs[d].copy()
        elif op == 0x10:
            pass
        elif op in (0x01, 0x02, 0x05):
            a, b = regs[s0], regs[s1]
            if op == 0x01:
                regs[d] = a + b
            elif op == 0x02:
                regs[d] = a - b
            else:
                regs[d] = a * np.uint64((w >> 21) & 0x1F) + b
        elif op in (0x09, 0x0A, 0x0B, 0x0C):
            cst = (w >> 15) & 0x7FF
            a = regs[s0]
            c = np.zeros_like(a)
            c[-1] = np.uint64(cst) << np.uint64(CST_SHIFT)
            if op == 0x09:
                regs[d] = a + c
            elif op == 0x0A:
                regs[d] = a - c
            elif op == 0x0B:
                regs[d] = c - a
            else:
                regs[d] = a * np.uint64(cst)
        else:
            raise ValueError(f"unknown DOp opcode {op:#x}")


def run_many(requests, ksk, oracle_bsk, luts, **ks_args):
    """requests: [(program words, src [n_src][N+1] u64, n_dst)] -> list of
    [n_dst][N+1] outputs.  Within a program, a run of PBS DOps none of which
    reads a register written earlier in the run is one level."""
    reqs = [_Req(*r) for r in requests]
    while True:
        pending = []  # (req, [pbs words])
        for r in reqs:
            while r.pc < len(r.words) and (r.words[r.pc] >> 26) < 0x30:
                _linear(r, r.words[r.pc])
                r.pc += 1
            if r.pc >= len(r.words):
                continue
            batch, written = [], set()
            while r.pc < len(r.words) and (r.words[r.pc] >> 26) >= 0x30:
                w = r.words[r.pc]
                if ((w >> 7) & 0x7F) in written:
                    break
                k = 1 << (((w >> 26) & 0x7) & 0x3)
                batch.append(w)
                written.update(range(w & 0x7F, (w & 0x7F) + k))
                r.pc += 1
            pending.append((r, batch))
        if not pending:
            break
        for k in (1, 2, 4, 8):
            items = [(r, w) for r, b in pending for w in b if 1 << (((w >> 26) & 0x7) & 0x3) == k]
            if not items:
                continue
            cts = np.stack([r.regs[(w >> 7) & 0x7F] for r, w in items])
            gids = np.array([(w >> 14) & 0xFFF for _, w in items], np.uint32)
            out = oracle_bsk.ks_pbs(ksk, cts, luts, gids, mlk=k, **ks_args)
            for j, (r, w) in enumerate(items):
                for m in range(k):
                    r.regs[(w & 0x7F) + m] = out[j * k + m]
    return [np.stack(r.dst) for r in reqs]


def run(program, src, n_dst, ksk, oracle_bsk, luts, **ks_args):
    return run_many([(program, src, n_dst)], ksk, oracle_bsk, luts, **ks_args)[0]
