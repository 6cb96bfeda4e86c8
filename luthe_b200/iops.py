"""Radix-integer IOps as DOp programs for the serving loop.

The reference expands integer operations (IOps, docs/iop.md) into digit
operations (DOps, docs/dop.md) in its firmware and TFHE-rs backend (the DOp
programs themselves are not in the reference).  Here the expansion is written
from the documented semantics: a 16-bit integer is 8 blocks (digits) of a
2-bit message with 2 carry bits of headroom and a padding bit; ALU DOps are
exact on the payload while it stays below 16; a PBS applies a 16-entry LUT and
cleans the noise.  Programs are 32-bit DOp words in the field layouts of
fw/ublaze/src/hpu_dop_fmt.h:49-117 (opcodes: include/luthe.h).

    ADD      a + b mod 2^16: blockwise ADD, then a carry chain of PBS_ML2
             (message and carry of a block from one blind rotation)
    ADD (prefix)  the same sum with the carries resolved by a parallel prefix
             of block carry states: 5 PBS levels instead of 8, 24 PBS
             instead of 8
    CMP_GT   a > k for a clear 16-bit k: per-block sign PBS, a 3-level tree of
             bivariate combine PBS (MSB block decides) whose root maps to {0, 1}
    MUL      a * b mod 2^16: schoolbook digit products (bivariate PBS on
             MAC-packed a_i * 4 + b_j, low and high halves), then per-column
             carry-save reduction in groups of up to 5 terms, earliest-ready
             terms first (101 PBS, 8 levels)

prog_add takes the fewest PBS, prog_add_prefix the fewest sequential PBS
levels; programs_for_load picks between them by load.
"""
import numpy as np

BLOCKS = 8
MSG_BITS = 2
OPC = dict(ADD=0x01, SUB=0x02, MAC=0x05, ADDS=0x09, SUBS=0x0A, SSUB=0x0B, MULS=0x0C, SYNC=0x10, LD=0x20, ST=0x21,
           PBS=0x30, PBS_ML2=0x31, PBS_ML4=0x32, PBS_ML8=0x33)
MEM_HEAP, MEM_SRC, MEM_DST = 1, 2, 3

# ------------------------------------------------------------------ LUTs
# 16-entry tables on the 4-bit payload x = carry*4 + msg (docs/dop.md:136-159 aliases)


def _many(*fs):
    """Many-LUT table: k functions of an input < 16/k, packed in consecutive blocks."""
    k = len(fs)
    span = 16 // k
    return [fs[b // span](b % span) for b in range(16)]


LUTS = {
    "None": [x for x in range(16)],
    "MsgOnly": [x & 3 for x in range(16)],
    "CarryInMsg": [x >> 2 for x in range(16)],
    "MultCarryMsgLsb": [((x >> 2) * (x & 3)) & 3 for x in range(16)],
    "MultCarryMsgMsb": [((x >> 2) * (x & 3)) >> 2 for x in range(16)],
    "ManyCarryMsg": _many(lambda x: x & 3, lambda x: x >> 2),
    "CmpCombine": [(x >> 2) if (x >> 2) != 1 else (x & 3) for x in range(16)],
    "IsTwo": [1 if x == 2 else 0 for x in range(16)],
    # the compare's last combine and the final "greater" test in one table
    "CmpCombineIsTwo": [1 if ((x >> 2) if (x >> 2) != 1 else (x & 3)) == 2 else 0 for x in range(16)],
    # carry state of a block sum s = a_i + b_i <= 6: 2 generates, 1 propagates, 0 stops
    "BlockState": [2 if x >= 4 else 1 if x == 3 else 0 for x in range(16)],
    "BlockState0": [2 if x >= 4 else 0 for x in range(16)],  # no carry into block 0
    "HalfMsg": [(x >> 1) & 3 for x in range(16)],             # (2 s + 2 c) / 2 mod 4
}
for _k in range(4):
    LUTS[f"Cmp{_k}"] = [0 if (x & 3) < _k else 1 if (x & 3) == _k else 2 for x in range(16)]
LUT_NAMES = list(LUTS)
LUT_ID = {name: i for i, name in enumerate(LUT_NAMES)}


def lut_tables():
    """[nlut][16] tables in LUT-id order (upload with luthe_lut_build per table)."""
    return [LUTS[name] for name in LUT_NAMES]


# ------------------------------------------------------------- assembler

def enc_arith(op, dst, s0, s1=0, mul=0):
    return (OPC[op] << 26) | ((mul & 0x1F) << 21) | ((s1 & 0x7F) << 14) | ((s0 & 0x7F) << 7) | (dst & 0x7F)


def enc_arith_msg(op, dst, s0, cst):
    return (OPC[op] << 26) | ((cst & 0x7FF) << 15) | ((s0 & 0x7F) << 7) | (dst & 0x7F)


def enc_mem(op, rid, mode, slot):
    return (OPC[op] << 26) | ((slot & 0xFFFF) << 10) | ((mode & 3) << 8) | (rid & 0x7F)


def enc_pbs(op, dst, src, gid):
    return (OPC[op] << 26) | ((gid & 0xFFF) << 14) | ((src & 0x7F) << 7) | (dst & 0x7F)


class Program:
    """DOp program builder with a register allocator over the 128-entry file.

    Freed registers are reused first in, first out.  The scheduler orders a
    write after every earlier read of the same register (write-after-read), so
    handing out the register freed last would make each new value wait for the
    PBS that read the old one: that way an earlier MUL program, 14 PBS levels
    deep by its data, took 45, and the compare 12 instead of 5.
    """

    def __init__(self, n_src, n_dst):
        self.words = []
        self.n_src, self.n_dst = n_src, n_dst
        self.free = list(range(128))  # least recently freed first

    def reg(self):
        return self.free.pop(0)

    def pair(self, k=2):
        """k consecutive registers starting at a multiple of k (many-LUT
        destination): of the aligned free blocks, the one freed longest ago."""
        pos = {r: i for i, r in enumerate(self.free)}
        blocks = [b for b in range(0, 128, k) if all(r in pos for r in range(b, b + k))]
        if not blocks:
            raise RuntimeError("register file exhausted")
        base = min(blocks, key=lambda b: max(pos[r] for r in range(b, b + k)))
        for r in range(base, base + k):
            self.free.remove(r)
        return base

    def release(self, *rs):
        for r in rs:
            if r not in self.free:
                self.free.append(r)

    def ld(self, r, src_block):
        self.words.append(enc_mem("LD", r, MEM_SRC, src_block))

    def st(self, dst_block, r):
        self.words.append(enc_mem("ST", r, MEM_DST, dst_block))

    def add(self, d, a, b):
        self.words.append(enc_arith("ADD", d, a, b))

    def mac(self, d, a, b, f):
        self.words.append(enc_arith("MAC", d, a, b, f))

    def pbs(self, d, s, lut):
        self.words.append(enc_pbs("PBS", d, s, LUT_ID[lut]))

    def pbs_ml2(self, d, s, lut):
        self.words.append(enc_pbs("PBS_ML2", d, s, LUT_ID[lut]))

    def array(self):
        return np.array(self.words, np.uint32)


def prog_add():
    """a (src blocks 0..7) + b (src 8..15) -> dst blocks 0..7, mod 2^16."""
    p = Program(2 * BLOCKS, BLOCKS)
    a = [p.reg() for _ in range(BLOCKS)]
    b = [p.reg() for _ in range(BLOCKS)]
    for i in range(BLOCKS):
        p.ld(a[i], i)
        p.ld(b[i], BLOCKS + i)
    carry = None
    for i in range(BLOCKS):
        p.add(a[i], a[i], b[i])                   # <= 6
        p.release(b[i])
        if carry is not None:
            p.add(a[i], a[i], carry)              # <= 7
            p.release(carry)
        if i < BLOCKS - 1:
            d = p.pair(2)
            p.pbs_ml2(d, a[i], "ManyCarryMsg")    # d: msg, d+1: carry
            p.st(i, d)
            p.release(d, a[i])
            carry = d + 1
        else:
            d = p.reg()
            p.pbs(d, a[i], "MsgOnly")
            p.st(i, d)
    return p.array()


def prog_add_prefix():
    """a + b mod 2^16 with the carries resolved by a parallel prefix: 5 PBS
    levels instead of the ripple chain's 8, for 24 PBS instead of 8.

    Level 1 classifies each block sum s_i = a_i + b_i (<= 6) as generate (2),
    propagate (1) or stop (0) (block 0: generate or stop, no carry comes in);
    three Sklansky rounds combine the states of blocks 0..i with the compare
    program's combine LUT (the upper state unless it propagates); the prefix
    of blocks 0..i-1 is then 0 or 2, and block i's digit is (2 s_i + prefix) / 2
    mod 4 from one more PBS.
    """
    p = Program(2 * BLOCKS, BLOCKS)
    a = [p.reg() for _ in range(BLOCKS)]
    b = [p.reg() for _ in range(BLOCKS)]
    for i in range(BLOCKS):
        p.ld(a[i], i)
        p.ld(b[i], BLOCKS + i)
    for i in range(BLOCKS):
        p.add(a[i], a[i], b[i])                   # s_i <= 6
        p.release(b[i])
    d = p.reg()
    p.pbs(d, a[0], "MsgOnly")
    p.st(0, d)
    p.release(d)
    pre = []
    for i in range(BLOCKS - 1):
        r = p.reg()
        p.pbs(r, a[i], "BlockState0" if i == 0 else "BlockState")
        pre.append(r)
    p.release(a[0])
    span = 1
    while span < BLOCKS - 1:                      # pre[i]: state of blocks (i - i mod 2 span) .. i
        new = list(pre)
        for i in range(BLOCKS - 1):
            if (i // span) % 2 == 1:
                j = (i // span) * span - 1        # last block of the lower half
                x = p.reg()
                p.mac(x, pre[i], pre[j], 4)       # hi * 4 + lo <= 10
                r = p.reg()
                p.pbs(r, x, "CmpCombine")
                p.release(x)
                new[i] = r
        p.release(*[old for old, nw in zip(pre, new) if old != nw])
        pre, span = new, 2 * span
    for i in range(1, BLOCKS):
        y = p.reg()
        p.mac(y, a[i], pre[i - 1], 2)             # 2 s_i + (0 or 2) <= 14
        d = p.reg()
        p.pbs(d, y, "HalfMsg")
        p.st(i, d)
        p.release(y, d, a[i])
    p.release(*pre)
    return p.array()


def prog_cmp_gt(k):
    """a (src blocks 0..7) > k (clear 16-bit) -> dst block 0 in {0, 1}."""
    p = Program(BLOCKS, 1)
    a = [p.reg() for _ in range(BLOCKS)]
    for i in range(BLOCKS):
        p.ld(a[i], i)
    cmp = []
    for i in range(BLOCKS):
        d = p.reg()
        p.pbs(d, a[i], f"Cmp{(k >> (2 * i)) & 3}")
        cmp.append(d)
        p.release(a[i])
    while len(cmp) > 1:                           # cmp[i]: block i, higher index = more significant
        nxt = []
        last = len(cmp) == 2                      # the root: combine and test "greater" at once
        for lo, hi in zip(cmp[0::2], cmp[1::2]):
            x = p.reg()
            p.mac(x, hi, lo, 4)                   # hi * 4 + lo <= 10
            d = p.reg()
            p.pbs(d, x, "CmpCombineIsTwo" if last else "CmpCombine")
            p.release(x, hi, lo)
            nxt.append(d)
        cmp = nxt
    p.st(0, cmp[0])
    return p.array()


def prog_mul():
    """a (src 0..7) * b (src 8..15) -> dst blocks 0..7, mod 2^16: 101 PBS in 8
    levels.

    Digit products a_i * b_j (i + j = k) as bivariate PBS on the MAC-packed
    a_i * 4 + b_j: the low half into column k, the high half into column k+1
    (level 1).  Each column is then reduced in groups of up to 5 terms (each
    <= 3, sum <= 15) to a message (stays) and a carry (to the next column; the
    top column keeps the message only), always grouping the terms that are
    ready earliest: carries arrive from the column below at later levels, and
    grouping in arrival order instead of readiness gave 14 levels for the same
    PBS count.
    """
    p = Program(2 * BLOCKS, BLOCKS)
    a = [p.reg() for _ in range(BLOCKS)]
    b = [p.reg() for _ in range(BLOCKS)]
    for i in range(BLOCKS):
        p.ld(a[i], i)
        p.ld(b[i], BLOCKS + i)
    cols = [[] for _ in range(BLOCKS)]            # (PBS level at which it is ready, register)
    for k in range(BLOCKS):
        for i in range(k + 1):                    # digit products a_i * b_j, i + j = k
            x = p.reg()
            p.mac(x, a[i], b[k - i], 4)           # a_i * 4 + b_j
            lo = p.reg()
            p.pbs(lo, x, "MultCarryMsgLsb")
            cols[k].append((1, lo))
            if k + 1 < BLOCKS:
                hi = p.reg()
                p.pbs(hi, x, "MultCarryMsgMsb")
                cols[k + 1].append((1, hi))
            p.release(x)
    p.release(*a, *b)
    for k in range(BLOCKS):
        terms = cols[k]
        while len(terms) > 1:
            terms.sort()
            grp, terms = terms[:5], terms[5:]
            level = max(lv for lv, _ in grp) + 1
            s = grp[0][1]
            for _, t in grp[1:]:
                p.add(s, s, t)
                p.release(t)
            m = p.reg()
            p.pbs(m, s, "MsgOnly")
            terms.append((level, m))
            if k + 1 < BLOCKS:
                c = p.reg()
                p.pbs(c, s, "CarryInMsg")
                cols[k + 1].append((level, c))
            p.release(s)
        p.st(k, terms[0][1])
        p.release(terms[0][1])
    return p.array()


def programs_for_load(in_flight, light=16):
    """(ADD, MUL) program builders for a request submitted while `in_flight`
    requests are queued or running: the prefix ADD while the loop is light
    (fewer sequential PBS, lower latency while the GPU has room), the ripple
    ADD once it is loaded (the prefix form's extra PBS then queue behind each
    other).  MUL has one form: its fewest-PBS program is also its shallowest."""
    return (prog_add_prefix if in_flight < light else prog_add), prog_mul


# ------------------------------------------------------ plaintext reference

def run_plain(words, src, n_dst):
    """Execute a DOp program on clear payloads (the 5-bit padded space) with
    the LUT semantics of a PBS; asserts that every PBS input stays below 16."""
    regs = [0] * 128
    dst = [0] * n_dst
    tables = lut_tables()
    for w in (int(x) for x in words):
        op = w >> 26
        d, s0, s1 = w & 0x7F, (w >> 7) & 0x7F, (w >> 14) & 0x7F
        if op == OPC["LD"]:
            regs[d] = src[(w >> 10) & 0xFFFF] % 32
        elif op == OPC["ST"]:
            dst[(w >> 10) & 0xFFFF] = regs[d]
        elif op == OPC["ADD"]:
            regs[d] = (regs[s0] + regs[s1]) % 32
        elif op == OPC["SUB"]:
            regs[d] = (regs[s0] - regs[s1]) % 32
        elif op == OPC["MAC"]:
            regs[d] = (regs[s0] * ((w >> 21) & 0x1F) + regs[s1]) % 32
        elif op in (OPC["PBS"], OPC["PBS_ML2"], OPC["PBS_ML4"], OPC["PBS_ML8"]):
            k = 1 << (op - OPC["PBS"])
            x = regs[s0]
            assert x < 16 // k, f"PBS input {x} out of range for {k} functions"
            t = tables[(w >> 14) & 0xFFF]
            for m in range(k):
                regs[d + m] = t[m * (16 // k) + x]
        elif op == OPC["SYNC"]:
            pass
        else:
            raise ValueError(f"opcode 0x{op:02x} not modelled")
    return dst


def to_blocks(v):
    return [(v >> (2 * i)) & 3 for i in range(BLOCKS)]


def from_blocks(bs):
    return sum((int(b) & 3) << (2 * i) for i, b in enumerate(bs))
