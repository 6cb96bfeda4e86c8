"""DOp programs of the radix IOps (no GPU): plaintext semantics, encodings and
register use."""
import random

import numpy as np
import pytest

from luthe_b200 import iops as I

EDGE = [0, 1, 3, 4, 255, 256, 0x5555, 0xAAAA, 0x7FFF, 0x8000, 0xFFFE, 0xFFFF]


@pytest.mark.parametrize("a,b", [(x, y) for x in EDGE for y in EDGE[::3]])
def test_add_and_mul_edges(a, b):
    src = I.to_blocks(a) + I.to_blocks(b)
    assert I.from_blocks(I.run_plain(I.prog_add(), src, 8)) == (a + b) % 65536
    assert I.from_blocks(I.run_plain(I.prog_mul(), src, 8)) == (a * b) % 65536
    assert I.from_blocks(I.run_plain(I.prog_add_prefix(), src, 8)) == (a + b) % 65536


@pytest.mark.parametrize("a,k", [(x, y) for x in EDGE for y in EDGE[::2]])
def test_cmp_edges(a, k):
    assert I.run_plain(I.prog_cmp_gt(k), I.to_blocks(a), 1) == [int(a > k)]


def test_random_programs():
    rng = random.Random(7)
    for _ in range(200):
        a, b, k = rng.randrange(65536), rng.randrange(65536), rng.randrange(65536)
        src = I.to_blocks(a) + I.to_blocks(b)
        assert I.from_blocks(I.run_plain(I.prog_add(), src, 8)) == (a + b) % 65536
        assert I.from_blocks(I.run_plain(I.prog_mul(), src, 8)) == (a * b) % 65536
        assert I.from_blocks(I.run_plain(I.prog_add_prefix(), src, 8)) == (a + b) % 65536
        assert I.run_plain(I.prog_cmp_gt(k), I.to_blocks(a), 1) == [int(a > k)]


def test_dop_field_layout():
    # fields LSB first (fw/ublaze/src/hpu_dop_fmt.h:56-99)
    w = I.enc_pbs("PBS_ML2", 6, 9, 5)
    assert w >> 26 == 0x31 and (w >> 14) & 0xFFF == 5 and (w >> 7) & 0x7F == 9 and w & 0x7F == 6
    assert (w >> 26) >> 4 == 0b11                      # kind PBS
    w = I.enc_arith("MAC", 1, 2, 3, 4)
    assert w >> 26 == 0x05 and (w >> 21) & 0x1F == 4 and (w >> 14) & 0x7F == 3
    assert (w >> 26) & 0b0100 and (w >> 26) & 0b0001   # MUL | ADD flags
    w = I.enc_mem("LD", 7, I.MEM_SRC, 300)
    assert (w >> 26) >> 4 == 0b10 and (w >> 10) & 0xFFFF == 300 and (w >> 8) & 3 == 2


def test_programs_fit_the_register_file():
    for prog in (I.prog_add(), I.prog_cmp_gt(0x1234), I.prog_mul(), I.prog_add_prefix()):
        for w in prog:
            w = int(w)
            assert w & 0x7F < 128
        assert len(prog) < 4096


def test_many_lut_table_layout():
    t = I.LUTS["ManyCarryMsg"]
    for x in range(8):
        assert t[x] == x & 3 and t[8 + x] == x >> 2


def _pbs_depth(words, ordered_reuse):
    """Critical path of a program in PBS levels (ALU DOps take no level), with
    the serving loop's dependency rules: read-after-write always, and with
    ordered_reuse also write-after-write and write-after-read, under which a
    write waits for every earlier reader of the register to finish."""
    done, reads_done, depth = {}, {}, 0
    for w in (int(x) for x in words):
        op, dst, s0, s1 = w >> 26, w & 0x7F, (w >> 7) & 0x7F, (w >> 14) & 0x7F
        if op >> 4 == 0b10:  # LD / ST
            srcs, dsts, cost = ([], [dst], 0) if op == I.OPC["LD"] else ([dst], [], 0)
        elif op >> 4 == 0b11:  # PBS, PBS_MLk: k destinations
            k = {I.OPC["PBS"]: 1, I.OPC["PBS_ML2"]: 2, I.OPC["PBS_ML4"]: 4, I.OPC["PBS_ML8"]: 8}[op]
            srcs, dsts, cost = [s0], list(range(dst, dst + k)), 1
        else:
            two = op in (I.OPC["ADD"], I.OPC["SUB"], I.OPC["MAC"])
            srcs, dsts, cost = ([s0, s1] if two else [s0]), [dst], 0
        start = max([done.get(s, 0) for s in srcs], default=0)
        if ordered_reuse:
            start = max([start] + [max(done.get(d, 0), reads_done.get(d, 0)) for d in dsts])
        end = start + cost
        for s in srcs:
            reads_done[s] = max(reads_done.get(s, 0), end)
        for d in dsts:
            done[d], reads_done[d] = end, 0
        depth = max(depth, end)
    return depth


def test_register_reuse_adds_no_pbs_level():
    """The allocator's register reuse lengthens no program's critical path:
    with write-after-read and write-after-write ordering the depth equals the
    data-only depth (ADD 8, compare 4, MUL 8, prefix ADD 5 PBS levels)."""
    for prog, want in ((I.prog_add(), 8), (I.prog_cmp_gt(0x1234), 4), (I.prog_mul(), 8), (I.prog_add_prefix(), 5)):
        assert _pbs_depth(prog, False) == want
        assert _pbs_depth(prog, True) == want


def test_prefix_add_exhaustive_carry_patterns():
    """Every pattern of per-block carry states: block sums 0..6 in each of the
    8 blocks would be 7^8 cases, so the 3^8 patterns of stop / propagate /
    generate (block sums 0, 3, 6) cover every prefix the Sklansky rounds see."""
    import itertools
    prog = I.prog_add_prefix()
    for states in itertools.product((0, 3, 6), repeat=I.BLOCKS):
        a = [min(s, 3) for s in states]
        b = [s - x for s, x in zip(states, a)]
        want = (I.from_blocks(a) + I.from_blocks(b)) % 65536
        assert I.from_blocks(I.run_plain(prog, a + b, 8)) == want, states


def test_pbs_counts():
    """PBS per program: the fewest-PBS forms and the prefix ADD."""
    count = lambda prog: sum(1 for w in prog if (int(w) >> 26) >> 4 == 0b11)
    assert [count(I.prog_add()), count(I.prog_cmp_gt(7)), count(I.prog_mul())] == [8, 15, 101]
    assert count(I.prog_add_prefix()) == 24


def test_programs_for_load():
    assert I.programs_for_load(0) == (I.prog_add_prefix, I.prog_mul)
    assert I.programs_for_load(15) == (I.prog_add_prefix, I.prog_mul)
    assert I.programs_for_load(16) == (I.prog_add, I.prog_mul)
    assert I.programs_for_load(3, light=2) == (I.prog_add, I.prog_mul)


def test_compare_exhaustive_on_block_patterns():
    """a > k for every pair of 8-block values drawn from digits {0, 2, 3}:
    each block is less, equal or greater in every position."""
    import itertools
    vals = [I.from_blocks(ds) for ds in itertools.product((0, 2, 3), repeat=4)]
    vals = [v | (v << 8) for v in vals] + [v << 8 for v in vals]
    for k in vals[::7]:
        prog = I.prog_cmp_gt(k)
        for a in vals:
            assert I.run_plain(prog, I.to_blocks(a), 1) == [int(a > k)], (a, k)
