"""The oracle's DOp-program interpreter (the checker of the serving loop):
the radix IOp programs of luthe_b200.iops decrypt to the integer results, and
running programs side by side equals running each alone."""
import numpy as np

import luthe_b200 as L
import oracle
from luthe_b200 import iops as I
from oracle import dops


def test_iop_programs_on_the_oracle():
    p = L.default_params(lwe_dim=32)
    keys = L.keygen(p, 77)
    ob = oracle.OracleBsk(keys["bsk"], p.lwe_dim, p.poly_size)
    luts = np.stack([L.lut_build(p, t) for t in I.lut_tables()])

    def enc(values, seed):
        blocks = [b for v in values for b in I.to_blocks(v)]
        return L.encrypt(p, keys["glwe_key"], np.array(blocks, np.uint32), seed)

    a, b, k = 0x9A3C, 0x0457, 0x9000
    reqs = [(I.prog_add(), enc([a, b], 1), 8), (I.prog_cmp_gt(k), enc([a], 2), 1), (I.prog_mul(), enc([a, b], 3), 8)]
    outs = dops.run_many(reqs, keys["ksk"], ob, luts)
    dec = [[int(x) for x in L.decrypt(p, keys["glwe_key"], o)] for o in outs]
    assert I.from_blocks(dec[0]) == (a + b) % 65536
    assert dec[1] == [int(a > k)]
    assert I.from_blocks(dec[2]) == (a * b) % 65536
    alone = dops.run(*reqs[0], keys["ksk"], ob, luts)
    assert np.array_equal(alone, outs[0])


def test_linear_dops_semantics():
    # ADDS/SUBS/SSUB/MULS place the constant at the body, cst << 59
    N = 8
    r0 = np.arange(N + 1, dtype=np.uint64) * np.uint64(3)
    prog = [I.enc_mem("LD", 0, I.MEM_SRC, 0), I.enc_arith_msg("ADDS", 1, 0, 5), I.enc_arith_msg("SUBS", 2, 0, 5),
            I.enc_arith_msg("SSUB", 3, 0, 5), I.enc_arith_msg("MULS", 4, 0, 5), I.enc_arith("SUB", 5, 1, 0)]
    prog += [I.enc_mem("ST", r, I.MEM_DST, r - 1) for r in range(1, 6)]
    out = dops.run(prog, r0[None, :], 5, None, None, None)
    c = np.zeros(N + 1, np.uint64)
    c[N] = np.uint64(5) << np.uint64(59)
    with np.errstate(over="ignore"):
        assert np.array_equal(out[0], r0 + c)
        assert np.array_equal(out[1], r0 - c)
        assert np.array_equal(out[2], c - r0)
        assert np.array_equal(out[3], r0 * np.uint64(5))
        assert np.array_equal(out[4], c)
