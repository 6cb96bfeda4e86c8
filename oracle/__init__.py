"""CPU oracle of the KS+PBS path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``tfhe_oracle.c``, the CPU restatement of the reference's
algorithms (each C function cites the reference file it follows).  Only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
this module, as the checker; the engine never does.

Parity pins: the full KS+PBS (key switch, blind rotation, sample extract)
equals the reference's test-vector generator's outputs word for word, on its
own keys and BSK files, with the generator's tie rule (``tests/golden``,
made by the reference's generator; tests/test_reference_pbs_pin.py); the
decomposer, monomial multiply, Solinas reduction, modulus switch and NTT are
also pinned stage by stage against the reference's Python models and
self-tests.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
P = 0xFFFFFFFF00000001
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            import importlib
            importlib.import_module("luthe_b200.build").build_oracle()
        L = ctypes.CDLL(LIB_PATH)
        vp, u64, u32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32
        L.or_gl_reduce128.argtypes = [u64, u64]
        L.or_gl_reduce128.restype = u64
        L.or_gl_mul.argtypes = [u64, u64]
        L.or_gl_mul.restype = u64
        L.or_gl_inv.argtypes = [u64]
        L.or_gl_inv.restype = u64
        L.or_decompose.argtypes = [u64, ctypes.c_int, ctypes.c_int, vp]
        L.or_decompose2.argtypes = [u64, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
        L.or_modsw_p_to_q.argtypes = [u64]
        L.or_modsw_p_to_q.restype = u64
        L.or_modsw_q_to_p.argtypes = [u64]
        L.or_modsw_q_to_p.restype = u64
        L.or_monomial.argtypes = [vp, u32, vp, u32]
        L.or_ntt_eval.argtypes = [vp, vp, u32]
        L.or_negacyclic_mul.argtypes = [vp, vp, vp, u32, u32]
        L.or_negacyclic_mul_schoolbook.argtypes = [vp, vp, vp, u32]
        L.or_keyswitch.argtypes = [vp, vp, u32, u32, u32, u32, u32, u32, vp, vp]
        L.or_keyswitch2.argtypes = [vp, vp, u32, u32, u32, u32, u32, u32, ctypes.c_int, vp, vp]
        L.or_bsk_prepare.argtypes = [vp, u32, u32]
        L.or_bsk_prepare.restype = vp
        L.or_bsk_prepare_eval.argtypes = [vp, u32, u32]
        L.or_bsk_prepare_eval.restype = vp
        L.or_ntt_inv_natural.argtypes = [vp, vp, u32]
        L.or_set_tie_rule.argtypes = [ctypes.c_int]
        L.or_bsk_free.argtypes = [vp]
        L.or_blind_rotate.argtypes = [vp, vp, vp, vp, vp, u32, u32]
        L.or_ks_pbs.argtypes = [vp, vp, vp, vp, vp, vp, u32, u32, u32, u32, u32]
        L.or_ks_pbs_ml.argtypes = [vp, vp, vp, vp, vp, vp, u32, u32, u32, u32, u32, u32]
        L.or_keygen.argtypes = [u32, u32, u32, u32, u32, u32, u64, vp, vp, vp, vp]
        L.or_encrypt.argtypes = [u32, u32, vp, vp, u64, u64, vp]
        L.or_decrypt.argtypes = [u32, u32, vp, vp, u64, vp]
        L.or_lut_build.argtypes = [u32, u32, vp, vp]
        L.or_num_threads.restype = ctypes.c_int
        L.or_set_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _p(a):
    assert a.flags.c_contiguous
    return a.ctypes.data


def decompose(v, base_log, level, gtv_top_tie=False):
    """Signed digits, LSB first.  gtv_top_tie selects the test-vector
    generator's rule for a top digit equal to B/2 (stays positive)."""
    d = np.zeros(level, np.int32)
    lib().or_decompose2(int(v), base_log, level, int(gtv_top_tie), _p(d))
    return [int(x) for x in d]


def modsw_p_to_q(a):
    return lib().or_modsw_p_to_q(int(a))


def modsw_q_to_p(x):
    return lib().or_modsw_q_to_p(int(x))


def reduce128(lo, hi):
    return lib().or_gl_reduce128(int(lo), int(hi))


def monomial(poly, e):
    poly = np.ascontiguousarray(poly, np.uint64)
    out = np.zeros_like(poly)
    lib().or_monomial(_p(poly), int(e), _p(out), poly.size)
    return out


def ntt_eval(poly):
    """A(psi^(2k+1)) for k in natural order, psi^64 = 8."""
    poly = np.ascontiguousarray(poly, np.uint64)
    out = np.zeros_like(poly)
    lib().or_ntt_eval(_p(poly), _p(out), poly.size)
    return out


def ntt_inv_natural(vals):
    """Coefficients of A from A(psi^(2k+1)), k in natural order (inverse of ntt_eval)."""
    vals = np.ascontiguousarray(vals, np.uint64)
    out = np.zeros_like(vals)
    lib().or_ntt_inv_natural(_p(vals), _p(out), vals.size)
    return out


def negacyclic_mul(a, b):
    a = np.ascontiguousarray(a, np.uint64)
    b = np.ascontiguousarray(b, np.uint64)
    N = a.shape[-1]
    out = np.zeros_like(a)
    lib().or_negacyclic_mul(_p(a), _p(b), _p(out), N, a.size // N)
    return out


def negacyclic_mul_schoolbook(a, b):
    a = np.ascontiguousarray(a, np.uint64)
    b = np.ascontiguousarray(b, np.uint64)
    out = np.zeros_like(a)
    lib().or_negacyclic_mul_schoolbook(_p(a), _p(b), _p(out), a.size)
    return out


def keyswitch(blwe, ksk, n, N, ks_bl=3, ks_lc=6, ks_w=21, gtv_top_tie=False):
    """Returns (out21[n+1], out2N[n+1]) for one BLWE of dimension N (k=1)."""
    blwe = np.ascontiguousarray(blwe, np.uint64)
    ksk = np.ascontiguousarray(ksk, np.uint32)
    o21 = np.zeros(n + 1, np.uint32)
    o2n = np.zeros(n + 1, np.uint32)
    lib().or_keyswitch2(_p(blwe), _p(ksk), n, N, ks_bl, ks_lc, ks_w, N, int(gtv_top_tie), _p(o21), _p(o2n))
    return o21, o2n


class OracleBsk:
    """BSK prepared in the oracle's own NTT domain."""

    def __init__(self, bsk_std_p, n, N, eval_domain=False):
        """bsk_std_p: [n][row][col][N] over Z_p, standard domain; or, with
        eval_domain, the evaluations BSK_i[row][col](psi^(2k+1)) in natural k."""
        self._bsk = np.ascontiguousarray(bsk_std_p, np.uint64)
        self.n, self.N = n, N
        prep = lib().or_bsk_prepare_eval if eval_domain else lib().or_bsk_prepare
        self.h = prep(_p(self._bsk), n, N)

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_bsk_free(self.h)
            self.h = None

    def blind_rotate(self, lwe2N, luts, lut_ids, pbs_bl=23):
        lwe2N = np.ascontiguousarray(lwe2N, np.uint32).reshape(-1, self.n + 1)
        luts = np.ascontiguousarray(luts, np.uint64)
        lut_ids = np.ascontiguousarray(lut_ids, np.uint32)
        out = np.zeros((lwe2N.shape[0], self.N + 1), np.uint64)
        lib().or_blind_rotate(self.h, _p(lwe2N), _p(luts), _p(lut_ids), _p(out), lwe2N.shape[0], pbs_bl)
        return out

    def ks_pbs(self, ksk, blwe_in, luts, lut_ids, ks_bl=3, ks_lc=6, ks_w=21, pbs_bl=23, mlk=1):
        """KS+PBS; with mlk > 1 (many-LUT) row c*mlk+m holds output m of input c."""
        ksk = np.ascontiguousarray(ksk, np.uint32)
        blwe_in = np.ascontiguousarray(blwe_in, np.uint64).reshape(-1, self.N + 1)
        luts = np.ascontiguousarray(luts, np.uint64)
        lut_ids = np.ascontiguousarray(lut_ids, np.uint32)
        out = np.zeros((blwe_in.shape[0] * mlk, self.N + 1), np.uint64)
        lib().or_ks_pbs_ml(self.h, _p(ksk), _p(blwe_in), _p(luts), _p(lut_ids), _p(out), blwe_in.shape[0], ks_bl,
                           ks_lc, ks_w, pbs_bl, mlk)
        return out


def set_tie_rule(generator):
    """Tie rule of the decompositions in every later blind rotation and
    KS+PBS of the oracle: the RTL's (False) or the reference generator's
    (True).  keyswitch() takes its rule as an argument instead."""
    lib().or_set_tie_rule(int(bool(generator)))


def keygen(n, N, seed, ks_bl=3, ks_lc=6, ks_w=21, pbs_bl=23):
    """Seeded keys without the engine library: {lwe_key, glwe_key, ksk, bsk}
    (the layouts and values of luthe_b200.keygen for the same seed)."""
    k = {"lwe_key": np.zeros(n, np.uint32), "glwe_key": np.zeros(N, np.uint32),
         "ksk": np.zeros((n + 1) * N * ks_lc, np.uint32), "bsk": np.zeros(n * 4 * N, np.uint64)}
    lib().or_keygen(n, N, ks_bl, ks_lc, ks_w, pbs_bl, seed, _p(k["lwe_key"]), _p(k["glwe_key"]), _p(k["ksk"]),
                    _p(k["bsk"]))
    return k


def encrypt(glwe_key, msgs, seed, bits=5):
    msgs = np.ascontiguousarray(msgs, np.uint32)
    N = glwe_key.size
    out = np.zeros((msgs.size, N + 1), np.uint64)
    lib().or_encrypt(N, bits, _p(np.ascontiguousarray(glwe_key, np.uint32)), _p(msgs), msgs.size, seed, _p(out))
    return out


def decrypt(glwe_key, blwe, bits=5):
    N = glwe_key.size
    blwe = np.ascontiguousarray(blwe, np.uint64).reshape(-1, N + 1)
    out = np.zeros(blwe.shape[0], np.uint32)
    lib().or_decrypt(N, bits, _p(np.ascontiguousarray(glwe_key, np.uint32)), _p(blwe), blwe.shape[0], _p(out))
    return out


def lut_build(N, table, bits=5):
    table = np.ascontiguousarray(table, np.uint32)
    out = np.zeros(2 * N, np.uint64)
    lib().or_lut_build(N, bits, _p(table), _p(out))
    return out


def set_threads(t):
    lib().or_set_threads(int(t))


def num_threads():
    return lib().or_num_threads()
