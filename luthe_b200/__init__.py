"""LUTHE-B200: a B200 (sm_100a) KS+PBS engine with the HPU's DOp surface.

This module loads the in-tree engine library (``libluthe.so``) through ctypes
and mirrors the reference's PBS/ALU operator interface:

* :class:`Engine` -- one device context with resident keys and LUTs; its
  methods are the batched DOps (``ks_pbs`` is ``PBS Dst Src LUT`` over a batch,
  ``lwe_op`` the linear DOps of pe_alu, plus the KS/BR/NTT stages on their own).
* :func:`keygen`, :func:`encrypt`, :func:`decrypt`, :func:`lut_build` -- host
  helpers for seeded key material and test data.

There is no fallback path: if the library is missing or the device cannot be
used, calls raise :class:`LutheError`.
"""
import ctypes
import json
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libluthe.so")

OK, E_PARAM, E_BUDGET, E_TIMEOUT, E_CUDA, E_STATE = range(6)
OP_ADD, OP_SUB, OP_MAC, OP_ADDS, OP_SUBS, OP_SSUB, OP_MULS = range(7)
# tie rule of the decompositions (luthe_set_tie_rule): the RTL's, or the
# reference test-vector generator's
TIE_RTL, TIE_GENERATOR = 0, 1

# exported symbols of include/luthe.h
SYMBOLS = [
    "luthe_params_default", "luthe_last_error", "luthe_ctx_create", "luthe_ctx_destroy", "luthe_device_bytes",
    "luthe_upload_bsk", "luthe_upload_bsk_eval", "luthe_set_tie_rule", "luthe_upload_ksk", "luthe_upload_luts", "luthe_reserve", "luthe_ks_pbs",
    "luthe_ks_pbs_host", "luthe_ks_pbs_graph", "luthe_ks_pbs_noalloc", "luthe_ks_pbs_ml", "luthe_keyswitch",
    "luthe_server_create", "luthe_server_destroy", "luthe_server_submit", "luthe_server_step",
    "luthe_server_fetch", "luthe_server_counters", "luthe_server_set_batching", "luthe_blind_rotate", "luthe_ntt_fwd",
    "luthe_ntt_inv", "luthe_ntt_mul", "luthe_lwe_op", "luthe_set_br_config", "luthe_autotune",
    "luthe_tuning_save", "luthe_tuning_load",
    "luthe_check_device_error", "luthe_measure_int_peak", "luthe_keygen", "luthe_encrypt", "luthe_decrypt", "luthe_lut_build",
]


class LutheError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"luthe error {code}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint32) for name in (
        "lwe_dim", "glwe_dim", "poly_size", "pbs_base_log", "pbs_level", "ks_base_log", "ks_level",
        "ks_width", "msg_width", "carry_width")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib():
    """The loaded engine library (built on first use if the sources are newer)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build
            build.build_engine()
        if not os.path.exists(LIB_PATH):
            raise LutheError(E_CUDA, f"engine library missing: {LIB_PATH}")
        L = ctypes.CDLL(LIB_PATH)
        vp, sz, u64, u32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint32
        P = ctypes.POINTER(Params)
        L.luthe_last_error.restype = ctypes.c_char_p
        L.luthe_params_default.argtypes = [P]
        L.luthe_ctx_create.argtypes = [P, ctypes.c_int, u64, ctypes.POINTER(vp)]
        L.luthe_ctx_destroy.argtypes = [vp]
        L.luthe_device_bytes.argtypes = [vp]
        L.luthe_device_bytes.restype = u64
        L.luthe_upload_bsk.argtypes = [vp, vp]
        L.luthe_upload_bsk_eval.argtypes = [vp, vp]
        L.luthe_set_tie_rule.argtypes = [vp, ctypes.c_int]
        L.luthe_upload_ksk.argtypes = [vp, vp]
        L.luthe_upload_luts.argtypes = [vp, vp, u32]
        L.luthe_reserve.argtypes = [vp, sz]
        for f in ("luthe_ks_pbs", "luthe_ks_pbs_graph", "luthe_ks_pbs_noalloc"):
            getattr(L, f).argtypes = [vp, vp, vp, vp, sz, vp]
        L.luthe_ks_pbs_host.argtypes = [vp, vp, vp, vp, sz]
        L.luthe_ks_pbs_ml.argtypes = [vp, vp, vp, vp, sz, u32, vp]
        pu32, pu64, pd = ctypes.POINTER(u32), ctypes.POINTER(u64), ctypes.POINTER(ctypes.c_double)
        L.luthe_server_create.argtypes = [vp, u64, u32, ctypes.POINTER(vp)]
        L.luthe_server_destroy.argtypes = [vp]
        L.luthe_server_submit.argtypes = [vp, vp, u32, vp, u32, u32, pu64]
        L.luthe_server_step.argtypes = [vp, pu32, pu32, pu32]
        L.luthe_server_fetch.argtypes = [vp, u64, vp, pd, pd]
        L.luthe_server_counters.argtypes = [vp, pu64, pu64, pu64, pu64]
        L.luthe_server_set_batching.argtypes = [vp, u32, u32]
        L.luthe_keyswitch.argtypes = [vp, vp, vp, vp, sz, vp]
        L.luthe_blind_rotate.argtypes = [vp, vp, vp, vp, sz, vp]
        L.luthe_ntt_fwd.argtypes = [vp, vp, vp, sz, vp]
        L.luthe_ntt_inv.argtypes = [vp, vp, vp, sz, vp]
        L.luthe_ntt_mul.argtypes = [vp, vp, vp, vp, sz, vp]
        L.luthe_lwe_op.argtypes = [vp, ctypes.c_int, vp, vp, vp, u64, sz, vp]
        L.luthe_set_br_config.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.luthe_autotune.argtypes = [vp, sz, ctypes.c_char_p, sz]
        L.luthe_tuning_save.argtypes = [vp, ctypes.c_char_p]
        L.luthe_tuning_load.argtypes = [vp, ctypes.c_char_p]
        L.luthe_check_device_error.argtypes = [vp]
        L.luthe_measure_int_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_double)]
        L.luthe_keygen.argtypes = [P, u64, vp, vp, vp, vp]
        L.luthe_encrypt.argtypes = [P, vp, vp, sz, u64, vp]
        L.luthe_decrypt.argtypes = [P, vp, vp, sz, vp]
        L.luthe_lut_build.argtypes = [P, vp, vp]
        _lib = L
    return _lib


def _check(code):
    if code != OK:
        raise LutheError(code, lib().luthe_last_error().decode())


def default_params(**over):
    p = Params()
    lib().luthe_params_default(ctypes.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p


# The reference's HPU parameter sets (hw/module/param/module/<name>/rtl/
# param_tfhe_definition_pkg.sv: N, GLWE_K, PBS_L, PBS_B_W, LWE_K, KS_L, KS_B_W,
# MOD_KSK_W).  All have N = 2048, k = 1, one PBS level, KSK modulus 2^21 and a
# 2-bit message + 2-bit carry payload.  "default" is the n = 804, KS 3 x 6 set
# that the gtv model runs by default and the benchmark is quoted on.
PARAM_SETS = {
    "default": dict(lwe_dim=804, pbs_base_log=23, ks_base_log=3, ks_level=6),
    # param_msg2_carry2_pfail64_132b_gaussian_1f72dba/rtl/param_tfhe_definition_pkg.sv:31-53
    "msg2_carry2_pfail64_132b_gaussian_1f72dba": dict(lwe_dim=804, pbs_base_log=23, ks_base_log=2, ks_level=8),
    # param_msg2_carry2_pfail64_132b_tuniform_7e47d8c/rtl/param_tfhe_definition_pkg.sv:31-53
    "msg2_carry2_pfail64_132b_tuniform_7e47d8c": dict(lwe_dim=839, pbs_base_log=23, ks_base_log=2, ks_level=7),
    # param_msg2_carry2_gaussian/rtl/param_tfhe_definition_pkg.sv:42-64
    "msg2_carry2_gaussian": dict(lwe_dim=834, pbs_base_log=23, ks_base_log=3, ks_level=5),
    # param_msg2_carry2_tuniform/rtl/param_tfhe_definition_pkg.sv:38-60
    "msg2_carry2_tuniform": dict(lwe_dim=887, pbs_base_log=22, ks_base_log=3, ks_level=5),
}


def param_set(name):
    """Params of one of the reference's named parameter sets (PARAM_SETS)."""
    if name not in PARAM_SETS:
        raise KeyError(f"unknown parameter set {name!r}; known: {sorted(PARAM_SETS)}")
    return default_params(**PARAM_SETS[name])


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        assert a.is_contiguous()
        return a.data_ptr()
    return int(a)


# ------------------------------------------------------------- host helpers

def keygen(params, seed):
    """Seeded keys: lwe_key[n], glwe_key[N], ksk[(n+1)*N*L] (u32), bsk[n*4*N] over Z_p."""
    n, N, L = params.lwe_dim, params.poly_size * params.glwe_dim, params.ks_level
    k = {
        "lwe_key": np.zeros(n, np.uint32),
        "glwe_key": np.zeros(N, np.uint32),
        "ksk": np.zeros((n + 1) * N * L, np.uint32),
        "bsk": np.zeros(n * 4 * params.poly_size, np.uint64),
    }
    _check(lib().luthe_keygen(ctypes.byref(params), seed, _ptr(k["lwe_key"]), _ptr(k["glwe_key"]),
                              _ptr(k["ksk"]), _ptr(k["bsk"])))
    return k


def encrypt(params, glwe_key, msgs, seed):
    msgs = np.ascontiguousarray(msgs, np.uint32)
    out = np.zeros((len(msgs), params.poly_size + 1), np.uint64)
    _check(lib().luthe_encrypt(ctypes.byref(params), _ptr(glwe_key), _ptr(msgs), len(msgs), seed, _ptr(out)))
    return out


def decrypt(params, glwe_key, blwe):
    blwe = np.ascontiguousarray(blwe, np.uint64).reshape(-1, params.poly_size + 1)
    out = np.zeros(blwe.shape[0], np.uint32)
    _check(lib().luthe_decrypt(ctypes.byref(params), _ptr(glwe_key), _ptr(blwe), blwe.shape[0], _ptr(out)))
    return out


def lut_build(params, table):
    table = np.ascontiguousarray(table, np.uint32)
    out = np.zeros(2 * params.poly_size, np.uint64)
    _check(lib().luthe_lut_build(ctypes.byref(params), _ptr(table), _ptr(out)))
    return out


def measure_int_peak(device=0):
    """(32-bit IMAD/s, Goldilocks mul/s) measured on `device` by probe kernels."""
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(lib().luthe_measure_int_peak(device, ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


# ------------------------------------------------------------------- engine

class Engine:
    """A device context holding the BSK, KSK and LUT memory of the HPU's pe_pbs.

    Device-pointer methods take torch CUDA tensors (or raw addresses) and a
    stream (torch stream, raw handle, or None for the default stream).
    """

    def __init__(self, params=None, device=0, hbm_budget=0):
        self.params = params or default_params()
        self._h = None
        h = ctypes.c_void_p()
        _check(lib().luthe_ctx_create(ctypes.byref(self.params), device, hbm_budget, ctypes.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            lib().luthe_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @staticmethod
    def _s(stream):
        if stream is None:
            return None
        return getattr(stream, "cuda_stream", stream)

    @property
    def device_bytes(self):
        return lib().luthe_device_bytes(self._h)

    def upload_keys(self, keys):
        self.upload_bsk(keys["bsk"])
        self.upload_ksk(keys["ksk"])

    def upload_bsk(self, bsk):
        bsk = np.ascontiguousarray(bsk, np.uint64)
        _check(lib().luthe_upload_bsk(self._h, _ptr(bsk)))

    def upload_bsk_eval(self, bsk_eval):
        """BSK in the evaluation domain, [n][row][col][k] = BSK_i[row][col](psi^(2k+1))
        (the form hpu_files.load_bsk returns for the HPU's bsk_nd_hwo files)."""
        bsk_eval = np.ascontiguousarray(bsk_eval, np.uint64)
        _check(lib().luthe_upload_bsk_eval(self._h, _ptr(bsk_eval)))

    def set_tie_rule(self, rule):
        """TIE_RTL (default) or TIE_GENERATOR: the decompositions' rule for a top
        digit equal to B/2 (luthe_set_tie_rule)."""
        _check(lib().luthe_set_tie_rule(self._h, rule))

    def upload_ksk(self, ksk):
        ksk = np.ascontiguousarray(ksk, np.uint32)
        _check(lib().luthe_upload_ksk(self._h, _ptr(ksk)))

    def upload_luts(self, luts):
        luts = np.ascontiguousarray(luts, np.uint64).reshape(-1, 2 * self.params.poly_size)
        _check(lib().luthe_upload_luts(self._h, _ptr(luts), luts.shape[0]))

    def reserve(self, count):
        _check(lib().luthe_reserve(self._h, count))

    def ks_pbs(self, d_in, d_ids, d_out, count, stream=None):
        _check(lib().luthe_ks_pbs(self._h, _ptr(d_in), _ptr(d_ids), _ptr(d_out), count, self._s(stream)))

    def ks_pbs_ml(self, d_in, d_ids, d_out, count, mlk, stream=None):
        """Many-LUT PBS: row c*mlk+m of d_out is function m of input c."""
        _check(lib().luthe_ks_pbs_ml(self._h, _ptr(d_in), _ptr(d_ids), _ptr(d_out), count, mlk, self._s(stream)))

    def ks_pbs_noalloc(self, d_in, d_ids, d_out, count, stream=None):
        """KS+PBS that allocates no device memory (fixed 4 MiB scratch; see
        luthe_ks_pbs_noalloc in include/luthe.h for the limit and the sharing)."""
        _check(lib().luthe_ks_pbs_noalloc(self._h, _ptr(d_in), _ptr(d_ids), _ptr(d_out), count, self._s(stream)))

    def ks_pbs_graph(self, d_in, d_ids, d_out, count, stream):
        _check(lib().luthe_ks_pbs_graph(self._h, _ptr(d_in), _ptr(d_ids), _ptr(d_out), count, self._s(stream)))

    def ks_pbs_host(self, blwe_in, lut_ids, out=None):
        blwe_in = np.ascontiguousarray(blwe_in, np.uint64).reshape(-1, self.params.poly_size + 1)
        lut_ids = np.ascontiguousarray(lut_ids, np.uint32)
        if out is None:
            out = np.empty_like(blwe_in)
        _check(lib().luthe_ks_pbs_host(self._h, _ptr(blwe_in), _ptr(lut_ids), _ptr(out), blwe_in.shape[0]))
        return out

    def keyswitch(self, d_in, d_out21, d_out2N, count, stream=None):
        _check(lib().luthe_keyswitch(self._h, _ptr(d_in), _ptr(d_out21), _ptr(d_out2N), count, self._s(stream)))

    def blind_rotate(self, d_lwe2N, d_ids, d_out, count, stream=None):
        _check(lib().luthe_blind_rotate(self._h, _ptr(d_lwe2N), _ptr(d_ids), _ptr(d_out), count, self._s(stream)))

    def ntt_fwd(self, d_in, d_out, count, stream=None):
        _check(lib().luthe_ntt_fwd(self._h, _ptr(d_in), _ptr(d_out), count, self._s(stream)))

    def ntt_inv(self, d_in, d_out, count, stream=None):
        _check(lib().luthe_ntt_inv(self._h, _ptr(d_in), _ptr(d_out), count, self._s(stream)))

    def ntt_mul(self, d_a, d_b, d_out, count, stream=None):
        _check(lib().luthe_ntt_mul(self._h, _ptr(d_a), _ptr(d_b), _ptr(d_out), count, self._s(stream)))

    def lwe_op(self, op, d_a, d_b, d_out, imm, count, stream=None):
        _check(lib().luthe_lwe_op(self._h, op, _ptr(d_a), _ptr(d_b), _ptr(d_out), imm, count, self._s(stream)))

    def set_br_config(self, cts_per_cta, ctas_per_sm=1):
        _check(lib().luthe_set_br_config(self._h, cts_per_cta, ctas_per_sm))

    def autotune(self, sample=0):
        """Time the blind rotation's launch forms on this device and keep the
        fastest (luthe_autotune); returns the record of trials and the choice."""
        buf = ctypes.create_string_buffer(1 << 16)
        _check(lib().luthe_autotune(self._h, sample, buf, 1 << 16))
        return json.loads(buf.value.decode())

    def tuning_save(self, path):
        _check(lib().luthe_tuning_save(self._h, str(path).encode()))

    def tuning_load(self, path):
        _check(lib().luthe_tuning_load(self._h, str(path).encode()))

    def check_device_error(self):
        _check(lib().luthe_check_device_error(self._h))


class Server:
    """Serving loop over an :class:`Engine`: DOp programs (see :mod:`luthe_b200.iops`)
    are submitted as requests and executed with continuous batching; ready PBS
    DOps of all in-flight requests share one KS+PBS launch per round."""

    def __init__(self, engine, pool_bytes=1 << 30, max_pbs=4096):
        self.engine = engine
        self.N = engine.params.poly_size
        h = ctypes.c_void_p()
        _check(lib().luthe_server_create(engine._h, pool_bytes, max_pbs, ctypes.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            lib().luthe_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, dops, src_blocks, n_dst):
        """Queue a request; returns its id.  src_blocks: [n_src][N+1] u64 BLWEs."""
        dops = np.ascontiguousarray(dops, np.uint32)
        src = np.ascontiguousarray(src_blocks, np.uint64).reshape(-1, self.N + 1)
        rid = ctypes.c_uint64()
        _check(lib().luthe_server_submit(self._h, _ptr(dops), dops.size, _ptr(src) if src.size else None,
                                         src.shape[0], n_dst, ctypes.byref(rid)))
        return rid.value

    def step(self):
        """One scheduling round; returns (completed, active, pending)."""
        c, a, p = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().luthe_server_step(self._h, ctypes.byref(c), ctypes.byref(a), ctypes.byref(p)))
        return c.value, a.value, p.value

    def fetch(self, rid, n_dst):
        """(output blocks, latency s, queueing s) of a finished request, or None."""
        out = np.zeros((n_dst, self.N + 1), np.uint64)
        lat, q = ctypes.c_double(), ctypes.c_double()
        code = lib().luthe_server_fetch(self._h, rid, _ptr(out), ctypes.byref(lat), ctypes.byref(q))
        if code == E_STATE:
            return None
        _check(code)
        return out, lat.value, q.value

    def set_batching(self, fill=0, window_us=0):
        """Hold ready PBS DOps while a lane is busy, fewer than `fill` are
        ready and the oldest waited less than `window_us` (0: off)."""
        _check(lib().luthe_server_set_batching(self._h, fill, window_us))

    def counters(self):
        v = [ctypes.c_uint64() for _ in range(4)]
        _check(lib().luthe_server_counters(self._h, *[ctypes.byref(x) for x in v]))
        return dict(zip(("rounds", "pbs", "alu", "launches"), (x.value for x in v)))

    def run(self, requests):
        """Submit all requests [(dops, src, n_dst)] now and step until done;
        returns the output blocks in submission order."""
        ids = [self.submit(*r) for r in requests]
        outs = {}
        while len(outs) < len(ids):
            self.step()
            for rid, r in zip(ids, requests):
                if rid not in outs:
                    got = self.fetch(rid, r[2])
                    if got is not None:
                        outs[rid] = got[0]
        return [outs[i] for i in ids]
