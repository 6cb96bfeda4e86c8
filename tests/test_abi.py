"""The C-ABI library loads without a GPU and exports what include/luthe.h declares;
host-side helpers behave.  No device compute is issued here."""
import os
import re
import subprocess

import numpy as np
import pytest

import luthe_b200 as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "luthe.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(luthe_\w+)\s*\(", src)))


def test_header_declares_python_symbol_list():
    assert header_functions() == sorted(L.SYMBOLS)


def test_library_exports_every_declared_symbol():
    L.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (luthe_\w+)", out))
    missing = [f for f in header_functions() if f not in exported]
    assert not missing, missing
    for f in header_functions():
        getattr(L.lib(), f)


def test_library_is_built_for_sm100a():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", L.LIB_PATH], capture_output=True,
                         text=True).stdout
    assert "sm_100a" in out


def test_default_params_match_the_parameter_set():
    p = L.default_params()
    assert p.as_dict() == dict(lwe_dim=804, glwe_dim=1, poly_size=2048, pbs_base_log=23, pbs_level=1,
                               ks_base_log=3, ks_level=6, ks_width=21, msg_width=2, carry_width=2)


def test_context_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(L.LutheError) as ei:
        L.Engine()
    assert ei.value.code == L.E_CUDA


def test_unsupported_params_rejected():
    with pytest.raises(L.LutheError) as ei:
        L.Engine(L.default_params(poly_size=1024))
    assert ei.value.code == L.E_PARAM


def test_encrypt_decrypt_roundtrip(params, keys):
    msgs = np.arange(16, dtype=np.uint32)
    ct = L.encrypt(params, keys["glwe_key"], msgs, 3)
    assert np.array_equal(L.decrypt(params, keys["glwe_key"], ct), msgs)


def test_keygen_is_deterministic(params):
    p = L.default_params(lwe_dim=16)
    a, b = L.keygen(p, 7), L.keygen(p, 7)
    for k in a:
        assert np.array_equal(a[k], b[k])
    assert np.all(a["bsk"] < np.uint64(0xFFFFFFFF00000001))


@pytest.mark.parametrize("name", ["default", "msg2_carry2_pfail64_132b_gaussian_1f72dba"])
def test_ksk_encrypts_key_digits(name):
    # KSK[x][y][z] is an LWE encryption of S_y 2^(21 - bl(L-z)) mod 2^21 under
    # the small key: level L-1 carries the most significant digit
    p = L.param_set(name)
    keys = L.keygen(p, 20261203)
    n, N, bl, lc = p.lwe_dim, p.poly_size, p.ks_base_log, p.ks_level
    K = keys["ksk"].reshape(n + 1, N, lc).astype(np.int64)
    s = keys["lwe_key"].astype(np.int64)
    for y in (0, 1, 1000):
        for z in range(lc):
            ph = (K[n, y, z] - int((K[:n, y, z] * s).sum())) % (1 << 21)
            err = (ph - int(keys["glwe_key"][y]) * (1 << (21 - bl * (lc - z))) + (1 << 20)) % (1 << 21) - (1 << 20)
            assert abs(err) < 100
