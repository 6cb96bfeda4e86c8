"""The oracle's own key generation, encryption, decryption and LUT builder
(used by the CPU reference timing, which loads nothing from the engine
library) give the engine's values for the same seed."""
import numpy as np

import luthe_b200 as L
import oracle


def test_oracle_keygen_equals_engine_keygen():
    p = L.default_params(lwe_dim=24, poly_size=256)
    a = oracle.keygen(24, 256, 9)
    b = L.keygen(p, 9)
    for k in ("lwe_key", "glwe_key", "ksk", "bsk"):
        assert np.array_equal(a[k], b[k]), k


def test_oracle_encrypt_decrypt_lut_equal_engine():
    p = L.default_params()
    keys = L.keygen(L.default_params(lwe_dim=4), 3)
    msgs = np.arange(40, dtype=np.uint32) % 16
    ct = oracle.encrypt(keys["glwe_key"], msgs, 5)
    assert np.array_equal(ct, L.encrypt(p, keys["glwe_key"], msgs, 5))
    assert np.array_equal(oracle.decrypt(keys["glwe_key"], ct), msgs)
    t = (np.arange(16, dtype=np.uint32) * 7) % 16
    assert np.array_equal(oracle.lut_build(2048, t), L.lut_build(p, t))
