"""The blind-rotation autotuner: it times the launch forms on this GPU, keeps
the fastest shape and batch-size cut-offs, saves them as JSON per device and
parameter set, and a later context loads them; results stay bit-exact."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import luthe_b200 as L
from conftest import from_dev, to_dev

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_autotune_choice_is_saved_loaded_and_exact(engine, params, keys, oracle_bsk, tmp_path):
    rng = np.random.default_rng(5)
    table = rng.integers(0, 16, 16).astype(np.uint32)
    luts = L.lut_build(params, table)[None, :]
    engine.upload_luts(luts)
    rec = engine.autotune(0)
    chosen = rec["chosen"]
    assert chosen["format"] == "luthe-tuning-1" and chosen["cts_per_cta"] in (1, 2)
    forms = {t["form"] for t in rec["trials"]}
    assert {"G1", "G2"} <= forms
    if chosen["cts_per_cta"] == 2:
        assert {"pair", "split", "wave", "wave+tail", "waves"} <= forms
    assert all(t["ms"] > 0 for t in rec["trials"])
    path = tmp_path / "tune.json"
    engine.tuning_save(path)
    assert json.loads(path.read_text()) == chosen
    # a context in a fresh process picks the file up from LUTHE_TUNING_DIR
    d = tmp_path / "dir"
    d.mkdir()
    (d / f"luthe_tune_{chosen['key']}.json").write_text(path.read_text())
    seen = tmp_path / "seen.json"
    code = "import sys, luthe_b200 as L; L.Engine().tuning_save(sys.argv[1])"
    env = dict(os.environ, LUTHE_TUNING_DIR=str(d))
    out = subprocess.run([sys.executable, "-c", code, str(seen)], cwd=ROOT, env=env, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert json.loads(seen.read_text()) == chosen
    # a file for another device or parameter set is refused
    bad = tmp_path / "bad.json"
    bad.write_text(path.read_text().replace(chosen["key"], "other_device"))
    with pytest.raises(L.LutheError):
        engine.tuning_load(bad)
    engine.tuning_load(path)
    # the tuned shape computes the same outputs as the oracle
    count = 2 * 148 + 60
    msgs = rng.integers(0, 16, count).astype(np.uint32)
    ct = L.encrypt(params, keys["glwe_key"], msgs, 55)
    ids = np.zeros(count, np.uint32)
    d_out = to_dev(np.zeros_like(ct))
    engine.ks_pbs(to_dev(ct), to_dev(ids), d_out, count)
    engine.check_device_error()
    got = from_dev(d_out, np.uint64)
    assert np.array_equal(got, oracle_bsk.ks_pbs(keys["ksk"], ct, luts, ids))
    engine.set_br_config(2, 1)  # back to the default shape for the other tests
