"""The athinput-driven driver (spd_k_b200/spdk_run, the reference's
src/main.cpp on the C ABI): run from a deck plus block/name=value overrides
it writes the reference's output files, compared here with the reference's
own outputs (the committed induction golden byte for byte, a hydro fixture
on the active elements)."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

from helpers import fixture, manifest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "spd_k_b200", "spdk_run")
M = manifest()


def run(args, out):
    env = dict(os.environ, SPD_OUTPUT_DIR=str(out))
    r = subprocess.run([DRIVER] + args, capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def test_induction_deck_reproduces_reference_golden(tmp_path):
    deck = tmp_path / "induction_loop.athinput"
    deck.write_text("<job>\nsystem = induction\nfallback = true\n<mesh>\np = 3\nnx1 = 8\nnx2 = 8\nnx3 = 8\n"
                    "<time>\ntlim = 0.2\ncfl = 0.8\n<output>\ndt = 0.1\n<induction>\nnu = 0.0025\n")
    out = run(["-i", str(deck)], tmp_path)
    assert "evolution: 17 steps" in out
    got = hashlib.sha256((tmp_path / "B2_cv_N8p3_2_0.dat").read_bytes()).hexdigest()
    assert got == M["goldens"]["induction_fv/B2_cv_N8p3_2_0.dat"]["sha256"]
    info = M["induction_cases"]["ind_golden_n8"]
    got_t = hashlib.sha256((tmp_path / info["troubles_output"]).read_bytes()).hexdigest()
    assert got_t == info["sha256_troubles"]


@pytest.mark.parametrize("case", ["blast2d_fallback", "sine2d_rk3"])
def test_hydro_overrides_reproduce_reference_fixture(tmp_path, case):
    info = M["cases"][case]
    out = run(info["overrides"], tmp_path)
    assert f"evolution: {info['steps']} steps" in out
    w = np.fromfile(tmp_path / info["output"])
    ref = fixture(case)                               # (5, 1, Ny, Nx, 1, n, n) active
    _, _, Ny, Nx, _, n, _ = ref.shape
    full = w.reshape(1, 6, 1, Ny + 2, Nx + 2, 1, n, n)[0, :5, :, 1:-1, 1:-1]
    assert np.array_equal(full, ref)
    assert np.all(np.isnan(w.reshape(1, 6, 1, Ny + 2, Nx + 2, 1, n, n)[0, :5, :, 0]))
