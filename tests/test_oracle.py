"""The CPU oracle against the reference's own outputs (no GPU).

Pins the C restatement in oracle/ to the reference: every fixture under
tests/golden was produced by the reference build (tests/golden/make_fixtures.py)
and must be reproduced bit for bit, including the raw dump bytes (ghost
elements and their NaNs); the 3D case must reproduce the reference's own
committed golden file byte for byte.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from helpers import (GOLDEN, fixture, manifest, oracle_run, reference_file_bytes, same_bits, sha256_bytes)

M = manifest()


@pytest.mark.parametrize("case", sorted(M["cases"]))
def test_oracle_reproduces_reference_fixture(case):
    info = M["cases"][case]
    w, steps, o, full = oracle_run(info["overrides"])
    assert steps == info["steps"]
    assert same_bits(w, fixture(case))
    assert sha256_bytes(reference_file_bytes(full)) == info["sha256"]


@pytest.mark.parametrize("case", sorted(M.get("viscous_cases", {})))
def test_oracle_reproduces_reference_viscous_fixture(case):
    """hydro/nu > 0 (src/hydro.cpp:420-572: interface states, gradients,
    viscous fluxes, interface sums; the diffusion dt limit), in 2D and 3D,
    ADER and SSP-RK2, with and without the fallback, beta given or default"""
    info = M["viscous_cases"][case]
    w, steps, o, full = oracle_run(info["overrides"])
    assert steps == info["steps"]
    assert same_bits(w, fixture(case))
    assert sha256_bytes(reference_file_bytes(full)) == info["sha256"]


def test_oracle_reproduces_reference_golden_3d():
    """tests/goldens/hydro_sd/W_cv_N8p3_1_0.dat of the reference: 3D sine
    wave, N=8, p=3, ADER, t=0.1 (its run_tests.py hydro_sd_3d case)."""
    want = M["goldens"]["hydro_sd/W_cv_N8p3_1_0.dat"]["sha256"]
    ov = ["job/fallback=false", "mesh/nx1=8", "mesh/nx2=8", "mesh/nx3=8", "time/tlim=0.1", "output/dt=0.1"]
    w, steps, o, full = oracle_run(ov)
    assert steps == 24
    assert sha256_bytes(reference_file_bytes(full)) == want


def test_oracle_analytic_l1_sine2d():
    """run_tests.py check_analytic: L1(rho) of the 2D sine wave at N=8,
    p=3, t=0.1 is below 3e-5 (reference measured 2.16e-5 in 3D)."""
    w, steps, o, _ = oracle_run(["job/fallback=false", "mesh/nx3=1", "time/tlim=0.1", "output/dt=0.1"])
    xf = o.array("fv_faces_x")[:, 0][2:-2]
    a, t = 2 * np.pi, o.t
    F = lambda x, y: -np.sin(a * (x + y - 2 * t)) / a ** 2
    X0, Y0 = np.meshgrid(xf[:-1], xf[:-1], indexing="ij")
    X1, Y1 = np.meshgrid(xf[1:], xf[1:], indexing="ij")
    exact = 1.0 + 0.125 * (F(X1, Y1) - F(X0, Y1) - F(X1, Y0) + F(X0, Y0)) / ((X1 - X0) * (Y1 - Y0))
    N, n = 8, 4
    rho = w[0, 0, :, :, 0].transpose(0, 2, 1, 3).reshape(N * n, N * n)  # (j,jj),(i,ii) -> y rows, x cols
    err = np.abs(rho - exact.T).mean()
    assert err < 3e-5


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "spd_K_ref")),
                    reason="reference build not present")
def test_oracle_matches_reference_binary_on_unseen_config():
    """A configuration no fixture covers (square advection, p=2, RK2,
    fallback, Von Neumann NAD, delta band, no blending), run by both."""
    from oracle import oracle as O
    ov = ["job/fallback=true", "mesh/p=2", "mesh/nx1=6", "mesh/nx2=6", "mesh/nx3=1",
          "problem/problem=square", "time/integrator=rk2", "fallback/NAD_neighbors=1st",
          "fallback/NAD=delta", "fallback/blending=false", "time/tlim=0.05", "output/dt=0.05"]
    with tempfile.TemporaryDirectory() as out:
        env = dict(os.environ, SPD_OUTPUT_DIR=out, OMP_NUM_THREADS="2")
        subprocess.run([O.REF_BIN] + ov, check=True, capture_output=True, env=env)
        ref = np.fromfile(os.path.join(out, "W_cv_N6p2_1_0.dat"))
    w, steps, o, full = oracle_run(ov)
    assert reference_file_bytes(full) == ref.tobytes()


def test_applied_induction_fallback_fixtures_are_not_the_plain_reference():
    """The applied-fallback fixtures (the reference with the upwind EMF step
    added, oracle/patch_indfb.py) flag troubles and differ from the plain
    reference on the same decks, so they pin the added step."""
    cases = M["indfb_cases"]
    plain = {"indfb_n8_p3_ader": "ind_golden_n8", "indfb_n6_p3_rk2": "ind_n6_p3_rk2_fv"}
    for name, info in cases.items():
        assert info["troubled_cells"] > 0
        if name in plain:
            other = M["induction_cases"][plain[name]]
            assert info["overrides"] == other["overrides"]
            assert info["sha256_B2_cv"] != other["sha256_B2_cv"]
    a = np.load(os.path.join(GOLDEN, "indfb_n6_p3_rk2.npz"))["B2_cv"]
    b = np.load(os.path.join(GOLDEN, "ind_n6_p3_rk2_fv.npz"))["B2_cv"]
    assert a.shape == b.shape and not np.array_equal(a, b)


@pytest.mark.skipif(not os.path.isdir(os.path.join(os.environ.get("SPDK_REFERENCE_ROOT", "/root/reference"), "src")),
                    reason="reference tree not present")
def test_applied_fallback_patch_recipe_applies():
    """oracle/patch_indfb.py finds each text it patches exactly once."""
    import importlib.util
    src = os.path.join(os.environ.get("SPDK_REFERENCE_ROOT", "/root/reference"), "src")
    spec = importlib.util.spec_from_file_location(
        "patch_indfb", os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "patch_indfb.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    with tempfile.TemporaryDirectory() as out:
        mod.main(src, out)
        text = open(os.path.join(out, "induction_ader.hpp")).read()
        assert text.count("spdk_apply_fallback(ader, X_dim, Y_dim, Z_dim);") == 1
        assert text.count("spdk_save_faces();") == 1
        assert sorted(os.listdir(out)) == ["induction_ader.hpp", "main.cpp", "spd_k.hpp"]
