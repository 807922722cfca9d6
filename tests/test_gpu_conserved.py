"""FP64 conservation sums (spdk_hydro_conserved): the domain integrals of
rho, the momenta and E from the sub-cell averages, compensated sums.

A uniform state integrates to its value times the box volume; periodic
runs without the fallback conserve every integral to FP64 round-off in the
plain form (2D and 3D) and to FP32 round-off in the precision form; the
sums are reproducible call to call.
"""
import numpy as np
import pytest

from helpers import gpu_config

pytestmark = pytest.mark.gpu

SINE = ["job/fallback=false", "mesh/p=3", "mesh/nx1=16", "mesh/nx2=16", "mesh/nx3=1", "time/tlim=0.1",
        "output/dt=0.1"]


def solver(ov, precision="fp64"):
    import spd_k_b200 as S
    c = gpu_config(ov)
    c["precision"] = precision
    return S.HydroSolver(c)


def test_uniform_state_integrates_to_value_times_volume():
    g = solver(SINE + ["mesh/x1len=2", "mesh/x2len=0.5"])
    E, V, npt = g.info.n_elements, g.nvar, g.npt
    vals = np.array([1.5, 0.25, -0.5, 3.0])
    u = np.broadcast_to(vals[None, :, None], (E, V, npt)).copy()
    g.write_u(u)
    s = g.conserved()
    assert np.allclose(s, vals * 1.0, rtol=1e-14, atol=1e-15), s
    assert np.array_equal(s, g.conserved())
    g.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 2e-14), ("fp32", 2e-6)])
def test_periodic_runs_conserve_every_integral(precision, tol):
    g = solver(SINE, precision)
    s0 = g.conserved()
    # rho = 1 + 0.125 sin(2 pi (x + y)), v = (1, 1), P = 1 on the unit box
    assert abs(s0[0] - 1.0) < 1e-6 and abs(s0[1] - 1.0) < 1e-6 and abs(s0[2] - 1.0) < 1e-6
    for _ in range(20):
        g.step()
    s1 = g.conserved()
    rel = np.abs(s1 - s0) / np.abs(s0)
    print(f"\n{precision}: integrals {s0} -> {s1}, relative change {rel}")
    assert (rel < tol).all(), rel
    g.close()


def test_3d_periodic_run_conserves_every_integral():
    g = solver(["job/fallback=false", "mesh/p=3", "mesh/nx1=6", "mesh/nx2=6", "mesh/nx3=6", "problem/problem=kh_noise"])
    s0 = g.conserved()
    for _ in range(3):
        g.step()
    s1 = g.conserved()
    scale = np.maximum(np.abs(s0), 1e-3 * np.abs(s0).max())
    assert (np.abs(s1 - s0) / scale < 1e-13).all(), (s0, s1)
    g.close()


def test_slab_solvers_are_rejected():
    import spd_k_b200 as S
    from spd_k_b200.api import SpdkError
    c = gpu_config(SINE + ["mesh/x2_bc=gradfree"])
    g = S.HydroSolver(dict(c, N=[16, 8, 1], slab_lo=4, slab_n=16))
    with pytest.raises(SpdkError, match="slab"):
        g.conserved()
    g.close()
