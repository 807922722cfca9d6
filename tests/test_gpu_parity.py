"""Parity of the sm_100a path with the reference, through the C ABI.

Bit-for-bit (IEEE value equality, NaN = NaN) against:
  - the reference's own outputs (tests/golden fixtures, made by the
    reference build), run with the reference's time loop and output clamping;
  - the oracle, step by step, from seeded random states that trip the
    trouble detector everywhere (every fallback path is exercised);
and, at the benchmark size (256x256, p=3), size-independent properties:
graph replay = step-by-step, run-to-run determinism, mass conservation while
the blast is inside the box, diagonal symmetry, positivity.
"""
import zlib

import numpy as np
import pytest

from helpers import (fixture, gpu_config, gpu_run, manifest, oracle_active, oracle_config, rel_l1, same_bits)

pytestmark = pytest.mark.gpu
M = manifest()


def solver(overrides, **extra):
    import spd_k_b200 as S
    return S.HydroSolver(dict(gpu_config(overrides), **extra))


@pytest.mark.parametrize("case", sorted(M["cases"]))
def test_matches_reference_fixture(case):
    info = M["cases"][case]
    w, steps, g = gpu_run(info["overrides"])
    ref = fixture(case)
    assert steps == info["steps"]
    assert same_bits(w, ref), rel_l1(ref, w)
    g.close()


@pytest.mark.parametrize("case", sorted(M.get("viscous_cases", {})))
def test_viscous_run_matches_reference_fixture(case):
    """hydro/nu > 0 (interface states, gradients, viscous fluxes, interface
    sums, diffusion dt limit), 2D/3D, ADER/SSP-RK2, with and without the
    fallback: the reference's W_cv and step count, bit for bit"""
    info = M["viscous_cases"][case]
    w, steps, g = gpu_run(info["overrides"])
    assert steps == info["steps"]
    assert same_bits(w, fixture(case)), rel_l1(fixture(case), w)
    g.close()


@pytest.mark.parametrize("case", sorted(M.get("bench_cases", {})))
def test_benchmark_geometry_matches_reference(case):
    """The benchmark workload itself (2D point blast, NAD+MUSCL, outflow) at
    64x64 and at the full 256x256 for a few steps: the reference's W_cv, bit
    for bit (signed zeros folded)."""
    import hashlib
    info = M["bench_cases"][case]
    w, steps, g = gpu_run(info["overrides"])
    assert steps == info["steps"]
    a4 = np.ascontiguousarray(w[[0, 1, 2, 4]]) + 0.0
    ref = np.load(f"tests/golden/{case}.npz")["W_cv"]
    assert same_bits(a4, ref), rel_l1(ref, a4)
    assert hashlib.sha256(a4.tobytes()).hexdigest() == info["sha256_signed_zero_folded"]
    g.close()


def test_config1_full_run_matches_reference():
    """2D sine wave 32x32, p=3, ADER, to t=1 (725 steps): the reference's
    result, bit for bit, and its L1 error against the exact solution."""
    import hashlib
    info = M["full_cases"]["config1_sine2d_32"]
    w, steps, g = gpu_run(info["overrides"])
    assert steps == info["steps"] == 725
    ref = np.load("tests/golden/config1_sine2d_32.npz")
    assert same_bits(w[0], ref["rho"]) and same_bits(w[4], ref["p"])
    act4 = np.ascontiguousarray(w[[0, 1, 2, 4]])
    assert hashlib.sha256(act4.tobytes()).hexdigest() == info["sha256_active_rho_vx_vy_p"]
    g.close()


def test_sine3d_matches_oracle_golden_config():
    """The configuration of the reference's committed 3D golden (the oracle
    reproduces that file byte for byte in the CPU suite)."""
    from helpers import oracle_run
    ov = ["job/fallback=false", "mesh/nx1=8", "mesh/nx2=8", "mesh/nx3=8", "time/tlim=0.1", "output/dt=0.1"]
    wo, so, o, _ = oracle_run(ov)
    wg, sg, g = gpu_run(ov)
    assert so == sg == 24
    assert same_bits(wg, wo)
    g.close()


def random_state(c, seed):
    """seeded primitive state -> conserved U in solver and oracle layouts"""
    rng = np.random.default_rng(seed)
    D = 3 if c["N"][2] > 1 else 2
    n = c["p"] + 1
    Nx, Ny, Nz = c["N"][0], c["N"][1], (c["N"][2] if D == 3 else 1)
    nz = n if D == 3 else 1
    shp = (Nz, Ny, Nx, nz, n, n)
    rho = rng.uniform(0.5, 1.5, shp)
    vel = [rng.uniform(-0.5, 0.5, shp) for _ in range(D)]
    p = rng.uniform(0.5, 1.5, shp)
    gm = c["gamma"]
    ek = sum(v * rho * v for v in vel)
    E = p / (gm - 1.0) + 0.5 * ek
    slots = [rho] + [rho * v for v in vel] + [E]
    mine = np.stack(slots, axis=3)  # (Nz,Ny,Nx,V,nz,n,n)
    ref = [rho] + [rho * v for v in vel] + ([np.zeros(shp)] if D == 2 else []) + [E]
    ref = np.stack(ref, axis=0)  # (5,Nz,Ny,Nx,nz,n,n)
    return mine, ref, D


def load_oracle_state(o, ref5, D):
    full = o.array("U_sp", copy=False)
    full[...] = 0.0
    full[0, 0] = 1.0          # ghost elements: a valid resting state
    full[0, 4] = 2.5
    if D == 2:
        full[0, :, :, 1:-1, 1:-1] = ref5
    else:
        full[0, :, 1:-1, 1:-1, 1:-1] = ref5
    o.call("primitives_to_cv")


RANDOM_CASES = {
    "2d_p3_fallback": ["job/fallback=true", "mesh/nx1=8", "mesh/nx2=8", "mesh/nx3=1"],
    "2d_p3_fallback_reflective": ["job/fallback=true", "mesh/nx1=8", "mesh/nx2=4", "mesh/nx3=1",
                                  "mesh/x1_bc=reflective", "mesh/x2_bc=gradfree"],
    "2d_p2_rk3_fallback": ["job/fallback=true", "mesh/p=2", "mesh/nx1=6", "mesh/nx2=6", "mesh/nx3=1",
                           "time/integrator=rk3"],
    "2d_p4_ader": ["job/fallback=false", "mesh/p=4", "mesh/nx1=4", "mesh/nx2=8", "mesh/nx3=1"],
    "2d_p5_fallback_noblend": ["job/fallback=true", "mesh/p=5", "mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=1",
                               "fallback/blending=false", "fallback/NAD_neighbors=1st"],
    "2d_p3_gravity_delta": ["job/fallback=true", "mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=1",
                            "hydro/g2=-0.5", "hydro/g1=0.25", "fallback/NAD=delta"],
    "3d_p2_fallback": ["job/fallback=true", "mesh/p=2", "mesh/nx1=3", "mesh/nx2=4", "mesh/nx3=2",
                       "mesh/x3_bc=reflective"],
    "3d_p3_rk2": ["job/fallback=false", "mesh/nx1=2", "mesh/nx2=3", "mesh/nx3=2", "time/integrator=rk2",
                  "hydro/g3=0.3"],
    # 3D tiles of 2x1x1 elements (p <= 3, even nx1), with the fallback
    "3d_p3_fallback_tile2": ["job/fallback=true", "mesh/nx1=2", "mesh/nx2=3", "mesh/nx3=2", "mesh/x2_bc=reflective"],
    "3d_p2_fallback_tile2": ["job/fallback=true", "mesh/p=2", "mesh/nx1=4", "mesh/nx2=3", "mesh/nx3=2",
                             "mesh/x1_bc=gradfree"],
    # FP64 tiles of 2x2x1 elements (p = 2, 3, even nx1 and nx2), with and
    # without the fallback
    "3d_p2_ader_tile22_423": ["job/fallback=false", "mesh/p=2", "mesh/nx1=4", "mesh/nx2=2", "mesh/nx3=3"],
    "3d_p2_fallback_tile22_443": ["job/fallback=true", "mesh/p=2", "mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=3",
                                  "mesh/x2_bc=reflective"],
    "3d_p3_fallback_tile22_443": ["job/fallback=true", "mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=3",
                                  "mesh/x1_bc=gradfree"],
    "3d_p3_ader_tile22_423": ["job/fallback=false", "mesh/nx1=4", "mesh/nx2=2", "mesh/nx3=3"],
    # viscous terms on every boundary kind, ADER and SSP-RK, with the fallback
    "2d_p3_viscous_fallback_reflective": ["job/fallback=true", "mesh/nx1=6", "mesh/nx2=4", "mesh/nx3=1",
                                          "mesh/x1_bc=reflective", "mesh/x2_bc=gradfree", "hydro/nu=0.02"],
    "2d_p2_rk3_viscous_beta": ["job/fallback=false", "mesh/p=2", "mesh/nx1=6", "mesh/nx2=6", "mesh/nx3=1",
                               "time/integrator=rk3", "hydro/nu=0.05", "hydro/beta=0.01"],
    "2d_p4_viscous_gravity": ["job/fallback=false", "mesh/p=4", "mesh/nx1=4", "mesh/nx2=6", "mesh/nx3=1",
                              "hydro/nu=0.01", "hydro/g2=-0.3", "mesh/x2_bc=reflective"],
    "3d_p2_viscous_fallback": ["job/fallback=true", "mesh/p=2", "mesh/nx1=3", "mesh/nx2=2", "mesh/nx3=3",
                               "mesh/x3_bc=reflective", "mesh/x1_bc=gradfree", "hydro/nu=0.01"],
}


@pytest.mark.parametrize("case", sorted(RANDOM_CASES))
def test_random_state_steps_match_oracle(case):
    from oracle import oracle as O
    ov = RANDOM_CASES[case]
    cg, co = gpu_config(ov), oracle_config(ov)
    mine, ref5, D = random_state(cg, seed=zlib.crc32(case.encode()))
    g = solver(ov)
    g.write_u(mine)
    o = O.Oracle(co)
    load_oracle_state(o, ref5, D)
    assert g.dt() == o.compute_dt()
    dt = o.compute_dt()
    for step in range(3):
        o.step(dt)
        g.step()
        dt = o.compute_dt()
        assert g.dt() == dt, f"dt after step {step + 1}"
        wo = oracle_active(o, "W_cv")
        wg = g.to_reference_slots(g.field_array(1))
        assert same_bits(wg, wo), (step, rel_l1(wo, wg))
        uo = oracle_active(o, "U_sp")
        ug = g.to_reference_slots(g.field_array(0))
        assert same_bits(ug, uo), (step, rel_l1(uo, ug))
    g.close()


def test_trouble_flags_match_oracle():
    """the last fallback slice's trouble aggregate, sub-cell by sub-cell"""
    from oracle import oracle as O
    ov = RANDOM_CASES["2d_p3_fallback"]
    cg, co = gpu_config(ov), oracle_config(ov)
    mine, ref5, D = random_state(cg, seed=7)
    g = solver(ov)
    g.write_u(mine)
    o = O.Oracle(co)
    load_oracle_state(o, ref5, D)
    dt = o.compute_dt()
    o.step(dt)
    g.step()
    g.sync()
    tr = o.array("troubles")[5, 0, 2:-2, 2:-2, 0, 0, 0, 0]  # (Y, X) aggregate over the active frame
    n = 4
    tg = g.read(2).reshape(8, 8, n, n).transpose(0, 2, 1, 3).reshape(8 * n, 8 * n)
    assert tr.sum() > 0
    assert np.array_equal(tg, tr)
    g.close()


def bench_overrides(N=256):
    import bench
    return bench.workload_overrides(N)


def test_graph_replay_equals_stepping_and_is_deterministic():
    ov = bench_overrides(64)
    a, b, c = solver(ov), solver(ov), solver(ov)
    a.steps(12)
    a.sync()
    for _ in range(12):
        b.step()
    c.steps(12)
    c.sync()
    ua, ub, uc = a.read(0), b.read(0), c.read(0)
    assert same_bits(ua, ub) and same_bits(ua, uc)
    assert a.dt() == b.dt() == c.dt()
    for s in (a, b, c):
        s.close()


def test_benchmark_size_properties():
    """256x256, p=3 point blast: 40 graph steps from the initial state."""
    g = solver(bench_overrides(256))
    w0 = g.field_array(1)
    n = 4
    g.steps(40)
    g.sync()
    w = g.field_array(1)
    u = g.field_array(0)
    assert np.all(np.isfinite(w)) and np.all(np.isfinite(u))
    # (W_cv may hold negative pressures: it averages point values of the
    # reconstructed polynomial; the reference shows the same at 64x64)
    # mass: sub-cell averages times sub-cell volumes (the blast is far from the edges)
    xg = (np.polynomial.legendre.leggauss(3)[0] + 1) / 2       # interior flux points
    xf = np.concatenate([[0.0], xg, [1.0]])
    hx = np.tile(np.diff(xf), 256) / 256                       # sub-cell widths
    vol = hx[:, None] * hx[None, :]
    def mass(a):
        rho = a[0, 0, :, :, 0].transpose(0, 2, 1, 3).reshape(256 * n, 256 * n)
        return float((rho * vol).sum())
    m0, m1 = mass(w0), mass(w)
    assert abs(m1 - m0) / m0 < 1e-12
    # symmetry of the blast about the diagonal x = y: x and y terms are
    # evaluated in a fixed order, and the trouble detector's yes/no decisions
    # amplify that round-off (the reference shows 2e-13 after 12 steps; by
    # 40 steps single flipped flags give local O(1e-2) differences), so the
    # check is on the L1 norm
    rho = w[0, 0, :, :, 0].transpose(0, 2, 1, 3).reshape(256 * n, 256 * n)
    assert np.abs(rho - rho.T).sum() < 1e-4 * np.abs(rho).sum()
    # the fallback is active around the blast
    tr = g.read(2)
    assert tr.sum() > 0
    g.close()
