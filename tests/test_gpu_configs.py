"""The workload configurations beyond the benchmark's, on the GPU.

* 3D Kelvin-Helmholtz, p=5 (216 points per element), seeded noise on the
  shear layer, NAD+SED+PAD with the MUSCL fallback: bit for bit against the
  oracle (6^3 elements, the size the oracle steps in seconds).
* 2D Rayleigh-Taylor at its full size (512 x 1536 elements, p=3, gravity
  -0.1, periodic x, reflective y; 12.6M DOF): a few steps of the plain FP64
  form, the FP32 form and the FP32 form with the learned indicator --
  size-independent properties: mass conserved to round-off (no mass crosses
  a periodic or reflective edge), densities positive and finite, the FP32
  form within 1e-4 relative L1 of FP64 per field (momentum components
  against the momentum's norm), mirror symmetry about
  x = 0.25 kept to 1e-12, and the indicator's a-priori flags scored against the
  same steps' a-posteriori labels.
"""
import numpy as np
import pytest

from helpers import gpu_config, oracle_active, oracle_config, rel_l1, same_bits

pytestmark = pytest.mark.gpu

KH3D = ["job/fallback=true", "mesh/p=5", "mesh/nx1=6", "mesh/nx2=6", "mesh/nx3=6", "problem/problem=kh_noise"]
KH_EXTRA = {"q": [1e-3], "seed": 20261203}
RTI = ["job/fallback=true", "mesh/p=3", "mesh/nx1=512", "mesh/nx2=1536", "mesh/nx3=1", "mesh/x1len=0.5",
       "mesh/x2len=1.5", "mesh/x1_bc=periodic", "mesh/x2_bc=reflective", "problem/problem=rti_top", "hydro/g2=-0.1"]


def test_kh3d_p5_noise_matches_oracle():
    import spd_k_b200 as S
    from oracle import oracle as O
    g = S.HydroSolver(dict(gpu_config(KH3D), **KH_EXTRA))
    o = O.Oracle(dict(oracle_config(KH3D), **KH_EXTRA))
    dt = o.compute_dt()
    assert g.dt() == dt
    for k in range(2):
        g.step()
        o.step(dt)
        dt = o.compute_dt()
        assert g.dt() == dt, f"dt after step {k + 1}"
        wg = g.to_reference_slots(g.field_array(S.FIELD_W_CV))
        assert same_bits(wg, oracle_active(o, "W_cv")), (k, rel_l1(oracle_active(o, "W_cv"), wg))
        ug = g.to_reference_slots(g.field_array(S.FIELD_U_SP))
        assert same_bits(ug, oracle_active(o, "U_sp")), k
    assert float(o.array("troubles")[5].sum()) > 0   # the fallback acted
    g.close()


def _mass_and_rho(g):
    n = g.p + 1
    Nx, Ny = g.N[0], g.N[1]
    xg = (np.polynomial.legendre.leggauss(n - 1)[0] + 1) / 2
    xf = np.concatenate([[0.0], xg, [1.0]])
    hx = np.tile(np.diff(xf), Nx) * (g.c["L"][0] / Nx)
    hy = np.tile(np.diff(xf), Ny) * (g.c["L"][1] / Ny)
    w = g.field_array(1)
    rho = w[0, 0, :, :, 0].transpose(0, 2, 1, 3).reshape(Ny * n, Nx * n)
    return float((rho * hy[:, None] * hx[None, :]).sum()), rho


def test_rti_full_size_properties_and_indicator():
    import os
    import spd_k_b200 as S
    from spd_k_b200.api import FIELD_ELEMENT_PREDICTED, FIELD_ELEMENT_TROUBLES
    from spd_k_b200.learned import Indicator, set_indicator
    weights = os.path.join(os.path.dirname(S.__file__), "data", "indicator_2d_p3.npz")
    steps = 4
    res = {}
    for form in ("fp64", "fp32", "fp32+learned"):
        c = dict(gpu_config(RTI), precision="fp32" if form != "fp64" else "fp64")
        g = S.HydroSolver(c)
        ind = None
        if form == "fp32+learned":
            ind = Indicator.load(weights)
            set_indicator(g, ind)
        m0, _ = _mass_and_rho(g)
        pred = lab = 0
        fp = fn = 0
        for _ in range(steps):
            g.step()
            if form == "fp32+learned":
                p_ = g.read(FIELD_ELEMENT_PREDICTED) > 0
                l_ = g.read(FIELD_ELEMENT_TROUBLES) > 0
                pred, lab = pred + int(p_.sum()), lab + int(l_.sum())
                fp, fn = fp + int((p_ & ~l_).sum()), fn + int((~p_ & l_).sum())
        g.sync()
        m1, rho = _mass_and_rho(g)
        u = g.field_array(0)
        assert np.all(np.isfinite(u)) and rho.min() > 0, form
        drift = abs(m1 - m0) / m0
        assert drift < (1e-12 if form == "fp64" else 1e-6), (form, drift)
        res[form] = (u, rho, g.read(S.FIELD_TROUBLES).sum(), pred, lab, fp, fn)
        g.close()
    u64, rho64, tr64 = res["fp64"][:3]
    assert tr64 > 0   # the density jump at y = 0.75 trips the detector
    # mirror symmetry about x = 0.25 (the perturbation is cos(4 pi x))
    # (the mirrored quadrature points round differently, and a detector
    # decision can turn that round-off into a local difference)
    sym = float(np.abs(rho64 - rho64[:, ::-1]).sum() / np.abs(rho64).sum())
    print(f"\nRTI 512x1536 mirror asymmetry (relative L1) after {steps} steps: {sym:.2e}")
    assert sym < 1e-12
    # density and energy against their own L1 norms; the momentum
    # components against the momentum's (the x momentum is born from the
    # perturbation and stays 1e-6 of the density after a few steps)
    u32 = res["fp32"][0]
    mom = float(np.abs(u64[1:3]).sum())
    errs = [float(np.abs(u32[v] - u64[v]).sum() / (mom if v in (1, 2) else np.abs(u64[v]).sum()))
            for v in range(u64.shape[0])]
    print(f"\nRTI 512x1536 fp32 vs fp64 relative L1 after {steps} steps: {errs}")
    assert max(errs) < 1e-4, errs
    pred, lab, fp, fn = res["fp32+learned"][3:]
    print(f"indicator on RTI: predicted {pred}, labelled {lab}, false positives {fp}, false negatives {fn}")
    assert lab > 0


KH64 = ["job/fallback=true", "mesh/p=5", "mesh/nx1=64", "mesh/nx2=64", "mesh/nx3=64", "problem/problem=kh_noise"]


def _mass3d(g):
    """total mass of a 3D run on the unit box: W_cv density sub-cell averages
    times the sub-cell volumes (faces at 0, the p Gauss-Legendre points and 1
    of each element), summed in FP64"""
    n = g.p + 1
    xg = (np.polynomial.legendre.leggauss(n - 1)[0] + 1) / 2
    hs = np.diff(np.concatenate([[0.0], xg, [1.0]]))   # sub-cell widths of one element (unit)
    Nx, Ny, Nz = g.N
    vol = (hs[:, None, None] * hs[None, :, None] * hs[None, None, :]) / (Nx * Ny * Nz)
    rho = g.field_array(1)[0]                          # (Nz, Ny, Nx, nz, ny, nx)
    return float((rho * vol[None, None, None]).sum())


def test_kh3d_64_p5_full_size():
    """The 3D Kelvin-Helmholtz configuration at its stated size (64^3 elements,
    p = 5: 56.6M DOF) in the plain FP64 form and the FP32 form: device memory,
    a few steps each (graph-replayed), mass conserved to round-off on the
    periodic box, finite state with positive density, the FP32 form within
    1e-5 relative L1 of FP64 per field after the same steps."""
    import time

    import torch

    import spd_k_b200 as S
    steps = 3
    res = {}
    for prec in ("fp64", "fp32"):
        g = S.HydroSolver(dict(gpu_config(KH64), precision=prec, **KH_EXTRA))
        mass0 = _mass3d(g)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.steps(steps)
        g.sync()
        ms = (time.perf_counter() - t0) * 1e3 / steps
        u = g.read(S.FIELD_U_SP)
        wcv = g.field_array(S.FIELD_W_CV)
        assert np.all(np.isfinite(u)) and float(wcv[0].min()) > 0, prec
        drift = abs(_mass3d(g) - mass0) / mass0
        assert drift < (1e-12 if prec == "fp64" else 1e-6), (prec, drift)
        res[prec] = (u, g.info.device_bytes, ms, drift)
        g.close()
    u64, mem64, ms64, d64 = res["fp64"]
    u32, mem32, ms32, d32 = res["fp32"]
    errs = [float(np.abs(u32.reshape(-1, 5, 216)[:, v] - u64.reshape(-1, 5, 216)[:, v]).sum() /
                  np.abs(u64.reshape(-1, 5, 216)[:, v]).sum()) for v in (0, 4)]
    print(f"\nKH 64^3 p=5: device memory fp64 {mem64 / 1e9:.1f} GB, fp32 {mem32 / 1e9:.1f} GB; "
          f"wall time per step fp64 {ms64:.1f} ms, fp32 {ms32:.1f} ms; mass drift fp64 {d64:.1e}, fp32 {d32:.1e}; "
          f"fp32 vs fp64 relative L1 (rho, E) {errs}")
    assert mem64 < 150e9 and mem32 < mem64
    assert max(errs) < 1e-5


def test_rti_indicator_over_a_long_run():
    """The Rayleigh-Taylor configuration at its full size, stepped well past
    the start: the learned indicator's false-positive and false-negative
    rates against the plain NAD run stepped alongside (same form, no
    indicator), every 100 steps, and the L1 difference of the two runs'
    densities at the end."""
    import os
    import spd_k_b200 as S
    from spd_k_b200.api import FIELD_ELEMENT_PREDICTED, FIELD_ELEMENT_TROUBLES
    from spd_k_b200.learned import Indicator, set_indicator
    weights = os.path.join(os.path.dirname(S.__file__), "data", "indicator_2d_p3.npz")
    c = dict(gpu_config(RTI), precision="fp32")
    plain, learned = S.HydroSolver(c), S.HydroSolver(c)
    ind = Indicator.load(weights)
    set_indicator(learned, ind)
    total, every = 1000, 100
    rows = []
    fp = fn = pos = neg = 0
    for k in range(1, total + 1):
        plain.step()
        learned.step()
        pred = learned.read(FIELD_ELEMENT_PREDICTED) > 0
        lab = plain.read(FIELD_ELEMENT_TROUBLES) > 0
        fp += int((pred & ~lab).sum())
        fn += int((~pred & lab).sum())
        pos += int(lab.sum())
        neg += int((~lab).sum())
        if k % every == 0:
            rows.append((k, plain.t if hasattr(plain, "t") else None, fp / max(neg, 1), fn / max(pos, 1), pos / every))
            fp = fn = pos = neg = 0
    wp, wl = plain.field_array(1), learned.field_array(1)
    l1 = [float(np.abs(wl[v] - wp[v]).sum() / np.abs(wp[v]).sum()) for v in range(wp.shape[0])]
    print("\nRTI 512x1536 fp32, learned indicator vs the plain run (per 100 steps): step, FPR, FNR, "
          "labelled elements per step")
    for k, _, fpr, fnr, lab in rows:
        print(f"  {k:5d}  FPR {fpr:.4f}  FNR {fnr:.4f}  labelled {lab:.0f}")
    print(f"  W_cv relative L1 learned vs plain after {total} steps: {l1}")
    assert all(np.isfinite(l1))
    set_indicator(learned, None)
    ind.close()
    plain.close()
    learned.close()
