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
