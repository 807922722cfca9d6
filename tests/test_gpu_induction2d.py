"""The 2D induction solver (spdk_induction2d_*): 2D field-loop advection.

Parity: the reference built with the loop's velocity and centre
(oracle/patch_loop2d.py) and run quasi-2D (nx3 = 2, periodic, B_z = 0) gives
B2_cv fixtures (tests/golden/loop2d_*.npz, made by make_fixtures.py
--loop2d); the FP64 form reproduces them bit for bit, ADER and SSP-RK2,
uniform and non-uniform element sizes. The precision form (FP32 state) is
compared with the FP64 form by their errors against the exact solution (the
initial field translated by v t). The full configuration -- [-1, 1]^2
periodic (as [0, 2]^2 with the loop at (1, 1)), 512^2 elements, p = 4,
v = (2, 1), A_z = 1e-3 (0.3 - r), to t = 1 -- runs in both forms.
"""
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN, same_bits

pytestmark = pytest.mark.gpu


def manifest_cases():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f).get("loop2d_cases", {})


def config_from_overrides(ov, precision="fp64"):
    from spd_k_b200.induction import field_loop_config
    d = dict(o.split("=", 1) for o in ov)
    c = field_loop_config(N=int(d["mesh/nx1"]), p=int(d["mesh/p"]), precision=precision,
                          integrator=d.get("time/integrator", "ader"))
    c["N"] = [int(d["mesh/nx1"]), int(d["mesh/nx2"])]
    c["L"] = [float(d["mesh/x1len"]), float(d["mesh/x2len"])]
    c["cfl"] = float(d["time/cfl"])
    return c, float(d["time/tlim"]), float(d["output/dt"])


@pytest.mark.parametrize("case", sorted(manifest_cases()))
def test_matches_patched_reference(case):
    from spd_k_b200.induction import Induction2D
    entry = manifest_cases()[case]
    c, tlim, dt_out = config_from_overrides(entry["overrides"])
    s = Induction2D(c)
    steps = s.evolve(tlim, dt_out)
    assert steps == entry["steps"]
    want = np.load(os.path.join(GOLDEN, case + ".npz"))["B2_cv"]
    got = s.b2_cv()
    assert got.shape == want.shape
    assert same_bits(got, want), np.abs(got - want).max()
    s.close()


def loop_error(N, p, t_end, precision):
    """L1 of (Bx, By) sub-cell averages at t_end against the initial field
    translated by v t_end (a whole number of elements here), relative to the
    initial field's L1"""
    from spd_k_b200.induction import Induction2D, field_loop_config
    c = field_loop_config(N=N, p=p, precision=precision)
    s = Induction2D(c)
    b0 = s.b2_cv()
    steps = s.evolve(t_end, t_end)
    b = s.b2_cv()
    s.close()
    L = c["L"][0]
    shift = [int(round(c["velocity"][d] * t_end / (L / N))) % N for d in range(2)]
    exact = np.roll(b0, shift=(shift[1], shift[0]), axis=(1, 2))
    err = [float(np.abs(b[v] - exact[v]).sum() / np.abs(exact[v]).sum()) for v in range(2)]
    return err, steps


def test_fp32_matches_fp64_error():
    """64^2, p = 4, to t = 0.5 (the loop moves by (1, 0.5)): both forms'
    errors against the translated initial field agree to 1 %"""
    e64, n64 = loop_error(64, 4, 0.5, "fp64")
    e32, n32 = loop_error(64, 4, 0.5, "fp32")
    print(f"\nloop 64^2 p=4 t=0.5: fp64 {e64}  fp32 {e32}  ({n64} steps)")
    assert n64 == n32
    for a, b in zip(e64, e32):
        assert a < 0.05
        assert abs(b - a) <= 0.01 * a


def test_field_loop_512_to_t1():
    """the full configuration in both forms: errors against the initial field
    translated by (2, 1), the loop's peak |B|^2 kept, FP32 within 1 % of FP64"""
    res = {}
    for prec in ("fp64", "fp32"):
        res[prec] = loop_error(512, 4, 1.0, prec)
    print(f"\nloop 512^2 p=4 t=1: fp64 {res['fp64']}  fp32 {res['fp32']}")
    (e64, n64), (e32, n32) = res["fp64"], res["fp32"]
    assert n64 == n32
    for a, b in zip(e64, e32):
        assert a < 0.01
        assert abs(b - a) <= 0.01 * a
