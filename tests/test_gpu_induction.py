"""The induction solver (src/induction_ader.hpp) on the GPU against the
reference's own CPU build: the reference's committed golden
(tests/goldens/induction_fv/B2_cv_N8p3_2_0.dat of the reference, 3D
magnetic loop, N=8, p=3, ADER with the FV corrector, t=0.2) byte for byte,
and small ADER / SSP-RK variants (tests/golden/ind_*.npz, made by
tests/golden/make_fixtures.py from oracle/_ref) bit for bit: B2_cv with its
ghost elements and, with the FV corrector, the trouble flags.
"""
import hashlib

import numpy as np
import pytest

from helpers import manifest

pytestmark = pytest.mark.gpu
M = manifest()
CASES = M.get("induction_cases", {})


def run_case(ov):
    from spd_k_b200.api import apply_overrides
    from spd_k_b200.induction import (FIELD_B2_CV, FIELD_TROUBLES, InductionSolver,
                                      induction_config_from_params)
    c = induction_config_from_params(apply_overrides({}, ov))
    g = InductionSolver(c)
    out = {}

    def grab(k, s):
        out[k] = {"B2_cv": s.read(FIELD_B2_CV)}
        if c["fallback"]:
            out[k]["troubles"] = s.read(FIELD_TROUBLES)

    g.run(c["tlim"], c["output_dt"], on_output=grab)
    return out, g


@pytest.mark.parametrize("case", sorted(CASES))
def test_induction_matches_reference(case):
    info = CASES[case]
    out, g = run_case(info["overrides"])
    idx = int(info["output"].split("_")[-2])
    assert g.n_step == info["steps"]
    last = out[idx]
    b2 = last["B2_cv"]
    if case == "ind_golden_n8":
        want = M["goldens"]["induction_fv/B2_cv_N8p3_2_0.dat"]["sha256"]
        assert hashlib.sha256(b2.tobytes()).hexdigest() == info["sha256_B2_cv"] == want
    else:
        ref = np.load(f"tests/golden/{case}.npz")
        assert b2.shape == ref["B2_cv"].shape
        bad = np.flatnonzero(b2 != ref["B2_cv"])
        assert bad.size == 0, (bad.size, bad[:8], np.abs(b2 - ref["B2_cv"]).max())
        assert hashlib.sha256(b2.tobytes()).hexdigest() == info["sha256_B2_cv"]
    if "sha256_troubles" in info:
        tr = last["troubles"]
        assert tr.sum() >= 0
        assert hashlib.sha256(tr.tobytes()).hexdigest() == info["sha256_troubles"], case
    g.close()


def test_divergence_free_and_field_loop_advected():
    """The curl form keeps div B at round-off; the loop is advected with
    v = (1, 1, 0) (|B|^2 is carried, not created)"""
    from spd_k_b200.induction import FIELD_B2_CV
    ov = M["induction_cases"]["ind_n4_p3_ader"]["overrides"]
    out, g = run_case(ov)
    n = 4
    b0 = out[0]["B2_cv"].reshape(4, 6, 6, 6, n, n, n)[:, 1:-1, 1:-1, 1:-1]
    b1 = g.read(FIELD_B2_CV).reshape(4, 6, 6, 6, n, n, n)[:, 1:-1, 1:-1, 1:-1]
    e0, e1 = b0[3].sum(), b1[3].sum()
    assert e0 > 0 and abs(e1 - e0) / e0 < 0.2
    assert np.all(np.isfinite(b1))
    g.close()


def _sd_divergence(g, p, N):
    """max |div B| h / max |B| at the solution points of the active
    elements, from the face fields and dfp_to_sp (spdk_build_matrices)"""
    import ctypes
    from spd_k_b200.api import load_library
    from spd_k_b200.induction import FIELD_BX_FP, FIELD_BY_FP, FIELD_BZ_FP
    L = load_library()
    n, E = p + 1, N + 2
    D = np.zeros(n * (n + 1))
    L.spdk_build_matrices.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 6
    assert L.spdk_build_matrices(p, 1, None, D.ctypes.data, None, None, None, None) == 0
    D = D.reshape(n, n + 1)
    bx = g.read(FIELD_BX_FP).reshape(E, E, E, n, n, n + 1)[1:-1, 1:-1, 1:-1]
    by = g.read(FIELD_BY_FP).reshape(E, E, E, n, n + 1, n)[1:-1, 1:-1, 1:-1]
    bz = g.read(FIELD_BZ_FP).reshape(E, E, E, n + 1, n, n)[1:-1, 1:-1, 1:-1]
    h = g.c["L"][0] / N
    d = (np.einsum("kjiabl,cl->kjiabc", bx, D) + np.einsum("kjialc,bl->kjiabc", by, D)
         + np.einsum("kjilbc,al->kjiabc", bz, D)) / h
    return float(np.abs(d).max() * h / max(np.abs(bx).max(), np.abs(by).max(), np.abs(bz).max()))


@pytest.mark.parametrize("case", sorted(M.get("indfb_cases", {})))
def test_applied_fallback_matches_patched_reference(case):
    """fallback/apply against the reference built with the same step added
    to its corrector (oracle/patch_indfb.py): B2_cv and the trouble flags
    of the last output bit for bit."""
    info = M["indfb_cases"][case]
    out, g = run_case(info["overrides"] + ["fallback/apply=true"])
    idx = int(info["output"].split("_")[-2])
    assert g.n_step == info["steps"]
    ref = np.load(f"tests/golden/{case}.npz")
    b2, tr = out[idx]["B2_cv"], out[idx]["troubles"]
    assert b2.shape == ref["B2_cv"].shape and tr.shape == ref["troubles"].shape
    bad = np.flatnonzero(tr != ref["troubles"])
    assert bad.size == 0, ("troubles", bad.size, bad[:8])
    bad = np.flatnonzero(b2 != ref["B2_cv"])
    assert bad.size == 0, (bad.size, bad[:8], np.abs(b2 - ref["B2_cv"]).max())
    assert int((tr.reshape(4, -1)[3] > 0).sum()) == info["troubled_cells"] > 0
    g.close()


def test_applied_fallback_keeps_div_b_and_limits_the_loop():
    """fallback/apply (no reference counterpart: the reference only
    detects): upwind EMFs on the edges of troubled sub-cells. Constrained
    transport keeps div B at round-off; the field loop's peak |B|^2 stays
    below the unlimited run's and the upwind edges dissipate |B|^2; the
    applied run is deterministic. Off (the default) the golden tests above
    hold byte for byte."""
    from spd_k_b200.api import SpdkError, apply_overrides
    from spd_k_b200.induction import FIELD_B2_CV, InductionSolver, induction_config_from_params
    ov = CASES["ind_golden_n8"]["overrides"]
    p, N, n = 3, 8, 4
    res = {}
    for apply in ("false", "true", "true"):
        c = induction_config_from_params(apply_overrides({}, ov + [f"fallback/apply={apply}"]))
        g = InductionSolver(c)
        g.run(c["tlim"], c["output_dt"])
        b2 = g.read(FIELD_B2_CV)
        res.setdefault(apply, []).append((b2, _sd_divergence(g, p, N)))
        g.close()
    (off, div_off), = res["false"]
    (on, div_on), (on2, _) = res["true"]
    assert div_off < 1e-12 and div_on < 1e-12
    assert np.array_equal(on, on2)
    a = off.reshape(4, N + 2, N + 2, N + 2, n, n, n)[:, 1:-1, 1:-1, 1:-1]
    b = on.reshape(4, N + 2, N + 2, N + 2, n, n, n)[:, 1:-1, 1:-1, 1:-1]
    assert not np.array_equal(a, b)
    assert b[3].max() < a[3].max()
    assert b[3].sum() < a[3].sum()
    with pytest.raises(SpdkError, match="fallback_apply"):
        c = induction_config_from_params(apply_overrides({}, ov + ["fallback/apply=true", "job/fallback=false"]))
        InductionSolver(c)
