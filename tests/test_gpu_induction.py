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
