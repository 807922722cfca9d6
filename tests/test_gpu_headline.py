"""The headline form on its own configuration.

The timed form is the precision form (FP32 state, FP64 islands) with the
learned a-priori indicator. Its claim is "at matched L1 error": on the full
2D point blast (256x256 elements, p=3, NAD+MUSCL, to t=0.05), the L1 error
of every conserved field's element means against an FP64 run on the
512x512 mesh must stay within 2x of the plain FP64 form's own error. The
FP32 form without the indicator is run beside them, and the indicator's
effect (limited elements, predicted elements) is reported.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T_END = 0.05
N = 256


def run_form(prec, learned):
    import bench
    import spd_k_b200 as S
    from helpers import gpu_config
    from spd_k_b200.api import FIELD_ELEMENT_PREDICTED, FIELD_ELEMENT_TROUBLES
    from spd_k_b200.learned import Indicator, set_indicator
    from test_gpu_precision import element_means
    ov = bench.workload_overrides(N) + [f"time/tlim={T_END!r}", f"output/dt={T_END!r}"]
    s = S.HydroSolver(dict(gpu_config(ov), precision=prec))
    ind = None
    if learned:
        ind = Indicator.load(os.path.join(os.path.dirname(S.__file__), "data", "indicator_2d_p3.npz"))
        set_indicator(s, ind, 0.5)
    s.run(T_END, T_END)
    assert abs(s.t - T_END) < 1e-12
    m = element_means(s)
    stats = {"steps": s.n_step}
    if learned:
        stats["predicted_last_step"] = int(s.read(FIELD_ELEMENT_PREDICTED).sum())
        stats["flagged_last_step"] = int(s.read(FIELD_ELEMENT_TROUBLES).sum())
        set_indicator(s, None)
        ind.close()
    s.close()
    return m, stats


def test_mixed_learned_matched_error_on_the_blast():
    from test_gpu_precision import blast_reference_means
    ref = blast_reference_means(N, T_END)
    V = ref.shape[0]
    err, stats = {}, {}
    for form, args in (("fp64", ("fp64", False)), ("fp32", ("fp32", False)), ("fp32+learned", ("fp32", True))):
        m, stats[form] = run_form(*args)
        assert np.all(np.isfinite(m))
        err[form] = [float(np.abs(m[i] - ref[i]).mean()) for i in range(V)]
    ratio = {k: [e / e0 for e, e0 in zip(v, err["fp64"])] for k, v in err.items()}
    print(f"\nblast {N}^2 p=3 to t={T_END}: L1 of element means (rho, m_x, m_y, E) vs FP64 {2 * N}^2")
    for k in err:
        print(f"  {k:13s} {err[k]}  ratio to fp64 {[round(r, 4) for r in ratio[k]]}  {stats[k]}")
    for e, e0 in zip(err["fp32+learned"], err["fp64"]):
        assert e <= 2.0 * e0
    for e, e0 in zip(err["fp32"], err["fp64"]):
        assert e <= 2.0 * e0
