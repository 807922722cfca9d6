"""The batched form (include/spdk_batch.h): many independent 2D problems of
uneven sizes and orders stepped by one launch per pass and order group,
captured as one graph per step.

Every member's state after the batched steps is bit-identical to the same
problem stepped alone with spdk_hydro_step (in the plain FP64 form, and in
the FP32 form against the FP32 single solver), before and after the
autotuner changes the tile shapes; the autotuner leaves the state as it
found it.
"""
import numpy as np
import pytest

from helpers import gpu_config, same_bits


def quadrant(N, p, seed, extra=()):
    rng = np.random.default_rng(seed)
    c = gpu_config(["job/fallback=true", f"mesh/p={p}", f"mesh/nx1={N[0]}", f"mesh/nx2={N[1]}", "mesh/nx3=1",
                    "mesh/x1_bc=gradfree", "mesh/x2_bc=gradfree", "problem/problem=quadrant",
                    "output/dt=-1", *extra])
    q = []
    for _ in range(4):
        q += [rng.uniform(0.1, 1.0), rng.uniform(0.1, 1.0), rng.uniform(-1, 1), rng.uniform(-1, 1)]
    c["q"] = q
    return c


def test_bad_batches_are_rejected_without_a_device():
    import spd_k_b200.batch as B
    from spd_k_b200.api import SpdkError
    good = quadrant((8, 8), 3, 0)
    for bad in (dict(good, N=[8, 8, 8]), dict(good, p=4), dict(good, integrator="rk3"), dict(good, N=[9, 8, 1])):
        with pytest.raises(SpdkError):
            B.Batch([good, bad])
    with pytest.raises(SpdkError):
        B.Batch([good, dict(good, precision="fp32")])


def ensemble(precision, fallback=True):
    cs = [quadrant((8, 12), 2, 1), quadrant((16, 8), 3, 2), quadrant((12, 12), 5, 3), quadrant((24, 16), 3, 4),
          quadrant((8, 8), 2, 5)]
    import bench
    blast = gpu_config(bench.workload_overrides(16))
    cs.append(blast)
    out = []
    for c in cs:
        c = dict(c, precision=precision, fallback=fallback)
        out.append(c)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision,fallback", [("fp64", True), ("fp32", True), ("fp64", False)])
def test_batch_matches_single_solvers(precision, fallback):
    import spd_k_b200 as S
    import spd_k_b200.batch as B
    cs = ensemble(precision, fallback)
    b = B.Batch(cs)
    info = b.info()
    assert info.n_problems == len(cs) and info.n_groups == 3
    b.steps(4)
    b.sync()
    singles = [S.HydroSolver(c) for c in cs]
    for s in singles:
        for _ in range(4):
            s.step()
        s.sync()
    for i, s in enumerate(singles):
        m = b.member(i)
        assert same_bits(m.read(0), s.read(0)), i
        assert same_bits(m.read(1), s.read(1)), i
        assert m.dt() == s.dt(), i
    # the autotuner restores the state and may change tiles; the results stay
    b.autotune(2)
    info2 = b.info()
    print("\ntiles:", list(info2.group_p[:info2.n_groups]), list(info2.group_tile[:info2.n_groups]))
    for i, s in enumerate(singles):
        assert same_bits(b.member(i).read(0), s.read(0)), i
    b.steps(3)
    b.sync()
    for s in singles:
        for _ in range(3):
            s.step()
        s.sync()
    for i, s in enumerate(singles):
        assert same_bits(b.member(i).read(1), s.read(1)), i
        s.close()
    b.close()


@pytest.mark.gpu
def test_batch_labels_match_single_solvers():
    """spdk_batch_record_labels: each member's per-element trouble labels of
    the last batched step equal the single solver's for the same step (the
    indicator's training data taken from the batched run); the state stays
    bit-identical with labels on."""
    import spd_k_b200 as S
    import spd_k_b200.batch as B
    from spd_k_b200.api import FIELD_ELEMENT_TROUBLES, SpdkError
    cs = ensemble("fp32", True)
    b = B.Batch(cs)
    b.record_labels(True)
    singles = [S.HydroSolver(c) for c in cs]
    flagged = 0
    for step in range(3):
        b.steps(1)
        b.sync()
        for s in singles:
            s.step()
            s.sync()
        for i, s in enumerate(singles):
            m = b.member(i)
            lb, ls = np.asarray(m.read(FIELD_ELEMENT_TROUBLES)), np.asarray(s.read(FIELD_ELEMENT_TROUBLES))
            assert np.array_equal(lb, ls), (step, i)
            flagged += int(lb.sum())
            assert same_bits(m.read(0), s.read(0)), (step, i)
    assert flagged > 0
    for s in singles:
        s.close()
    b.close()
    with pytest.raises(SpdkError):
        nb = B.Batch(ensemble("fp64", False)[:2])
        try:
            nb.record_labels(True)
        finally:
            nb.close()
