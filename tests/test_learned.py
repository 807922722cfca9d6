"""The learned a-priori troubled-cell indicator.

CPU: the FP64 restatement (oracle/mlp_oracle.py) is checked against central
finite differences and torch's BF16 rounding.
GPU: the feature rows of a solver state equal the restatement's bit for
bit; the FP32-accumulating forward/backward kernels give the restatement's
loss and gradient to FP32 round-off; the network trained on the GPU from
the solver's own NAD labels predicts troubled elements of an unseen run,
and wired into the solver it sends them to the fallback a priori (reported:
false-positive and false-negative rates, L1 difference from the plain run;
asserted: its error against a refined FP64 run stays within 2x of the plain
run's, in FP64 and in the FP32 form).
"""
import numpy as np
import pytest

from oracle import mlp_oracle as MO


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    n_in, B = 7, 13
    theta = rng.normal(0, 0.3, MO.layout(n_in)["n"])
    X = rng.normal(0, 1, (B, n_in))
    y = (rng.uniform(size=B) < 0.4).astype(float)
    w = rng.uniform(0.5, 2.0, B)
    _, g = MO.loss_grad(theta, X, y, w)
    idx = rng.choice(len(theta), 40, replace=False)
    for q in idx:
        e = np.zeros_like(theta)
        e[q] = 1e-6
        fd = (MO.loss_grad(theta + e, X, y, w)[0] - MO.loss_grad(theta - e, X, y, w)[0]) / 2e-6
        assert abs(fd - g[q]) <= 1e-7 + 1e-5 * abs(fd), q


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(1)
    a = np.concatenate([rng.normal(0, 1, 5000), rng.normal(0, 1e-3, 5000), [0.0, -0.0, 1.0, 3.0039062]])
    a = a.astype(np.float32)
    want = torch.from_numpy(a).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(MO.bf16_bits(a), want)


# ---------------------------------------------------------------------- GPU
def blast(N, precision="fp64"):
    import bench
    import spd_k_b200 as S
    from helpers import gpu_config
    return S.HydroSolver(dict(gpu_config(bench.workload_overrides(N)), precision=precision))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_features_match_oracle(precision):
    from spd_k_b200.learned import features
    g = blast(32, precision)
    for _ in range(6):
        g.step()
    x = features(g).cpu().numpy().view(np.uint16)
    u = g.read(0).reshape(g.info.n_elements, g.info.nvar, g.info.n_points)
    want = MO.features(u, 2, g.p, list(g.N), [1, 1, 1], g.c["gamma"])
    assert x.shape == want.shape and x.shape[1] == 40
    assert np.array_equal(x, want)
    g.close()


@pytest.mark.gpu
def test_gradient_matches_cpu_oracle():
    import torch
    from spd_k_b200.learned import Indicator
    rng = np.random.default_rng(3)
    n_in, B = 40, 3000
    ind = Indicator(n_in, seed=7)
    theta = rng.normal(0, 0.2, ind.n_params).astype(np.float32)
    ind.set_params(theta)
    Xf = rng.normal(0, 1, (B, n_in)).astype(np.float32)
    Xb = MO.bf16_bits(Xf)
    y = (rng.uniform(size=B) < 0.3).astype(np.float32)
    w = rng.uniform(0.5, 2.0, B).astype(np.float32)
    X = torch.from_numpy(Xb.view(np.int16)).cuda()
    loss, grad = ind.loss_grad(X, torch.from_numpy(y).cuda(), torch.from_numpy(w).cuda())
    loss, grad = float(loss.item()), grad.cpu().numpy().astype(np.float64)
    # FP64 on the BF16-rounded parameters and inputs the kernels use
    th64 = MO.bf16_round(theta)
    l_ref, g_ref = MO.loss_grad(th64, MO.bits_to_float(Xb), y.astype(np.float64), w.astype(np.float64))
    assert abs(loss - l_ref) <= 1e-5 * abs(l_ref)
    assert np.linalg.norm(grad - g_ref) <= 1e-4 * np.linalg.norm(g_ref)
    p_gpu = ind.predict(X).cpu().numpy()
    p_ref, _ = MO.forward(th64, MO.bits_to_float(Xb))
    assert np.max(np.abs(p_gpu - p_ref)) < 1e-5
    ind.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,N", [("fp64", 32), ("fp32", 32), ("fp64", 30), ("fp32", 30)])
def test_solver_indicator_flags_match_oracle(precision, N):
    """The solver's indicator builds the feature rows on chip and runs the
    network on the tensor cores (one pass over 4 x 4 element tiles when the
    element counts allow, else element means first); its flags equal the
    restatement's features -> forward -> p > threshold except within 1e-5
    of the threshold."""
    from spd_k_b200.learned import Indicator, set_indicator
    from spd_k_b200.api import FIELD_ELEMENT_PREDICTED
    rng = np.random.default_rng(5)
    g = blast(N, precision)
    for _ in range(6):
        g.step()
    ind = Indicator(40, seed=2)
    theta = rng.normal(0, 0.3, ind.n_params).astype(np.float32)
    ind.set_params(theta)
    u = g.read(0).reshape(g.info.n_elements, g.info.nvar, g.info.n_points)
    X = MO.bits_to_float(MO.features(u, 2, g.p, list(g.N), [1, 1, 1], g.c["gamma"]))
    p_ref, _ = MO.forward(MO.bf16_round(theta), X)
    # the uniform background gives many elements one value: threshold in
    # the middle of the distinct values
    thr = float(np.median(np.unique(p_ref)))
    set_indicator(g, ind, thr)
    g.step()                                       # flags of the state before the step
    pred = g.read(FIELD_ELEMENT_PREDICTED)
    want = p_ref > thr
    clear = np.abs(p_ref - thr) > 1e-5
    assert 0 < want.sum() < len(want)
    assert np.array_equal(pred[clear] > 0, want[clear])
    # later steps take the features the previous step's last update stored,
    # stepped one by one and by graph replay
    for advance in (lambda: g.step(), lambda: g.steps(1)):
        advance()
        g.sync()
        u = g.read(0).reshape(g.info.n_elements, g.info.nvar, g.info.n_points)
        X = MO.bits_to_float(MO.features(u, 2, g.p, list(g.N), [1, 1, 1], g.c["gamma"]))
        p_ref, _ = MO.forward(MO.bf16_round(theta), X)
        advance()
        g.sync()
        pred = g.read(FIELD_ELEMENT_PREDICTED)
        clear = np.abs(p_ref - thr) > 1e-5
        assert np.array_equal(pred[clear] > 0, (p_ref > thr)[clear])
    set_indicator(g, None)
    g.close()
    ind.close()


def _rates(pred, lab):
    tp = float(np.sum((pred > 0) & (lab > 0)))
    fp = float(np.sum((pred > 0) & (lab == 0)))
    fn = float(np.sum((pred == 0) & (lab > 0)))
    neg, pos = float(np.sum(lab == 0)), float(np.sum(lab > 0))
    return {"fpr": fp / max(neg, 1), "fnr": fn / max(pos, 1), "precision": tp / max(tp + fp, 1), "pos": pos}


@pytest.mark.gpu
def test_trained_indicator_predicts_and_feeds_the_fallback():
    import torch
    from spd_k_b200.learned import Indicator, collect, features, set_indicator
    from spd_k_b200.api import FIELD_ELEMENT_PREDICTED, FIELD_ELEMENT_TROUBLES
    # training data: the solver's own NAD labels on the 64x64 blast
    g = blast(64)
    X, y = collect(g, 150)
    g.close()
    pos = float(y.sum().item())
    assert pos > 100
    w = torch.where(y > 0, 0.5 * len(y) / pos, 0.5 * len(y) / (len(y) - pos)).float()
    ind = Indicator(X.shape[1], seed=1)
    hist = ind.fit(X, y, w, epochs=25)
    assert hist[-1] < 0.5 * hist[0], hist
    # unseen run: the 96x96 blast
    g = blast(96)
    Xt, yt = collect(g, 120, every=5)
    pt = ind.predict(Xt).cpu().numpy()
    r = _rates(pt > 0.5, yt.cpu().numpy())
    print(f"\nheld-out (96x96): {r}")
    assert r["fnr"] < 0.2 and r["fpr"] < 0.1
    g.close()
    # wired into the solver: the predicted elements are troubled a priori
    # in every slice; NAD still runs everywhere
    plain, learned = blast(64), blast(64)
    set_indicator(learned, ind, 0.5)
    stats = []
    for s in range(60):
        plain.step()
        learned.step()
        pred = learned.read(FIELD_ELEMENT_PREDICTED)
        lab = plain.read(FIELD_ELEMENT_TROUBLES)
        tr = learned.read(2).reshape(-1, 16).max(axis=1)
        assert np.all(tr[pred > 0] == 1)          # predicted elements went to the fallback
        stats.append(_rates(pred, lab))
    wp, wl = plain.field_array(1), learned.field_array(1)
    l1 = [float(np.abs(wl[v] - wp[v]).sum() / np.abs(wp[v]).sum()) for v in range(4)]
    fpr = np.mean([s["fpr"] for s in stats])
    fnr = np.mean([s["fnr"] for s in stats])
    print(f"in the loop (against the plain run's labels): mean FPR {fpr:.4f}, FNR {fnr:.4f}; "
          f"W_cv relative L1 vs plain {l1}")
    assert fnr < 0.3 and fpr < 0.01
    set_indicator(learned, None)
    plain.close()
    learned.close()
    # the error the a-priori limiting adds: element means of (rho, m, E) at
    # t = 0.005 against an FP64 run on the 128x128 mesh, with and without
    # the indicator (and in the FP32 form with it: the mixed + learned form)
    from test_gpu_precision import element_means
    t_end = 0.005
    import bench
    import spd_k_b200 as S
    from helpers import gpu_config

    def run(N, prec, with_ind):
        ov = bench.workload_overrides(N) + [f"time/tlim={t_end!r}", f"output/dt={t_end!r}"]
        s = S.HydroSolver(dict(gpu_config(ov), precision=prec))
        if with_ind:
            set_indicator(s, ind, 0.5)
        s.run(t_end, t_end)
        m = element_means(s)
        if with_ind:
            set_indicator(s, None)
        s.close()
        return m
    ref = run(128, "fp64", False)
    V = ref.shape[0]
    ref = ref.reshape(V, 64, 2, 64, 2).mean(axis=(2, 4))
    err = {}
    for k in (("fp64", False), ("fp64", True), ("fp32", True)):
        m = run(64, *k)
        err[k] = [float(np.abs(m[i] - ref[i]).mean()) for i in range(V)]
    print(f"L1 of element means vs FP64 128x128: {err}")
    for k in (("fp64", True), ("fp32", True)):
        for e, e0 in zip(err[k], err[("fp64", False)]):
            assert e <= 2.0 * e0
    ind.close()
