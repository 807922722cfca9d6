"""Train the learned troubled-cell indicator on the GPU and save its weights.

    python -m spd_k_b200.train_indicator [--out spd_k_b200/data/indicator_2d_p3.npz]

Training data are the solver's own a-posteriori NAD/SED/PAD labels (per
element, any sub-cell in any slice of the step) paired with the feature
rows of the state before the step, from the two configurations the
indicator serves: the 2D point blast (gamma = 1.4, outflow boundaries,
p = 3) at 64^2 and 128^2, stepped alone, and the batched run of the seeded
four-quadrant Riemann ensemble (sides 64..512, rho, P in U[0.1, 1], v in
U[-1, 1]; its p = 3 members among the first 64 problems, FP32 form, labels
recorded by the batch itself, spdk_batch_record_labels). Classes are
balanced by weight; the network is trained with the library's own BF16/FP32
forward and backward kernels.
"""
import argparse
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def blast_overrides(N):
    p0 = 0.4 / (math.pi * 0.01 ** 2)
    return ["job/fallback=true", "mesh/p=3", f"mesh/nx1={N}", f"mesh/nx2={N}", "mesh/nx3=1",
            "mesh/x1_bc=gradfree", "mesh/x2_bc=gradfree", "time/cfl=0.8", "time/integrator=ader",
            "hydro/gamma=1.4", "problem/problem=spherical_blast", "problem/d0=1.0", f"problem/p0={p0!r}",
            "problem/p1=1e-5", "problem/radius=0.01", "fallback/tolerance=1e-5", "output/dt=-1"]


def gather(verbose=True):
    import torch
    from . import HydroSolver
    from .api import apply_overrides, config_from_params
    from .learned import collect
    runs = [(config_from_params(apply_overrides({}, blast_overrides(64))), 200, 1),
            (config_from_params(apply_overrides({}, blast_overrides(128))), 300, 3)]
    xs, ys = [], []
    for c, steps, every in runs:
        g = HydroSolver(c)
        X, y = collect(g, steps, every)
        g.close()
        xs.append(X)
        ys.append(y)
        if verbose:
            print(f"{c['problem']} {c['N'][0]}^2: {X.shape[0]} rows, {int(y.sum().item())} troubled", flush=True)
    X, y = batched_rows(verbose=verbose)
    xs.append(X)
    ys.append(y)
    return torch.cat(xs), torch.cat(ys)


def batched_rows(count=64, p=3, steps=100, every=25, verbose=True):
    """(X, y) from the batched run of the ensemble's order-p members among
    its first `count` problems: feature rows of every member before each
    `every`-th step and the labels the batched step records"""
    import torch
    from .api import FIELD_ELEMENT_TROUBLES
    from .batch import Batch
    from .learned import features
    from .workloads import riemann_ensemble
    cfgs = [c for c in riemann_ensemble(count, precision="fp32") if c["p"] == p]
    b = Batch(cfgs)
    b.record_labels(True)
    xs, ys = [], []
    for s in range(steps):
        take = s % every == 0
        if take:
            b.sync()
            rows = [features(b.member(i)) for i in range(len(cfgs))]
        b.steps(1)
        if take:
            b.sync()
            for i in range(len(cfgs)):
                lab = np.asarray(b.member(i).read(FIELD_ELEMENT_TROUBLES), dtype=np.float32)
                xs.append(rows[i])
                ys.append(torch.from_numpy(lab).cuda())
    b.close()
    X, y = torch.cat(xs), torch.cat(ys)
    if verbose:
        print(f"batched ensemble, {len(cfgs)} p={p} problems: {X.shape[0]} rows, {int(y.sum().item())} troubled",
              flush=True)
    return X, y


def main():
    import torch
    from .learned import Indicator
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "data", "indicator_2d_p3.npz"))
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args()
    X, y = gather()
    pos = float(y.sum().item())
    w = torch.where(y > 0, 0.5 * len(y) / pos, 0.5 * len(y) / (len(y) - pos)).float()
    ind = Indicator(X.shape[1], seed=args.seed)
    hist = ind.fit(X, y, w, epochs=args.epochs)
    p = ind.predict(X).cpu().numpy()
    lab = y.cpu().numpy()
    fp = float(np.sum((p > 0.5) & (lab == 0))) / max(float(np.sum(lab == 0)), 1)
    fn = float(np.sum((p <= 0.5) & (lab > 0))) / max(pos, 1)
    print(f"loss {hist[0]:.4f} -> {hist[-1]:.4f}; training-set FPR {fp:.4f} FNR {fn:.4f}")
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    ind.save(args.out)
    print(args.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
