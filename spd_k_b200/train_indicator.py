"""Train the learned troubled-cell indicator on the GPU and save its weights.

    python -m spd_k_b200.train_indicator [--out spd_k_b200/data/indicator_2d_p3.npz]

Training data are the solver's own a-posteriori NAD/SED/PAD labels (per
element, any sub-cell in any slice of the step) paired with the feature
rows of the state before the step, from two families run by this library:
the 2D point blast (gamma = 1.4, outflow boundaries, p = 3) at 64^2 and
128^2, and seeded four-quadrant Riemann problems (rho, P in U[0.1, 1],
v in U[-1, 1]) at 64^2. Classes are balanced by weight; the network is
trained with the library's own BF16/FP32 forward and backward kernels.
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


def quadrant_config(N, seed):
    """a seeded four-quadrant Riemann problem (quadrant IC: q[4 k .. 4 k + 3]
    = rho, P, vx, vy of quadrant k)"""
    from .api import apply_overrides, config_from_params
    rng = np.random.default_rng(seed)
    ov = ["job/fallback=true", "mesh/p=3", f"mesh/nx1={N}", f"mesh/nx2={N}", "mesh/nx3=1",
          "mesh/x1_bc=gradfree", "mesh/x2_bc=gradfree", "problem/problem=quadrant", "hydro/gamma=1.4",
          "output/dt=-1"]
    c = config_from_params(apply_overrides({}, ov))
    q = []
    for _ in range(4):
        q += [rng.uniform(0.1, 1.0), rng.uniform(0.1, 1.0), rng.uniform(-1, 1), rng.uniform(-1, 1)]
    c["q"] = q
    return c


def gather(verbose=True):
    import torch
    from . import HydroSolver
    from .api import apply_overrides, config_from_params
    from .learned import collect
    runs = [(config_from_params(apply_overrides({}, blast_overrides(64))), 200, 1),
            (config_from_params(apply_overrides({}, blast_overrides(128))), 300, 3)]
    runs += [(quadrant_config(64, s), 120, 2) for s in range(6)]
    xs, ys = [], []
    for c, steps, every in runs:
        g = HydroSolver(c)
        X, y = collect(g, steps, every)
        g.close()
        xs.append(X)
        ys.append(y)
        if verbose:
            print(f"{c['problem']} {c['N'][0]}^2: {X.shape[0]} rows, {int(y.sum().item())} troubled", flush=True)
    return torch.cat(xs), torch.cat(ys)


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
