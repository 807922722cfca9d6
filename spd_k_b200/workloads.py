"""Named workloads that step one solver on the GPU, for timing and profiling.

    python -m spd_k_b200.workloads <name> [--N n] [--p p] [--precision fp64|fp32]
                                         [--steps k] [--learned path]

Each workload builds its solver through the package's public API, takes
one untimed step (set-up kernels and first-step paths run there), then
`--steps` steps, and prints one line: the workload, the steps and the
milliseconds per step (wall clock, the device synchronized on both sides).
The names:

  blast2d      spherical blast, 2D, N^2 elements, ADER + NAD/SED/MUSCL
               fallback, gradfree boundaries (the headline deck; --learned
               sets the BF16 a-priori indicator)
  blast3d      the same blast in 3D, N^3 elements
  kh3d         Kelvin-Helmholtz with seeded noise, 3D, N^3 elements
  viscous2d    2D Kelvin-Helmholtz with hydro/nu = 0.02 and the fallback
  batched      the first N problems of the seeded four-quadrant Riemann
               ensemble (sides {64..512}, p in {2, 3, 5}), one batched step
  mlp_train    Adam steps of the indicator network on 65536 random rows
  induction3d  the 3D magnetic loop (v = (1, 1, 0)), N^3, the FV corrector
               with detection (--apply 1: the applied fallback)
  induction2d  the 2D field loop, N^2, v = (2, 1), periodic
  divergence   the FP32 divergence contraction of one blast slice (N^2
               elements x 4 variables, p = 3) on CUDA cores (--mode 0) or
               3xTF32 tensor cores (--mode 1)
"""
import argparse
import ctypes
import math
import os
import time

P0_BLAST = 0.4 / (math.pi * 0.01 ** 2)  # (gamma-1) E / (pi r^2), E = 1, r = 0.01
DEFAULT_INDICATOR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "indicator_2d_p3.npz")


def blast_overrides(N=256, p=3, dims=2):
    """the spherical blast deck: rho 1, p = P0_BLAST inside r = 0.01 and
    1e-5 outside, gamma 1.4, gradfree boundaries, ADER + NAD(1e-5)"""
    z = [f"mesh/nx3={N}", "mesh/x3_bc=gradfree"] if dims == 3 else ["mesh/nx3=1"]
    return [
        "job/system=hydro", "job/fallback=true", f"mesh/p={p}", f"mesh/nx1={N}", f"mesh/nx2={N}",
        *z, "mesh/x1_bc=gradfree", "mesh/x2_bc=gradfree", "time/cfl=0.8",
        "time/integrator=ader", "hydro/gamma=1.4", "problem/problem=spherical_blast",
        "problem/d0=1.0", f"problem/p0={P0_BLAST!r}", "problem/p1=1e-5", "problem/radius=0.01",
        "fallback/tolerance=1e-5", "output/dt=-1",
    ]


def riemann_ensemble(count, seed=2024, precision="fp32", side=(64, 512)):
    """seeded ensemble of four-quadrant Riemann problems: element counts per
    side uniform in {side[0], side[0] + 8, ..., side[1]} (multiples of 8 so
    every autotuner tile divides them), p uniform in {2, 3, 5}, rho and P in
    U[0.1, 1], v in U[-1, 1], gamma 1.4, HLLC + NAD/MUSCL fallback, outflow.
    The first k problems of a seed are the same whatever count is asked for."""
    import numpy as np
    from spd_k_b200.api import apply_overrides, config_from_params
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nx, ny = (int(v) for v in rng.integers(side[0] // 8, side[1] // 8 + 1, 2) * 8)
        p = int(rng.choice([2, 3, 5]))
        ov = ["job/fallback=true", f"mesh/p={p}", f"mesh/nx1={nx}", f"mesh/nx2={ny}", "mesh/nx3=1",
              "mesh/x1_bc=gradfree", "mesh/x2_bc=gradfree", "problem/problem=quadrant", "hydro/gamma=1.4",
              "output/dt=-1"]
        c = config_from_params(apply_overrides({}, ov))
        q = []
        for _ in range(4):
            q += [rng.uniform(0.1, 1.0), rng.uniform(0.1, 1.0), rng.uniform(-1, 1), rng.uniform(-1, 1)]
        c["q"] = q
        c["precision"] = precision
        out.append(c)
    return out


def hydro_config(name, N, p, precision):
    from spd_k_b200.api import apply_overrides, config_from_params
    if name == "blast2d":
        ov = blast_overrides(N, p, 2)
    elif name == "blast3d":
        ov = blast_overrides(N, p, 3)
    elif name == "kh3d":
        ov = ["job/fallback=true", f"mesh/p={p}", f"mesh/nx1={N}", f"mesh/nx2={N}", f"mesh/nx3={N}",
              "problem/problem=kh_noise"]
    elif name == "viscous2d":
        ov = ["job/fallback=true", f"mesh/p={p}", f"mesh/nx1={N}", f"mesh/nx2={N}", "mesh/nx3=1",
              "problem/problem=kelvin_helmholtz", "hydro/nu=0.02"]
    else:
        raise ValueError(name)
    c = config_from_params(apply_overrides({}, ov))
    c["precision"] = precision
    return c


def _timed(fn, steps):
    """milliseconds per call of fn over `steps` calls, the device
    synchronized on both sides"""
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) * 1e3 / max(steps, 1)


def run(args):
    import torch
    torch.cuda.init()
    name, steps = args.name, args.steps
    if name in ("blast2d", "blast3d", "kh3d", "viscous2d"):
        from spd_k_b200.api import HydroSolver
        N = args.N or {"blast2d": 256, "blast3d": 32, "kh3d": 16, "viscous2d": 128}[name]
        p = args.p or {"kh3d": 5}.get(name, 3)
        g = HydroSolver(hydro_config(name, N, p, args.precision))
        ind = None
        if args.learned:
            from spd_k_b200.learned import Indicator, set_indicator
            ind = Indicator.load(args.learned)  # outlives the solver that uses it
            set_indicator(g, ind, 0.5)
        g.step()
        ms = _timed(g.step, steps)
        g.close()
        if ind is not None:
            ind.close()
        desc = f"{name} N={N} p={p} {args.precision}" + (" learned" if args.learned else "")
    elif name == "batched":
        from spd_k_b200.batch import Batch
        cfgs = riemann_ensemble(args.N or 16, precision=args.precision)
        b = Batch(cfgs)
        b.autotune()
        b.steps(1)
        ms = _timed(lambda: b.steps(1), steps)
        b.close()
        desc = f"batched {len(cfgs)} problems {args.precision}"
    elif name == "mlp_train":
        import numpy as np
        from spd_k_b200.learned import Indicator
        n_in = int(np.load(DEFAULT_INDICATOR)["n_in"])
        gen = torch.Generator(device="cuda").manual_seed(5)
        X = torch.randint(-3000, 3000, (65536, n_in), dtype=torch.int16, device="cuda", generator=gen)
        y = (torch.rand(65536, device="cuda", generator=gen) < 0.2).float()
        ind = Indicator(n_in)
        ind.fit(X, y, epochs=1)
        ms = _timed(lambda: ind.fit(X, y, epochs=1), steps)
        ind.close()
        desc = f"mlp_train 65536 rows x {n_in}, batch 4096 (one epoch per step)"
    elif name == "induction3d":
        from spd_k_b200.api import apply_overrides
        from spd_k_b200.induction import InductionSolver, induction_config_from_params
        N, p = args.N or 16, args.p or 3
        ov = ["job/system=induction", "induction/nu=0.0025", "time/cfl=0.8", "job/fallback=true", f"mesh/p={p}",
              f"mesh/nx1={N}", f"mesh/nx2={N}", f"mesh/nx3={N}"] + (["fallback/apply=true"] if args.apply else [])
        g = InductionSolver(induction_config_from_params(apply_overrides({}, ov)))
        g.step()
        ms = _timed(g.step, steps)
        g.close()
        desc = f"induction3d N={N} p={p} fallback" + (" applied" if args.apply else " detection")
    elif name == "induction2d":
        from spd_k_b200.induction import Induction2D, field_loop_config
        N, p = args.N or 512, args.p or 4
        g = Induction2D(field_loop_config(N=N, p=p, precision=args.precision))
        g.step()
        ms = _timed(g.step, steps)
        g.close()
        desc = f"induction2d N={N} p={p} {args.precision}"
    elif name == "divergence":
        from spd_k_b200.api import load_library
        L = load_library()
        f = L.spdk_study_divergence
        f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_longlong] + [ctypes.c_void_p] * 4
        N = args.N or 256
        count = N * N * 4
        gen = torch.Generator(device="cuda").manual_seed(3)
        fx = torch.randn(count, 4, 5, device="cuda", generator=gen)
        fy = torch.randn(count, 4, 5, device="cuda", generator=gen)
        out = torch.empty(count, 4, 4, device="cuda")
        st = torch.cuda.current_stream().cuda_stream

        def call():
            if f(args.mode, 3, count, fx.data_ptr(), fy.data_ptr(), out.data_ptr(), st) != 0:
                raise RuntimeError("spdk_study_divergence failed")
        call()
        ms = _timed(call, steps)
        desc = f"divergence {count} element-variables, mode {args.mode}"
    else:
        raise SystemExit(f"unknown workload {name!r}")
    print(f"{desc}: {steps} steps, {ms:.4f} ms/step", flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("name")
    ap.add_argument("--N", type=int, default=0)
    ap.add_argument("--p", type=int, default=0)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--learned", default=None)
    ap.add_argument("--apply", type=int, default=0)
    ap.add_argument("--mode", type=int, default=0)
    return run(ap.parse_args(argv))


if __name__ == "__main__":
    main()
