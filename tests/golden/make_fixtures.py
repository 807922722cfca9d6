"""Generate the parity fixtures from the reference's own CPU build.

Runs oracle/_ref/spd_K_ref (the reference sources compiled unmodified; see
oracle/Makefile) on small configurations given as block/name=value
overrides of the reference defaults, and stores, per case:
  <case>.npz     the active region of W_cv (slots rho, vx, vy, vz, p) at the
                 last output, shape (5, Nz, Ny, Nx, nz, ny, nx), and the
                 output time and step count
  manifest.json  the overrides, the output index and the SHA-256 of the
                 reference's raw output file
It also records the SHA-256 of the reference's committed goldens
(tests/goldens/ in the reference tree) and the induction solver's outputs
(INDUCTION_CASES). Needs the reference tree; run once:
    python tests/golden/make_fixtures.py [--induction | --viscous | --loop2d | --indfb]
"""
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "spd_K_ref")
# the reference tree: SPDK_REFERENCE_ROOT, by default where this build keeps it
REF_TREE = os.environ.get("SPDK_REFERENCE_ROOT", "/root/reference")

BLAST = ["problem/problem=spherical_blast", "hydro/gamma=1.6666666666667"]
CASES = {
    # the reference's own regression set (tests/run_tests.py:44-143), 2D, small
    "sine2d_ader": ["job/fallback=false", "mesh/nx3=1", "time/tlim=0.1", "output/dt=0.1"],
    "sine2d_rk3": ["job/fallback=false", "mesh/nx3=1", "time/integrator=rk3", "time/tlim=0.1", "output/dt=0.1"],
    "sine2d_fallback": ["job/fallback=true", "mesh/nx3=1", "time/tlim=0.1", "output/dt=0.1"],
    "blast2d_fallback": ["job/fallback=true", "mesh/nx3=1", *BLAST, "time/tlim=0.02", "output/dt=0.02"],
    "blast2d_rk3_fallback": ["job/fallback=true", "mesh/nx3=1", *BLAST, "time/integrator=rk3",
                             "time/tlim=0.02", "output/dt=0.02"],
    "implosion2d_reflective": ["job/fallback=true", "mesh/nx1=8", "mesh/nx2=8", "mesh/nx3=1",
                               "mesh/x1len=0.3", "mesh/x2len=0.3", "mesh/x1_bc=reflective",
                               "mesh/x2_bc=reflective", "problem/problem=implosion", "time/tlim=0.05",
                               "output/dt=0.05"],
    # the point-blast geometry of the benchmark workload at 16x16
    "blast2d_gradfree_p3": ["job/fallback=true", "mesh/nx1=16", "mesh/nx2=16", "mesh/nx3=1",
                            "mesh/x1_bc=gradfree", "mesh/x2_bc=gradfree", "problem/problem=spherical_blast",
                            "problem/p0=1273.2395447351628", "problem/p1=1e-5", "problem/radius=0.05",
                            "time/tlim=0.002", "output/dt=0.002"],
    "kh2d_p2": ["job/fallback=true", "mesh/p=2", "mesh/nx1=8", "mesh/nx2=8", "mesh/nx3=1",
                "problem/problem=kelvin_helmholtz", "time/tlim=0.05", "output/dt=0.05"],
    "rti2d_gravity": ["job/fallback=true", "mesh/nx1=4", "mesh/nx2=8", "mesh/nx3=1", "mesh/x1len=0.5",
                      "mesh/x2len=1.0", "mesh/x2_bc=reflective", "problem/problem=rti", "hydro/g2=-0.1",
                      "time/tlim=0.05", "output/dt=0.05"],
    # 1-D profile problems run as quasi-2D strips
    "sod2d_p4": ["job/fallback=true", "mesh/p=4", "mesh/nx1=16", "mesh/nx2=2", "mesh/nx3=1",
                 "mesh/x1_bc=gradfree", "problem/problem=sod_shock_tube", "time/tlim=0.05", "output/dt=0.05"],
}
# viscous runs (hydro/nu > 0): the reference's viscous terms, served by the
# prototype-level path (the fused solver rejects nu > 0)
VISCOUS_CASES = {
    "sine2d_viscous": ["job/fallback=false", "mesh/p=3", "mesh/nx1=8", "mesh/nx2=8", "mesh/nx3=1", "hydro/nu=0.01",
                       "time/tlim=0.02", "output/dt=0.02"],
    "kh2d_viscous_fallback": ["job/fallback=true", "mesh/p=2", "mesh/nx1=6", "mesh/nx2=6", "mesh/nx3=1",
                              "hydro/nu=0.005", "problem/problem=kelvin_helmholtz", "time/tlim=0.02",
                              "output/dt=0.02"],
    "sine3d_viscous_rk2_beta": ["job/fallback=false", "mesh/p=2", "mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=3",
                                "hydro/nu=0.02", "hydro/beta=0.003", "time/integrator=rk2", "time/tlim=0.01",
                                "output/dt=0.01"],
}
# full-size run of the plain-method CPU-runnable configuration (2D sine,
# 32x32, p=3, ADER, LLF, to t=1): only rho and p are stored, with the
# SHA-256 of the active rho, vx, vy, p slots
FULL_CASES = {
    "config1_sine2d_32": ["job/fallback=false", "mesh/nx1=32", "mesh/nx2=32", "mesh/nx3=1",
                          "time/tlim=1.0", "output/dt=1.0"],
}
# the benchmark workload (2D point blast, NAD+MUSCL, gradfree) at reduced
# and full size for a few steps; the run ends at 0.999 x steps x dt0 with
# output clamping, as the reference driver does
BENCH_CASES = {"bench_blast_64": (64, 12), "bench_blast_256": (256, 10)}
GOLDENS = {
    "hydro_sd/W_cv_N8p3_1_0.dat": "reference golden: 3D sine wave, N=8, p=3, ADER, t=0.1",
    "induction_fv/B2_cv_N8p3_2_0.dat": "reference golden: 3D induction loop with fallback, t=0.2",
}


# the 3D induction solver (magnetic loop advected at v = (1, 1, 0),
# src/induction_ader.hpp): the reference golden deck (sha only) and small
# variants; stored per case: the full B2_cv file (ghost elements included)
# and, with the FV path, the full troubles file of the last output
INDUCTION_BASE = ["job/system=induction", "induction/nu=0.0025", "time/cfl=0.8"]
INDUCTION_CASES = {
    "ind_golden_n8": ["job/fallback=true", "mesh/p=3", "mesh/nx1=8", "mesh/nx2=8", "mesh/nx3=8",
                      "time/tlim=0.2", "output/dt=0.1"],
    "ind_n4_p3_ader": ["job/fallback=false", "mesh/p=3", "mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=4",
                       "time/tlim=0.1", "output/dt=0.05"],
    "ind_n6_p3_rk2_fv": ["job/fallback=true", "mesh/p=3", "mesh/nx1=6", "mesh/nx2=6", "mesh/nx3=6",
                         "time/integrator=rk2", "time/tlim=0.1", "output/dt=0.05"],
    "ind_n4_p2_rk3": ["job/fallback=false", "mesh/p=2", "mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=4",
                      "time/integrator=rk3", "time/tlim=0.1", "output/dt=0.05"],
    "ind_n4_p4_rk2_gradfree": ["job/fallback=false", "mesh/p=4", "mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=4",
                               "time/integrator=rk2", "mesh/x1_bc=gradfree", "mesh/x2_bc=gradfree",
                               "mesh/x3_bc=gradfree", "time/tlim=0.05", "output/dt=0.05"],
}
# (the reference's FV induction path writes past its FV arrays in the ghost
# fill of staggered fields and crashes at N = 4 for p = 2..4; the FV cases
# above are ones it completes)


def induction_fixtures(manifest):
    for name, ov in INDUCTION_CASES.items():
        ov = INDUCTION_BASE + ov
        with tempfile.TemporaryDirectory() as out:
            env = dict(os.environ, SPD_OUTPUT_DIR=out + "/", OMP_NUM_THREADS="8")
            r = subprocess.run([REF_BIN] + ov, capture_output=True, text=True, env=env, check=True)
            files = [f for f in os.listdir(out) if f.startswith("B2_cv_")]
            last = max(files, key=lambda f: int(f.split("_")[-2]))
            idx = int(last.split("_")[-2])
            steps = int(r.stdout.split("evolution: ")[1].split(" steps")[0])
            entry = {"overrides": ov, "output": last, "steps": steps,
                     "sha256_B2_cv": sha256(os.path.join(out, last))}
            tr = [f for f in os.listdir(out) if f.startswith("troubles_") and int(f.split("_")[-2]) == idx]
            if tr:
                entry["troubles_output"] = tr[0]
                entry["sha256_troubles"] = sha256(os.path.join(out, tr[0]))
            if name != "ind_golden_n8":
                arrays = {"B2_cv": np.fromfile(os.path.join(out, last))}
                if tr:
                    arrays["troubles"] = np.fromfile(os.path.join(out, tr[0]))
                np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
            manifest.setdefault("induction_cases", {})[name] = entry
            print(name, last, steps, flush=True)


# the applied induction fallback (upwind EMFs on the edges of troubled
# sub-cells, no reference counterpart): the reference with that step added
# to its corrector (oracle/patch_indfb.py, make -C oracle indfb); the GPU
# runs the same decks with fallback/apply=true
INDFB_BIN = os.path.join(ROOT, "oracle", "_ref", "spd_K_indfb")
INDFB_CASES = {
    "indfb_n8_p3_ader": INDUCTION_CASES["ind_golden_n8"],
    "indfb_n6_p3_rk2": INDUCTION_CASES["ind_n6_p3_rk2_fv"],
    "indfb_n8_p2_ader": ["job/fallback=true", "mesh/p=2", "mesh/nx1=8", "mesh/nx2=8", "mesh/nx3=8",
                         "time/tlim=0.1", "output/dt=0.05"],
    "indfb_n8_p4_rk3": ["job/fallback=true", "mesh/p=4", "mesh/nx1=8", "mesh/nx2=8", "mesh/nx3=8",
                        "time/integrator=rk3", "time/tlim=0.05", "output/dt=0.05"],
}
# (like the plain reference, the patched build crashes in the FV ghost fill
# at N = 6 for p = 2 and 4; these are decks it completes)


def indfb_fixtures(manifest):
    for name, ov in INDFB_CASES.items():
        ov = INDUCTION_BASE + ov
        with tempfile.TemporaryDirectory() as out:
            env = dict(os.environ, SPD_OUTPUT_DIR=out + "/", OMP_NUM_THREADS="8")
            r = subprocess.run([INDFB_BIN] + ov, capture_output=True, text=True, env=env, check=True)
            files = [f for f in os.listdir(out) if f.startswith("B2_cv_")]
            last = max(files, key=lambda f: int(f.split("_")[-2]))
            idx = int(last.split("_")[-2])
            steps = int(r.stdout.split("evolution: ")[1].split(" steps")[0])
            tr = [f for f in os.listdir(out) if f.startswith("troubles_") and int(f.split("_")[-2]) == idx][0]
            troubles = np.fromfile(os.path.join(out, tr))
            np.savez_compressed(os.path.join(HERE, name + ".npz"), B2_cv=np.fromfile(os.path.join(out, last)),
                                troubles=troubles)
            manifest.setdefault("indfb_cases", {})[name] = {
                "overrides": ov, "output": last, "steps": steps, "sha256_B2_cv": sha256(os.path.join(out, last)),
                "troubled_cells": int((troubles.reshape(4, -1)[3] > 0).sum())}
            print(name, last, steps, flush=True)


# 2D field-loop advection (the 2D induction solver): quasi-2D runs (nx3 = 2,
# periodic, B_z = 0) of the reference built with v = (2, 1, 0) and the loop
# centred at (1, 1) on [0, 2]^2 (oracle/patch_loop2d.py, make -C oracle
# loop2d); induction/nu = 0 (no resistive dt cap), fallback off
LOOP2D_BIN = os.path.join(ROOT, "oracle", "_ref", "spd_K_loop2d")
LOOP2D_BASE = ["job/system=induction", "induction/nu=0", "job/fallback=false", "mesh/x1len=2", "mesh/x2len=2",
               "mesh/x3len=1", "mesh/nx3=2", "time/cfl=0.8"]
LOOP2D_CASES = {
    "loop2d_n16_p4_ader": ["mesh/p=4", "mesh/nx1=16", "mesh/nx2=16", "time/tlim=0.1", "output/dt=0.1"],
    "loop2d_n12_p3_rk2": ["mesh/p=3", "mesh/nx1=12", "mesh/nx2=12", "time/integrator=rk2", "time/tlim=0.1",
                          "output/dt=0.1"],
    "loop2d_n8x12_p2_ader": ["mesh/p=2", "mesh/nx1=8", "mesh/nx2=12", "time/tlim=0.15", "output/dt=0.05"],
}


def loop2d_fixtures(manifest):
    for name, ov in LOOP2D_CASES.items():
        ov = LOOP2D_BASE + ov
        p = int([o for o in ov if o.startswith("mesh/p=")][0].split("=")[1])
        nx = int([o for o in ov if o.startswith("mesh/nx1=")][0].split("=")[1])
        ny = int([o for o in ov if o.startswith("mesh/nx2=")][0].split("=")[1])
        n = p + 1
        with tempfile.TemporaryDirectory() as out:
            env = dict(os.environ, SPD_OUTPUT_DIR=out + "/", OMP_NUM_THREADS="8")
            r = subprocess.run([LOOP2D_BIN] + ov, capture_output=True, text=True, env=env, check=True)
            files = [f for f in os.listdir(out) if f.startswith("B2_cv_")]
            last = max(files, key=lambda f: int(f.split("_")[-2]))
            steps = int(r.stdout.split("evolution: ")[1].split(" steps")[0])
            b = np.fromfile(os.path.join(out, last)).reshape(4, 4, ny + 2, nx + 2, n, n, n)
            act = b[:, 1:3, 1:-1, 1:-1]          # the two active z elements
            # the run is z-independent: both z elements are equal, and the z
            # sub-cell rows differ only by the rounding of the z averaging weights
            assert np.array_equal(act[:, 0], act[:, 1]), name
            scale = np.abs(act[:, 0]).max()
            assert all(np.abs(act[:, 0, :, :, 0] - act[:, 0, :, :, kk]).max() <= 1e-13 * scale for kk in range(n)), name
            np.savez_compressed(os.path.join(HERE, name + ".npz"),
                                B2_cv=np.ascontiguousarray(act[:, 0, :, :, 0]))
            manifest.setdefault("loop2d_cases", {})[name] = {
                "overrides": ov, "output": last, "steps": steps, "sha256_B2_cv": sha256(os.path.join(out, last)),
                "velocity": [2.0, 1.0], "center": [1.0, 1.0]}
            print(name, last, steps, flush=True)


def sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        h.update(f.read())
    return h.hexdigest()


def hydro_case(name, ov, entries):
    """run the reference on one hydro case; W_cv of the last output (active
    elements) into <name>.npz and its manifest entry into entries"""
    if True:
        with tempfile.TemporaryDirectory() as out:
            env = dict(os.environ, SPD_OUTPUT_DIR=out, OMP_NUM_THREADS="8")
            r = subprocess.run([REF_BIN] + ov, capture_output=True, text=True, env=env, check=True)
            files = sorted(f for f in os.listdir(out) if f.startswith("W_cv_"))
            last = max(files, key=lambda f: int(f.split("_")[-2]))
            raw = np.fromfile(os.path.join(out, last))
            # shape from the coordinate files: active faces per direction
            def n_el(axis):
                fs = [f for f in os.listdir(out) if f.startswith(axis + "_N")]
                return int(fs[0].split("_N")[1].split("p")[0]), int(fs[0].split("p")[1].split("_")[0])
            (Nx, p), (Ny, _), (Nz, _) = n_el("X"), n_el("Y"), n_el("Z")
            n = p + 1
            act = lambda N: N > 1
            shape = (1, 6, Nz + 2 if act(Nz) else 1, Ny + 2, Nx + 2, n if act(Nz) else 1, n, n)
            w = raw.reshape(shape)[0, :5]
            w = w[:, 1:-1] if act(Nz) else w
            w = w[:, :, 1:-1, 1:-1]
            steps = int(r.stdout.split("evolution: ")[1].split(" steps")[0])
            np.savez_compressed(os.path.join(HERE, name + ".npz"), W_cv=np.ascontiguousarray(w))
            entries[name] = {"overrides": ov, "output": last, "steps": steps,
                             "sha256": sha256(os.path.join(out, last)), "shape": list(w.shape)}
            print(name, last, w.shape, steps, flush=True)


def main():
    if not os.path.exists(REF_BIN):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    manifest = {"cases": {}, "goldens": {}}
    for name, ov in CASES.items():
        hydro_case(name, ov, manifest["cases"])
    for name, ov in VISCOUS_CASES.items():
        hydro_case(name, ov, manifest.setdefault("viscous_cases", {}))
    for name, ov in FULL_CASES.items():
        with tempfile.TemporaryDirectory() as out:
            env = dict(os.environ, SPD_OUTPUT_DIR=out, OMP_NUM_THREADS="8")
            r = subprocess.run([REF_BIN] + ov, capture_output=True, text=True, env=env, check=True)
            last = sorted(f for f in os.listdir(out) if f.startswith("W_cv_"))[-1]
            raw = np.fromfile(os.path.join(out, last))
            N = 32
            w = raw.reshape(1, 6, 1, N + 2, N + 2, 1, 4, 4)[0, :5, :, 1:-1, 1:-1]
            act4 = np.ascontiguousarray(w[[0, 1, 2, 4]])
            steps = int(r.stdout.split("evolution: ")[1].split(" steps")[0])
            np.savez_compressed(os.path.join(HERE, name + ".npz"), rho=np.ascontiguousarray(w[0]),
                                p=np.ascontiguousarray(w[4]))
            manifest["full_cases"] = manifest.get("full_cases", {})
            manifest["full_cases"][name] = {"overrides": ov, "output": last, "steps": steps,
                                            "sha256_active_rho_vx_vy_p": hashlib.sha256(act4.tobytes()).hexdigest()}
            print(name, last, steps, flush=True)
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as O
    for name, (N, steps) in BENCH_CASES.items():
        ov = bench.workload_overrides(N)
        dt0 = O.Oracle(O.config_from_params(O.apply_overrides({}, ov))).compute_dt()
        tend = steps * dt0 * 0.999
        ov = [x for x in ov if not x.startswith("output/")] + [f"time/tlim={tend!r}", f"output/dt={tend!r}"]
        with tempfile.TemporaryDirectory() as out:
            env = dict(os.environ, SPD_OUTPUT_DIR=out, OMP_NUM_THREADS="8")
            r = subprocess.run([REF_BIN] + ov, capture_output=True, text=True, env=env, check=True)
            raw = np.fromfile(os.path.join(out, f"W_cv_N{N}p3_1_0.dat"))
            w = raw.reshape(1, 6, 1, N + 2, N + 2, 1, 4, 4)[0, :5, :, 1:-1, 1:-1]
            a4 = np.ascontiguousarray(w[[0, 1, 2, 4]]) + 0.0   # +0.0 folds signed zeros
            nsteps = int(r.stdout.split("evolution: ")[1].split(" steps")[0])
            np.savez_compressed(os.path.join(HERE, name + ".npz"), W_cv=a4)
            manifest.setdefault("bench_cases", {})[name] = {
                "overrides": ov, "steps": nsteps, "slots": "rho, vx, vy, p",
                "sha256_signed_zero_folded": hashlib.sha256(a4.tobytes()).hexdigest()}
            print(name, nsteps, flush=True)
    induction_fixtures(manifest)
    for rel, what in GOLDENS.items():
        path = os.path.join(REF_TREE, "tests", "goldens", rel)
        if os.path.exists(path):
            manifest["goldens"][rel] = {"sha256": sha256(path), "what": what}
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    if "--viscous" in sys.argv:
        # regenerate only the viscous fixtures, keeping the rest of the manifest
        with open(os.path.join(HERE, "manifest.json")) as f:
            m = json.load(f)
        for name, ov in VISCOUS_CASES.items():
            hydro_case(name, ov, m.setdefault("viscous_cases", {}))
        with open(os.path.join(HERE, "manifest.json"), "w") as f:
            json.dump(m, f, indent=1)
    elif "--indfb" in sys.argv:
        # regenerate only the applied induction fallback fixtures
        with open(os.path.join(HERE, "manifest.json")) as f:
            m = json.load(f)
        indfb_fixtures(m)
        with open(os.path.join(HERE, "manifest.json"), "w") as f:
            json.dump(m, f, indent=1)
    elif "--loop2d" in sys.argv:
        # regenerate only the 2D field-loop fixtures, keeping the rest of the manifest
        with open(os.path.join(HERE, "manifest.json")) as f:
            m = json.load(f)
        loop2d_fixtures(m)
        with open(os.path.join(HERE, "manifest.json"), "w") as f:
            json.dump(m, f, indent=1)
    elif "--induction" in sys.argv:
        # regenerate only the induction fixtures, keeping the rest of the manifest
        with open(os.path.join(HERE, "manifest.json")) as f:
            m = json.load(f)
        induction_fixtures(m)
        with open(os.path.join(HERE, "manifest.json"), "w") as f:
            json.dump(m, f, indent=1)
    else:
        sys.exit(main())
