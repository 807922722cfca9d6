"""C ABI and host-side set-up of libspdk_cuda.so (no GPU needed).

- the library loads and exports every function include/spdk.h declares;
- argument validation fails cleanly before any device call;
- the transform matrices and the initial condition computed by the
  product's host code are bit-identical to the oracle's (and therefore to
  the reference's, which the oracle reproduces bit for bit).
"""
import ctypes
import os
import re

import numpy as np
import pytest

from helpers import gpu_config, oracle_config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "spdk.h")


PROTO_HEADER = os.path.join(ROOT, "include", "spdk_proto.h")
INDUCTION_HEADER = os.path.join(ROOT, "include", "spdk_induction.h")
LEARNED_HEADER = os.path.join(ROOT, "include", "spdk_learned.h")
BATCH_HEADER = os.path.join(ROOT, "include", "spdk_batch.h")


def declared_functions(paths=(HEADER, PROTO_HEADER, INDUCTION_HEADER, LEARNED_HEADER, BATCH_HEADER)):
    names = set()
    for path in paths:
        text = re.sub(r"/\*.*?\*/", "", open(path).read(), flags=re.S)
        names |= set(re.findall(r"\b(spdk_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from spd_k_b200.api import load_library
    return load_library()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 40
    for n in names:
        assert hasattr(lib, n), n


def test_abi_version(lib):
    ver = int(re.search(r"#define SPDK_ABI_VERSION (\d+)", open(HEADER).read()).group(1))
    assert lib.spdk_abi_version() == ver


def test_bad_config_is_rejected_without_a_device(lib):
    from spd_k_b200.api import make_config
    c = gpu_config(["mesh/nx3=1", "mesh/p=9"])
    cfg = make_config(c)
    h = ctypes.c_void_p()
    rc = lib.spdk_hydro_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == -1
    assert b"p must be" in lib.spdk_last_error()
    c = gpu_config(["mesh/nx1=1"])
    rc = lib.spdk_hydro_create(ctypes.byref(make_config(c)), ctypes.byref(h))
    assert rc == -1
    c = gpu_config(["mesh/nx3=1", "hydro/nu=-0.1"])
    rc = lib.spdk_hydro_create(ctypes.byref(make_config(c)), ctypes.byref(h))
    assert rc == -1 and b"nu must be" in lib.spdk_last_error()


def test_viscosity_parameters_follow_the_reference_defaults():
    """hydro/nu opts in, hydro/beta defaults to -2/3 nu (src/main.cpp:236-237)"""
    from spd_k_b200.api import make_config
    c = gpu_config(["hydro/nu=0.03"])
    cfg = make_config(c)
    assert cfg.nu == 0.03 and cfg.beta == -2. / 3 * 0.03
    cfg = make_config(gpu_config(["hydro/nu=0.03", "hydro/beta=0.5"]))
    assert cfg.beta == 0.5
    assert make_config(gpu_config([])).nu == 0.0


@pytest.mark.parametrize("p", range(1, 8))
@pytest.mark.parametrize("ader", [1, 0])
def test_matrices_match_oracle(lib, p, ader):
    from oracle import oracle as O
    n, nf = p + 1, p + 2
    bufs = {k: np.zeros(s) for k, s in [("sp_to_fp", nf * n), ("dfp_to_sp", n * nf), ("sp_to_cv", n * n),
                                         ("cv_to_sp", n * n), ("invader", n * n), ("wt", n)]}
    P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    lib.spdk_build_matrices.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.POINTER(ctypes.c_double)] * 6
    assert lib.spdk_build_matrices(p, ader, *(P(bufs[k]) for k in
                                              ("sp_to_fp", "dfp_to_sp", "sp_to_cv", "cv_to_sp", "invader", "wt"))) == 0
    o = O.Oracle(oracle_config([f"mesh/p={p}", "mesh/nx1=2", "mesh/nx2=2", "mesh/nx3=1",
                                "time/integrator=" + ("ader" if ader else "rk3")]))
    for k in ("sp_to_fp", "dfp_to_sp", "sp_to_cv", "cv_to_sp"):
        assert np.array_equal(bufs[k], o.array(k).ravel()), k
    if ader:
        assert np.array_equal(bufs["invader"], o.array("invader").ravel())
        assert np.array_equal(bufs["wt"], o.array("wt").ravel())


IC_CASES = [
    ["mesh/nx1=6", "mesh/nx2=4", "mesh/nx3=1"],
    ["mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=1", "problem/problem=spherical_blast"],
    ["mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=4", "problem/problem=spherical_blast", "mesh/p=2"],
    ["mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=1", "problem/problem=kelvin_helmholtz"],
    ["mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=1", "problem/problem=implosion", "mesh/x1len=0.3", "mesh/x2len=0.3"],
    ["mesh/nx1=4", "mesh/nx2=8", "mesh/nx3=1", "problem/problem=rti", "hydro/g2=-0.1"],
    ["mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=1", "problem/problem=sedov", "mesh/p=4"],
    ["mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=1", "problem/problem=square"],
    ["mesh/nx1=8", "mesh/nx2=2", "mesh/nx3=1", "problem/problem=sod_shock_tube"],
    ["mesh/nx1=8", "mesh/nx2=2", "mesh/nx3=1", "problem/problem=shu_osher", "mesh/x1len=2"],
    ["mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=1", "problem/problem=user"],
    ["mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=2", "problem/problem=kh_noise", "mesh/p=5"],
    ["mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=1", "problem/problem=rti_top", "hydro/g2=-0.1"],
    # large enough (>= 2^22 point evaluations) for the host-threaded quadrature
    ["mesh/nx1=128", "mesh/nx2=136", "mesh/nx3=1", "problem/problem=rti_top", "hydro/g2=-0.1"],
    ["mesh/nx1=6", "mesh/nx2=6", "mesh/nx3=6", "problem/problem=kh_noise", "mesh/p=5"],
]


@pytest.mark.parametrize("ov", IC_CASES, ids=lambda ov: "_".join(x.split("=")[1] for x in ov))
def test_initial_condition_matches_oracle(lib, ov):
    from oracle import oracle as O
    from spd_k_b200.api import make_config
    extra = {"q": [1e-3], "seed": 12345}
    cg = dict(gpu_config(ov), **extra)
    co = dict(oracle_config(ov), **extra)
    if cg["problem"] == "quadrant":
        pass
    D = 3 if cg["N"][2] > 1 else 2
    V, n = D + 2, cg["p"] + 1
    npt = n ** D
    E = cg["N"][0] * cg["N"][1] * (cg["N"][2] if D == 3 else 1)
    out = np.zeros(E * V * npt)
    lib.spdk_initial_wcv.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t]
    cfg = make_config(cg)
    assert lib.spdk_initial_wcv(ctypes.byref(cfg), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size) == 0
    o = O.Oracle(co)
    w = o.array("W_cv")[0]  # oracle initial W_cv (the constructor keeps it)
    w = w[:, 1:-1] if D == 3 else w
    w = w[:, :, 1:-1, 1:-1]
    Nx, Ny, Nz = cg["N"][0], cg["N"][1], (cg["N"][2] if D == 3 else 1)
    nz = n if D == 3 else 1
    mine = out.reshape(Nz, Ny, Nx, V, nz, n, n).transpose(3, 0, 1, 2, 4, 5, 6)
    slots = [0, 1, 2, 3, 4] if D == 3 else [0, 1, 2, 4]
    assert np.array_equal(mine, w[slots])


def test_driver_rejects_bad_command_lines_without_a_device(tmp_path):
    """spdk_run parses like src/main.cpp: -i <deck>, block/name=value
    overrides, anything else is an error; configuration errors end the run
    before any device call"""
    import subprocess
    drv = os.path.join(ROOT, "spd_k_b200", "spdk_run")
    env = dict(os.environ, SPD_OUTPUT_DIR=str(tmp_path))
    for args, msg in ((["bogus"], "unrecognized argument"), (["job/system=mhd"], "unknown system"),
                      (["mesh/nx1=1"], "x-direction must be active"),
                      (["time/integrator=rk4"], "unknown integrator"),
                      (["mesh/x1_bc=open"], "unknown boundary"),
                      (["-i", str(tmp_path / "missing.athinput")], "cannot open input file")):
        r = subprocess.run([drv] + args, capture_output=True, text=True, env=env, timeout=60)
        assert r.returncode == 1 and msg in r.stderr, (args, r.stderr)


def test_fv_faces_match_oracle(lib):
    from oracle import oracle as O
    c = oracle_config(["mesh/nx1=6", "mesh/nx2=4", "mesh/nx3=1", "mesh/x1len=0.3", "mesh/p=4"])
    o = O.Oracle(c)
    for d, (N, L, act) in enumerate(((6, 0.3, 1), (4, 1.0, 1), (1, 1.0, 0))):
        want = o.array("fv_faces_" + "xyz"[d]).reshape(-1)
        n = len(want) if act else 1
        out = np.zeros(n)
        assert lib.spdk_fv_faces(N, 4, ctypes.c_double(L), act, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 ctypes.c_size_t(n)) == 0
        if act:
            assert np.array_equal(out, want)
