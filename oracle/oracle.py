"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``liboracle.so`` (the C restatement in spdk_oracle.c) and drives it
with the reference's own time loop (src/hydro_ader.hpp:215-273), so tests
and the CPU baseline can compare the CUDA path against it. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import this.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "spd_K_ref")

PERIODIC, GRADFREE, REFLECTIVE = 0, 1, 2
ADER, RK = 0, 1
PROBLEMS = {
    "sine_wave": 0, "sedov": 1, "spherical_blast": 2, "square": 3,
    "sod_shock_tube": 4, "shu_osher": 5, "kelvin_helmholtz": 6,
    "implosion": 7, "rti": 8, "user": 9,
    # project problems (no reference counterpart)
    "kh_noise": 10, "quadrant": 11, "rti_top": 12,
}
BCS = {"periodic": PERIODIC, "gradfree": GRADFREE, "reflective": REFLECTIVE}


class OrcCfg(ctypes.Structure):
    _fields_ = [
        ("p", ctypes.c_int), ("N", ctypes.c_int * 3), ("L", ctypes.c_double * 3),
        ("bc", ctypes.c_int * 3), ("integrator", ctypes.c_int), ("rk_order", ctypes.c_int),
        ("fallback", ctypes.c_int), ("gamma", ctypes.c_double), ("cfl", ctypes.c_double),
        ("g", ctypes.c_double * 3), ("nad_tolerance", ctypes.c_double),
        ("nad_delta", ctypes.c_int), ("nad_moore", ctypes.c_int), ("sed", ctypes.c_int),
        ("blending", ctypes.c_int), ("problem", ctypes.c_int),
        ("amp", ctypes.c_double), ("v1", ctypes.c_double), ("v2", ctypes.c_double),
        ("v3", ctypes.c_double), ("d0", ctypes.c_double), ("d1", ctypes.c_double),
        ("p0", ctypes.c_double), ("p1", ctypes.c_double), ("radius", ctypes.c_double),
        ("sigma", ctypes.c_double), ("dir", ctypes.c_int),
        ("cx", ctypes.c_double), ("cy", ctypes.c_double), ("cz", ctypes.c_double),
        ("q", ctypes.c_double * 16), ("seed", ctypes.c_ulonglong), ("nu", ctypes.c_double), ("beta", ctypes.c_double),
    ]


# per-problem <problem> defaults: src/main.cpp:31-65
# (amp, v1, v2, v3, d0, d1, p0, p1, radius, sigma, dir)
PROBLEM_DEFAULTS = {
    "sine_wave": (0.125, 1.0, 1.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0),
    "square": (0.0, 1.0, 1.0, 0.0, 1.0, 2.0, 1.0, 0.0, 0.25, 0.0, 0),
    "sod_shock_tube": (0.0, 0.0, 0.0, 0.0, 1.0, 0.125, 1.0, 0.1, 0.5, 0.0, 0),
    "shu_osher": (0.2, 0.0, 0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0),
    "kelvin_helmholtz": (0.1, 0.5, 0.0, 0.0, 1.0, 2.0, 2.5, 0.0, 0.0, 0.05 / math.sqrt(2.0), 0),
    "implosion": (0.0, 0.0, 0.0, 0.0, 1.0, 0.125, 1.0, 0.14, 0.15, 0.0, 0),
    "sedov": (0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.1, 0.0, 0),
    "spherical_blast": (0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 10.0, 0.1, 0.1, 0.0, 0),
    "rti": (0.025, 0.0, 0.0, 0.0, 2.0, 1.0, 1.0, 0.0, 0.5, 0.0, 0),
    "user": (0.5, 1.0, 0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.5, 0.1, 0),
    "kh_noise": (0.01, 0.5, 0.0, 0.0, 1.0, 2.0, 2.5, 0.0, 0.25, 0.0, 0),
    "quadrant": (0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0, 0.0, 0.0, 0),
    "rti_top": (0.01, 0.0, 0.0, 0.0, 2.0, 1.0, 2.5, 0.0, 0.75, 0.0, 0),
}
PP_NAMES = ("amp", "v1", "v2", "v3", "d0", "d1", "p0", "p1", "radius", "sigma", "dir")


def parse_athinput(text):
    """block -> {name: value-string}; last assignment wins
    (src/parameter_input.cpp:24-73)."""
    params, block = {}, None
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if not line:
            continue
        if line.startswith("<"):
            block = line[1:line.index(">")].strip()
            params.setdefault(block, {})
            continue
        name, value = line.split("=", 1)
        params.setdefault(block, {})[name.strip()] = value.strip()
    return params


def apply_overrides(params, overrides):
    for o in overrides:
        bn, value = o.split("=", 1)
        block, name = bn.split("/", 1)
        params.setdefault(block.strip(), {})[name.strip()] = value.strip()
    return params


def _get(params, block, name, default, conv):
    v = params.get(block, {}).get(name)
    return default if v is None else conv(v)


def _bool(v):
    v = v.lower()
    if v in ("true", "yes", "on", "1"):
        return True
    if v in ("false", "no", "off", "0"):
        return False
    raise ValueError(f"not a boolean: {v}")


def config_from_params(params):
    """RunConfig + mesh exactly as src/main.cpp:126-189 builds them."""
    g = lambda b, n, d, c=float: _get(params, b, n, d, c)
    p = g("mesh", "p", 3, int)
    N = [g("mesh", "nx1", 8, int), g("mesh", "nx2", 8, int), g("mesh", "nx3", 8, int)]
    L = [g("mesh", "x1len", 1.0), g("mesh", "x2len", 1.0), g("mesh", "x3len", 1.0)]
    problem = g("problem", "problem", "sine_wave", str)
    integ = g("time", "integrator", "ader", str)
    c = dict(
        p=p, N=N, L=L,
        cfl=g("time", "cfl", 0.8), gamma=g("hydro", "gamma", 1.4),
        g=[g("hydro", "g1", 0.0), g("hydro", "g2", 0.0), g("hydro", "g3", 0.0)],
        fallback=g("job", "fallback", True, _bool),
        nad_tolerance=g("fallback", "tolerance", 1e-5),
        nad_delta=g("fallback", "NAD", "relative", str) == "delta",
        nad_moore=g("fallback", "NAD_neighbors", "2nd", str) == "2nd",
        sed=g("fallback", "SED", True, _bool),
        blending=g("fallback", "blending", True, _bool),
        problem=problem,
        bc=[g("mesh", "x1_bc", "periodic", str), g("mesh", "x2_bc", "periodic", str),
            g("mesh", "x3_bc", "periodic", str)],
        integrator=integ,
        tlim=g("time", "tlim", 0.1),
        output_dt=g("output", "dt", None),
        system=g("job", "system", "hydro", str),
    )
    dflt = PROBLEM_DEFAULTS[problem]
    for name, d in zip(PP_NAMES, dflt):
        c[name] = g("problem", name, d, int if name == "dir" else float)
    c["cx"], c["cy"], c["cz"] = 0.5 * L[0], 0.5 * L[1], 0.5 * L[2]
    # src/main.cpp:236-237: hydro/nu, hydro/beta = -2./3*nu by default
    c["nu"] = g("hydro", "nu", 0.0)
    c["beta"] = g("hydro", "beta", -2. / 3 * c["nu"])
    return c


def make_cfg(c):
    """dict (config_from_params keys) -> OrcCfg."""
    o = OrcCfg()
    o.p = c["p"]
    for d in range(3):
        o.N[d] = c["N"][d]
        o.L[d] = c["L"][d]
        o.bc[d] = BCS[c["bc"][d]] if isinstance(c["bc"][d], str) else c["bc"][d]
        o.g[d] = c["g"][d]
    integ = c.get("integrator", "ader")
    if integ == "ader":
        o.integrator, o.rk_order = ADER, 3
    else:
        o.integrator, o.rk_order = RK, int(integ[2])
    o.fallback = int(c["fallback"])
    o.gamma, o.cfl = c["gamma"], c["cfl"]
    o.nad_tolerance = c["nad_tolerance"]
    o.nad_delta, o.nad_moore = int(c["nad_delta"]), int(c["nad_moore"])
    o.sed, o.blending = int(c["sed"]), int(c["blending"])
    o.problem = PROBLEMS[c["problem"]]
    for name in PP_NAMES:
        setattr(o, name, c[name])
    o.cx, o.cy, o.cz = c["cx"], c["cy"], c["cz"]
    for i, v in enumerate(c.get("q", [])):
        o.q[i] = v
    o.seed = c.get("seed", 0)
    o.nu = c.get("nu", 0.0)
    o.beta = c.get("beta", -2. / 3 * o.nu)
    return o


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(OrcCfg)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_compute_dt.restype = ctypes.c_double
        L.orc_compute_dt.argtypes = [ctypes.c_void_p]
        for f in ("orc_step", "orc_update_prediction", "orc_update_solution", "orc_fv_update"):
            getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_double]
        for f in ("orc_copy_ader", "orc_solve_fluxes", "orc_primitives_to_cv"):
            getattr(L, f).argtypes = [ctypes.c_void_p]
        L.orc_array.restype = ctypes.POINTER(ctypes.c_double)
        L.orc_array.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
        _lib = L
    return _lib


class Oracle:
    """One hydro solver instance (the reference's Hydro_ader constructor:
    matrices, ICs, W_sp/U_sp; src/hydro_ader.hpp:76-213)."""

    def __init__(self, c):
        self.c = c
        self._cfg = make_cfg(c)
        self.h = lib().orc_create(ctypes.byref(self._cfg))
        self.t = 0.0
        self.n_step = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def array(self, name, copy=True):
        dims = (ctypes.c_int * 8)()
        ptr = lib().orc_array(self.h, name.encode(), dims)
        if not ptr:
            raise KeyError(name)
        shape = tuple(dims)
        n = int(np.prod(shape))
        a = np.ctypeslib.as_array(ptr, shape=(n,)).reshape(shape)
        return a.copy() if copy else a

    def set_array(self, name, values):
        a = self.array(name, copy=False)
        a[...] = np.asarray(values, dtype=np.float64).reshape(a.shape)

    def compute_dt(self):
        return lib().orc_compute_dt(self.h)

    def step(self, dt):
        lib().orc_step(self.h, dt)

    def call(self, name, *args):
        getattr(lib(), "orc_" + name)(self.h, *args)

    def run(self, t_end, dt_output=None, max_steps=None, on_output=None):
        """src/hydro_ader.hpp:215-273: dt from the constructor, optional
        output clamping of dt, output index 0 written at construction."""
        outputs = dt_output is not None and dt_output > 0
        dt = self.compute_dt()
        t_output = dt_output if outputs else None
        n_out = 0
        if outputs and on_output:
            on_output(n_out, self)
        if outputs:
            n_out += 1
        steps = 0
        while self.t < t_end:
            self.step(dt)
            self.t += dt
            self.n_step += 1
            steps += 1
            dt = self.compute_dt()
            if outputs:
                if self.t >= t_output:
                    t_output = self.t + dt_output
                    if on_output:
                        on_output(n_out, self)
                    n_out += 1
                if self.t + dt > t_output:
                    dt = t_output - self.t
            if max_steps is not None and steps >= max_steps:
                break
        return dt


def run_reference(input_file, overrides, outdir, threads=None, timeout=3600):
    """Run the reference's own CPU build (oracle/_ref/spd_K_ref) with an
    athinput deck; returns its stdout."""
    env = dict(os.environ, SPD_OUTPUT_DIR=outdir)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    r = subprocess.run([REF_BIN, "-i", input_file] + list(overrides), env=env,
                       capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])
    return r.stdout


def load_dump(path, shape=None):
    a = np.fromfile(path)
    return a if shape is None else a.reshape(shape)
