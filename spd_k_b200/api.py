"""Python host interface of the spd_K B200 solver (ctypes over libspdk_cuda.so).

Mirrors the reference's driver-facing objects: ``HydroSolver`` is
``Hydro_ader`` (constructor = set-up, ``step`` = one pass of the
time_evolution loop body, ``evolve`` = time_evolution), configured from the
same athinput blocks (src/main.cpp:126-189). There is no CPU fallback: if the
CUDA library is missing or no GPU is present, construction raises.
"""
import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspdk_cuda.so")

BC = {"periodic": 0, "gradfree": 1, "reflective": 2}
PROBLEMS = {
    "sine_wave": 0, "sedov": 1, "spherical_blast": 2, "square": 3,
    "sod_shock_tube": 4, "shu_osher": 5, "kelvin_helmholtz": 6,
    "implosion": 7, "rti": 8, "user": 9, "kh_noise": 10, "quadrant": 11,
    "rti_top": 12,
}
FIELD_U_SP, FIELD_W_CV, FIELD_TROUBLES, FIELD_THETA = 0, 1, 2, 3
FIELD_ELEMENT_TROUBLES, FIELD_ELEMENT_PREDICTED = 4, 5
# arithmetic of the solver: the plain FP64 form (bitwise the reference) or
# the FP32 precision form (FP64 kept for pressure recovery, detector bounds, dt)
PRECISIONS = {"fp64": 0, "fp32": 1}
PRECISIONS_BY_ID = {v: k for k, v in PRECISIONS.items()}

# per-problem <problem> defaults (src/main.cpp:31-65):
# amp, v1, v2, v3, d0, d1, p0, p1, radius, sigma, dir
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


class HydroConfig(ctypes.Structure):
    """spdk_hydro_config (include/spdk.h)."""
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
        ("q", ctypes.c_double * 16), ("seed", ctypes.c_ulonglong),
        ("precision", ctypes.c_int), ("device", ctypes.c_int),
        ("nu", ctypes.c_double), ("beta", ctypes.c_double),
        ("slab_lo", ctypes.c_int), ("slab_n", ctypes.c_int),
    ]


class HydroInfo(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int), ("p", ctypes.c_int), ("n_points", ctypes.c_int),
        ("nvar", ctypes.c_int), ("N", ctypes.c_int * 3), ("n_elements", ctypes.c_longlong),
        ("n_dof", ctypes.c_longlong), ("n_time_slices", ctypes.c_int),
        ("launches_per_step", ctypes.c_int), ("device_bytes", ctypes.c_size_t),
    ]


class CheckpointInfo(ctypes.Structure):
    """spdk_checkpoint_info (include/spdk.h)"""
    _fields_ = [("t", ctypes.c_double), ("t_output", ctypes.c_double), ("steps", ctypes.c_longlong),
                ("outputs", ctypes.c_longlong)]


EXPORTS = (
    "spdk_last_error", "spdk_abi_version", "spdk_hydro_create", "spdk_hydro_destroy",
    "spdk_hydro_get_info", "spdk_hydro_get_dt", "spdk_hydro_set_dt", "spdk_hydro_step",
    "spdk_hydro_steps", "spdk_hydro_evolve", "spdk_hydro_evolve_from", "spdk_hydro_sync", "spdk_hydro_read",
    "spdk_hydro_write",
)

_lib = None


class SpdkError(RuntimeError):
    pass


def load_library(path=LIB_PATH):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise SpdkError(f"{path} is missing: build it with `python -m spd_k_b200.build`")
    L = ctypes.CDLL(path)
    L.spdk_last_error.restype = ctypes.c_char_p
    L.spdk_abi_version.restype = ctypes.c_int
    L.spdk_hydro_create.argtypes = [ctypes.POINTER(HydroConfig), ctypes.POINTER(ctypes.c_void_p)]
    L.spdk_hydro_destroy.argtypes = [ctypes.c_void_p]
    L.spdk_hydro_get_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(HydroInfo)]
    L.spdk_hydro_get_dt.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
    L.spdk_hydro_set_dt.argtypes = [ctypes.c_void_p, ctypes.c_double]
    L.spdk_hydro_step.argtypes = [ctypes.c_void_p]
    L.spdk_hydro_steps.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.spdk_hydro_evolve.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                    ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_double)]
    L.spdk_hydro_evolve_from.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_double)]
    L.spdk_hydro_sync.argtypes = [ctypes.c_void_p]
    L.spdk_hydro_read.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                  ctypes.c_size_t]
    L.spdk_hydro_write.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                   ctypes.c_size_t]
    ci = ctypes.POINTER(CheckpointInfo)
    L.spdk_hydro_checkpoint.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ci]
    L.spdk_hydro_checkpoint_async.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ci]
    L.spdk_hydro_checkpoint_wait.argtypes = [ctypes.c_void_p]
    L.spdk_hydro_restore.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ci]
    ip = ctypes.POINTER(ctypes.c_int)
    L.spdk_checkpoint_peek.argtypes = [ctypes.c_char_p, ci, ip, ip, ip, ip, ip]
    L.spdk_hydro_rows.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    L.spdk_hydro_slab_dt.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.spdk_hydro_conserved.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise SpdkError(f"spdk error {rc}: {_lib.spdk_last_error().decode()}")


def checkpoint_peek(path):
    """spdk_checkpoint_peek: a checkpoint's header, without a solver or a GPU"""
    L = load_library()
    info = CheckpointInfo()
    prec, p, integ, rk = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    N = (ctypes.c_int * 3)()
    _check(L.spdk_checkpoint_peek(os.fsencode(path), ctypes.byref(info), ctypes.byref(prec), ctypes.byref(p), N,
                                  ctypes.byref(integ), ctypes.byref(rk)))
    return {"t": info.t, "t_output": info.t_output, "steps": info.steps, "outputs": info.outputs,
            "precision": PRECISIONS_BY_ID.get(prec.value, prec.value), "p": p.value, "N": list(N),
            "integrator": integ.value, "rk_order": rk.value}


def parse_athinput(text):
    """block -> {name: value} (src/parameter_input.cpp:24-73)."""
    params, block = {}, None
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if not line:
            continue
        if line.startswith("<"):
            block = line[1:line.index(">")].strip()
            params.setdefault(block, {})
            continue
        if "=" not in line or block is None:
            raise ValueError(f"bad athinput line: {line!r}")
        name, value = line.split("=", 1)
        params[block][name.strip()] = value.strip()
    return params


def apply_overrides(params, overrides):
    for o in overrides:
        bn, value = o.split("=", 1)
        block, name = bn.split("/", 1)
        params.setdefault(block.strip(), {})[name.strip()] = value.strip()
    return params


def _bool(v):
    v = v.lower()
    if v in ("true", "yes", "on", "1"):
        return True
    if v in ("false", "no", "off", "0"):
        return False
    raise ValueError(f"not a boolean: {v}")


def config_from_params(params):
    """Run configuration with the reference's defaults (src/main.cpp:126-189)."""
    def g(b, n, d, conv=float):
        v = params.get(b, {}).get(n)
        return d if v is None else conv(v)
    L = [g("mesh", "x1len", 1.0), g("mesh", "x2len", 1.0), g("mesh", "x3len", 1.0)]
    problem = g("problem", "problem", "sine_wave", str)
    c = dict(
        p=g("mesh", "p", 3, int),
        N=[g("mesh", "nx1", 8, int), g("mesh", "nx2", 8, int), g("mesh", "nx3", 8, int)],
        L=L, cfl=g("time", "cfl", 0.8), gamma=g("hydro", "gamma", 1.4),
        g=[g("hydro", "g1", 0.0), g("hydro", "g2", 0.0), g("hydro", "g3", 0.0)],
        fallback=g("job", "fallback", True, _bool),
        nad_tolerance=g("fallback", "tolerance", 1e-5),
        nad_delta=g("fallback", "NAD", "relative", str) == "delta",
        nad_moore=g("fallback", "NAD_neighbors", "2nd", str) == "2nd",
        sed=g("fallback", "SED", True, _bool), blending=g("fallback", "blending", True, _bool),
        problem=problem,
        bc=[g("mesh", "x1_bc", "periodic", str), g("mesh", "x2_bc", "periodic", str),
            g("mesh", "x3_bc", "periodic", str)],
        integrator=g("time", "integrator", "ader", str),
        tlim=g("time", "tlim", 0.1), output_dt=g("output", "dt", None),
        system=g("job", "system", "hydro", str),
    )
    for name, d in zip(PP_NAMES, PROBLEM_DEFAULTS[problem]):
        c[name] = g("problem", name, d, int if name == "dir" else float)
    c["cx"], c["cy"], c["cz"] = 0.5 * L[0], 0.5 * L[1], 0.5 * L[2]
    # src/main.cpp:236-237: viscosity is opt-in (hydro/nu > 0); beta = -2/3 nu by default
    c["nu"] = g("hydro", "nu", 0.0)
    c["beta"] = g("hydro", "beta", -2. / 3 * c["nu"])
    return c


def make_config(c, device=0):
    o = HydroConfig()
    o.p = c["p"]
    for d in range(3):
        o.N[d] = c["N"][d]
        o.L[d] = c["L"][d]
        o.bc[d] = BC[c["bc"][d]] if isinstance(c["bc"][d], str) else int(c["bc"][d])
        o.g[d] = c["g"][d]
    integ = c.get("integrator", "ader")
    if integ == "ader":
        o.integrator, o.rk_order = 0, 3
    elif integ.startswith("rk") and len(integ) == 3 and integ[2] in "123":
        o.integrator, o.rk_order = 1, int(integ[2])
    else:
        raise ValueError(f"unknown integrator {integ!r} (ader, rk1, rk2, rk3)")
    o.fallback = int(bool(c["fallback"]))
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
    o.seed = int(c.get("seed", 0))
    prec = c.get("precision", "fp64")
    if prec not in PRECISIONS:
        raise ValueError(f"unknown precision {prec!r} ({', '.join(PRECISIONS)})")
    o.precision = PRECISIONS[prec]
    o.device = device
    o.nu = c.get("nu", 0.0)
    o.beta = c.get("beta", -2. / 3 * o.nu)
    o.slab_lo, o.slab_n = int(c.get("slab_lo", 0)), int(c.get("slab_n", 0))
    return o


class HydroSolver:
    """GPU solver instance (the reference's Hydro_ader)."""

    def __init__(self, c, device=0):
        L = load_library()
        self.c = c
        self._cfg = make_config(c, device)
        h = ctypes.c_void_p()
        _check(L.spdk_hydro_create(ctypes.byref(self._cfg), ctypes.byref(h)))
        self.h = h
        info = HydroInfo()
        _check(L.spdk_hydro_get_info(self.h, ctypes.byref(info)))
        self.info = info
        self.ndim, self.p, self.npt, self.nvar = info.ndim, info.p, info.n_points, info.nvar
        self.N = tuple(info.N)
        self.t = 0.0
        self.n_step = 0

    @classmethod
    def attach(cls, handle, c):
        """a non-owning view of a solver handle owned elsewhere (a batch member)"""
        self = cls.__new__(cls)
        self.c = c
        self.h = handle
        self._owner = False
        info = HydroInfo()
        _check(_lib.spdk_hydro_get_info(self.h, ctypes.byref(info)))
        self.info = info
        self.ndim, self.p, self.npt, self.nvar = info.ndim, info.p, info.n_points, info.nvar
        self.N = tuple(info.N)
        self.t = 0.0
        self.n_step = 0
        return self

    def close(self):
        if not getattr(self, "_owner", True):
            self.h = None
            return
        if getattr(self, "h", None):
            _lib.spdk_hydro_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def n_dof(self):
        return self.info.n_dof

    def dt(self):
        v = ctypes.c_double()
        _check(_lib.spdk_hydro_get_dt(self.h, ctypes.byref(v)))
        return v.value

    def set_dt(self, dt):
        _check(_lib.spdk_hydro_set_dt(self.h, dt))

    def step(self):
        _check(_lib.spdk_hydro_step(self.h))

    def rows_to(self, lo, hi, buf):
        """element rows [lo, hi) of U_sp along the slab axis -> device tensor buf
        (solver arithmetic), ordered on the solver stream"""
        _check(_lib.spdk_hydro_rows(self.h, 0, lo, hi, ctypes.c_void_p(buf.data_ptr())))

    def rows_from(self, lo, hi, buf):
        """device tensor buf -> element rows [lo, hi) of U_sp"""
        _check(_lib.spdk_hydro_rows(self.h, 1, lo, hi, ctypes.c_void_p(buf.data_ptr())))

    def slab_dt(self, lo, hi):
        """next dt = minimum of the CFL / diffusion candidates over element rows
        [lo, hi) of the current W_cv; returns it"""
        _check(_lib.spdk_hydro_slab_dt(self.h, lo, hi))
        return self.dt()

    def steps(self, n):
        _check(_lib.spdk_hydro_steps(self.h, n))

    def sync(self):
        _check(_lib.spdk_hydro_sync(self.h))

    def evolve(self, t_end, dt_output=None, t0=None, t_output=None):
        """time_evolution on the device (spdk_hydro_evolve); with t0 (and the
        next output time t_output) it resumes a run (spdk_hydro_evolve_from)"""
        steps, t = ctypes.c_longlong(), ctypes.c_double()
        if t0 is None:
            _check(_lib.spdk_hydro_evolve(self.h, t_end, dt_output or -1.0, ctypes.byref(steps), ctypes.byref(t)))
        else:
            t_out0 = t_output if t_output is not None else -1.0
            _check(_lib.spdk_hydro_evolve_from(self.h, t0, t_out0, t_end, dt_output or -1.0, ctypes.byref(steps),
                                               ctypes.byref(t)))
        self.t = t.value
        self.n_step += steps.value
        return steps.value

    def conserved(self):
        """FP64 domain integrals of (rho, m_1..m_D, E), compensated sums"""
        a = np.empty(self.nvar, dtype=np.float64)
        _check(_lib.spdk_hydro_conserved(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self.nvar))
        return a

    def read(self, field, out=None):
        cells = self.info.n_elements * self.npt
        if field in (FIELD_U_SP, FIELD_W_CV):
            count = cells * self.nvar
        elif field in (FIELD_ELEMENT_TROUBLES, FIELD_ELEMENT_PREDICTED):
            count = self.info.n_elements
        else:
            count = cells
        a = out if out is not None else np.empty(count, dtype=np.float64)
        _check(_lib.spdk_hydro_read(self.h, field, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), count))
        return a

    def checkpoint(self, path, t=0.0, t_output=0.0, steps=0, outputs=0, wait=True):
        """spdk_hydro_checkpoint (wait=True) or spdk_hydro_checkpoint_async"""
        info = CheckpointInfo(t, t_output, steps, outputs)
        fn = _lib.spdk_hydro_checkpoint if wait else _lib.spdk_hydro_checkpoint_async
        _check(fn(self.h, os.fsencode(path), ctypes.byref(info)))

    def checkpoint_wait(self):
        _check(_lib.spdk_hydro_checkpoint_wait(self.h))

    def restore(self, path):
        """spdk_hydro_restore; returns the stored bookkeeping as a dict"""
        info = CheckpointInfo()
        _check(_lib.spdk_hydro_restore(self.h, os.fsencode(path), ctypes.byref(info)))
        return {"t": info.t, "t_output": info.t_output, "steps": info.steps, "outputs": info.outputs}

    def write_u(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64).ravel()
        _check(_lib.spdk_hydro_write(self.h, FIELD_U_SP, u.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     u.size))

    def run(self, t_end, dt_output=None, on_output=None):
        """time_evolution driven from Python (src/hydro_ader.hpp:215-273):
        one blocking dt read per step, dt clamped to output times, and
        on_output(index, solver) at construction and every output time."""
        outputs = dt_output is not None and dt_output > 0
        dt = self.dt()
        t_output = dt_output if outputs else None
        n_out = 0
        if outputs:
            if on_output:
                on_output(n_out, self)
            n_out += 1
        while self.t < t_end:
            self.step()
            self.t += dt
            self.n_step += 1
            dt = self.dt()
            if outputs:
                if self.t >= t_output:
                    t_output = self.t + dt_output
                    if on_output:
                        on_output(n_out, self)
                    n_out += 1
                if self.t + dt > t_output:
                    dt = t_output - self.t
                    self.set_dt(dt)
        self.t_output = t_output
        return dt

    # ---- layout helpers -------------------------------------------------
    def field_array(self, field):
        """field as (V, Nz, Ny, Nx, nz, ny, nx) (cell fields: V = 1)."""
        n = self.p + 1
        Nx, Ny, Nz = self.N
        nz = n if self.ndim == 3 else 1
        a = self.read(field)
        V = self.nvar if field in (FIELD_U_SP, FIELD_W_CV) else 1
        a = a.reshape(Nz, Ny, Nx, V, nz, n, n)
        return np.ascontiguousarray(a.transpose(3, 0, 1, 2, 4, 5, 6))

    def to_reference_slots(self, a):
        """(V, ...) solver slots -> reference slot order (rho, mx, my, mz, E):
        a 2D run gets an all-zero mz slot."""
        if self.ndim == 3:
            return a
        z = np.zeros_like(a[:1])
        return np.concatenate([a[:3], z, a[3:]], axis=0)
