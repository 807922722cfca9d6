"""Python binding of the induction solver (include/spdk_induction.h).

The reference builds an Induction_ader for job/system = induction
(src/main.cpp:227-249); InductionSolver is that object on the GPU, driven by
the same athinput parameters (mesh, time, output, fallback, induction/nu).
"""
import ctypes

import numpy as np

from .api import BC, SpdkError, config_from_params, load_library

FIELD_B2_CV, FIELD_TROUBLES, FIELD_BX_FP, FIELD_BY_FP, FIELD_BZ_FP = 0, 1, 2, 3, 4


class InductionConfig(ctypes.Structure):
    _fields_ = [
        ("p", ctypes.c_int), ("N", ctypes.c_int * 3), ("L", ctypes.c_double * 3), ("bc", ctypes.c_int * 3),
        ("integrator", ctypes.c_int), ("rk_order", ctypes.c_int), ("fallback", ctypes.c_int),
        ("cfl", ctypes.c_double), ("nu", ctypes.c_double), ("nad_tolerance", ctypes.c_double),
        ("nad_delta", ctypes.c_int), ("nad_moore", ctypes.c_int), ("sed", ctypes.c_int), ("device", ctypes.c_int),
        ("fallback_apply", ctypes.c_int),
    ]


def induction_config_from_params(params):
    """the hydro run configuration plus induction/nu (src/main.cpp:227-229)"""
    c = config_from_params(params)
    v = params.get("induction", {}).get("nu")
    c["nu"] = 0.0025 if v is None else float(v)
    a = params.get("fallback", {}).get("apply")
    c["fallback_apply"] = a is not None and a.strip().lower() in ("true", "1", "yes", "on")
    return c


def make_induction_config(c, device=0):
    o = InductionConfig()
    o.p = c["p"]
    for d in range(3):
        o.N[d] = c["N"][d]
        o.L[d] = c["L"][d]
        o.bc[d] = BC[c["bc"][d]] if isinstance(c["bc"][d], str) else int(c["bc"][d])
    integ = c.get("integrator", "ader")
    if integ == "ader":
        o.integrator, o.rk_order = 0, 3
    elif integ.startswith("rk") and len(integ) == 3 and integ[2] in "123":
        o.integrator, o.rk_order = 1, int(integ[2])
    else:
        raise ValueError(f"unknown integrator {integ!r} (ader, rk1, rk2, rk3)")
    o.fallback = int(bool(c["fallback"]))
    o.cfl, o.nu = c["cfl"], c["nu"]
    o.nad_tolerance = c["nad_tolerance"]
    o.nad_delta, o.nad_moore, o.sed = int(c["nad_delta"]), int(c["nad_moore"]), int(c["sed"])
    o.device = device
    o.fallback_apply = int(bool(c.get("fallback_apply", False)))
    return o


def _lib():
    L = load_library()
    if not getattr(L, "_induction_types", False):
        vp = ctypes.c_void_p
        L.spdk_induction_create.argtypes = [ctypes.POINTER(InductionConfig), ctypes.POINTER(vp)]
        L.spdk_induction_destroy.argtypes = [vp]
        L.spdk_induction_get_dt.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.spdk_induction_set_dt.argtypes = [vp, ctypes.c_double]
        L.spdk_induction_step.argtypes = [vp]
        L.spdk_induction_evolve.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_longlong),
                                            ctypes.POINTER(ctypes.c_double)]
        L.spdk_induction_field_size.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
        L.spdk_induction_read.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t]
        L._induction_types = True
    return L


def _check(L, rc):
    if rc != 0:
        raise SpdkError(f"spdk error {rc}: {L.spdk_last_error().decode()}")


class InductionSolver:
    """GPU induction solver (the reference's Induction_ader)."""

    def __init__(self, c, device=0):
        L = _lib()
        self.c = c
        self._cfg = make_induction_config(c, device)
        h = ctypes.c_void_p()
        _check(L, L.spdk_induction_create(ctypes.byref(self._cfg), ctypes.byref(h)))
        self.h = h
        self.t = 0.0
        self.n_step = 0

    def close(self):
        if getattr(self, "h", None):
            _lib().spdk_induction_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def dt(self):
        v = ctypes.c_double()
        L = _lib()
        _check(L, L.spdk_induction_get_dt(self.h, ctypes.byref(v)))
        return v.value

    def step(self):
        L = _lib()
        _check(L, L.spdk_induction_step(self.h))

    def evolve(self, t_end, dt_output=None):
        L = _lib()
        steps, t = ctypes.c_longlong(), ctypes.c_double()
        _check(L, L.spdk_induction_evolve(self.h, t_end, dt_output or -1.0, ctypes.byref(steps), ctypes.byref(t)))
        self.n_step += steps.value
        self.t = t.value
        return steps.value

    def run(self, t_end, dt_output=None, on_output=None):
        """time_evolution (src/induction_ader.hpp:222-272) driven from
        Python: on_output(index, solver) at construction and at every output
        time, dt clamped to the output times"""
        L = _lib()
        outputs = dt_output is not None and dt_output > 0
        t_output = dt_output if outputs else None
        n_out = 0
        if outputs:
            if on_output:
                on_output(n_out, self)
            n_out += 1
        dt = self.dt()
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
                    _check(L, L.spdk_induction_set_dt(self.h, dt))

    def read(self, field):
        L = _lib()
        n = ctypes.c_size_t()
        _check(L, L.spdk_induction_field_size(self.h, field, ctypes.byref(n)))
        a = np.empty(n.value, dtype=np.float64)
        _check(L, L.spdk_induction_read(self.h, field, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n.value))
        return a


# ---------------------------------------------------------------------------
# 2D induction solver (include/spdk_induction.h, spdk_induction2d_*)
# ---------------------------------------------------------------------------
FIELD2_BX, FIELD2_BY, FIELD2_B2_CV = 0, 1, 2


class Induction2DConfig(ctypes.Structure):
    _fields_ = [
        ("p", ctypes.c_int), ("N", ctypes.c_int * 2), ("L", ctypes.c_double * 2), ("integrator", ctypes.c_int),
        ("rk_order", ctypes.c_int), ("cfl", ctypes.c_double), ("velocity", ctypes.c_double * 2),
        ("loop_center", ctypes.c_double * 2), ("loop_A0", ctypes.c_double), ("loop_R", ctypes.c_double),
        ("precision", ctypes.c_int), ("device", ctypes.c_int),
    ]


class Induction2DInfo(ctypes.Structure):
    _fields_ = [("p", ctypes.c_int), ("N", ctypes.c_int * 2), ("n_elements", ctypes.c_longlong),
                ("n_face_values", ctypes.c_longlong), ("n_time_slices", ctypes.c_int),
                ("launches_per_step", ctypes.c_int)]


def field_loop_config(N=512, p=4, L=2.0, velocity=(2.0, 1.0), center=(1.0, 1.0), A0=1e-3, R=0.3, cfl=0.8,
                      integrator="ader", precision="fp64"):
    """the 2D field-loop advection: [0, L]^2 periodic (the box [-1, 1]^2 shifted
    by 1 when L = 2 and the centre is (1, 1)), A_z = A0 (R - r) inside r <= R"""
    return dict(p=p, N=[N, N], L=[L, L], velocity=list(velocity), center=list(center), A0=A0, R=R, cfl=cfl,
                integrator=integrator, precision=precision)


def make_induction2d_config(c, device=0):
    o = Induction2DConfig()
    o.p = c["p"]
    for d in range(2):
        o.N[d] = c["N"][d]
        o.L[d] = c["L"][d]
        o.velocity[d] = c["velocity"][d]
        o.loop_center[d] = c["center"][d]
    integ = c.get("integrator", "ader")
    if integ == "ader":
        o.integrator, o.rk_order = 0, 3
    elif integ.startswith("rk") and len(integ) == 3 and integ[2] in "123":
        o.integrator, o.rk_order = 1, int(integ[2])
    else:
        raise ValueError(f"unknown integrator {integ!r} (ader, rk1, rk2, rk3)")
    o.cfl = c["cfl"]
    o.loop_A0, o.loop_R = c["A0"], c["R"]
    prec = c.get("precision", "fp64")
    if prec not in ("fp64", "fp32"):
        raise ValueError(f"unknown precision {prec!r}")
    o.precision = 0 if prec == "fp64" else 1
    o.device = device
    return o


def _lib2():
    L = load_library()
    if not getattr(L, "_induction2d_types", False):
        vp = ctypes.c_void_p
        L.spdk_induction2d_create.argtypes = [ctypes.POINTER(Induction2DConfig), ctypes.POINTER(vp)]
        L.spdk_induction2d_destroy.argtypes = [vp]
        L.spdk_induction2d_get_info.argtypes = [vp, ctypes.POINTER(Induction2DInfo)]
        L.spdk_induction2d_get_dt.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.spdk_induction2d_set_dt.argtypes = [vp, ctypes.c_double]
        L.spdk_induction2d_step.argtypes = [vp]
        L.spdk_induction2d_sync.argtypes = [vp]
        L.spdk_induction2d_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.spdk_induction2d_evolve.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_longlong),
                                              ctypes.POINTER(ctypes.c_double)]
        L.spdk_induction2d_read.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t]
        L._induction2d_types = True
    return L


class Induction2D:
    """GPU 2D induction solver: field-loop advection with a uniform in-plane
    velocity (a quasi-2D run of the reference's Induction_ader)."""

    def __init__(self, c, device=0):
        L = _lib2()
        self.c = c
        self._cfg = make_induction2d_config(c, device)
        h = ctypes.c_void_p()
        _check(L, L.spdk_induction2d_create(ctypes.byref(self._cfg), ctypes.byref(h)))
        self.h = h
        info = Induction2DInfo()
        _check(L, L.spdk_induction2d_get_info(self.h, ctypes.byref(info)))
        self.info = info
        self.p, self.N = c["p"], list(c["N"])
        self.t = 0.0
        self.n_step = 0

    def close(self):
        if getattr(self, "h", None):
            _lib2().spdk_induction2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def dt(self):
        v = ctypes.c_double()
        L = _lib2()
        _check(L, L.spdk_induction2d_get_dt(self.h, ctypes.byref(v)))
        return v.value

    def step(self):
        L = _lib2()
        _check(L, L.spdk_induction2d_step(self.h))

    def sync(self):
        L = _lib2()
        _check(L, L.spdk_induction2d_sync(self.h))

    def stream(self):
        """the cudaStream_t handle the solver launches on"""
        L = _lib2()
        sp = ctypes.c_void_p()
        _check(L, L.spdk_induction2d_get_stream(self.h, ctypes.byref(sp)))
        return sp.value

    def evolve(self, t_end, dt_output=None):
        L = _lib2()
        steps, t = ctypes.c_longlong(), ctypes.c_double()
        _check(L, L.spdk_induction2d_evolve(self.h, t_end, dt_output or -1.0, ctypes.byref(steps), ctypes.byref(t)))
        self.n_step += steps.value
        self.t = t.value
        return steps.value

    def read(self, field):
        n, nf, E = self.p + 1, self.p + 2, self.info.n_elements
        count = E * n * nf if field in (FIELD2_BX, FIELD2_BY) else 4 * E * n * n
        a = np.empty(count, dtype=np.float64)
        L = _lib2()
        _check(L, L.spdk_induction2d_read(self.h, field, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), count))
        return a

    def b2_cv(self):
        """(4, Ny, Nx, n, n): Bx, By, Bz, |B|^2 sub-cell averages"""
        n = self.p + 1
        a = self.read(FIELD2_B2_CV).reshape(self.N[1], self.N[0], 4, n, n)
        return np.ascontiguousarray(a.transpose(2, 0, 1, 3, 4))
