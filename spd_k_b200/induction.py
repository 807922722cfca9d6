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
