"""Python binding of the prototype-level C ABI (include/spdk_proto.h).

Each function takes device tensors in the reference's own layout (torch
float64 CUDA tensors: SD arrays with 8 dims (t, var, k, j, i, kk, jj, ii),
FV arrays with 4 dims (var, K, J, I), matrices 2 dims, vectors 1 dim) and
enqueues the matching libspdk_cuda.so export on the current torch stream.
Names and argument order follow src/prototypes.hpp; the reference's global
cfg is the ProtoCfg argument.
"""
import ctypes

from .api import SpdkError, load_library


class SD(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("ext", ctypes.c_int * 8)]


class FV(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("ext", ctypes.c_int * 4)]


class Mat(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("rows", ctypes.c_int), ("cols", ctypes.c_int)]


class Vec(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("n", ctypes.c_int)]


class ProtoCfg(ctypes.Structure):
    _fields_ = [
        ("p", ctypes.c_int), ("active", ctypes.c_int * 3), ("gamma", ctypes.c_double),
        ("cfl", ctypes.c_double), ("g", ctypes.c_double * 3), ("nad_tolerance", ctypes.c_double),
        ("nad_delta", ctypes.c_int), ("nad_moore", ctypes.c_int), ("sed", ctypes.c_int),
    ]


PERIODIC, GRADFREE, REFLECTIVE = 0, 1, 2
# normal / transverse momentum slots of each direction (src/hydro_ader.hpp:282-287)
V123 = ((1, 2, 3), (2, 3, 1), (3, 1, 2))


def _check_tensor(t, ndim):
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise SpdkError("expected a contiguous float64 CUDA tensor")
    if t.dim() != ndim:
        raise SpdkError(f"expected {ndim} dims, got {t.dim()}")


def sd(t):
    _check_tensor(t, 8)
    return SD(t.data_ptr(), (ctypes.c_int * 8)(*t.shape))


def fv(t):
    _check_tensor(t, 4)
    return FV(t.data_ptr(), (ctypes.c_int * 4)(*t.shape))


def mat(t):
    _check_tensor(t, 2)
    return Mat(t.data_ptr(), t.shape[0], t.shape[1])


def vec(t):
    _check_tensor(t, 1)
    return Vec(t.data_ptr(), t.shape[0])


def proto_cfg(c):
    """ProtoCfg from a solver configuration dict (spd_k_b200.config_from_params)."""
    o = ProtoCfg()
    o.p = c["p"]
    N = c["N"]
    for d in range(3):
        o.active[d] = 1 if N[d] > 1 else 0
        o.g[d] = c["g"][d]
    o.gamma, o.cfl = c["gamma"], c["cfl"]
    o.nad_tolerance = c["nad_tolerance"]
    o.nad_delta, o.nad_moore, o.sed = int(c["nad_delta"]), int(c["nad_moore"]), int(c["sed"])
    return o


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _call(name, *args):
    L = load_library()
    rc = getattr(L, name)(*args, _stream())
    if rc != 0:
        raise SpdkError(f"{name}: {L.spdk_last_error().decode()} (status {rc})")


def _r(x):
    return ctypes.byref(x)


def _opt(make, t):
    return ctypes.byref(make(t)) if t is not None else None


D = ctypes.c_double
I = ctypes.c_int


def transform_a_to_b_1d(a, b, m, dim):
    _call("spdk_transform_a_to_b_1d", _r(sd(a)), _r(sd(b)), _r(mat(m)), I(dim))


def transform_a_to_b_1d_slice(a, b, m, dim, t):
    _call("spdk_transform_a_to_b_1d_slice", _r(sd(a)), _r(sd(b)), _r(mat(m)), I(dim), I(t))


def transform_a_to_b(a, b, tmp, m, cfg):
    _call("spdk_transform_a_to_b", _r(sd(a)), _r(sd(b)), _r(sd(tmp)), _r(mat(m)), _r(cfg))


def combine_solution(u, u0, a):
    _call("spdk_combine_solution", _r(sd(u)), _r(sd(u0)), D(a))


def update_prediction(u, ua, fx, fy, fz, dfp_to_sp, invader, w, dt, dx, dy, dz, cfg):
    _call("spdk_update_prediction", _r(sd(u)), _r(sd(ua)), _r(sd(fx)), _r(sd(fy)), _r(sd(fz)), _r(mat(dfp_to_sp)),
          _r(mat(invader)), _r(vec(w)), D(dt), D(dx), D(dy), D(dz), _r(cfg))


def update_solution(u, ua, fx, fy, fz, dfp_to_sp, w, dt, dx, dy, dz, cfg):
    _call("spdk_update_solution", _r(sd(u)), _r(sd(ua)), _r(sd(fx)), _r(sd(fy)), _r(sd(fz)), _r(mat(dfp_to_sp)),
          _r(vec(w)), D(dt), D(dx), D(dy), D(dz), _r(cfg))


def compute_primitives(u, w, cfg):
    if u.dim() == 8:
        _call("spdk_compute_primitives", _r(sd(u)), _r(sd(w)), _r(cfg))
    else:
        _call("spdk_fv_compute_primitives", _r(fv(u)), _r(fv(w)), _r(cfg))


def compute_conservatives(w, u, cfg):
    if w.dim() == 8:
        _call("spdk_compute_conservatives", _r(sd(w)), _r(sd(u)), _r(cfg))
    else:
        _call("spdk_fv_compute_conservatives", _r(fv(w)), _r(fv(u)), _r(cfg))


def compute_fluxes(u, f, v1, v2, v3, cfg):
    _call("spdk_compute_fluxes", _r(sd(u)), _r(sd(f)), I(v1), I(v2), I(v3), _r(cfg))


def compute_dt(w, dx, dy, dz, nu, out, cfg):
    """min over active points into the 1-element device tensor `out`"""
    import torch
    if not (out.is_cuda and out.dtype == torch.float64 and out.numel() >= 1):
        raise SpdkError("out must be a float64 CUDA tensor")
    _call("spdk_compute_dt", _r(sd(w)), D(dx), D(dy), D(dz), D(nu), ctypes.c_void_p(out.data_ptr()), _r(cfg))


def sd_riemann_solver(u, f, v1, v2, v3, dim, viscous, cfg):
    _call("spdk_sd_riemann_solver", _r(sd(u)), _r(sd(f)), I(v1), I(v2), I(v3), I(dim), I(int(viscous)), _r(cfg))


def sd_rusanov_solver(u, f, dim):
    _call("spdk_sd_rusanov_solver", _r(sd(u)), _r(sd(f)), I(dim))


def compute_gradient(u, du, h, dfp_to_sp, dim, cfg):
    _call("spdk_compute_gradient", _r(sd(u)), _r(sd(du)), D(h), _r(mat(dfp_to_sp)), I(dim), _r(cfg))


def compute_viscous_flux(u, du1, v1, du2, v2, du3, v3, sp_to_fp, nu, beta, dim, cfg):
    _call("spdk_compute_viscous_flux", _r(sd(u)), _r(sd(du1)), I(v1), _r(sd(du2)), I(v2), _r(sd(du3)), I(v3),
          _r(mat(sp_to_fp)), D(nu), D(beta), I(dim), _r(cfg))


def boundaries_sd(u, dim, bc_type):
    _call("spdk_boundaries_sd", _r(sd(u)), I(dim), I(bc_type))


def boundaries_fv(u, dim, bc_type, alignment=0, a_dim=0):
    _call("spdk_boundaries_fv", _r(fv(u)), I(dim), I(bc_type), I(alignment), I(a_dim))


def face_integral(f_fp, f, tmp, sp_to_cv, dim, t, cfg):
    _call("spdk_face_integral", _r(sd(f_fp)), _r(fv(f)), _opt(sd, tmp), _r(mat(sp_to_cv)), I(dim), I(t), _r(cfg))


def fv_update_solution(u_old, u_new, u_cv, fx, xf, fy, yf, fz, zf, w, t, dt, update, cfg):
    _call("spdk_fv_update_solution", _r(fv(u_old)), _r(fv(u_new)), _r(sd(u_cv)), _opt(fv, fx), _opt(vec, xf),
          _opt(fv, fy), _opt(vec, yf), _opt(fv, fz), _opt(vec, zf), _r(vec(w)), I(t), D(dt), I(int(update)), _r(cfg))


def detect_troubles(w_new, w_old, troubles, ax, ay, az, xc, xf, yc, yf, zc, zf, pad, limit_mask, cfg):
    _call("spdk_detect_troubles", _r(fv(w_new)), _r(fv(w_old)), _r(fv(troubles)), _opt(fv, ax), _opt(fv, ay),
          _opt(fv, az), _opt(vec, xc), _opt(vec, xf), _opt(vec, yc), _opt(vec, yf), _opt(vec, zc), _opt(vec, zf),
          I(int(pad)), I(limit_mask), _r(cfg))


def apply_blending(troubles, theta, cfg):
    _call("spdk_apply_blending", _r(fv(troubles)), _r(fv(theta)), _r(cfg))


def blending_ring(theta_in, theta_out, cfg):
    _call("spdk_blending_ring", _r(fv(theta_in)), _r(fv(theta_out)), _r(cfg))


def theta_from_troubles(troubles, theta):
    _call("spdk_theta_from_troubles", _r(fv(troubles)), _r(fv(theta)))


def fallback_fluxes(w_old, theta, xc, xf, fx, yc, yf, fy, zc, zf, fz, ader, w, dt, cfg):
    _call("spdk_fallback_fluxes", _r(fv(w_old)), _r(fv(theta)), _opt(vec, xc), _opt(vec, xf), _opt(fv, fx),
          _opt(vec, yc), _opt(vec, yf), _opt(fv, fy), _opt(vec, zc), _opt(vec, zf), _opt(fv, fz), I(ader),
          _r(vec(w)), D(dt), _r(cfg))
