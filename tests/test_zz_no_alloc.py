"""The allocation-free step against the allocating solver.

spdk_hydro_step_noalloc is for callers that cannot allocate device memory
when they step -- a host that owns every device byte through its own pool, a
plugin running inside someone else's stream capture, a real-time loop -- so
it keeps its working storage in a fixed array inside the library. Called
here through the C ABI on caller-owned buffers, it must reproduce
spdk_hydro_step (the allocating entry point) bit for bit -- state, W_cv and
the next dt -- on two calls in a row, for ADER and SSP-RK1/3, 2D and 3D,
in place and on separate input/output buffers, and at the largest problem
its fixed array accepts; after every clean call its status word reads 0.
The file is collected last, so a failure here leaves every other test run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = {
    "ader_2d_p3": ["job/fallback=false", "mesh/nx1=16", "mesh/nx2=8", "mesh/nx3=1",
                   "problem/problem=kelvin_helmholtz"],
    "rk3_2d_p2_gravity": ["job/fallback=false", "mesh/p=2", "mesh/nx1=8", "mesh/nx2=8", "mesh/nx3=1",
                          "time/integrator=rk3", "problem/problem=rti", "hydro/g2=-0.1",
                          "mesh/x2_bc=reflective"],
    "ader_3d_p2": ["job/fallback=false", "mesh/p=2", "mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=4",
                   "problem/problem=spherical_blast"],
    "rk1_2d_p3": ["job/fallback=false", "mesh/nx1=8", "mesh/nx2=12", "mesh/nx3=1", "time/integrator=rk1",
                  "problem/problem=kelvin_helmholtz"],
    # the largest ADER p=3 2D problem the fixed array holds: 2 (p+1) states of
    # 60x68 elements = 16,711,680 bytes of the 16,776,960 available
    "ader_2d_p3_largest": ["job/fallback=false", "mesh/nx1=60", "mesh/nx2=68", "mesh/nx3=1",
                           "problem/problem=kelvin_helmholtz"],
}
# separate input and output buffers, no W_cv output
SEPARATE = {"ader_2d_p3", "rk3_2d_p2_gravity"}


def bind(lib):
    f = lib.spdk_hydro_step_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p] * 6
    return f


def status(lib, stream):
    f = lib.spdk_hydro_noalloc_status
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
    st = ctypes.c_int(-1)
    rc = f(ctypes.byref(st), stream)
    assert rc == 0, lib.spdk_last_error().decode()
    return st.value


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_step_matches_allocating_step(case):
    import torch

    import spd_k_b200 as S
    from spd_k_b200.api import apply_overrides, config_from_params, make_config

    c = config_from_params(apply_overrides({}, CASES[case]))
    ref = S.HydroSolver(c)
    lib = S.load_library()
    step = bind(lib)
    cfg = make_config(c)
    dev = torch.device("cuda:0")
    u = torch.from_numpy(ref.read(S.FIELD_U_SP)).to(dev)   # caller-owned buffers
    separate = case in SEPARATE
    u_out = torch.empty_like(u) if separate else u
    w = None if separate else torch.empty_like(u)
    dt = torch.tensor([ref.dt()], dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        u_before = u.cpu().numpy() if separate else None
        rc = step(ctypes.addressof(cfg), u.data_ptr(), u_out.data_ptr(), None if w is None else w.data_ptr(),
                  dt.data_ptr(), stream.cuda_stream)
        assert rc == 0, lib.spdk_last_error().decode()
        assert status(lib, stream.cuda_stream) == 0, f"device-detected fault in call {call + 1}"
        ref.step()
        torch.cuda.synchronize(dev)
        assert np.array_equal(u_out.cpu().numpy(), ref.read(S.FIELD_U_SP)), f"U_sp differs after call {call + 1}"
        if w is not None:
            assert np.array_equal(w.cpu().numpy(), ref.read(S.FIELD_W_CV)), f"W_cv differs after call {call + 1}"
        assert float(dt.item()) == ref.dt(), f"next dt differs after call {call + 1}"
        if separate:
            assert np.array_equal(u.cpu().numpy(), u_before), f"input buffer changed by call {call + 1}"
            u, u_out = u_out, u   # the next call reads this call's output
    ref.close()


def test_noalloc_rejects_oversized_and_fallback_configs():
    import spd_k_b200 as S
    from spd_k_b200.api import apply_overrides, config_from_params, make_config

    lib = S.load_library()
    step = bind(lib)
    big = make_config(config_from_params(apply_overrides({}, ["job/fallback=false", "mesh/nx1=512",
                                                                "mesh/nx2=512", "mesh/nx3=1"])))
    rc = step(ctypes.addressof(big), 16, 16, None, 16, None)
    assert rc == -1 and b"working storage" in lib.spdk_last_error()
    # one element past the largest accepted problem's working storage
    over = make_config(config_from_params(apply_overrides({}, ["job/fallback=false", "mesh/nx1=64",
                                                                 "mesh/nx2=64", "mesh/nx3=1"])))
    rc = step(ctypes.addressof(over), 16, 16, None, 16, None)
    assert rc == -1 and b"working storage" in lib.spdk_last_error()
    fb = make_config(config_from_params(apply_overrides({}, ["job/fallback=true", "mesh/nx3=1"])))
    rc = step(ctypes.addressof(fb), 16, 16, None, 16, None)
    assert rc == -1 and b"fallback" in lib.spdk_last_error()
    slab = make_config(config_from_params(apply_overrides({}, ["job/fallback=false", "mesh/nx3=1",
                                                                 "mesh/x2_bc=gradfree"])))
    slab.slab_n = slab.N[1] + 4
    slab.slab_lo = 2
    rc = step(ctypes.addressof(slab), 16, 16, None, 16, None)
    assert rc == -1 and b"slab" in lib.spdk_last_error()
