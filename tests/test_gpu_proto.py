"""The prototype-level C ABI (include/spdk_proto.h) against the oracle.

A host drives the exported functions in the order the reference's
Hydro_ader does (src/hydro_ader.hpp:215-586), on device arrays in the
reference's own layout (ghost elements and FV ghost frames included), and
every array is compared bit for bit (IEEE equality, NaN = NaN) with the
oracle's after the same sub-step: the flux pass, the Picard update, and
whole ADER / SSP-RK steps with and without the fallback, from seeded states
that trip the trouble detector.
"""
import zlib

import numpy as np
import pytest

from helpers import gpu_config, oracle_config, same_bits

pytestmark = pytest.mark.gpu

SD_NAMES = ["U_sp", "W_sp", "W_cv", "U_cv", "U_ader_sp", "U_ader_fp_x", "U_ader_fp_y", "U_ader_fp_z",
            "F_ader_fp_x", "F_ader_fp_y", "F_ader_fp_z"]
FV_NAMES = ["troubles", "theta", "U_new", "U_old", "W_new", "W_old", "F_x", "F_y", "F_z",
            "alpha_x", "alpha_y", "alpha_z"]
VEC_NAMES = ["wt", "fv_faces_x", "fv_faces_y", "fv_faces_z", "fv_centers_x", "fv_centers_y", "fv_centers_z"]
MAT_NAMES = ["sp_to_fp", "dfp_to_sp", "sp_to_cv", "cv_to_sp", "invader"]


class Mirror:
    """device copies of every oracle array, in the oracle's (reference) layout"""

    def __init__(self, o, c):
        import torch
        self.o, self.c = o, c
        self.act = [1 if n > 1 else 0 for n in c["N"]]
        self.a = {}
        for name in SD_NAMES:
            self.a[name] = torch.from_numpy(o.array(name)).cuda()
        for name in FV_NAMES:
            self.a[name] = torch.from_numpy(o.array(name).reshape(o.array(name).shape[:4]).copy()).cuda()
        for name in VEC_NAMES:
            self.a[name] = torch.from_numpy(o.array(name).reshape(-1).copy()).cuda()
        for name in MAT_NAMES:
            if c["integrator"] != "ader" and name == "invader":
                continue
            self.a[name] = torch.from_numpy(o.array(name).reshape(o.array(name).shape[:2]).copy()).cuda()
        if c.get("nu", 0.0) > 0:
            for x in "xyz":
                self.a["dU" + x + "_sp"] = torch.from_numpy(o.array("dU" + x + "_sp")).cuda()
        self.a["T_sweep"] = torch.zeros_like(self.a["U_sp"])
        self.a["U0_sp"] = torch.zeros_like(self.a["U_sp"])
        self.a["theta_tmp"] = torch.zeros_like(self.a["theta"])
        for x in "xyz":
            self.a["T_fp_" + x] = torch.zeros_like(self.a["F_ader_fp_" + x][:1]).contiguous()
        self.dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda")

    def __getitem__(self, k):
        return self.a[k]

    def same(self, name):
        g = self.a[name].cpu().numpy()
        r = self.o.array(name).reshape(g.shape)
        return same_bits(g, r)


def dirs(M):
    return [d for d in range(3) if M.act[d]]


def xyz(M, prefix):
    return [M[prefix + "xyz"[d]] if M.act[d] else None for d in range(3)]


def solve_fluxes(M, P, cfg):
    """src/hydro_ader.hpp:278-289, with the viscous terms of :284-288 and
    :383-405 when hydro/nu > 0"""
    nu = M.c.get("nu", 0.0)
    fp = ["U_ader_fp_" + x for x in "xyz"]
    for d in dirs(M):
        P.transform_a_to_b_1d(M["U_ader_sp"], M[fp[d]], M["sp_to_fp"], d)
    for d in dirs(M):
        P.compute_fluxes(M[fp[d]], M["F_ader_fp_" + "xyz"[d]], *P.V123[d], cfg)
    for d in dirs(M):
        P.boundaries_sd(M[fp[d]], d, BC[M.c["bc"][d]])
    for d in dirs(M):
        P.sd_riemann_solver(M[fp[d]], M["F_ader_fp_" + "xyz"[d]], *P.V123[d], d, int(nu > 0), cfg)
    if nu > 0:
        dU = [M["dU" + x + "_sp"] for x in "xyz"]
        for d in dirs(M):
            P.compute_gradient(M[fp[d]], dU[d], h(M)[d], M["dfp_to_sp"], d, cfg)
        for d in dirs(M):
            v1, v2, v3 = P.V123[d]
            P.compute_viscous_flux(M[fp[d]], dU[d], v1, dU[(d + 1) % 3], v2, dU[(d + 2) % 3], v3, M["sp_to_fp"], nu,
                                   M.c["beta"], d, cfg)
        for d in dirs(M):
            P.boundaries_sd(M[fp[d]], d, BC[M.c["bc"][d]])
        for d in dirs(M):
            P.sd_rusanov_solver(M[fp[d]], M["F_ader_fp_" + "xyz"[d]], d)


def flux_args(M):
    return [M["F_ader_fp_" + x] for x in "xyz"]


def h(M):
    return [M.c["L"][d] / M.c["N"][d] for d in range(3)]


def copy_ader(M):
    nt = M["U_ader_sp"].shape[0]
    for t in range(nt):
        M["U_ader_sp"][t].copy_(M["U_sp"][0])


BC = {"periodic": 0, "gradfree": 1, "reflective": 2}


def fv_boundaries(M, P, name):
    for d in dirs(M):
        P.boundaries_fv(M[name], d, BC[M.c["bc"][d]])


def fv_update(M, P, cfg, dt):
    """src/hydro_ader.hpp:500-575"""
    mask = (1 << 0) | (1 << 4)
    P.transform_a_to_b(M["U_sp"], M["U_cv"], M["T_sweep"], M["sp_to_cv"], cfg)
    F = xyz(M, "F_")
    Xf = xyz(M, "fv_faces_")
    Xc = xyz(M, "fv_centers_")
    A = xyz(M, "alpha_")
    nt = M["F_ader_fp_x"].shape[0]
    for t in range(nt):
        for d in dirs(M):
            x = "xyz"[d]
            both = all(M.act[e] for e in range(3) if e != d)
            P.face_integral(M["F_ader_fp_" + x], M["F_" + x], M["T_fp_" + x] if both else None, M["sp_to_cv"], d, t,
                            cfg)
        P.fv_update_solution(M["U_old"], M["U_new"], M["U_cv"], F[0], Xf[0], F[1], Xf[1], F[2], Xf[2], M["wt"], t, dt,
                             0, cfg)
        fv_boundaries(M, P, "U_old")
        fv_boundaries(M, P, "U_new")
        P.compute_primitives(M["U_new"], M["W_new"], cfg)
        P.compute_primitives(M["U_old"], M["W_old"], cfg)
        P.detect_troubles(M["W_new"], M["W_old"], M["troubles"], A[0], A[1], A[2], Xc[0], Xf[0], Xc[1], Xf[1], Xc[2],
                          Xf[2], 1, mask, cfg)
        fv_boundaries(M, P, "troubles")
        if M.c["blending"]:
            P.apply_blending(M["troubles"], M["theta_tmp"], cfg)
            P.blending_ring(M["theta_tmp"], M["theta"], cfg)
        else:
            P.theta_from_troubles(M["troubles"], M["theta"])
        fv_boundaries(M, P, "theta")
        P.fallback_fluxes(M["W_old"], M["theta"], Xc[0], Xf[0], F[0], Xc[1], Xf[1], F[1], Xc[2], Xf[2], F[2], t,
                          M["wt"], dt, cfg)
        P.fv_update_solution(M["U_old"], M["U_new"], M["U_cv"], F[0], Xf[0], F[1], Xf[1], F[2], Xf[2], M["wt"], t, dt,
                             1, cfg)
    P.transform_a_to_b(M["U_cv"], M["U_sp"], M["T_sweep"], M["cv_to_sp"], cfg)


def step(M, P, cfg, dt):
    """src/hydro_ader.hpp:234-325 (ADER_step / RK_step + primitives to W_cv)"""
    dx, dy, dz = h(M)
    c = M.c
    if c["integrator"] == "ader":
        copy_ader(M)
        nt = M["U_ader_sp"].shape[0]
        for a in range(nt):
            solve_fluxes(M, P, cfg)
            if a < nt - 1:
                P.update_prediction(M["U_sp"], M["U_ader_sp"], *flux_args(M), M["dfp_to_sp"], M["invader"], M["wt"],
                                    dt, dx, dy, dz, cfg)
        if c["fallback"]:
            fv_update(M, P, cfg, dt)
        else:
            P.update_solution(M["U_sp"], M["U_ader_sp"], *flux_args(M), M["dfp_to_sp"], M["wt"], dt, dx, dy, dz, cfg)
    else:
        order = int(c["integrator"][2])
        rk_a = {1: [0.0], 2: [0.0, 0.5], 3: [0.0, 0.75, 1.0 / 3.0]}[order]
        M["U0_sp"].copy_(M["U_sp"])
        for st in range(order):
            copy_ader(M)
            solve_fluxes(M, P, cfg)
            if c["fallback"]:
                fv_update(M, P, cfg, dt)
            else:
                P.update_solution(M["U_sp"], M["U_ader_sp"], *flux_args(M), M["dfp_to_sp"], M["wt"], dt, dx, dy, dz,
                                  cfg)
            if rk_a[st] > 0:
                P.combine_solution(M["U_sp"], M["U0_sp"], rk_a[st])
    P.compute_primitives(M["U_sp"], M["W_sp"], cfg)
    P.transform_a_to_b(M["W_sp"], M["W_cv"], M["T_sweep"], M["sp_to_cv"], cfg)
    P.compute_dt(M["W_cv"], dx, dy, dz, c.get("nu", 0.0), M.dt_dev, cfg)


CASES = {
    "2d_p3_ader_fallback": ["job/fallback=true", "mesh/nx1=6", "mesh/nx2=5", "mesh/nx3=1"],
    "2d_p2_rk3_fallback_reflective": ["job/fallback=true", "mesh/p=2", "mesh/nx1=4", "mesh/nx2=6", "mesh/nx3=1",
                                      "time/integrator=rk3", "mesh/x1_bc=reflective", "mesh/x2_bc=gradfree"],
    "2d_p4_ader_gravity_delta_noblend": ["job/fallback=true", "mesh/p=4", "mesh/nx1=4", "mesh/nx2=4", "mesh/nx3=1",
                                         "hydro/g2=-0.5", "fallback/NAD=delta", "fallback/blending=false"],
    "2d_p3_ader_nofallback": ["job/fallback=false", "mesh/nx1=4", "mesh/nx2=6", "mesh/nx3=1", "hydro/g1=0.2"],
    "3d_p2_ader_fallback": ["job/fallback=true", "mesh/p=2", "mesh/nx1=3", "mesh/nx2=3", "mesh/nx3=2",
                            "mesh/x3_bc=reflective"],
    "3d_p3_rk2_gravity": ["job/fallback=false", "mesh/nx1=2", "mesh/nx2=3", "mesh/nx3=2", "time/integrator=rk2",
                          "hydro/g3=0.3"],
    # viscous terms (hydro/nu > 0): interface states, gradients, viscous
    # fluxes, interface sums and the diffusion dt limit
    "2d_p3_ader_viscous_fallback": ["job/fallback=true", "mesh/nx1=5", "mesh/nx2=4", "mesh/nx3=1", "hydro/nu=0.02"],
    "2d_p2_rk3_viscous_reflective": ["job/fallback=false", "mesh/p=2", "mesh/nx1=4", "mesh/nx2=5", "mesh/nx3=1",
                                     "time/integrator=rk3", "mesh/x2_bc=reflective", "mesh/x1_bc=gradfree",
                                     "hydro/nu=0.05", "hydro/beta=0.01"],
    "3d_p2_ader_viscous": ["job/fallback=false", "mesh/p=2", "mesh/nx1=3", "mesh/nx2=2", "mesh/nx3=3",
                           "mesh/x3_bc=reflective", "hydro/nu=0.01"],
}


def random_oracle(ov, seed):
    """oracle with a seeded random state that trips the detector (the same
    construction as the fused path's parity tests)"""
    from oracle import oracle as O
    from test_gpu_parity import load_oracle_state, random_state
    cg, co = gpu_config(ov), oracle_config(ov)
    _, ref5, D = random_state(cg, seed)
    o = O.Oracle(co)
    load_oracle_state(o, ref5, D)
    return o, co


@pytest.mark.parametrize("case", sorted(CASES))
def test_prototype_steps_match_oracle(case):
    import torch
    import spd_k_b200.proto as P
    o, c = random_oracle(CASES[case], zlib.crc32(case.encode()))
    M = Mirror(o, c)
    cfg = P.proto_cfg(c)
    dt = o.compute_dt()
    for n in range(2):
        step(M, P, cfg, dt)
        o.step(dt)
        torch.cuda.synchronize()
        for name in ("U_sp", "W_cv", "W_sp"):
            assert M.same(name), (case, n, name)
        if c["fallback"]:
            for name in ("troubles", "theta", "U_new", "W_old", "F_x", "F_y"):
                assert M.same(name), (case, n, name)
        dt_o = o.compute_dt()
        assert M.dt_dev.item() == dt_o, (case, n)
        dt = dt_o
    if c["fallback"]:
        assert float(o.array("troubles")[5].sum()) > 0


def test_flux_pass_and_prediction_match_oracle():
    """one flux pass (transform to flux points, fluxes, ghost interface fill,
    LLF) and one Picard update, array by array"""
    import torch
    import spd_k_b200.proto as P
    o, c = random_oracle(["job/fallback=true", "mesh/nx1=5", "mesh/nx2=4", "mesh/nx3=1", "hydro/g1=0.3",
                          "mesh/x2_bc=reflective"], 5)
    M = Mirror(o, c)
    cfg = P.proto_cfg(c)
    dt = o.compute_dt()
    o.call("copy_ader")
    o.call("solve_fluxes")
    copy_ader(M)
    solve_fluxes(M, P, cfg)
    torch.cuda.synchronize()
    for name in ("U_ader_sp", "U_ader_fp_x", "U_ader_fp_y", "F_ader_fp_x", "F_ader_fp_y"):
        assert M.same(name), name
    o.call("update_prediction", dt)
    P.update_prediction(M["U_sp"], M["U_ader_sp"], *flux_args(M), M["dfp_to_sp"], M["invader"], M["wt"], dt,
                        *h(M), cfg)
    torch.cuda.synchronize()
    assert M.same("U_ader_sp")


def test_viscous_flux_pass_matches_oracle():
    """one flux pass with hydro/nu > 0: after the interface states, the
    gradients at the solution points, the viscous fluxes (with their ghost
    fill) and the interface sums, every array equals the oracle's"""
    import torch
    import spd_k_b200.proto as P
    o, c = random_oracle(["job/fallback=false", "mesh/nx1=4", "mesh/nx2=5", "mesh/nx3=1", "hydro/nu=0.03",
                          "mesh/x1_bc=reflective", "mesh/x2_bc=gradfree"], 11)
    M = Mirror(o, c)
    cfg = P.proto_cfg(c)
    o.call("copy_ader")
    o.call("solve_fluxes")
    copy_ader(M)
    solve_fluxes(M, P, cfg)
    torch.cuda.synchronize()
    for name in ("dUx_sp", "dUy_sp", "U_ader_fp_x", "U_ader_fp_y", "F_ader_fp_x", "F_ader_fp_y"):
        assert M.same(name), name
    assert float(np.abs(o.array("dUx_sp")).max()) > 0


def test_bad_arguments_are_rejected():
    import torch
    import spd_k_b200.proto as P
    from spd_k_b200.api import SpdkError
    a = torch.zeros((1, 5, 3, 3, 1, 2, 2), dtype=torch.float64, device="cuda")  # 7 dims
    with pytest.raises(SpdkError):
        P.boundaries_sd(a, 0, 0)
    u = torch.zeros((1, 5, 1, 4, 4, 1, 3, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(SpdkError):
        P.boundaries_sd(u, 0, 7)          # unknown boundary type
    f = torch.zeros((5, 1, 8, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(SpdkError):
        P.boundaries_fv(f, 0, 0, alignment=1, a_dim=0)
    cfg = P.ProtoCfg()
    with pytest.raises(SpdkError):
        P.compute_fluxes(u, u, 1, 1, 3, cfg)
