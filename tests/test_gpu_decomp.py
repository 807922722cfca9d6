"""Slab domain decomposition on the GPU: 2 and 3 slab solvers (one process,
one GPU) stepped with the owned-row dt minimum and a halo exchange after
every step equal the undecomposed solver bit for bit -- owned rows of U_sp
and the agreed dt after every step -- on the benchmark geometry with the
fallback, in both arithmetic forms, in 3D, and with the viscous terms under
SSP-RK3."""
import numpy as np
import pytest

from helpers import gpu_config, same_bits

pytestmark = pytest.mark.gpu

BLAST = ["job/fallback=true", "mesh/nx1=64", "mesh/nx2=64", "mesh/nx3=1", "mesh/x1_bc=gradfree",
         "mesh/x2_bc=gradfree", "problem/problem=spherical_blast", "problem/p0=1273.2395447351628",
         "problem/p1=1e-5", "problem/radius=0.01"]
CASES = {
    "blast64_fp64_2slabs": (BLAST, "fp64", 2, 8),
    "blast64_fp64_3slabs": (BLAST, "fp64", 3, 8),
    "blast64_fp32_2slabs": (BLAST, "fp32", 2, 8),
    "blast3d_p2_2slabs": (["job/fallback=true", "mesh/p=2", "mesh/nx1=6", "mesh/nx2=6", "mesh/nx3=24",
                           "mesh/x3_bc=gradfree", "problem/problem=spherical_blast"], "fp64", 2, 5),
    "viscous_rk3_reflective_2slabs": (["job/fallback=false", "mesh/p=2", "mesh/nx1=8", "mesh/nx2=20", "mesh/nx3=1",
                                       "mesh/x2_bc=reflective", "time/integrator=rk3", "hydro/nu=0.002",
                                       "problem/problem=kelvin_helmholtz"], "fp64", 2, 6),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_decomposed_run_equals_the_whole_domain(case):
    import spd_k_b200 as S
    from spd_k_b200.decomp import SlabGroup
    ov, prec, ranks, steps = CASES[case]
    c = dict(gpu_config(ov), precision=prec)
    whole = S.HydroSolver(c)
    grp = SlabGroup(c, ranks)
    assert grp.dt() == whole.dt()
    for k in range(steps):
        whole.step()
        dt = grp.step()
        assert dt == whole.dt(), f"dt after step {k + 1}"
        assert same_bits(grp.owned(S.FIELD_U_SP), whole.field_array(S.FIELD_U_SP)), f"U_sp after step {k + 1}"
    if c["fallback"]:
        assert whole.read(S.FIELD_TROUBLES).sum() > 0     # the limiter was active
    grp.close()
    whole.close()


def test_too_narrow_a_halo_is_not_exact():
    """the halo must cover the step's dependency radius: one row per side is
    not enough for the limited blast, and the owned rows drift"""
    import spd_k_b200 as S
    from spd_k_b200.decomp import SlabGroup
    c = dict(gpu_config(BLAST), precision="fp64")
    whole = S.HydroSolver(c)
    grp = SlabGroup(c, 2, halo=1)
    for _ in range(8):
        whole.step()
        grp.step()
    assert not same_bits(grp.owned(S.FIELD_U_SP), whole.field_array(S.FIELD_U_SP))
    grp.close()
    whole.close()
