"""spdk_hydro_evolve (time_evolution, src/hydro_ader.hpp:215-273) runs its
loop on the device: the step's dt, t, the clamping of dt to output times
and the stop test are evaluated by the step's last kernel, and the host
launches captured steps in batches. It must take exactly the steps of the
host loop (one blocking dt read per step, the reference's structure) and
leave the same state, next dt and time, bit for bit -- with and without
output clamping, in both arithmetic forms, with the learned indicator and
with SSP-RK -- and stepping on afterwards must continue identically."""
import numpy as np
import pytest

from helpers import gpu_config, same_bits

pytestmark = pytest.mark.gpu

BLAST = ["job/fallback=true", "mesh/nx1=32", "mesh/nx2=32", "mesh/nx3=1", "mesh/x1_bc=gradfree",
         "mesh/x2_bc=gradfree", "problem/problem=spherical_blast"]
CASES = {
    "blast_fp64": (BLAST, "fp64", False, 0.004, None),
    "blast_fp64_outputs": (BLAST, "fp64", False, 0.004, 0.0007),
    "blast_fp32_learned_outputs": (BLAST, "fp32", True, 0.004, 0.001),
    "sine_rk3_fp64": (["job/fallback=false", "mesh/nx1=8", "mesh/nx2=8", "mesh/nx3=1", "time/integrator=rk3"],
                      "fp64", False, 0.05, 0.02),
}


def make(ov, prec, learned):
    import os
    import spd_k_b200 as S
    from spd_k_b200.learned import Indicator, set_indicator
    g = S.HydroSolver(dict(gpu_config(ov), precision=prec))
    if learned:
        # the solver borrows the network: keep it alive as long as the solver
        g.indicator = Indicator.load(os.path.join(os.path.dirname(S.__file__), "data", "indicator_2d_p3.npz"))
        set_indicator(g, g.indicator)
    return g


@pytest.mark.parametrize("case", sorted(CASES))
def test_device_loop_equals_host_loop(case):
    import spd_k_b200 as S
    ov, prec, learned, t_end, dt_out = CASES[case]
    host, dev = make(ov, prec, learned), make(ov, prec, learned)
    host.run(t_end, dt_out)                 # Python loop: step + blocking dt per step
    n = dev.evolve(t_end, dt_out)           # spdk_hydro_evolve
    assert n == host.n_step and n > 0
    assert dev.t == host.t
    assert dev.dt() == host.dt()
    assert same_bits(dev.field_array(S.FIELD_U_SP), host.field_array(S.FIELD_U_SP))
    assert same_bits(dev.field_array(S.FIELD_W_CV), host.field_array(S.FIELD_W_CV))
    for _ in range(3):                      # the gate is open again afterwards
        host.step()
        dev.step()
    assert dev.dt() == host.dt()
    assert same_bits(dev.field_array(S.FIELD_U_SP), host.field_array(S.FIELD_U_SP))
    # a second evolve call starts its clock at 0 again, as time_evolution does
    n2 = dev.evolve(t_end / 4)
    assert n2 > 0
    host.close()
    dev.close()


def test_evolve_to_zero_takes_no_step():
    import spd_k_b200 as S
    g = make(BLAST, "fp64", False)
    u0 = g.field_array(S.FIELD_U_SP)
    assert g.evolve(0.0) == 0
    assert same_bits(g.field_array(S.FIELD_U_SP), u0)
    g.close()
