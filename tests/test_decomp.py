"""Slab domain decomposition (spd_k_b200.decomp) on CPU: the partition, the
exchange plan and the dependency radius, and two gloo ranks driving
SlabRank over a CPU stand-in solver whose step has the same structure (a
stencil of known radius, a per-row dt candidate) -- the decomposed run
equals the undecomposed one exactly. The GPU solver's own decomposed runs
are in tests/test_gpu_decomp.py."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from spd_k_b200 import decomp as DC


def test_partition_owns_every_row_once_with_halos_inside_the_domain():
    for rows, ranks, halo in ((64, 2, 13), (64, 3, 13), (256, 8, 13), (10, 1, 50)):
        sl = DC.slab_partition(rows, ranks, halo)
        assert sl[0].own_lo == 0 and sl[-1].own_hi == rows
        for a, b in zip(sl, sl[1:]):
            assert a.own_hi == b.own_lo
        for s in sl:
            assert 0 <= s.ext_lo <= s.own_lo < s.own_hi <= s.ext_hi <= rows
            if ranks > 1:
                assert s.own_lo - s.ext_lo in (0, halo) and s.ext_hi - s.own_hi in (0, halo)
    with pytest.raises(ValueError):
        DC.slab_partition(20, 3, 8)      # a slab of 6 rows cannot feed a halo of 8


def test_exchange_plan_fills_every_halo_row_from_its_owner():
    sl = DC.slab_partition(64, 3, 13)
    plan = DC.exchange_plan(sl)
    for r, s in enumerate(sl):
        want = set(range(s.ext_lo, s.own_lo)) | set(range(s.own_hi, s.ext_hi))
        got = set()
        for src, dst, lo, hi in plan:
            if dst == r:
                assert all(sl[src].own_lo <= q < sl[src].own_hi for q in range(lo, hi))
                got |= set(range(lo, hi))
        assert got == want


def test_step_radius_follows_the_step_structure():
    base = dict(p=3, N=[64, 64, 1], fallback=True, integrator="ader")
    assert DC.step_radius(base) == 4 + 4 * 2          # 4 Picard passes, 4 slices of 6 sub-cells
    assert DC.step_radius(dict(base, fallback=False)) == 4
    assert DC.step_radius(dict(base, integrator="rk3", fallback=False)) == 3
    assert DC.step_radius(dict(base, nu=0.01, fallback=False)) == 8
    assert DC.step_radius(dict(base, p=1)) == 2 + 2 * 3
    c = dict(base, bc=["gradfree", "periodic", "periodic"])
    with pytest.raises(ValueError):
        DC.slab_config(c, DC.slab_partition(64, 2, 13)[0])


class StencilRows:
    """CPU stand-in for a slab solver: rows of values, a step of radius 2
    (a nonlinear 5-point stencil with copied edges) and a dt candidate per
    row, with the slab solver's methods"""

    def __init__(self, rows, width, lo, seed=7):
        g = torch.Generator().manual_seed(seed)
        full = torch.rand(rows + lo + 64, width, generator=g, dtype=torch.float64)
        self.u = full[lo:lo + rows].clone()
        self.dt_value = 0.0

    def step(self):
        u = self.u
        p = torch.cat([u[:1], u[:1], u, u[-1:], u[-1:]])
        self.u = 0.2 * (p[:-4] + p[1:-3] + p[2:-2] + p[3:-1] + p[4:]) + 0.01 * torch.sin(p[2:-2] * p[1:-3])

    def dt(self):
        return float(1.0 / (1.0 + self.u.abs().max()))

    def slab_dt(self, lo, hi):
        self.dt_value = float(1.0 / (1.0 + self.u[lo:hi].abs().max()))
        return self.dt_value

    def set_dt(self, dt):
        self.dt_value = dt

    def rows_to(self, lo, hi, buf):
        buf.copy_(self.u[lo:hi].reshape(-1))

    def rows_from(self, lo, hi, buf):
        self.u[lo:hi] = buf.reshape(hi - lo, -1)

    def sync(self):
        pass


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q, steps):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    rows, width, halo = 40, 5, 2 + 1
    slabs = DC.slab_partition(rows, world, halo)
    s = slabs[rank]
    g = StencilRows(s.rows, width, s.ext_lo)
    r = DC.SlabRank(dist, slabs, g, width, lambda n: torch.empty(n, dtype=torch.float64))
    dts = [r.agree_dt(initial=True)]
    for _ in range(steps):
        dts.append(r.step())
    lo, hi = s.local(s.own_lo, s.own_hi)
    q.put((rank, g.u[lo:hi].clone(), dts))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_equal_the_undecomposed_run():
    steps, world = 6, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_rank, args=(r, world, port, q, steps)) for r in range(world)]
    for p in ps:
        p.start()
    out = sorted((q.get(timeout=120) for _ in ps), key=lambda o: o[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = StencilRows(40, 5, 0)
    dts = [ref.slab_dt(0, 40)]
    for _ in range(steps):
        ref.step()
        dts.append(ref.slab_dt(0, 40))
    got = torch.cat([o[1] for o in out])
    assert torch.equal(got, ref.u)
    assert out[0][2] == out[1][2] == dts
