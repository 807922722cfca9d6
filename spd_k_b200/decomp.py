"""Slab domain decomposition of one hydro problem across ranks.

The reference's MPI decomposition is disabled (src/boundary.cpp:3-24); this
is the B200 replacement, one rank per GPU. The domain's slowest active axis
(y in 2D, z in 3D, which must be non-periodic) is cut into slabs of owned
element rows. Each rank's solver holds its owned rows plus `halo` rows on
every internal side, with the whole domain's geometry and initial condition
(spdk_hydro_config slab_lo / slab_n). A step of a slab solver is exact on
every row farther from its internal edges than the step's dependency radius
(step_radius); with halo >= that radius the owned rows equal the
undecomposed run's bit for bit. After each step:

1. dt: each rank's minimum over its owned rows (spdk_hydro_slab_dt), then
   the minimum over ranks (the all-reduce of the reference's compute_dt
   under MPI, src/hydro.cpp:255-259);
2. halo exchange: across each internal edge, each side sends the rows of
   the other's halo (they lie in its owned rows), once per step.

Nothing is exchanged inside a step: the halo covers the step's dependency
radius, so the fused kernels run unchanged (communication-avoiding, at the
price of recomputing the halo rows).

Two drivers share the partition and the exchange plan:
* SlabGroup: every slab in one process (one GPU or several), exchanging by
  device copies;
* SlabRank: one slab per torch.distributed rank (NCCL on GPUs), exchanging
  by point-to-point sends and receives and all-reducing dt.
"""
from dataclasses import dataclass


@dataclass(frozen=True)
class Slab:
    own_lo: int   # owned element rows [own_lo, own_hi) of the domain
    own_hi: int
    ext_lo: int   # rows held by the slab's solver [ext_lo, ext_hi)
    ext_hi: int

    @property
    def rows(self):
        return self.ext_hi - self.ext_lo

    def local(self, lo, hi):
        """domain rows -> rows of the slab's solver"""
        return lo - self.ext_lo, hi - self.ext_lo


def step_radius(c):
    """element rows per side that one step's result depends on.

    Each SD evaluation (a Picard pass or an RK stage) reads the face traces
    of the neighbouring element (radius 1; 2 with the viscous terms, whose
    face fluxes use the neighbours' gradients). Each fallback slice updates
    a sub-cell from candidates up to 6 sub-cells away (NAD box 1, SED 3,
    theta blending and ring 2) and W_old up to 2 away."""
    n = c["p"] + 1
    integ = c.get("integrator", "ader")
    evals, slices = (n, n) if integ == "ader" else (int(integ[2]), int(integ[2]))
    per_eval = 2 if c.get("nu", 0.0) > 0 else 1
    per_slice = -(-6 // n) if c["fallback"] else 0
    return evals * per_eval + slices * per_slice


def slab_axis(c):
    return 2 if c["N"][2] > 1 else 1


def slab_partition(rows, ranks, halo):
    """owned rows as even as possible; halo rows on internal sides only.
    Every slab must own at least `halo` rows so that a neighbour's halo lies
    in its owned rows."""
    if ranks < 1 or rows < ranks:
        raise ValueError(f"cannot cut {rows} rows into {ranks} slabs")
    base, extra = divmod(rows, ranks)
    out, lo = [], 0
    for r in range(ranks):
        hi = lo + base + (1 if r < extra else 0)
        if ranks > 1 and hi - lo < halo:
            raise ValueError(f"slab {r} owns {hi - lo} rows, fewer than the halo of {halo}")
        out.append(Slab(lo, hi, max(0, lo - halo), min(rows, hi + halo)))
        lo = hi
    return out


def exchange_plan(slabs):
    """(src, dst, lo, hi): domain rows [lo, hi) that slab src sends to slab
    dst after every step (src owns them, dst holds them as halo)"""
    plan = []
    for r in range(len(slabs) - 1):
        a, b = slabs[r], slabs[r + 1]
        if b.ext_lo < a.own_hi:
            plan.append((r, r + 1, b.ext_lo, a.own_hi))
        if a.ext_hi > b.own_lo:
            plan.append((r + 1, r, b.own_lo, a.ext_hi))
    return plan


def slab_config(c, slab):
    """the solver configuration of one slab (domain geometry, slab rows)"""
    ax = slab_axis(c)
    if c["bc"][ax] == "periodic":
        raise ValueError("the slab axis (y in 2D, z in 3D) must not be periodic")
    N = list(c["N"])
    rows = N[ax]
    N[ax] = slab.rows
    return dict(c, N=N, slab_lo=slab.ext_lo, slab_n=rows)


def default_halo(c):
    return step_radius(c) + 1


class SlabGroup:
    """All slabs of a decomposed run in this process (devices: one per slab,
    or the same GPU for all). step() advances every slab, agrees on dt and
    refreshes the halos; owned() gathers the owned rows of a field."""

    def __init__(self, c, ranks, devices=None, halo=None):
        from .api import HydroSolver
        self.c = c
        self.halo = default_halo(c) if halo is None else halo
        rows = c["N"][slab_axis(c)]
        self.slabs = slab_partition(rows, ranks, self.halo)
        self.plan = exchange_plan(self.slabs)
        devices = devices or [0] * ranks
        self.solvers = [HydroSolver(slab_config(c, s), device=d) for s, d in zip(self.slabs, devices)]
        self.devices = devices
        self.n_step = 0
        self.agree_dt(initial=True)

    def agree_dt(self, initial=False):
        """the minimum over slabs of each slab's owned-row dt. At creation
        every held row is exact, so each solver's own dt (the constructor's,
        from the FP64 initial W_cv in both forms) is already a minimum over
        correct rows, and the minimum of those is the whole domain's."""
        if initial:
            dts = [g.dt() for g in self.solvers]
        else:
            dts = [g.slab_dt(*s.local(s.own_lo, s.own_hi)) for g, s in zip(self.solvers, self.slabs)]
        dt = min(dts)
        for g in self.solvers:
            g.set_dt(dt)
        return dt

    def exchange(self):
        import torch
        for src, dst, lo, hi in self.plan:
            gs, gd = self.solvers[src], self.solvers[dst]
            buf = torch.empty(self.row_values(gs) * (hi - lo), dtype=self.dtype(gs),
                              device=f"cuda:{self.devices[src]}")
            gs.rows_to(*self.slabs[src].local(lo, hi), buf)
            gs.sync()
            if self.devices[dst] != self.devices[src]:
                buf = buf.to(f"cuda:{self.devices[dst]}")
                torch.cuda.synchronize(self.devices[dst])
            gd.rows_from(*self.slabs[dst].local(lo, hi), buf)
            gd.sync()

    def step(self):
        for g in self.solvers:
            g.step()
        dt = self.agree_dt()
        self.exchange()
        self.n_step += 1
        return dt

    def dt(self):
        return self.solvers[0].dt()

    @staticmethod
    def row_values(g):
        return g.info.n_elements // g.N[slab_axis_of(g)] * g.nvar * g.npt

    @staticmethod
    def dtype(g):
        import torch
        return torch.float32 if g.c.get("precision", "fp64") == "fp32" else torch.float64

    def owned(self, field=0):
        """a field ([element][var][point] order) of the owned rows of every
        slab, concatenated in domain order"""
        import numpy as np
        parts = []
        for g, s in zip(self.solvers, self.slabs):
            a = g.field_array(field)
            ax = slab_axis(self.c)
            lo, hi = s.local(s.own_lo, s.own_hi)
            parts.append(a[:, lo:hi] if ax == 2 else a[:, :, lo:hi])
        return np.concatenate(parts, axis=1 if slab_axis(self.c) == 2 else 2)

    def close(self):
        for g in self.solvers:
            g.close()


def slab_axis_of(g):
    return 2 if g.ndim == 3 else 1


class SlabRank:
    """One slab per torch.distributed rank. `solver` is the rank's slab
    solver (a HydroSolver made from slab_config, or any object with the same
    step / slab_dt / set_dt / rows_to / rows_from / sync methods); `make_buf`
    allocates a 1-D exchange buffer of n values (device tensors for NCCL,
    CPU tensors for gloo)."""

    def __init__(self, dist, slabs, solver, row_values, make_buf):
        self.dist = dist
        self.rank = dist.get_rank()
        self.slabs = slabs
        self.slab = slabs[self.rank]
        self.plan = exchange_plan(slabs)
        self.g = solver
        self.row_values = row_values
        self.make_buf = make_buf

    def agree_dt(self, initial=False):
        """own-row minimum (at creation: the solver's own dt, every held row
        being exact then), then the minimum over ranks"""
        dt = self.g.dt() if initial else self.g.slab_dt(*self.slab.local(self.slab.own_lo, self.slab.own_hi))
        t = self.make_buf(1)
        t.fill_(dt)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)
        dt = float(t[0].item())
        self.g.set_dt(dt)
        return dt

    def exchange(self):
        """every rank posts its sends and receives of the plan in plan order
        (the same on every rank), then waits for all of them"""
        ops, recvs = [], []
        for src, dst, lo, hi in self.plan:
            if src == self.rank:
                buf = self.make_buf(self.row_values * (hi - lo))
                self.g.rows_to(*self.slab.local(lo, hi), buf)
                self.g.sync()
                ops.append(self.dist.P2POp(self.dist.isend, buf, dst))
            elif dst == self.rank:
                buf = self.make_buf(self.row_values * (hi - lo))
                ops.append(self.dist.P2POp(self.dist.irecv, buf, src))
                recvs.append((lo, hi, buf))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        for lo, hi, buf in recvs:
            if buf.is_cuda:
                import torch
                torch.cuda.current_stream(buf.device).synchronize()
            self.g.rows_from(*self.slab.local(lo, hi), buf)
            self.g.sync()

    def step(self):
        self.g.step()
        dt = self.agree_dt()
        self.exchange()
        return dt
