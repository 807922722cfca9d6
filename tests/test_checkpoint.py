"""Checkpoint / restart (include/spdk.h, spdk_checkpoint.cu; no reference
counterpart).

CPU: the header reader (spdk_checkpoint_peek) on files made here, and its
errors. GPU: a solver restored from a checkpoint and stepped on equals the
run that was never interrupted, bit for bit (U_sp and dt), in the plain
FP64 form, the FP32 form, the FP32 form with the learned indicator and an
SSP-RK3 run; the asynchronous checkpoint captures the state of the moment
it is called while the solver keeps stepping; a checkpoint is refused by a
solver of another configuration; the driver restarted from its own
mid-run checkpoint writes the uninterrupted run's final output file byte
for byte.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

from helpers import gpu_config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "spd_k_b200", "spdk_run")

HEADER_V1 = "<8s18IQ3d2q2d112x"   # the 256-byte header, version 1
# version 2: box lengths, gravity, nu, beta, NAD tolerance, four fallback
# switches, slab_lo, slab_n
HEADER_V2 = "<8s18IQ3d2q2d3d3d3d6i16x"


def fake_checkpoint(path, magic=b"SPDKCKP1", version=1, t=0.125, t_output=0.25, steps=17, outputs=3):
    ints = [version, 1, 2, 3, 64, 48, 1, 4, 16, 0, 1, 1, 1, 1, 0, 4, 0, 0]
    count = 64 * 48 * 4 * 16
    common = (magic, *ints, count, t, 1e-4, t_output, steps, outputs, 1.4, 0.8)
    if version == 2:
        hd = struct.pack(HEADER_V2, *common, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1e-5, 0, 1, 1, 1, 0, 0)
    else:
        hd = struct.pack(HEADER_V1, *common)
    assert len(hd) == 256
    with open(path, "wb") as f:
        f.write(hd)
        f.write(np.zeros(count, dtype=np.float32).tobytes())


@pytest.mark.parametrize("version", [1, 2])
def test_peek_reads_the_header(tmp_path, version):
    from spd_k_b200.api import checkpoint_peek
    path = tmp_path / "c.spdk"
    fake_checkpoint(path, version=version)
    info = checkpoint_peek(str(path))
    assert info == {"t": 0.125, "t_output": 0.25, "steps": 17, "outputs": 3, "precision": "fp32", "p": 3,
                    "N": [64, 48, 1], "integrator": 0, "rk_order": 1}


@pytest.mark.parametrize("bad,code", [("magic", -1), ("version", -1), ("short", -5), ("missing", -5)])
def test_peek_rejects_bad_files(tmp_path, bad, code):
    from spd_k_b200.api import SpdkError, checkpoint_peek
    path = tmp_path / "c.spdk"
    if bad == "magic":
        fake_checkpoint(path, magic=b"NOTACKPT")
    elif bad == "version":
        fake_checkpoint(path, version=9)
    elif bad == "short":
        path.write_bytes(b"SPDKCKP1" + bytes(20))
    with pytest.raises(SpdkError, match=f"spdk error {code}"):
        checkpoint_peek(str(path))


# ---------------------------------------------------------------------- GPU
def blast(side, **kw):
    import bench
    import spd_k_b200 as S
    return S.HydroSolver(dict(gpu_config(bench.workload_overrides(side)), **kw))


def same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp64", "fp32", "fp32+indicator", "rk3"])
def test_restart_continues_bit_for_bit(tmp_path, form):
    kw = {"precision": "fp64" if form in ("fp64", "rk3") else "fp32"}
    if form == "rk3":
        kw.update(integrator="rk3", fallback=False)
    ind = None
    if form == "fp32+indicator":
        from spd_k_b200.learned import Indicator, set_indicator
        ind = Indicator.load(os.path.join(ROOT, "spd_k_b200", "data", "indicator_2d_p3.npz"))
    a = blast(32, **kw)
    if ind:
        set_indicator(a, ind, 0.5)
    for _ in range(3):
        a.step()
    a.steps(3)
    path = str(tmp_path / "a.spdk")
    a.checkpoint(path, t=0.5, t_output=0.75, steps=6, outputs=2)
    for _ in range(2):
        a.step()
    a.steps(3)
    a.sync()
    b = blast(32, **kw)
    if ind:
        set_indicator(b, ind, 0.5)
    info = b.restore(path)
    assert info == {"t": 0.5, "t_output": 0.75, "steps": 6, "outputs": 2}
    for _ in range(2):
        b.step()
    b.steps(3)
    b.sync()
    assert same_bits(a.read(0), b.read(0))
    assert same_bits(a.read(1), b.read(1))
    assert a.dt() == b.dt()
    for s in (a, b):
        if ind:
            set_indicator(s, None)
        s.close()
    if ind:
        ind.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_async_checkpoint_snapshots_the_moment_of_the_call(tmp_path, precision):
    a = blast(32, precision=precision)
    a.steps(4)
    a.sync()
    u4, dt4 = a.read(0), a.dt()
    path = str(tmp_path / "async.spdk")
    a.checkpoint(path, t=1.0, steps=4, wait=False)
    a.steps(5)                                     # steps overlap the write
    a.checkpoint_wait()
    a.sync()
    b = blast(32, precision=precision)
    b.restore(path)
    assert same_bits(b.read(0), u4) and b.dt() == dt4
    b.steps(5)
    b.sync()
    assert same_bits(a.read(0), b.read(0)) and a.dt() == b.dt()
    a.close()
    b.close()


@pytest.mark.gpu
def test_restore_refuses_another_configuration(tmp_path):
    from spd_k_b200.api import SpdkError
    a = blast(32)
    path = str(tmp_path / "c.spdk")
    a.checkpoint(path)
    for kw in ({"precision": "fp32"}, {"N": [32, 16, 1]}, {"p": 2}, {"L": [2.0, 1.0, 1.0]},
               {"g": [0.0, -0.1, 0.0]}, {"nad_tolerance": 1e-4}, {"sed": False}):
        b = blast(32, **kw)
        with pytest.raises(SpdkError, match="another configuration"):
            b.restore(path)
        b.close()
    a.close()


@pytest.mark.gpu
def test_driver_restart_reproduces_the_final_output(tmp_path):
    base = ["job/fallback=true", "mesh/nx1=16", "mesh/nx2=16", "mesh/nx3=1", "mesh/x1_bc=gradfree",
            "mesh/x2_bc=gradfree", "problem/problem=spherical_blast", "problem/p0=1273.2395447351628",
            "problem/p1=1e-5", "problem/radius=0.05", "time/tlim=0.004", "output/dt=0.001"]
    full, part = tmp_path / "full", tmp_path / "part"
    full.mkdir()
    part.mkdir()

    def run(args, out):
        env = dict(os.environ, SPD_OUTPUT_DIR=str(out))
        r = subprocess.run([DRIVER] + args, capture_output=True, text=True, env=env, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        return r.stdout

    out1 = run(base + ["output/checkpoint_dt=0.0015"], full)
    ckpts = sorted(full.glob("checkpoint_*.spdk"), key=lambda p: int(p.stem.split("_")[1]))
    assert len(ckpts) >= 2
    mid = ckpts[0]
    out2 = run(base + [f"job/restart={mid}"], part)
    assert "restarted from" in out2
    finals = sorted(full.glob("W_cv_N16p3_*_0.dat"), key=lambda p: int(p.stem.split("_")[3]))
    last = finals[-1].name
    assert (part / last).read_bytes() == (full / last).read_bytes()
    steps_full = int(out1.split("evolution: ")[1].split(" steps")[0])
    steps_part = int(out2.split("evolution: ")[1].split(" steps")[0])
    assert steps_part == steps_full


@pytest.mark.gpu
@pytest.mark.parametrize("dt_out", [None, 0.0007])
def test_evolve_resumes_a_restored_run(tmp_path, dt_out):
    """spdk_hydro_evolve_from continues a restored run at the checkpoint's t
    and next output time: the same steps and state as one uninterrupted
    device loop."""
    import spd_k_b200 as S
    t_mid, t_end = 0.0015, 0.004
    a = blast(32)
    a.run(t_mid, dt_out)
    path = str(tmp_path / "mid.spdk")
    a.checkpoint(path, t=a.t, t_output=a.t_output or 0.0, steps=a.n_step)
    b = blast(32)
    info = b.restore(path)
    n_b = b.evolve(t_end, dt_out, t0=info["t"], t_output=info["t_output"] if dt_out else None)
    c = blast(32)
    n_c = c.evolve(t_end, dt_out)
    assert a.n_step + n_b == n_c
    assert b.t == c.t and b.dt() == c.dt()
    assert same_bits(b.read(S.FIELD_U_SP), c.read(S.FIELD_U_SP))
    # already past t_end: no step, t stays
    assert b.evolve(t_end, dt_out, t0=t_end, t_output=t_end) == 0 and b.t == t_end
    for s in (a, b, c):
        s.close()
