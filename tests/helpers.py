"""Shared test helpers: run a configuration given as block/name=value
overrides through the oracle (CPU checker) or the GPU solver with the
reference's time loop, and compare states bit for bit."""
import hashlib
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def fixture(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))["W_cv"]


def oracle_config(overrides):
    from oracle import oracle as O
    return O.config_from_params(O.apply_overrides({}, overrides))


def gpu_config(overrides):
    from spd_k_b200.api import apply_overrides, config_from_params
    return config_from_params(apply_overrides({}, overrides))


def oracle_active(o, name="W_cv"):
    """oracle array -> active region (5, Nz, Ny, Nx, nz, ny, nx)."""
    a = o.array(name)[0]
    a = a[:, 1:-1] if a.shape[1] > 1 else a
    return np.ascontiguousarray(a[:, :, 1:-1, 1:-1])


def oracle_run(overrides):
    """(W_cv of the last output, steps, oracle) through the reference loop."""
    from oracle import oracle as O
    c = oracle_config(overrides)
    o = O.Oracle(c)
    out = {}
    o.run(c["tlim"], c["output_dt"], on_output=lambda n, s: out.__setitem__(n, s.array("W_cv")))
    last = out[max(out)]
    a = last[0]
    a = a[:, 1:-1] if a.shape[1] > 1 else a
    return np.ascontiguousarray(a[:, :, 1:-1, 1:-1]), o.n_step, o, last


def reference_file_bytes(w_full):
    """Reference-format W_cv dump (6 slots; slot 5 is identically zero) from
    an oracle W_cv array of shape (1, 5, ...)."""
    full = np.zeros((1, 6) + w_full.shape[2:], dtype=np.float64)
    full[:, :5] = w_full
    return full.tobytes()


def sha256_bytes(b):
    return hashlib.sha256(b).hexdigest()


def gpu_run(overrides, device=0):
    """(W_cv at the last output in reference slot order, steps, solver)."""
    import spd_k_b200 as S
    c = gpu_config(overrides)
    g = S.HydroSolver(c, device=device)
    out = {}
    g.run(c["tlim"], c["output_dt"],
          on_output=lambda n, s: out.__setitem__(n, s.to_reference_slots(s.field_array(S.FIELD_W_CV))))
    return out[max(out)], g.n_step, g


def same_bits(a, b):
    """Equal as IEEE values, NaN matching NaN (signed zeros compare equal)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def rel_l1(a, b):
    """relative L1 difference per conserved/primitive slot"""
    return [float(np.abs(a[v] - b[v]).sum() / max(np.abs(a[v]).sum(), 1e-300)) for v in range(a.shape[0])]
