"""Python binding of the batched form (include/spdk_batch.h)."""
import ctypes

from .api import HydroConfig, HydroSolver, SpdkError, load_library, make_config


class BatchInfo(ctypes.Structure):
    _fields_ = [
        ("n_problems", ctypes.c_int), ("n_groups", ctypes.c_int), ("n_dof", ctypes.c_longlong),
        ("launches_per_step", ctypes.c_int), ("group_p", ctypes.c_int * 8), ("group_tile", ctypes.c_int * 8),
        ("group_size", ctypes.c_int * 8), ("device_bytes", ctypes.c_size_t),
    ]


def _lib():
    L = load_library()
    if not getattr(L, "_batch_types", False):
        vp = ctypes.c_void_p
        L.spdk_batch_create.argtypes = [ctypes.POINTER(HydroConfig), ctypes.c_int, ctypes.POINTER(vp)]
        L.spdk_batch_destroy.argtypes = [vp]
        L.spdk_batch_autotune.argtypes = [vp, ctypes.c_int]
        L.spdk_batch_steps.argtypes = [vp, ctypes.c_int]
        L.spdk_batch_sync.argtypes = [vp]
        L.spdk_batch_get_info.argtypes = [vp, ctypes.POINTER(BatchInfo)]
        L.spdk_batch_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.spdk_batch_member.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp)]
        L.spdk_batch_record_labels.argtypes = [vp, ctypes.c_int]
        L._batch_types = True
    return L


def _check(L, rc):
    if rc != 0:
        raise SpdkError(f"spdk error {rc}: {L.spdk_last_error().decode()}")


def problem_dof(c):
    """solution points of a configuration dict (active elements x (p+1)^d)"""
    n = c["p"] + 1
    active = [N for N in c["N"] if N > 1]
    e = 1
    for N in active:
        e *= N
    return e * n ** len(active)


def partition(configs, world):
    """Greedy size-balanced split of independent problems across ranks
    (longest processing time first: problems in decreasing DOF, each to the
    rank with the least DOF so far, ties to the lower rank and the lower
    index). Deterministic, so every rank computes the same split without a
    collective; returns one list of problem indices per rank, each in
    increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(configs)), key=lambda i: (-problem_dof(configs[i]), i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += problem_dof(configs[i])
    return [sorted(p) for p in parts]


def waves(configs, max_dof):
    """consecutive groups of the configurations of at most max_dof DOF each
    (a single problem larger than max_dof forms a group of its own): an
    ensemble larger than the device holds runs wave after wave"""
    out, cur, cur_dof = [], [], 0
    for c in configs:
        d = problem_dof(c)
        if cur and cur_dof + d > max_dof:
            out.append(cur)
            cur, cur_dof = [], 0
        cur.append(c)
        cur_dof += d
    if cur:
        out.append(cur)
    return out


def shard(configs, rank, world):
    """(indices, configurations) of this rank's part of the ensemble"""
    idx = partition(configs, world)[rank]
    return idx, [configs[i] for i in idx]


class Batch:
    """Many independent 2D problems (configuration dicts) stepped together."""

    def __init__(self, configs, device=0):
        L = _lib()
        self.configs = list(configs)
        arr = (HydroConfig * len(self.configs))(*[make_config(c, device) for c in self.configs])
        h = ctypes.c_void_p()
        _check(L, L.spdk_batch_create(arr, len(self.configs), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _lib().spdk_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def autotune(self, steps=3):
        L = _lib()
        _check(L, L.spdk_batch_autotune(self.h, steps))

    def steps(self, n):
        L = _lib()
        _check(L, L.spdk_batch_steps(self.h, n))

    def sync(self):
        L = _lib()
        _check(L, L.spdk_batch_sync(self.h))

    def info(self):
        L = _lib()
        i = BatchInfo()
        _check(L, L.spdk_batch_get_info(self.h, ctypes.byref(i)))
        return i

    def stream(self):
        L = _lib()
        s = ctypes.c_void_p()
        _check(L, L.spdk_batch_get_stream(self.h, ctypes.byref(s)))
        return s.value

    def record_labels(self, on=True):
        """every replayed step also writes each member's per-element trouble
        labels (read with member(i).read(FIELD_ELEMENT_TROUBLES))"""
        L = _lib()
        _check(L, L.spdk_batch_record_labels(self.h, 1 if on else 0))

    def member(self, i):
        """a read-only solver view of problem i (read after sync())"""
        L = _lib()
        m = ctypes.c_void_p()
        _check(L, L.spdk_batch_member(self.h, i, ctypes.byref(m)))
        return HydroSolver.attach(m, self.configs[i])
