"""Python binding of the learned troubled-cell indicator (include/spdk_learned.h).

    ind = Indicator(n_in)                       # seeded BF16 MLP, 2 x 64 GELU
    X, y = collect(solver, steps)               # feature rows + NAD labels, on the GPU
    ind.fit(X, y)                               # GPU training (own fwd/bwd kernels, Adam)
    solver.set_indicator(ind, threshold)        # a-priori flags every step

Feature rows are BF16 bit patterns in int16 torch CUDA tensors; labels and
weights float32 CUDA tensors. torch is only the device-memory plumbing here:
every computation runs in libspdk_cuda.so.
"""
import ctypes

import numpy as np

from .api import FIELD_ELEMENT_PREDICTED, FIELD_ELEMENT_TROUBLES, SpdkError, load_library

HIDDEN = 64


def _lib():
    L = load_library()
    if not getattr(L, "_learned_types", False):
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.spdk_mlp_create.argtypes = [i, i, ctypes.c_ulonglong, ctypes.POINTER(vp)]
        L.spdk_mlp_destroy.argtypes = [vp]
        L.spdk_mlp_num_params.argtypes = [vp, ctypes.POINTER(i)]
        L.spdk_mlp_get_params.argtypes = [vp, ctypes.POINTER(f), i]
        L.spdk_mlp_set_params.argtypes = [vp, ctypes.POINTER(f), i]
        L.spdk_mlp_forward.argtypes = [vp, vp, i, vp, vp]
        L.spdk_mlp_loss_grad.argtypes = [vp, vp, vp, vp, i, vp, vp, vp]
        L.spdk_mlp_train_step.argtypes = [vp, vp, vp, vp, i, f, vp, vp]
        L.spdk_hydro_feature_size.argtypes = [vp, ctypes.POINTER(i)]
        L.spdk_hydro_features.argtypes = [vp, vp, ctypes.c_size_t]
        L.spdk_hydro_set_indicator.argtypes = [vp, vp, f]
        L._learned_types = True
    return L


def _check(L, rc):
    if rc != 0:
        raise SpdkError(f"spdk error {rc}: {L.spdk_last_error().decode()}")


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def layout(n_in):
    """offsets of W1 [n_in][64], b1, W2 [64][64], b2, w3 [64], b3 in the parameter vector"""
    o = {"W1": 0, "b1": n_in * HIDDEN}
    o["W2"] = o["b1"] + HIDDEN
    o["b2"] = o["W2"] + HIDDEN * HIDDEN
    o["w3"] = o["b2"] + HIDDEN
    o["b3"] = o["w3"] + HIDDEN
    o["n"] = o["b3"] + 1
    return o


class Indicator:
    """The BF16 MLP on the GPU."""

    def __init__(self, n_in, seed=1):
        L = _lib()
        h = ctypes.c_void_p()
        _check(L, L.spdk_mlp_create(n_in, HIDDEN, seed, ctypes.byref(h)))
        self.h, self.n_in = h, n_in
        n = ctypes.c_int()
        _check(L, L.spdk_mlp_num_params(h, ctypes.byref(n)))
        self.n_params = n.value

    def close(self):
        if getattr(self, "h", None):
            _lib().spdk_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        a = np.empty(self.n_params, dtype=np.float32)
        L = _lib()
        _check(L, L.spdk_mlp_get_params(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.n_params))
        return a

    def set_params(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        L = _lib()
        _check(L, L.spdk_mlp_set_params(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.n_params))

    def predict(self, X):
        import torch
        p = torch.empty(X.shape[0], dtype=torch.float32, device=X.device)
        L = _lib()
        _check(L, L.spdk_mlp_forward(self.h, _ptr(X), X.shape[0], _ptr(p), _stream()))
        return p

    def loss_grad(self, X, y, w=None):
        import torch
        loss = torch.zeros(1, dtype=torch.float32, device=X.device)
        grad = torch.zeros(self.n_params, dtype=torch.float32, device=X.device)
        L = _lib()
        _check(L, L.spdk_mlp_loss_grad(self.h, _ptr(X), _ptr(y), _ptr(w), X.shape[0], _ptr(loss), _ptr(grad),
                                       _stream()))
        return loss, grad

    def fit(self, X, y, w=None, epochs=30, batch=4096, lr=3e-3, seed=0):
        """minibatch Adam on the GPU; returns the mean loss of each epoch"""
        import torch
        L = _lib()
        g = torch.Generator(device="cpu").manual_seed(seed)
        loss = torch.zeros(1, dtype=torch.float32, device=X.device)
        hist = []
        n = X.shape[0]
        for _ in range(epochs):
            perm = torch.randperm(n, generator=g).to(X.device)
            tot, cnt = 0.0, 0
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                xb, yb = X[idx].contiguous(), y[idx].contiguous()
                wb = w[idx].contiguous() if w is not None else None
                _check(L, L.spdk_mlp_train_step(self.h, _ptr(xb), _ptr(yb), _ptr(wb), xb.shape[0], lr, _ptr(loss),
                                                _stream()))
                tot += float(loss.item()) * xb.shape[0]
                cnt += xb.shape[0]
            hist.append(tot / cnt)
        return hist

    def save(self, path):
        np.savez(path, params=self.params(), n_in=self.n_in)

    @classmethod
    def load(cls, path):
        d = np.load(path)
        ind = cls(int(d["n_in"]))
        ind.set_params(d["params"])
        return ind


def features(solver):
    """feature rows of the solver's current state (int16 CUDA tensor [E][n_in])"""
    import torch
    L = _lib()
    n = ctypes.c_int()
    _check(L, L.spdk_hydro_feature_size(solver.h, ctypes.byref(n)))
    E = solver.info.n_elements
    x = torch.empty((E, n.value), dtype=torch.int16, device="cuda")
    _check(L, L.spdk_hydro_features(solver.h, _ptr(x), E * n.value))
    solver.sync()
    return x


def element_flags(solver, field=FIELD_ELEMENT_TROUBLES):
    return solver.read(field)


def collect(solver, steps, every=1):
    """(X, y): feature rows of the state before each step and the label that
    step produces (1 if NAD/SED/PAD flagged any sub-cell of the element in
    any slice), for `steps` steps of the solver"""
    import torch
    xs, ys = [], []
    for s in range(steps):
        x = features(solver) if s % every == 0 else None
        solver.step()
        if x is not None:
            lab = np.asarray(solver.read(FIELD_ELEMENT_TROUBLES), dtype=np.float32)
            xs.append(x)
            ys.append(torch.from_numpy(lab).cuda())
    return torch.cat(xs), torch.cat(ys)


def set_indicator(solver, ind, threshold=0.5):
    L = _lib()
    _check(L, L.spdk_hydro_set_indicator(solver.h, ind.h if ind is not None else None, threshold))
