"""The divergence contraction of the FP32 Picard pass on tensor cores
(spdk_study_divergence mode 1: mma.sync TF32 with the 3xTF32 split) against
the CUDA-core form (mode 0) and an FP64 evaluation on the host: both FP32
forms within FP32 round-off of the FP64 values."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tensor_core_divergence_matches_cuda_cores():
    import torch

    import spd_k_b200 as S
    L = S.load_library()
    f = L.spdk_study_divergence
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_longlong] + [ctypes.c_void_p] * 4
    L.spdk_build_matrices.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 6
    rng = np.random.default_rng(5)
    count = 4099   # not a multiple of a warp's 16 element-variables
    fx = rng.normal(0, 1, (count, 4, 5)).astype(np.float32)
    fy = rng.normal(0, 1, (count, 4, 5)).astype(np.float32)
    D = np.zeros(20)
    assert L.spdk_build_matrices(3, 1, None, D.ctypes.data, None, None, None, None) == 0
    D = D.reshape(4, 5)
    want = np.einsum("ejl,il->eji", fx.astype(np.float64), D) + np.einsum("eil,jl->eji", fy.astype(np.float64), D)
    dev = torch.device("cuda:0")
    tx, ty = torch.from_numpy(fx).to(dev), torch.from_numpy(fy).to(dev)
    out = {}
    for mode in (0, 1):
        o = torch.full((count, 4, 4), float("nan"), dtype=torch.float32, device=dev)
        rc = f(mode, 3, count, tx.data_ptr(), ty.data_ptr(), o.data_ptr(), torch.cuda.current_stream().cuda_stream)
        assert rc == 0, L.spdk_last_error()
        torch.cuda.synchronize()
        out[mode] = o.cpu().numpy().astype(np.float64)
    scale = np.abs(want).max()
    for mode in (0, 1):
        err = np.abs(out[mode] - want).max() / scale
        print(f"\nmode {mode}: max |error| / max |value| = {err:.2e}")
        assert np.all(np.isfinite(out[mode])) and err < 1e-5
