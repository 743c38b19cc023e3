"""Helpers shared by the GPU tests: numpy <-> torch device buffers and
direct C-ABI calls."""
import numpy as np


def dev(a, device="cuda"):
    """numpy array -> contiguous torch CUDA tensor with the same bytes."""
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    elif a.dtype == np.uint64:
        a = a.view(np.int64)
    return torch.from_numpy(a.copy()).to(device)


def host(t, dtype=None):
    import torch
    torch.cuda.synchronize()
    a = t.detach().cpu().numpy()
    return a.view(dtype) if dtype is not None else a


def empty(shape, dtype, device="cuda"):
    import torch
    tmap = {np.float32: torch.float32, np.uint32: torch.int32, np.int32: torch.int32,
            np.float64: torch.float64, np.uint8: torch.uint8, np.int64: torch.int64}
    return torch.zeros(shape, dtype=tmap[np.dtype(dtype).type], device=device)


def stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def random_model(L, q, seed, sigma=0.3):
    rng = np.random.default_rng(seed)
    J = rng.normal(0, sigma, size=(L * (L - 1) // 2, q * q)).astype("<f4")
    return J
