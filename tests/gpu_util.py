"""Device buffers for the GPU tests (torch allocates and uploads; cuda-python's runtime binding
copies from raw device pointers that the library hands out)."""
import numpy as np


def to_device(a: np.ndarray):
    import torch

    a = np.ascontiguousarray(a)
    t = torch.empty(max(a.nbytes, 16), dtype=torch.uint8, device="cuda")
    if a.nbytes:
        t[: a.nbytes].copy_(torch.from_numpy(a.view(np.uint8).reshape(-1)))
    return t


def from_device(ptr: int, dtype, count: int) -> np.ndarray:
    """Copies `count` elements of `dtype` from a device pointer into a new numpy array."""
    import torch
    from cuda.bindings import runtime as rt

    dtype = np.dtype(dtype)
    out = np.empty(count, dtype)
    if count == 0:
        return out
    torch.cuda.synchronize()
    (err,) = rt.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == rt.cudaError_t.cudaSuccess, err
    return out
