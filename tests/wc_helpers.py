"""Shared helpers of the GPU tests: numpy <-> CUDA tensors with unsigned
bit patterns, and canonical multisets."""
import numpy as np

_SIGNED = {1: np.uint8, 4: np.int32, 8: np.int64}
_UNSIGNED = {1: np.uint8, 4: np.uint32, 8: np.uint64}


def dev(a):
    """numpy unsigned array -> CUDA tensor holding the same bits"""
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(_SIGNED[a.itemsize])).cuda()


def host(t, nbytes=None):
    """CUDA tensor -> numpy unsigned array of the same bits"""
    a = t.detach().cpu().numpy()
    return a.view(_UNSIGNED[a.itemsize if nbytes is None else nbytes])


def empty_dev(n, nbytes, fill=0):
    import torch
    dt = {1: torch.uint8, 4: torch.int32, 8: torch.int64}[nbytes]
    t = torch.empty(n, dtype=dt, device="cuda")
    if nbytes == 1:
        t.fill_(fill)
    else:
        t.fill_(np.array(fill, dtype=_UNSIGNED[nbytes]).view(_SIGNED[nbytes]).item())
    return t


def sorted_pairs(keys, values=None):
    order = np.argsort(keys, kind="stable")
    return (keys[order], None if values is None else values[order])


def copy_device_words(ptr, count, nbytes):
    """Copy `count` words of `nbytes` at device pointer `ptr` to numpy."""
    import ctypes
    import torch
    torch.cuda.synchronize()
    cudart = ctypes.CDLL("libcudart.so.12")
    out = np.empty(count, dtype=_UNSIGNED[nbytes])
    rc = cudart.cudaMemcpy(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(ptr),
                           ctypes.c_size_t(count * nbytes), ctypes.c_int(2))
    assert rc == 0, rc
    return out
