"""Device buffers for the C ABI: torch tensors used as raw HBM storage.

Field elements, points and indices travel as numpy ``uint64`` arrays on the
host (limb layout of include/lzk.h) and as ``torch.int64`` tensors of the
same shape on the device (same bytes).  torch only provides the memory and
the stream; every computation happens in liblzk_b200.so.
"""
import numpy as np
import torch


def stream_ptr(stream=None):
    """cudaStream_t of a torch stream (current stream when None) as int."""
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def to_device(a, device="cuda"):
    """numpy array (uint64/uint32/...) -> device tensor with the same bytes."""
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        t = torch.from_numpy(a.view(np.int64))
    elif a.dtype == np.uint32:
        t = torch.from_numpy(a.view(np.int32))
    else:
        t = torch.from_numpy(a)
    return t.to(device, non_blocking=False)


def empty(shape, device="cuda", dtype=torch.int64):
    return torch.empty(shape, dtype=dtype, device=device)


def zeros(shape, device="cuda", dtype=torch.int64):
    return torch.zeros(shape, dtype=dtype, device=device)


def to_host(t):
    """device tensor -> numpy array, int64 viewed back as uint64."""
    a = t.detach().cpu().numpy()
    if a.dtype == np.int64:
        return a.view(np.uint64)
    if a.dtype == np.int32:
        return a.view(np.uint32)
    return a


def ptr(t):
    return None if t is None else t.data_ptr()
