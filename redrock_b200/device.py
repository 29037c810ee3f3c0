"""Device plumbing: torch owns device memory and streams, the C ABI computes.

Nothing here computes results on the host: arrays are moved to the GPU,
pointers are handed to librr_b200.so, and the status word written by the
kernels is checked after the stream is synchronised.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("redrock_b200 needs a CUDA device (B200, sm_100a); none is visible")
    _lib.lib()


def device():
    require_cuda()
    return torch.device("cuda", torch.cuda.current_device())


def stream_handle(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes_void(s.cuda_stream)


def ctypes_void(v):
    return None if v in (0, None) else int(v)


def is_device_tensor(a):
    return isinstance(a, torch.Tensor) and a.is_cuda


def to_device(a, dtype=torch.float64, dev=None):
    """numpy / list / tensor -> contiguous CUDA tensor (pinned H2D for numpy)."""
    dev = dev or device()
    if isinstance(a, torch.Tensor):
        return a.to(device=dev, dtype=dtype).contiguous()
    arr = np.ascontiguousarray(np.asarray(a), dtype=_np_dtype(dtype))
    t = torch.from_numpy(arr)
    if arr.nbytes >= (1 << 20):
        t = t.pin_memory()
    return t.to(dev, non_blocking=True)


def capture_graph(fn):
    """Capture fn()'s launches as a CUDA graph on a side stream and return
    (graph, fn's result).  Unlike torch.cuda.graph, this leaves torch's
    device and pinned-host caches alone (no empty_cache before the capture),
    so pinned buffers and cached blocks stay warm for the work around the
    graph; allocations inside fn come from the graph's private pool and
    live as long as the graph."""
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        g.capture_begin()
        try:
            out = fn()
        finally:
            g.capture_end()
    torch.cuda.current_stream().wait_stream(side)
    return g, out


def to_numpy(t):
    if isinstance(t, torch.Tensor):
        return t.detach().cpu().numpy()
    return np.asarray(t)


def _np_dtype(dtype):
    return {torch.float64: np.float64, torch.float32: np.float32, torch.int32: np.int32,
            torch.int64: np.int64, torch.uint8: np.uint8}[dtype]


def ptr(t):
    if t is None:
        return None
    return t.data_ptr()


class StatusWord:
    """One device int the kernels set on bad data or a timed-out wait."""

    def __init__(self, dev=None):
        self.t = torch.zeros(1, dtype=torch.int32, device=dev or device())

    @property
    def ptr(self):
        return self.t.data_ptr()

    def reset(self):
        self.t.zero_()

    def check(self, what):
        code = int(self.t.item())
        if code:
            self.t.zero_()
            _lib.check(code, what)


def struct_bytes(structs):
    """ctypes structure list -> numpy uint8 buffer (for device upload)."""
    import ctypes
    if not structs:
        return np.zeros(0, dtype=np.uint8)
    n = len(structs)
    arr = (type(structs[0]) * n)(*structs)
    return np.frombuffer(bytes(arr), dtype=np.uint8).copy()
