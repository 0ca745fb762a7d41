"""Device copies of host table bytes for the served loop (torch allocations).

``upload(data)`` copies one table to the device and returns (device address,
handle); dropping the handle (``free``) returns the memory to torch's caching
allocator.  The copy has finished when ``upload`` returns, so a job submitted
on another stream may read it at once.
"""
from __future__ import annotations

import numpy as np


class TorchUploader:
    def __init__(self, device: int = 0):
        import torch
        self.torch = torch
        self.device = device
        self.stream = torch.cuda.Stream(device)

    def upload(self, data):
        torch = self.torch
        a = data if isinstance(data, np.ndarray) else np.frombuffer(data, np.uint8)
        src = torch.from_numpy(a) if a.flags.writeable else torch.from_numpy(a.copy())
        if not src.is_pinned():
            src = src.pin_memory()
        with torch.cuda.stream(self.stream):
            dst = torch.empty(max(16, a.size + 16), dtype=torch.uint8,
                              device=f"cuda:{self.device}")
            dst[:a.size].copy_(src, non_blocking=True)
        self.stream.synchronize()
        return dst.data_ptr(), dst

    @staticmethod
    def free(handle):
        del handle
