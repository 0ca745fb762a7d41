"""Device copies of host table bytes for the served loop (torch allocations).

``upload(data)`` starts copying one table to the device on the uploader's own
stream and returns (device address, handle) at once; ``ready(handle)`` waits
until that copy has finished, which the loop does before it submits the first
job that reads the table (on another stream).  Dropping the handle (``free``)
returns the memory to torch's caching allocator, which may hand it out again
for work on the uploader's stream at once: it knows nothing of the engine's
streams.  So ``free(handle)`` may only be called after every job that read the
table has completed (the served loop drops a table only after the waits of
the jobs that read it); the copy itself is ordered on the uploader's stream.
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
            done = torch.cuda.Event()
            done.record(self.stream)
        # the source stays referenced until the copy is known to be done
        return dst.data_ptr(), [dst, src, done]

    @staticmethod
    def ready(handle):
        if handle[1] is not None:
            handle[2].synchronize()
            handle[1] = None

    @staticmethod
    def free(handle):
        del handle
