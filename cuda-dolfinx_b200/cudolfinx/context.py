"""Device context (mirrors python/cudolfinx/context.py:29-35).

The reference creates a PETSc CUDA device and retains the primary CUDA
context of device 0 (cpp/cudolfinx/common/CUDA.cpp:28-52).  Here one engine
context per device is created on first use; work is issued on torch's current
CUDA stream of that device.
"""
from __future__ import annotations

import torch

from . import _lib

_contexts: dict[int, "Context"] = {}


class Context:
    def __init__(self, device: int):
        self.device = device
        h = _lib.out_handle()
        _lib.check(_lib.lib.fe_context_create(device, h), "fe_context_create")
        self.handle = h.value
        self._upload = None
        self._download = None

    # Transfers run on two side streams, host->device and device->host (two
    # copy engines), ordered against the compute stream with events, so a
    # coefficient upload overlaps the kernels that do not read it and a
    # read-back overlaps the next assembly.
    def upload_stream(self) -> torch.cuda.Stream:
        if self._upload is None:
            self._upload = torch.cuda.Stream(device=self.device)
        return self._upload

    def download_stream(self) -> torch.cuda.Stream:
        if self._download is None:
            self._download = torch.cuda.Stream(device=self.device)
        return self._download

    def join_transfers(self):
        """Make the current stream wait for every transfer issued so far (e.g.
        before timing or reading results on the current stream)."""
        cur = torch.cuda.current_stream(self.device)
        for st in (self._upload, self._download):
            if st is not None:
                cur.wait_stream(st)

    def torch_stream(self) -> torch.cuda.Stream:
        return torch.cuda.current_stream(self.device)

    def synchronize(self):
        """Wait for the device (transfers included) and raise if a kernel
        reported an error word."""
        _lib.check(_lib.lib.fe_context_synchronize(self.handle), "fe_context_synchronize")

    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    @property
    def torch_device(self):
        return torch.device("cuda", self.device)


def get_cuda_context(device: int | None = None) -> Context:
    """Return the engine context of ``device`` (default: torch's current device)."""
    if not torch.cuda.is_available():
        raise RuntimeError("cudolfinx_b200 needs a CUDA device (B200, sm_100a); none is visible")
    if device is None:
        device = torch.cuda.current_device()
    ctx = _contexts.get(device)
    if ctx is None:
        ctx = Context(device)
        _contexts[device] = ctx
    return ctx
