"""SL-BDF2 steps on a state that lives in pinned HOST memory.

``HostStateStepper.step`` wraps ``slc_step_bdf2_host`` (C ABI): every call
uploads that step's V^n and V^{n-1}, runs the step with its exact bulk shift
on the GPU, and downloads V^{n+1}, p and (u_bulk, forcing).  The copies run
on two copy streams in chunks, overlapped with the compute and with each
other; feeding a step's V^{n+1} back as the next step's V^n pipelines the
round trip chunk by chunk.  Results are on the host once the current CUDA
stream has completed (``torch.cuda.current_stream().synchronize()``).
"""

from __future__ import annotations

import torch

from . import _native as N


def pinned_like(t):
    """A page-locked host tensor of t's shape and dtype."""
    return torch.empty(t.shape, dtype=t.dtype, device="cpu").pin_memory()


class HostStateStepper:
    def __init__(self, flow):
        if flow.sl_bdf2_pressure != "noninc":
            raise ValueError("the host-state step is the non-incremental pressure form "
                             "(sl.bdf2_pressure: noninc)")
        self.flow = flow
        self._shapes = [tuple(t.shape) for t in (flow.u, flow.v, flow.w, flow.p)]

    def _check(self, ts, shapes, name):
        for t, s in zip(ts, shapes):
            if not isinstance(t, torch.Tensor) or t.device.type != "cpu":
                raise ValueError(f"{name}: host tensors expected")
            if t.dtype != torch.float64 or tuple(t.shape) != s or not t.is_contiguous():
                raise ValueError(f"{name}: contiguous float64 {s} expected")

    def step(self, cur, prev, nxt, p, bulk2, dt):
        """cur, prev, nxt: (u, v, w) host triples; p host pressure; bulk2 a
        2-element float64 host tensor receiving (u_bulk, forcing)."""
        self._check(cur, self._shapes[:3], "cur")
        self._check(prev, self._shapes[:3], "prev")
        self._check(nxt, self._shapes[:3], "next")
        self._check([p], self._shapes[3:], "p")
        if bulk2.dtype != torch.float64 or bulk2.numel() != 2 or bulk2.device.type != "cpu":
            raise ValueError("bulk2: a 2-element float64 host tensor expected")
        pc, k1 = N.ptr_array(cur)
        pp, k2 = N.ptr_array(prev)
        pn, k3 = N.ptr_array(nxt)
        stream = N.stream_of(self.flow.u)
        import ctypes
        self.flow._grid.call("slc_step_bdf2_host", pc, pp, pn, ctypes.c_void_p(p.data_ptr()),
                             ctypes.c_void_p(bulk2.data_ptr()), float(self.flow.U_bulk), float(dt),
                             stream)

    def stats(self):
        """How the host-state calls ran (slc_host_step_stats): calls streamed by
        x slab, calls run whole, slabs of the last call, and slabs of the last
        call recomputed after all of V^n arrived.  Synchronises."""
        import ctypes
        out = (ctypes.c_int64 * 4)()
        N.check(N.lib().slc_host_step_stats(self.flow._grid.handle, out), self.flow._grid.handle)
        return {"streamed_calls": out[0], "whole_calls": out[1], "slabs": out[2],
                "deferred_slabs": out[3]}
