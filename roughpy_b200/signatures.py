"""Batched path signatures on the GPU.

``signature(increments, offsets, depth, mode)`` computes, for every stream
``s`` with increment rows ``offsets[s]:offsets[s+1]``, the Chen product
``exp(x_0) (x) exp(x_1) (x) ...`` in the dense truncated free tensor algebra:
the quantity RoughPy's ``Context.compute_signature`` /
``LiteContext::compute_signature`` (algebra/src/lite_context.h:542-563)
returns for one stream, for thousands of uneven streams in one launch.

Modes: ``"f64"`` (float64 throughout) and ``"f32c"`` (float32 storage and
products with compensated accumulation of the running signature).
"""
from __future__ import annotations

import ctypes
import json

import numpy as np
import torch

from . import _lib

MODES = {"f64": _lib.F64, "f32c": _lib.F32}


def tensor_size(width: int, depth: int) -> int:
    n = int(_lib.lib.rpyb_tensor_size(int(width), int(depth)))
    if n < 0:
        raise ValueError(_lib.last_error())
    return n


def offsets_from_lengths(lengths) -> np.ndarray:
    lengths = np.asarray(lengths, dtype=np.int64)
    off = np.zeros(lengths.shape[0] + 1, dtype=np.int64)
    np.cumsum(lengths, out=off[1:])
    return off


def longest_first(offsets) -> np.ndarray:
    """Processing order for the device work queue: streams by length, longest first."""
    offsets = np.asarray(offsets, dtype=np.int64)
    lengths = np.diff(offsets)
    return np.argsort(-lengths, kind="stable").astype(np.int64)


class SignaturePlan:
    """One batch layout (offsets + processing order) with its launch schedule.

    Wraps ``rpyb_sig_plan``: the schedule (lane shape, warps per block and
    the time-segment length that splits long streams across the GPU) comes
    from ``RPYB_SIG_SCHEDULE``, the tuning cache, or -- with ``tune`` -- from
    timing the candidates once for this layout's (width, depth, length, batch)
    bucket.  Reusable across calls with the same stream lengths; ``run``
    allocates nothing.  One run at a time per plan.
    """

    def __init__(self, offsets, width: int, depth: int, mode: str = "f32c", device="cuda",
                 tune: bool = True):
        if mode not in MODES:
            raise ValueError(f"mode must be one of {sorted(MODES)}")
        self.width = int(width)
        self.depth = int(depth)
        self.mode = mode
        self.code = MODES[mode]
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        if off.ndim != 1 or off.shape[0] < 1 or np.any(np.diff(off) < 0) or off[0] != 0:
            raise ValueError("offsets must be a non-decreasing int array starting at 0")
        self.n_streams = int(off.shape[0] - 1)
        self.total = int(off[-1])
        self.max_len = int(np.diff(off).max()) if self.n_streams else 0
        self.offsets_host = off
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.offsets = torch.from_numpy(off).to(self.device)
        self.order = torch.from_numpy(longest_first(off)).to(self.device)
        self.size = tensor_size(self.width, self.depth)
        self.dtype = torch.float64 if self.code == _lib.F64 else torch.float32
        self._handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            s = torch.cuda.current_stream(self.device).cuda_stream
            _lib.check(_lib.lib.rpyb_sig_plan_create(
                self.code, self.width, self.depth, self.n_streams, off.ctypes.data,
                _lib.SIG_PLAN_TUNE if tune else 0, s, ctypes.byref(self._handle)))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            _lib.lib.rpyb_sig_plan_free(h)
            self._handle = None

    def schedule(self) -> dict:
        """The plan's launch schedule (lane shape g, warps per block, segment
        length, work items, merge levels, and where the choice came from)."""
        buf = ctypes.create_string_buffer(1024)
        _lib.lib.rpyb_sig_plan_describe(self._handle, buf, len(buf))
        return json.loads(buf.value.decode())

    def _check_inputs(self, increments):
        if increments.dtype != self.dtype:
            raise TypeError(f"increments must be {self.dtype} for mode {self.mode}")
        if not increments.is_cuda or not increments.is_contiguous():
            raise ValueError("increments must be a contiguous CUDA tensor")
        if increments.numel() != self.total * self.width:
            raise ValueError("increments do not match the offsets")

    def run(self, increments: torch.Tensor, out: torch.Tensor | None = None,
            stream: torch.cuda.Stream | None = None, report_error: bool = False):
        """Launch on device tensors (no host synchronisation).

        With ``report_error`` the call returns ``(out, err)``: ``err[s]`` is
        stream s's largest per-level relative error against the float64 GPU
        path run on the same increments (zeros in "f64" mode, which is its
        own reference); the first such call allocates the float64 buffers."""
        self._check_inputs(increments)
        if out is None:
            out = torch.empty((self.n_streams, self.size), dtype=self.dtype, device=self.device)
        err = None
        if report_error:
            err = torch.zeros(self.n_streams, dtype=torch.float64, device=self.device)
        if self.n_streams:
            s = (stream or torch.cuda.current_stream(self.device)).cuda_stream
            _lib.check(_lib.lib.rpyb_sig_plan_run(
                self._handle, increments.data_ptr() if self.total else None, out.data_ptr(),
                out.stride(0) if out.dim() > 1 else self.size,
                err.data_ptr() if err is not None else None, s))
        return (out, err) if report_error else out

    def capture(self, increments: torch.Tensor, out: torch.Tensor | None = None):
        """Capture one launch into a CUDA graph: returns ``(graph, out)``.

        ``increments`` and ``out`` become the graph's static buffers: refill
        ``increments`` in place (same layout) and call ``graph.replay()`` to
        recompute ``out``.  A launch is a work-queue reset and one persistent
        kernel on the plan's own workspace, so the graph holds no allocation;
        what replay saves is the per-call launch overhead, which dominates for
        small batches.  The first launch runs outside the capture, on a side
        stream, so that one-time set-up (module loading, kernel attributes)
        stays out of the graph."""
        if out is None:
            out = torch.empty((self.n_streams, self.size), dtype=self.dtype, device=self.device)
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self.run(increments, out, stream=side)
        torch.cuda.current_stream(self.device).wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.run(increments, out)
        return graph, out

    def run_host_pipelined(self, inc_host: torch.Tensor, out_host: torch.Tensor,
                           n_chunks: int = 8) -> torch.Tensor:
        """End-to-end call on host buffers through ``rpyb_signature_host``:
        chunked, with the copies in both directions overlapping the kernels.
        Pass pinned tensors; synchronise the current stream before reading."""
        if inc_host.is_cuda or out_host.is_cuda:
            raise ValueError("run_host_pipelined takes host tensors")
        if inc_host.dtype != self.dtype or out_host.dtype != self.dtype:
            raise TypeError(f"host buffers must be {self.dtype}")
        if not inc_host.is_contiguous() or inc_host.numel() != self.total * self.width:
            raise ValueError("increments do not match the offsets")
        key = int(n_chunks)
        if getattr(self, "_host_key", None) != key:
            nbytes = int(_lib.lib.rpyb_signature_host_device_bytes(
                self.code, self.width, self.depth, self.n_streams,
                self.offsets_host.ctypes.data, key))
            if nbytes < 0:
                raise ValueError(_lib.last_error())
            self._host_buf = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=self.device)
            self._host_key = key
        _lib.check(_lib.lib.rpyb_signature_host(
            self.code, self.width, self.depth, self.n_streams, self.offsets_host.ctypes.data,
            inc_host.data_ptr(), out_host.data_ptr(), out_host.stride(0), key,
            self._host_buf.data_ptr(), self._host_buf.numel(),
            torch.cuda.current_stream(self.device).cuda_stream))
        return out_host

    def run_host(self, inc_host: torch.Tensor, out_host: torch.Tensor, inc_dev: torch.Tensor,
                 out_dev: torch.Tensor) -> torch.Tensor:
        """End-to-end call from (pinned) host buffers on the current stream:
        host->device copy of the increments, the signature launch, and the
        device->host copy of the signatures.  Asynchronous; synchronise the
        stream before reading ``out_host``."""
        inc_dev.copy_(inc_host, non_blocking=True)
        self.run(inc_dev, out_dev)
        out_host.copy_(out_dev, non_blocking=True)
        return out_host


def signature(increments, offsets=None, depth: int = 2, mode: str = "f32c", width=None):
    """Signatures of a batch of streams.

    ``increments``: array ``[total, width]`` (NumPy or torch; a single stream
    may be given as ``[L, width]`` with ``offsets=None``).  Returns a tensor
    ``[n_streams, tensor_size]`` on the GPU (or NumPy for NumPy input).
    """
    is_numpy = isinstance(increments, np.ndarray)
    dt = np.float64 if mode == "f64" else np.float32
    if is_numpy:
        inc = torch.from_numpy(np.ascontiguousarray(increments, dtype=dt)).cuda()
    else:
        inc = increments.to(dtype=torch.float64 if mode == "f64" else torch.float32).contiguous()
        if not inc.is_cuda:
            inc = inc.cuda()
    if inc.dim() != 2:
        raise ValueError("increments must be two-dimensional [rows, width]")
    w = int(width or inc.shape[1])
    if offsets is None:
        offsets = np.array([0, inc.shape[0]], dtype=np.int64)
    plan = SignaturePlan(offsets, w, depth, mode, device=inc.device)
    out = plan.run(inc)
    if is_numpy:
        return out.cpu().numpy()
    return out


class _SignatureFunction(torch.autograd.Function):
    """Batched signatures with the hand-written adjoint kernel as backward."""

    @staticmethod
    def forward(ctx, increments, plan, checkpoint_every):
        out = plan.run(increments.contiguous())
        ctx.save_for_backward(increments)
        ctx.plan = plan
        ctx.checkpoint_every = int(checkpoint_every)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        (inc,) = ctx.saved_tensors
        plan = ctx.plan
        grad = grad_out.to(inc.dtype).contiguous()
        grad_inc = torch.empty_like(inc)
        ws_bytes = int(_lib.lib.rpyb_signature_backward_workspace_size(
            plan.code, plan.width, plan.depth, plan.n_streams, plan.max_len,
            ctx.checkpoint_every))
        if ws_bytes < 0:
            raise ValueError(_lib.last_error())
        ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=inc.device)
        _lib.check(_lib.lib.rpyb_signature_backward(
            plan.code, plan.width, plan.depth, plan.n_streams, plan.offsets.data_ptr(),
            plan.max_len, inc.data_ptr(), grad.data_ptr(), grad.stride(0), grad_inc.data_ptr(),
            ctx.checkpoint_every, ws.data_ptr(), ws.numel(),
            torch.cuda.current_stream(inc.device).cuda_stream))
        return grad_inc, None, None


def signature_with_grad(increments: torch.Tensor, plan: SignaturePlan,
                        checkpoint_every: int = 64) -> torch.Tensor:
    """Differentiable batched signatures: forward by the signature kernel,
    backward by the reverse Chen product kernel (states recomputed from
    checkpoints every ``checkpoint_every`` steps)."""
    return _SignatureFunction.apply(increments, plan, checkpoint_every)
