"""CUDA-graph captured NUFFT operators.

A captured operator owns static device buffers (input, output, workspace) for
one plan and batch size; `forward` / `adjoint` copy the caller's data into
the static input (or take what the caller wrote there: `x_in`, `y_in`) and
replay the graph, so a steady-state call is one graph launch (the FFT passes
and the interpolation or gridding kernel) with no host-side argument
processing. This replaces the reference's
per-call Python dispatch (src/deepmr/fft/nufft.py:450-606) for serving and
iterative reconstructions that apply the same operator many times.
"""

import torch

from .. import _lib


class CapturedNUFFT:
    """Forward and adjoint NUFFT of `plan` for a fixed batch, captured in CUDA graphs.

    Parameters
    ----------
    plan : NUFFTPlan
        Plan from ``plan_nufft`` (on a CUDA device).
    batch : int
        Number of images per call (coils x ...), frames excluded.
    weight : torch.Tensor, optional
        Per-sample density weight applied by both operators (``(total,)`` or
        broadcastable to the plan's sample shape).
    deterministic : bool
        Gridding mode of the adjoint.
    """

    def __init__(self, plan, batch, weight=None, deterministic=False):
        interp = plan.interpolator
        self.plan = plan
        self.dev = interp.device
        self.batch = int(batch)
        ndim = plan.ndim
        F = interp.nframes
        self.image_shape = (self.batch,) + ((F,) if F > 1 else ()) + tuple(int(s) for s in plan.shape)
        from .nufft import _kspace_shape

        self.kspace_shape = tuple(_kspace_shape(interp, (self.batch,)))
        self.x_in = torch.zeros(self.image_shape, dtype=torch.complex64, device=self.dev)
        self.y_out = torch.zeros(self.kspace_shape, dtype=torch.complex64, device=self.dev)
        self.y_in = torch.zeros(self.kspace_shape, dtype=torch.complex64, device=self.dev)
        self.x_out = torch.zeros(self.image_shape, dtype=torch.complex64, device=self.dev)
        self.ws = interp.workspace(self.batch)
        if weight is not None:
            w = torch.as_tensor(weight, dtype=torch.float32).to(self.dev)
            self.w = w.reshape(-1).contiguous() if w.numel() == interp.total else None
            if self.w is None:
                raise ValueError("captured operators take a per-sample weight of `total` elements")
        else:
            self.w = None
        self.det = int(bool(deterministic))
        self._ndim = ndim
        self.g_fwd = self._capture(self._run_forward)
        self.g_adj = self._capture(self._run_adjoint)

    def _run_forward(self):
        L = _lib.lib()
        _lib.check(L.dmr_nufft_forward(self.plan.interpolator.handle, _lib.ptr(self.x_in), 0,
                                       _lib.ptr(self.y_out), self.batch, _lib.ptr(self.w), 0,
                                       _lib.ptr(self.ws), self.ws.numel(), _lib.stream_ptr(self.dev)))

    def _run_adjoint(self):
        L = _lib.lib()
        _lib.check(L.dmr_nufft_adjoint(self.plan.interpolator.handle, _lib.ptr(self.y_in), 0,
                                       _lib.ptr(self.x_out), self.batch, _lib.ptr(self.w), 0, self.det,
                                       _lib.ptr(self.ws), self.ws.numel(), _lib.stream_ptr(self.dev)))

    def _capture(self, fn):
        with torch.cuda.device(self.dev):
            s = torch.cuda.Stream(self.dev)
            s.wait_stream(torch.cuda.current_stream(self.dev))
            with torch.cuda.stream(s):
                fn()  # warm-up outside capture: kernel attributes, cuFFT plan
                fn()
            torch.cuda.current_stream(self.dev).wait_stream(s)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                fn()
        return graph

    def forward(self, image=None):
        """image -> kspace (a view of the static output: copy it to keep it).
        Without ``image`` (or given ``x_in`` itself) the operator reads what
        the caller wrote into ``x_in``, and no copy runs."""
        if image is not None and image is not self.x_in:
            self.x_in.copy_(torch.as_tensor(image).reshape(self.image_shape))
        self.g_fwd.replay()
        return self.y_out

    def adjoint(self, kspace=None):
        """kspace -> image (a view of the static output: copy it to keep it).
        Without ``kspace`` (or given ``y_in`` itself) the operator reads what
        the caller wrote into ``y_in``, and no copy runs."""
        if kspace is not None and kspace is not self.y_in:
            self.y_in.copy_(torch.as_tensor(kspace).reshape(self.kspace_shape))
        self.g_adj.replay()
        return self.x_out


def frames_split(kspace, plan):
    """Split flat uneven-frame k-space ``(..., total)`` into a list of per-frame views."""
    offs = plan.interpolator.frame_offsets
    return [kspace[..., int(offs[f]):int(offs[f + 1])] for f in range(len(offs) - 1)]


def frames_concat(parts):
    """Concatenate per-frame k-space ``[(..., M_f)]`` into ``(..., total)``."""
    return torch.cat([torch.as_tensor(p) for p in parts], dim=-1)


__all__ = ["CapturedNUFFT", "frames_split", "frames_concat"]
