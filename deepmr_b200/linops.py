"""Linear operators of the reference's CG-SENSE callers, on this library.

Drop-ins for the parts of ``deepmr.linops`` and ``deepmr.recon`` that a
non-Cartesian CG-SENSE reconstruction goes through:

* ``NUFFTOp`` / ``NUFFTAdjointOp`` / ``NUFFTGramOp``
  (src/deepmr/linops/nufft.py:12-241): density weights enter as their square
  root on both sides, as in the reference; the Gram operator is the Toeplitz
  self-adjoint with a width-6 kernel (the reference's default there);
* ``SenseOp`` / ``SenseAdjointOp`` (src/deepmr/linops/coil.py:11-205) with the
  reference's map layouts ((nsets, nslices, ncoils, ny, nx) in 2D,
  (nsets, ncoils, nz, ny, nx) in 3D) and its multicontrast axis rules;
* the operator algebra they are composed with (``Linop`` with ``.H``, ``+``,
  ``-``, ``*``; ``Add``, ``Compose``, ``Multiply``, ``Identity``:
  src/deepmr/linops/base.py:10-247);
* ``EncodingOp`` (src/deepmr/recon/alg/linop.py:9-148), non-Cartesian branch
  with given coil maps.

The composition ``C.H * NUFFTGramOp * C`` of one set of coil maps (one slice)
with a single-frame Toeplitz kernel, which is the normal operator EncodingOp
builds with ``toeplitz=True``, runs as one fused SENSE + Toeplitz call
(``dmr_sense_normal``: coil expansion fused into the zero-pad kernel, coil sum
into the crop kernel) instead of three operators with per-coil intermediates;
``deepmr_b200.optim.cg_solve`` recognises it and keeps the whole CG on the
device. Every operator computes on a CUDA device; results return on the
input's device like the NUFFT functions.

Differences from the reference: ``Multiply.H`` is the adjoint of the scaled
operator (conj(a) A^H; the reference returns the unadjointed operator, which
agrees for the real scalings CG uses on self-adjoint operators);
``EncodingOp`` needs coil maps (ESPIRiT calibration is not part of this
library) and covers the non-Cartesian branch only.
"""

__all__ = ["Linop", "Add", "Compose", "Multiply", "Identity", "NUFFTOp", "NUFFTAdjointOp", "NUFFTGramOp",
           "SenseOp", "SenseAdjointOp", "SenseGramOp", "EncodingOp"]

import numpy as np
import torch
import torch.nn as nn

from . import fft as _fft
from . import recon as _recon


class Linop(nn.Module):
    """Linear operator y = A x with ``.H`` (adjoint), ``+``, ``-`` and ``*``
    (composition with an operator, scaling by a scalar, application to a tensor)."""

    def __init__(self, ndim):
        super().__init__()
        self.ndim = ndim

    def _adjoint_linop(self):
        raise NotImplementedError

    @property
    def H(self):
        return self._adjoint_linop()

    def __add__(self, other):
        return Add([self, other])

    def __sub__(self, other):
        return Add([self, -other])

    def __neg__(self):
        return Multiply(self, -1)

    def __mul__(self, other):
        if np.isscalar(other) or (isinstance(other, torch.Tensor) and other.dim() == 0):
            return Multiply(self, other)
        if isinstance(other, Linop):
            return Compose([self, other])
        if isinstance(other, torch.Tensor):
            return self(other)
        raise NotImplementedError(f"cannot multiply a Linop by {type(other)}")

    def __rmul__(self, other):
        if np.isscalar(other) or (isinstance(other, torch.Tensor) and other.dim() == 0):
            return Multiply(self, other)
        return NotImplemented

    def to(self, *args, **kwargs):
        for k, v in list(self.__dict__.items()):
            if isinstance(v, torch.Tensor):
                self.__dict__[k] = v.to(*args, **kwargs)
        return self


def _same_ndim(linops):
    nd = {op.ndim for op in linops}
    if len(nd) != 1:
        raise ValueError("all operators must have the same spatial dimensionality")
    return nd.pop()


class Add(Linop):
    """(A + B) x = A x + B x."""

    def __init__(self, linops):
        super().__init__(_same_ndim(linops))
        self.linops = list(linops)

    def forward(self, x):
        out = self.linops[0](x)
        for op in self.linops[1:]:
            out = out + op(x)
        return out

    def to(self, *args, **kwargs):
        return Add([op.to(*args, **kwargs) for op in self.linops])

    def _adjoint_linop(self):
        return Add([op.H for op in self.linops])


class Compose(Linop):
    """(A B) x = A (B x). C^H * NUFFTGramOp * C is fused (see the module docstring)."""

    def __init__(self, linops):
        super().__init__(_same_ndim(linops))
        flat = []
        for op in linops:
            flat.extend(op.linops if isinstance(op, Compose) else [op])
        self.linops = flat
        self.fused = SenseGramOp.from_chain(flat)

    def forward(self, x):
        if self.fused is not None:
            return self.fused(x)
        for op in self.linops[::-1]:
            x = op(x)
        return x

    def to(self, *args, **kwargs):
        return Compose([op.to(*args, **kwargs) for op in self.linops])

    def _adjoint_linop(self):
        return Compose([op.H for op in self.linops[::-1]])


class Multiply(Linop):
    """(a A) x = A (a x)."""

    def __init__(self, linop, a):
        super().__init__(linop.ndim)
        self.linop = linop
        self.a = a

    def forward(self, x):
        return self.linop(x * self.a)

    def to(self, *args, **kwargs):
        return Multiply(self.linop.to(*args, **kwargs), self.a)

    def _adjoint_linop(self):
        a = self.a.conj() if isinstance(self.a, torch.Tensor) else np.conj(self.a)
        return Multiply(self.linop.H, a)


class Identity(Linop):
    """I x = x."""

    def forward(self, x):
        return x

    def _adjoint_linop(self):
        return self


# ---------------------------------------------------------------------------
# NUFFT operators (src/deepmr/linops/nufft.py:12-241)
# ---------------------------------------------------------------------------
def _sqrt_weight(weight, device):
    if weight is None:
        return None
    return torch.as_tensor(weight, dtype=torch.float32).to(_recon._nufft.compute_device(device)) ** 0.5


class NUFFTOp(Linop):
    """Forward NUFFT: image (..., [ncontrasts,] *shape) -> k-space (..., [ncontrasts,] nviews, nsamples)."""

    def __init__(self, coord=None, shape=None, basis_adjoint=None, weight=None, device="cpu",
                 threadsperblock=128, width=4, oversamp=1.25):
        super().__init__(coord.shape[-1] if coord is not None else None)
        self.nufft_plan = (_fft.plan_nufft(coord, shape, width, oversamp, device)
                           if coord is not None and shape is not None else None)
        self.weight = _sqrt_weight(weight, device)
        self.basis_adjoint = None if basis_adjoint is None else torch.as_tensor(basis_adjoint)
        self.threadsperblock = threadsperblock

    def forward(self, x):
        return _fft.apply_nufft(x, self.nufft_plan, self.basis_adjoint, self.weight,
                                threadsperblock=self.threadsperblock)

    def _adjoint_linop(self):
        op = NUFFTAdjointOp(basis=None if self.basis_adjoint is None else self.basis_adjoint.conj().T,
                            threadsperblock=self.threadsperblock)
        op.ndim, op.nufft_plan, op.weight = self.ndim, self.nufft_plan, self.weight
        return op


class NUFFTAdjointOp(Linop):
    """Adjoint NUFFT: k-space (..., [ncontrasts,] nviews, nsamples) -> image (..., [ncontrasts,] *shape)."""

    def __init__(self, coord=None, shape=None, basis=None, weight=None, device="cpu", threadsperblock=128,
                 width=4, oversamp=1.25, **kwargs):
        super().__init__(coord.shape[-1] if coord is not None else None)
        self.nufft_plan = (_fft.plan_nufft(coord, shape, width, oversamp, device)
                           if coord is not None and shape is not None else None)
        self.weight = _sqrt_weight(weight, device)
        self.basis = None if basis is None else torch.as_tensor(basis)
        self.threadsperblock = threadsperblock

    def forward(self, y):
        return _fft.apply_nufft_adj(y, self.nufft_plan, self.basis, self.weight,
                                    threadsperblock=self.threadsperblock)

    def _adjoint_linop(self):
        op = NUFFTOp(basis_adjoint=None if self.basis is None else self.basis.conj().T,
                     threadsperblock=self.threadsperblock)
        op.ndim, op.nufft_plan, op.weight = self.ndim, self.nufft_plan, self.weight
        return op


class NUFFTGramOp(Linop):
    """Toeplitz self-adjoint NUFFT^H NUFFT (up to the reference's kernel normalisation)."""

    def __init__(self, coord, shape, basis=None, weight=None, device="cpu", threadsperblock=128, width=6,
                 **kwargs):
        super().__init__(coord.shape[-1])
        self.toeplitz_kern = _fft.plan_toeplitz_nufft(coord, shape, basis, weight, width, device)
        self.threadsperblock = threadsperblock

    def forward(self, x):
        return _fft.apply_nufft_selfadj(x, self.toeplitz_kern, threadsperblock=self.threadsperblock)

    def _adjoint_linop(self):
        return self


# ---------------------------------------------------------------------------
# coil operators (src/deepmr/linops/coil.py:11-205)
# ---------------------------------------------------------------------------
def _coil_axis(ndim, multicontrast):
    """Coil axis of the expanded images, counted from the end."""
    return -(ndim + 2) if multicontrast else -(ndim + 1)


class SenseOp(Linop):
    """Multiply an image by the coil maps: (nslices, ..., *shape) -> (nsets, nslices, ncoils, ..., *shape)
    (2D) or (nsets, ncoils, ..., *shape) (3D)."""

    def __init__(self, ndim, sensmap, device=None, multicontrast=True):
        super().__init__(ndim)
        s = torch.as_tensor(sensmap)
        self.device = s.device if device is None else device
        self.sensmap = s.to(self.device)
        self.multicontrast = multicontrast
        if multicontrast:
            self.sensmap = self.sensmap.unsqueeze(-ndim - 1)

    def forward(self, x):
        isnumpy = isinstance(x, np.ndarray)
        x = torch.as_tensor(x)
        y = self.sensmap.to(x.device) * x.unsqueeze(_coil_axis(self.ndim, self.multicontrast))
        return y.numpy(force=True) if isnumpy else y

    def _adjoint_linop(self):
        s = self.sensmap.squeeze(-self.ndim - 1) if self.multicontrast else self.sensmap
        return SenseAdjointOp(self.ndim, s, self.device, self.multicontrast)


class SenseAdjointOp(Linop):
    """Coil combination: sum over coils (and sets) of conj(maps) * images."""

    def __init__(self, ndim, sensmap, device=None, multicontrast=True):
        super().__init__(ndim)
        s = torch.as_tensor(sensmap)
        self.device = s.device if device is None else device
        self.sensmap = s.to(self.device)
        self.multicontrast = multicontrast
        if multicontrast:
            self.sensmap = self.sensmap.unsqueeze(-ndim - 1)

    def forward(self, y):
        isnumpy = isinstance(y, np.ndarray)
        y = torch.as_tensor(y)
        x = (self.sensmap.to(y.device).conj() * y).sum(_coil_axis(self.ndim, self.multicontrast)).sum(0)
        return x.numpy(force=True) if isnumpy else x

    def _adjoint_linop(self):
        s = self.sensmap.squeeze(-self.ndim - 1) if self.multicontrast else self.sensmap
        return SenseOp(self.ndim, s, self.device, self.multicontrast)


class SenseGramOp(Linop):
    """Fused C^H T C (+ lamda I) for one set of coil maps and a single-frame
    Toeplitz kernel: one dmr_sense_normal call per application.

    Input and output are the combined image as the unfused composition takes
    it: (nslices = 1, *shape) in 2D, (*shape) in 3D (a leading axis of size 1
    is kept as given)."""

    def __init__(self, sense, gram, lamda=0.0):
        super().__init__(gram.ndim)
        self.sense, self.gram, self.lamda = sense, gram, float(lamda)
        maps = sense.sensmap
        self.maps = maps.reshape((-1,) + tuple(maps.shape[-self.ndim:]))
        self._normal = None

    @staticmethod
    def from_chain(ops):
        """The fused operator for [SenseAdjointOp, NUFFTGramOp, SenseOp] with the
        same maps, one set / slice and a single-frame kernel, else None."""
        if len(ops) != 3:
            return None
        ca, gram, c = ops
        if not (isinstance(ca, SenseAdjointOp) and isinstance(gram, NUFFTGramOp) and isinstance(c, SenseOp)):
            return None
        if c.multicontrast or ca.multicontrast or ca.sensmap.shape != c.sensmap.shape:
            return None
        if not torch.equal(ca.sensmap, c.sensmap):
            return None
        nd = c.ndim
        lead = c.sensmap.shape[:-nd - 1]  # (nsets, nslices) in 2D, (nsets,) in 3D
        if int(np.prod(lead)) != 1:
            return None
        kv = gram.toeplitz_kern.value
        if kv.dim() > nd and int(np.prod(kv.shape[:-nd])) != 1:
            return None
        return SenseGramOp(c, gram.toeplitz_kern)

    def normal(self, device):
        if self._normal is None or self._normal.dev != device:
            self._normal = _recon.SenseNormal(self.maps.to(device), self.gram, self.lamda)
        return self._normal

    def forward(self, x):
        isnumpy = isinstance(x, np.ndarray)
        xt = torch.as_tensor(x)
        dev = _recon._nufft.compute_device(xt.device if xt.device.type == "cuda" else None)
        op = self.normal(dev)
        xin = xt.to(dev, torch.complex64).reshape(op.ishape).contiguous()
        out = torch.empty_like(xin)
        op.apply(xin, out, op.workspace())
        out = out.reshape(xt.shape)
        if xt.device != out.device:
            out = out.to(xt.device)
        return out.numpy(force=True) if isnumpy else out

    def _adjoint_linop(self):
        return self

    def with_lamda(self, lamda):
        return SenseGramOp(self.sense, self.gram, self.lamda + float(lamda))


# ---------------------------------------------------------------------------
# encoding operator (src/deepmr/recon/alg/linop.py:9-148)
# ---------------------------------------------------------------------------
def EncodingOp(data, mask=None, traj=None, dcf=None, shape=None, nsets=1, basis=None, device=None,
               cal_data=None, sensmap=None, toeplitz=False):
    """E and E^H E of a non-Cartesian acquisition with given coil maps.

    data (..., ncoils, ncontrasts, nviews, nsamples) only supplies the coil
    count; traj (ncontrasts, nviews, nsamples, ndim) or (nviews, nsamples,
    ndim); dcf density weights; shape the image matrix; sensmap the coil maps
    in SenseOp's layout. toeplitz=True gives E^H E = C^H NUFFTGramOp C (fused)."""
    if mask is not None:
        raise NotImplementedError("Cartesian (mask) encoding operators are not part of this library")
    if traj is None or shape is None:
        raise ValueError("non-Cartesian encoding needs traj and shape")
    ncoils = data.shape[-4]
    if device is None:
        device = data.device
    traj = torch.as_tensor(traj)
    ndim = traj.shape[-1]
    F = NUFFTOp(traj, tuple(shape)[-ndim:], basis, dcf, device=device)
    FHF = NUFFTGramOp(traj, tuple(shape)[-ndim:], basis, dcf, device=device) if toeplitz else F.H * F
    if ncoils == 1:
        return F, FHF
    if sensmap is None:
        raise NotImplementedError("coil-map calibration (ESPIRiT) is not part of this library: pass sensmap")
    C = SenseOp(ndim, sensmap, multicontrast=traj.dim() >= 4)
    return F * C, C.H * FHF * C
