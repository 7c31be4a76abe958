"""Coil calibration on this library's NUFFT — drop-in for the reference's
``deepmr.recon.calib`` callers of ``deepmr.fft``.

* ``find_acs`` (src/deepmr/recon/calib/acs.py:11-152): the calibration k-space
  region. Non-Cartesian data: the samples of the first view within radius
  ``min(shape) // 2`` (the same sample positions are taken from every view),
  density-weighted, gridded with the adjoint NUFFT at oversampling 2 on the
  calibration grid and Fourier-transformed back to k-space. Cartesian data:
  the largest sampled box around the k-space centre (grown isotropically,
  then stretched per axis), Fourier-transformed along its slice axis.
* ``espirit_cal`` (src/deepmr/recon/calib/espirit.py:14-223): ESPIRiT maps
  from that region. Hankel matrix of k x k (x k) blocks of the central r-point
  region, its right singular vectors above ``t`` times the largest singular
  value as k-space kernels, their images on the calibration grid, and per
  voxel the left singular vectors of the kernel images (eigenvalues
  ``s**2 > c`` kept), Fourier-resampled to the image size and normalised by
  the root sum of squares of the first set.
* ``resize``, ``resample``, ``rss``, ``fermi``: the signal helpers those use
  (src/deepmr/_signal/resize.py:11-211, subspace.py:9-70, filter.py:8-100).

The NUFFT and the FFTs run on the data's device (the GPU for CUDA tensors).
ESPIRiT's two SVDs (the Hankel matrix, a few hundred rows, and the per-voxel
ncoils x nkernels kernel images) run in LAPACK on the host, as the reference's
CPU path does: a singular vector's phase is arbitrary per voxel, and the
Fourier resampling to the image grid mixes neighbouring voxels, so the maps
depend on the SVD's phase convention (another SVD, e.g. the GPU's, gives maps
that differ beyond rounding after the resampling although each voxel's
vectors agree up to phase).
"""

__all__ = ["find_acs", "espirit_cal", "resize", "resample", "rss", "fermi"]

import numpy as np
import torch

from . import fft as _fft


# ---------------------------------------------------------------------------
# signal helpers
# ---------------------------------------------------------------------------
def _expanded(ishape, oshape):
    """Input and output shapes on the same number of axes: the output's
    leading axes are the input's (or 1), the input keeps its own shape."""
    ishape, oshape = list(ishape), list(oshape)
    n = max(len(ishape), len(oshape))
    pi = [1] * (n - len(ishape)) + ishape
    po = [1] * (n - len(oshape)) + oshape
    big = [max(a, b) for a, b in zip(pi, po)]
    return big[: n - len(ishape)] + ishape, big[: n - len(oshape)] + oshape


def resize(input, oshape):
    """Centred zero-pad / crop of the trailing axes to `oshape`."""
    isnumpy = isinstance(input, np.ndarray)
    x = torch.as_tensor(input)
    if isinstance(oshape, int):
        oshape = [oshape]
    ish, osh = _expanded(x.shape, oshape)
    if ish == osh:
        return input
    src, dst = [], []
    for i, o in zip(ish, osh):
        si, so = max(i // 2 - o // 2, 0), max(o // 2 - i // 2, 0)
        n = min(i - si, o - so)
        src.append(slice(si, si + n))
        dst.append(slice(so, so + n))
    out = torch.zeros(osh, dtype=x.dtype, device=x.device)
    out[tuple(dst)] = x.reshape(ish)[tuple(src)]
    return out.numpy(force=True) if isnumpy else out


def fermi(ndim, size, width=None):
    """Isotropic Fermi window of `size` points per axis, half maximum at
    radius ``width // 2``, transition scale 20 * size, peak 1."""
    width = size if width is None else width
    radius = int(width // 2)
    ax = torch.arange(int(-size // 2), int(size // 2), dtype=torch.float32)
    grids = torch.meshgrid(*([ax] * ndim), indexing="xy")
    r = torch.stack(grids, 0).pow(2).sum(0).sqrt()
    w = 1.0 / (1.0 + torch.exp(r - radius) / (20 * size))
    return w / w.max()


def _cfft(x, dims, inverse=False):
    op = torch.fft.ifftn if inverse else torch.fft.fftn
    return torch.fft.fftshift(op(torch.fft.ifftshift(x, dim=dims), dim=dims, norm="ortho"), dim=dims)


def resample(input, oshape, filt=True, polysmooth=False):
    """Fourier resampling of the trailing len(oshape) axes (centred FFT,
    centred pad / crop, Fermi window when any axis grows, inverse FFT;
    magnitude for real input)."""
    isnumpy = isinstance(input, np.ndarray)
    x = torch.as_tensor(input)
    if isinstance(oshape, int):
        oshape = [oshape]
    dims = list(range(-len(oshape), 0))
    real = bool(torch.isreal(x).all())
    spec = _cfft(x, dims)
    ish, osh = _expanded(x.shape, oshape)
    window = None
    if filt and any(o > i for o, i in zip(osh, ish)):
        window = resize(fermi(len(oshape), max(osh), min(osh)), osh)
    spec = resize(spec, osh)
    if window is not None:
        spec = spec * window.to(spec.device)
    out = _cfft(spec, dims, inverse=True)
    if real:
        out = out.abs()
    return out.numpy(force=True) if isnumpy else out


def rss(input, axis=None, keepdim=False):
    """Root sum of squares (complex dtype kept, as the reference's)."""
    isnumpy = isinstance(input, np.ndarray)
    x = torch.as_tensor(input)
    if axis is None:
        return (x * x.conj()).sum() ** 0.5
    out = (x * x.conj()).sum(dim=axis, keepdim=keepdim) ** 0.5
    return out.numpy() if isnumpy else out


# ---------------------------------------------------------------------------
# calibration region
# ---------------------------------------------------------------------------
def find_acs(data, shape=None, coord=None, dcf=None):
    """Calibration k-space ``(ncoils, nz, ny, nx)`` (acs.py:11-51)."""
    if coord is None:
        return _cartesian_acs(data)
    return _noncartesian_acs(data, shape, coord, dcf)


def _cartesian_acs(kspace):
    """Largest fully sampled box around the centre of
    ``(nslices, ncoils, ncontrasts, ny, nx)`` data, contrasts summed
    (acs.py:54-114)."""
    ksp = kspace.sum(axis=-3)
    istorch = isinstance(ksp, torch.Tensor)
    device = ksp.device if istorch else None
    ksp = (ksp.numpy(force=True) if istorch else np.asarray(ksp)).astype(np.complex64)
    ksp = np.moveaxis(ksp, 1, -1)  # coils last
    mask = np.abs(ksp[..., 0]) > 0
    box = [[n // 2, n // 2 + 1] for n in mask.shape]

    def full(b):
        return bool(np.all(mask[tuple(slice(lo, hi) for lo, hi in b)]))

    # grow every side at once while the box stays inside and sampled
    while all(lo > 0 and hi < n for (lo, hi), n in zip(box, mask.shape)) and \
            full([[lo - 1, hi + 1] for lo, hi in box]):
        box = [[lo - 1, hi + 1] for lo, hi in box]
    # then each axis on its own, left then right
    for a in range(mask.ndim):
        while box[a][0] > 0 and full([[lo - (d == a), hi] for d, (lo, hi) in enumerate(box)]):
            box[a][0] -= 1
        while box[a][1] < mask.shape[a] and full([[lo, hi + (d == a)] for d, (lo, hi) in enumerate(box)]):
            box[a][1] += 1
    sub = ksp[tuple(slice(lo, hi) for lo, hi in box) + (slice(None),)].copy()
    sub = np.moveaxis(sub, -1, 1)
    if istorch:
        sub = torch.as_tensor(sub, device=device, dtype=torch.complex64)
    sub = sub.swapaxes(0, 1)  # (ncoils, nz, ny, nx)
    return _fft.fft(sub, axes=(1,))


def _noncartesian_acs(kspace, cal_shape, coord, dcf):
    """acs.py:117-152: contrasts folded into views, central samples of the
    first view's radius profile, adjoint NUFFT at oversampling 2, back to
    k-space with a centred FFT over the last three axes."""
    ndim = coord.shape[-1]
    ksp = kspace.reshape(*kspace.shape[:2], 1, -1, kspace.shape[-1])
    crd = coord.reshape(1, -1, *coord.shape[-2:])
    radius = (crd[0, 0] ** 2).sum(axis=-1) ** 0.5
    sel = radius <= min(cal_shape) // 2
    ksp = ksp[..., sel]
    crd = crd[..., sel, :]
    if dcf is not None:
        ksp = dcf.reshape(1, -1, dcf.shape[-1])[..., sel] * ksp
    grid = _fft.nufft_adj(ksp, crd, cal_shape, oversamp=2.0).squeeze()
    if grid.ndim != 4:
        grid = grid[None, ...]
    if ndim == 2:
        grid = grid.swapaxes(0, 1)
    grid = _fft.fft(grid, axes=range(-3, 0))
    return torch.as_tensor(grid, dtype=torch.complex64)


# ---------------------------------------------------------------------------
# ESPIRiT
# ---------------------------------------------------------------------------
def espirit_cal(data, coord=None, dcf=None, shape=None, k=6, r=24, t=0.02, c=0.0, nsets=1):
    """ESPIRiT coil maps and the central r-point calibration data
    (espirit.py:14-148). Returns ``(maps, calib)``."""
    isnumpy = isinstance(data, np.ndarray)
    while len(data.shape) < 5:
        data = data[None, ...]
    if coord is not None:
        ndim = coord.shape[-1]
        shape = ndim * [shape] if np.isscalar(shape) else list(shape)[-ndim:]
        shape = [int(s) for s in shape]
    else:
        ndim = 2
        shape = list(data.shape[-2:])
    # calibration grid: 1/16, 1/8, 1/4, 1/2 of the image from 1024, 512, 256, 128 up; else 64
    big = max(shape)
    div = 16 if big >= 1024 else 8 if big >= 512 else 4 if big >= 256 else 2 if big >= 128 else 0
    cshape = [s // div for s in shape] if div else [64] * ndim
    cal = find_acs(data, cshape, coord, dcf)
    maps = _espirit(cal.clone(), k, r, t, c)
    maps = maps[[0]] if nsets == 1 else maps[:nsets]
    maps = resample(maps, shape)  # (nsets, ncoils, nz, ny, nx)
    maps = maps / rss(maps, axis=1, keepdim=True)[[0]]
    if ndim == 2:
        maps = maps.swapaxes(1, 2)
    if isnumpy:
        maps = maps.numpy(force=True)
    return maps, resize(cal, ndim * [r])


def _espirit(X, k, r, t, c):
    """espirit.py:152-223 on calibration data X ``(ncoils, nz, ny, nx)``:
    maps ``(neigen, ncoils, nz, ny, nx)``."""
    X = X.permute(3, 2, 1, 0)  # (nx, ny, nz, ncoils)
    dims = X.shape[:3]
    nc = X.shape[3]
    live = [n > 1 for n in dims]
    p = sum(live)
    # central r-point region (whole axis when it has one point)
    region = tuple(slice(n // 2 - r // 2, n // 2 + r // 2) if on else slice(0, 1) for n, on in zip(dims, live))
    C = X[region].to(torch.complex64)
    # Hankel matrix: one row per k-block position (x outer, z inner), the
    # block's (x, y, z, coil) values in C order along the row
    ksz = [k if on else 1 for on in live]
    blocks = C
    for a in range(3):
        blocks = blocks.unfold(a, ksz[a], 1)  # (.., .., .., nc, kx, ky, kz)
    A = blocks.permute(0, 1, 2, 4, 5, 6, 3).reshape(-1, ksz[0] * ksz[1] * ksz[2] * nc)
    _, S, VH = torch.linalg.svd(A.cpu(), full_matrices=True)
    V = VH.conj().t().to(X.device)
    nker = int(torch.sum(S >= t * S[0]))
    V = V[:, :nker]
    # kernels placed at the centre of the calibration grid, flipped and
    # conjugated, to image space
    kernels = torch.zeros(tuple(dims) + (nc, nker), dtype=torch.complex64, device=X.device)
    centre = tuple(slice(n // 2 - k // 2, n // 2 + k // 2) if on else slice(0, 1) for n, on in zip(dims, live))
    kernels[centre] = V.reshape(ksz[0], ksz[1], ksz[2], nc, nker)
    npts = dims[0] * dims[1] * dims[2]
    kimg = _fft.fft(kernels.flip(0).flip(1).flip(2).conj(), (0, 1, 2)) * npts**0.5 / (k**p) ** 0.5
    # per voxel: left singular vectors of its (ncoils x nker) kernel image
    u, s, _ = torch.linalg.svd(kimg.reshape(-1, nc, nker).cpu(), full_matrices=True)
    keep = s**2 > c
    u = (keep[:, None, :] * u).to(X.device)
    return u.view(dims[0], dims[1], dims[2], nc, nc).permute(4, 3, 2, 1, 0)
