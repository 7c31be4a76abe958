"""Density compensation estimates for non-Cartesian trajectories, the
preprocessing callers that produce the NUFFT adjoint's density weights
(src/deepmr/_design/grad/utils/dcf.py): ``voronoi`` (Voronoi cell sizes,
dcf.py:75-160), ``analytical_dcf`` (|k|, dcf.py:20-31) and
``angular_compensation`` (dcf.py:34-72).

Host code: the Voronoi diagram comes from Qhull through
``scipy.spatial.Voronoi``, as in the reference; the cell measures, the spike
clipping, the edge extrapolation and the normalisation follow the reference's
arithmetic step by step, so results agree with it to float32 rounding:

* a 2D cell's measure is its polygon area (shoelace over the region's vertices
  in Qhull order, dcf.py:257-276);
* a 3D cell's measure is the reference's formula, the sum over all pairs
  (i, j) of |(B_i x C_i) . A_j| / 6 with A, B, C the region's vertices 0..n-3,
  1..n-2, 2..n-1 minus vertex 0 (dcf.py:290-306) -- all pairs, not only
  i = j, exactly as the reference computes it;
* open cells (a vertex at infinity) get 0;
* of repeated coordinates only the first occurrence is measured; the others
  keep 0 (the reference's redistribution, dcf.py:227-236 and 335-345,
  compares group ids with point indices and leaves the weights unchanged)
  until the normalisation sets zeros to 1.

Differences, outside what the reference can run: torch input is accepted and
returned as torch (the reference's ``coord.detach().numpy`` without a call
fails), and complex coordinates ``kx + 1j ky`` become (..., 2) (the
reference stacks them along the first axis and then fails in Qhull).
"""

import numpy as np
import torch

__all__ = ["analytical_dcf", "angular_compensation", "voronoi"]


def analytical_dcf(coord):
    """|k| per sample: ``(coord ** 2).sum(-1) ** 0.5`` (dcf.py:20-31)."""
    return (coord**2).sum(axis=-1) ** 0.5


def angular_compensation(wi, coord, rotation_axis):
    """Through-plane correction of in-plane weights ``wi`` (npts,) for 3D
    projections (dcf.py:34-72): shot n's coordinates (nproj, npts, 3) without
    its rotation axis give |k| per sample, multiplied into ``wi`` and
    normalised to sum 1."""
    cang = np.stack([np.delete(coord[n], rotation_axis[n], axis=-1) for n in range(len(rotation_axis))], axis=0)
    out = wi[None, :] * analytical_dcf(cang)
    out /= np.sum(out)
    return out


def voronoi(coord, nshots=1, fix_edge=False, ratio=0.1):
    """Voronoi density compensation (dcf.py:75-160).

    Args:
        coord: (..., 2) or (..., 3) coordinates (numpy or torch; complex
            ``kx + 1j ky`` accepted).
        nshots: > 1 treats ``coord`` (npts, 2) as one interleaf of ``nshots``
            uniformly rotated ones; the diagram covers all of them and the
            first interleaf's weights are returned.
        fix_edge: replace the zero weights of open cells by a cubic fit of the
            weight against |k|^2 over the outer samples (|k|^2 > 0.6 max).
        ratio: spike clipping: weights above the value at rank
            ``round((1 - (1 - ratio) * 0.98) * M)`` in descending order are
            clipped to it.

    Returns:
        float32 weights of shape ``coord.shape[:-1]`` (one interleaf for
        nshots > 1), scaled so that the sample nearest k = 0 weighs
        1 / nshots; torch in, torch out (same device).
    """
    device = None
    if isinstance(coord, torch.Tensor):
        device = coord.device
        coord = coord.detach().cpu().numpy()
    coord = np.array(coord, copy=True)
    if np.iscomplexobj(coord):
        coord = np.stack((coord.real, coord.imag), axis=-1)
    if nshots > 1:
        coord = _rotated_interleaves(coord, nshots)

    cabs = ((coord[0] if nshots > 1 else coord) ** 2).sum(axis=-1) ** 0.5
    k0 = np.argmin(cabs)
    ishape = coord.shape[:-1]
    pts = coord.reshape(-1, coord.shape[-1])

    # repeated coordinates: only the first occurrence of each is measured
    _, first, counts = np.unique(pts, return_index=True, return_counts=True, axis=0)
    if np.any(counts > 1):
        wi = np.zeros(pts.shape[0], dtype=np.float32)
        wi[first] = _cell_weights(pts[first], fix_edge, ratio)
    else:
        wi = _cell_weights(pts, fix_edge, ratio)
    wi = np.nan_to_num(wi, posinf=0.0, neginf=0.0)

    wi = wi.reshape(ishape)
    if nshots > 1:
        wi = wi[0]
    wi = _normalize(wi)
    wi = (1 / wi[k0] / nshots) * wi
    wi = wi.squeeze()
    if device is not None:
        wi = torch.as_tensor(wi, dtype=torch.float32, device=device)
    return wi


def _rotated_interleaves(coord, nshots):
    """``nshots`` copies of one 2D interleaf (npts, 2) rotated about z by
    2 pi s / nshots, as float32 (nshots, npts, 2) (the reference's uniform
    tilt and projection, tilt.py:14-54, 196-215, 255-290)."""
    ang = (np.arange(nshots) * (2 * np.pi / nshots)) % (2 * np.pi)
    c, s = np.cos(ang), np.sin(ang)
    # rotation about the unit z axis: rows (c, -s, 0), (s, c, 0), (0, 0, 1)
    R = np.zeros((nshots, 3, 3))
    R[:, 0, 0], R[:, 0, 1] = c, -s
    R[:, 1, 0], R[:, 1, 1] = s, c
    R[:, 2, 2] = 1.0
    k = coord.T
    k3 = np.stack((k[0], k[1], 0 * k[1]), axis=0)
    out = np.einsum("bij,j...->bi...", R, k3).swapaxes(0, 1)[:2]
    return out.astype(np.float32).transpose(1, 2, 0)


def _cell_weights(pts, fix_edge, ratio):
    """Cell measures of distinct points, clipped (dcf.py:239-254)."""
    from scipy.spatial import Voronoi

    vor = Voronoi(pts)
    verts = vor.vertices
    measure = _area2d if pts.shape[-1] == 2 else _volume3d
    wi = np.zeros(pts.shape[0], dtype=np.float32)
    for m in range(pts.shape[0]):
        region = vor.regions[vor.point_region[m]]
        if len(region) and min(region) >= 0:
            wi[m] = measure(verts[np.asarray(region, dtype=np.int64)])

    # clip spikes: the threshold is the value at rank round(r * M), descending;
    # r moves towards 1 while that value is not finite
    fufa = 0.98
    while True:
        r = 1 - (1 - ratio) * fufa
        thld = wi[np.argsort(wi)[::-1][round(r * wi.size)]]
        if np.isfinite(thld):
            break
        fufa **= 2
    wi[wi > thld] = thld

    if fix_edge:
        # open cells at the edge: cubic fit of the weight against |k|^2
        rho = np.sum(pts**2, axis=-1)
        good = rho > 0.6 * np.max(rho)
        poly = np.polynomial.Polynomial.fit(rho[good], wi[good], 3)
        wi[wi == 0] = poly(rho[wi == 0])
    return wi


def _area2d(p):
    """Area of a convex polygon from its vertices in order (shoelace)."""
    x, y = p[:, 0], p[:, 1]
    return abs(np.sum(x * (np.roll(y, -1) - np.roll(y, 1)))) / 2.0


def _volume3d(p):
    """The reference's 3D cell measure: sum over all pairs (i, j) of
    |(B_i x C_i) . A_j| / 6, A, B, C = vertices 0..n-3, 1..n-2, 2..n-1 minus
    vertex 0."""
    a = p[:-2] - p[0]
    b = p[1:-1] - p[0]
    c = p[2:] - p[0]
    return np.sum(np.abs(np.cross(b, c) @ a.T)) / 6.0


def _normalize(w):
    """Weights -> their normalised inverse's inverse, zeros counted as 1
    (dcf.py:164-172)."""
    total = np.sum(w)
    w[np.isclose(w, 0.0)] = 1.0
    inv = total / w
    inv = inv / np.sum(inv)
    inv[np.isclose(inv, 0.0)] = 1.0
    return 1 / inv
