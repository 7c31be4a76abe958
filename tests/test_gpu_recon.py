"""CG-SENSE on the device and the continuous-batching server (GPU).

The reconstruction is checked against the oracle restatement of the
reference's cg_solve + SENSE + Toeplitz normal operator (oracle/cg_ref.py);
serving is checked to give each request the same result alone and in a mix.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(torch.as_tensor(a).detach().cpu(), dtype=np.complex128).ravel()
    b = np.asarray(torch.as_tensor(b).detach().cpu(), dtype=np.complex128).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def small_recon():
    from deepmr_b200 import synth
    from oracle import nufft_ref as R

    N, C = 64, 8
    coord = synth.radial_2d(80, 128, N)
    dcf = synth.ramp_dcf(coord)
    maps = torch.as_tensor(synth.coil_maps(C, (N, N), seed=0))
    x = maps * torch.as_tensor(synth.ellipse_phantom(N, seed=1)).to(torch.complex64)
    y = R.apply_nufft(x, R.plan_nufft(torch.as_tensor(coord), N, 4, 1.25))
    y = y + 1e-2 * synth.complex_gaussian(tuple(y.shape), seed=2)
    return dict(N=N, C=C, coord=coord, dcf=dcf, maps=maps, y=y)


def test_sense_normal_vs_oracle(small_recon):
    import deepmr_b200.fft as F
    from deepmr_b200 import recon, synth
    from oracle import cg_ref, nufft_ref as R

    d = small_recon
    gram = F.plan_toeplitz_nufft(torch.as_tensor(d["coord"]), d["N"], dcf=d["dcf"], width=6, device="cuda")
    op = recon.SenseNormal(d["maps"].cuda(), gram, lamda=0.05)
    x = synth.complex_gaussian((d["N"], d["N"]), seed=5)
    out = torch.empty(x.shape, dtype=torch.complex64, device="cuda")
    op.apply(x.cuda(), out, op.workspace())
    ogram = R.plan_toeplitz(torch.as_tensor(d["coord"]), d["N"], dcf=d["dcf"], width=6)
    assert rel(out, cg_ref.sense_normal(x, d["maps"], ogram, 0.05)) < 1e-5


def test_cg_sense_vs_oracle(small_recon):
    from deepmr_b200 import recon
    from oracle import cg_ref

    d = small_recon
    x = recon.cg_sense(d["y"], d["coord"], (d["N"], d["N"]), d["maps"], d["dcf"], niter=20)
    x_ref, _, _ = cg_ref.cg_sense(d["y"], d["coord"], d["N"], d["maps"], d["dcf"], niter=20)
    # 20 CG steps amplify fp32 rounding differences; float64 inner products here,
    # complex64 in the reference
    assert rel(x, x_ref) < 1e-4, rel(x, x_ref)


def test_cg_sense_vs_reference_fixture(load_golden):
    """CG-SENSE against the reference's own recon pipeline: EncodingOp with
    toeplitz=True, AHy = E^H(dcf**0.5 y) and cg_solve for 20 iterations
    (src/deepmr/recon/alg/linop.py:108-148, classic_recon.py:153-174,
    optim/cg.py:16-221), run by tests/golden/make_golden.py on a 128^2,
    8-coil, 96 x 256 radial acquisition. Tolerance 1e-5 relative L2 for AHy
    and for the 20-iteration solution."""
    from deepmr_b200 import recon

    g = load_golden("cgsense2d")
    N = int(g["shape"])
    maps = torch.as_tensor(g["maps"]).cuda()
    plan = recon._nufft.plan_nufft(torch.as_tensor(g["coord"]), (N, N), 4, 1.25, "cuda")
    dcf = torch.as_tensor(g["dcf"]).cuda()
    ahy = recon.sense_adjoint(torch.as_tensor(g["kspace"]).cuda(), plan, maps, dcf)
    assert rel(ahy, g["ahy"]) < 1e-5, rel(ahy, g["ahy"])
    x = recon.cg_sense(g["kspace"], g["coord"], (N, N), maps, g["dcf"], niter=int(g["niter"]))
    e = rel(x, g["x_cg"])
    print(f"CG-SENSE vs reference: AHy {rel(ahy, g['ahy']):.2e}, 20 iterations {e:.2e}")
    assert e < 1e-5, e


def test_encoding_op_cg_solve_dropin(load_golden):
    """The reference's CG-SENSE caller code, unchanged, on the drop-in operators:
    E, EHE = EncodingOp(..., toeplitz=True); AHy = E.H(dcf**0.5 * y);
    cg_solve(AHy, EHE, niter=20) (src/deepmr/recon/alg/classic_recon.py:133-174).
    EHE is fused (one dmr_sense_normal per application, CG on the device); the
    same iteration through the generic torch CG (a plain callable operator)
    agrees too. Tolerance 1e-5 against the reference's output."""
    from deepmr_b200 import linops, optim

    g = load_golden("cgsense2d")
    N = int(g["shape"])
    maps = torch.as_tensor(g["maps"])
    coord, dcf = torch.as_tensor(g["coord"]), torch.as_tensor(g["dcf"]).cuda()
    y = torch.as_tensor(g["kspace"]).cuda()
    data = torch.zeros((maps.shape[0], 1) + tuple(y.shape[1:]), dtype=torch.complex64, device="cuda")
    E, EHE = linops.EncodingOp(data, traj=coord, dcf=dcf, shape=(N, N), sensmap=maps[None, None].cuda(),
                               toeplitz=True, device="cuda")
    assert EHE.fused is not None
    img = E.H(dcf**0.5 * y[None, None])
    assert tuple(img.shape) == (1, N, N)
    assert rel(img[0], g["ahy"]) < 1e-5, rel(img[0], g["ahy"])
    out, _ = optim.cg_solve(img, EHE, niter=int(g["niter"]), tol=0.0, ndim=2)
    assert tuple(out.shape) == (1, N, N) and out.device.type == "cuda"
    assert rel(out[0], g["x_cg"]) < 1e-5, rel(out[0], g["x_cg"])
    # generic CG (complex64 inner products, as the reference) over the same operator
    out2, _ = optim.cg_solve(img, lambda v: EHE(v), niter=int(g["niter"]), tol=0.0, ndim=2)
    assert rel(out2[0], g["x_cg"]) < 1e-5, rel(out2[0], g["x_cg"])
    # unfused composition (three operators) gives the same normal operator
    v = img.clone()
    unfused = linops.Compose([EHE.linops[0], EHE.linops[1], linops.Identity(2), EHE.linops[2]])
    assert unfused.fused is None
    assert rel(unfused(v), EHE(v)) < 1e-5


def _requests():
    from deepmr_b200 import recon

    return recon.synthetic_requests(6, rate_hz=1000.0, seed=3, sizes=(48, 64, 96), coils=(4, 8), niter=8)


def test_serving_results_identical_alone_and_in_mix():
    from deepmr_b200 import recon

    reqs = _requests()
    server = recon.ReconServer(device="cuda", max_active=6, deterministic=True)
    server.prepare(reqs)
    mixed = server.run(reqs, realtime=False)
    assert mixed.peak_active > 1  # the work really overlapped
    alone = server.run_sequential(reqs, realtime=False)
    one_slot = recon.ReconServer(device="cuda", max_active=1, deterministic=True)
    one_slot.prepare(reqs)
    single = one_slot.run(reqs, realtime=False)
    for r in reqs:
        assert torch.equal(mixed.results[r.rid], alone.results[r.rid]), r.rid
        assert torch.equal(single.results[r.rid], alone.results[r.rid]), r.rid


def test_serving_atomic_gridding_same_alone_and_in_mix_within_tolerance():
    """The default server grids AHy with atomics: results agree to float32 rounding."""
    from deepmr_b200 import recon

    reqs = _requests()
    server = recon.ReconServer(device="cuda", max_active=6)
    server.prepare(reqs)
    mixed = server.run(reqs, realtime=False)
    alone = server.run_sequential(reqs, realtime=False)
    det = recon.ReconServer(device="cuda", max_active=6, deterministic=True)
    det.prepare(reqs)
    ref = det.run_sequential(reqs, realtime=False)
    for r in reqs:
        assert rel(mixed.results[r.rid], alone.results[r.rid]) < 1e-5, r.rid
        assert rel(mixed.results[r.rid], ref.results[r.rid]) < 1e-5, r.rid


def test_serving_admission_respects_budget():
    from deepmr_b200 import recon

    reqs = _requests()
    budget = max(recon.working_set_bytes(r) for r in reqs)
    server = recon.ReconServer(device="cuda", max_active=6, hbm_budget=budget)
    server.prepare(reqs)
    stats = server.run(reqs, realtime=False)
    assert 0 < stats.peak_bytes <= budget and len(stats.results) == len(reqs) and not stats.errors
    s = stats.summary()
    assert s["requests"] == len(reqs) and s["p99_ms"] >= s["p50_ms"] > 0
    # results come back on the host
    assert all(x.device.type == "cpu" for x in stats.results.values())


def test_serving_error_statuses_and_the_rest_served():
    """Cancelled (before and while running), malformed and over-budget requests
    produce an error status; the others' results equal the plain path's."""
    import dataclasses

    import numpy as np

    from deepmr_b200 import recon

    reqs = _requests()
    budget = max(recon.working_set_bytes(r) for r in reqs)
    bad_coord = np.array(reqs[0].coord, dtype=np.float32, copy=True)
    bad_coord[0, 0, 0] = np.nan
    extra = [
        dataclasses.replace(reqs[1], rid=100, cancelled=True),
        dataclasses.replace(reqs[0], rid=101, traj_key="nan-coords", coord=bad_coord),
        dataclasses.replace(reqs[2], rid=102, shape=(512, 512), maps_key="big",
                            maps=np.zeros((reqs[2].kspace.shape[0], 512, 512), np.complex64)),
        dataclasses.replace(reqs[3], rid=103),
    ]

    class CancelWhileRunning(recon.ReconServer):
        def _start(self, req, nbytes, now):
            a = super()._start(req, nbytes, now)
            if req.rid == 103:
                req.cancel()
            return a

    server = CancelWhileRunning(device="cuda", max_active=6, hbm_budget=budget, deterministic=True)
    server.prepare(reqs)
    stats = server.run(reqs + extra, realtime=False)
    assert stats.errors[100] == "cancelled" and stats.errors[103] == "cancelled"
    assert stats.errors[101].startswith("malformed coordinates")
    assert "exceeds the HBM budget" in stats.errors[102]
    assert set(stats.results) == {r.rid for r in reqs}
    ref = server.run_sequential(reqs, realtime=False)
    for r in reqs:
        assert torch.equal(stats.results[r.rid], ref.results[r.rid]), r.rid
