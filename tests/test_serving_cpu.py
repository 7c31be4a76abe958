"""Host-side admission of the CG-SENSE server (no GPU): FIFO order, slots, the
HBM budget, and the error statuses of cancelled, malformed and over-budget
requests (the server's `run` turns a rejection into `ServeStats.errors`)."""

import numpy as np
import pytest

from deepmr_b200.recon import Admission, ReconRequest, working_set_bytes


def _req(rid, n=16, coils=2, arrival=0.0, coord=None, kshape=None, maps_shape=None, dcf=None, traj="t"):
    if coord is None:
        coord = np.random.default_rng(rid).uniform(-n / 2, n / 2, (4, 8, 2)).astype(np.float32)
    kshape = tuple(coord.shape[:-1]) if kshape is None else kshape
    ksp = np.zeros((coils,) + kshape, np.complex64)
    maps = np.zeros(maps_shape if maps_shape is not None else (coils, n, n), np.complex64)
    return ReconRequest(rid, ksp, traj, coord, (n, n), f"m{n}x{coils}", maps, dcf, 4, 0.0, arrival)


def _adm(budget=1 << 40, max_active=4, known=()):
    return Admission(budget, max_active, working_set_bytes, known)


def test_fifo_admission_and_arrival():
    adm = _adm()
    pending = [_req(0, arrival=0.0), _req(1, arrival=5.0)]
    d = adm.take(pending, now=1.0, realtime=True, nactive=0, used=0)
    assert d[0] == "admit" and d[1].rid == 0 and d[2] == working_set_bytes(d[1])
    assert adm.take(pending, now=1.0, realtime=True, nactive=1, used=d[2]) is None  # not arrived yet
    d = adm.take(pending, now=1.0, realtime=False, nactive=1, used=d[2])
    assert d[0] == "admit" and d[1].rid == 1 and pending == []


def test_slots_and_budget_hold_the_queue():
    r = _req(0)
    nb = working_set_bytes(r)
    adm = _adm(budget=int(1.5 * nb), max_active=2)
    pending = [r, _req(1)]
    assert adm.take(pending, 0.0, False, 0, 0)[0] == "admit"
    # one active: the second does not fit beside it, and waits (FIFO)
    assert adm.take(pending, 0.0, False, 1, nb) is None and len(pending) == 1
    # nothing active: it runs alone
    assert adm.take(pending, 0.0, False, 0, 0)[0] == "admit"
    adm = _adm(max_active=1)
    pending = [_req(2)]
    assert adm.take(pending, 0.0, False, 1, 0) is None


def test_over_budget_request_is_rejected_not_admitted():
    small, big = _req(0, n=8), _req(1, n=64, coils=8)
    adm = _adm(budget=working_set_bytes(small) + 1)
    pending = [big, small]
    kind, req, why = adm.take(pending, 0.0, False, 0, 0)
    assert kind == "reject" and req.rid == 1 and "exceeds the HBM budget" in why
    assert adm.take(pending, 0.0, False, 0, 0)[0] == "admit"


def test_cancelled_request_gets_a_status():
    r = _req(0)
    r.cancel()
    pending = [r, _req(1)]
    adm = _adm()
    assert adm.take(pending, 0.0, False, 0, 0) == ("reject", r, "cancelled")
    assert adm.take(pending, 0.0, False, 0, 0)[1].rid == 1


@pytest.mark.parametrize("bad", ["nan", "inf", "dims"])
def test_malformed_coordinates_get_a_status(bad):
    coord = np.zeros((4, 8, 2), np.float32)
    if bad == "nan":
        coord[1, 3, 0] = np.nan
    elif bad == "inf":
        coord[2, 0, 1] = np.inf
    else:
        coord = np.zeros((4, 8, 3), np.float32)
    r = _req(0, coord=coord, kshape=(4, 8))
    kind, _, why = _adm().take([r], 0.0, False, 0, 0)
    assert kind == "reject" and why.startswith("malformed coordinates")


def test_malformed_shapes_get_a_status():
    adm = _adm()
    r = _req(0, kshape=(4, 9))
    assert adm.validate(r).startswith("malformed k-space")
    r = _req(1, maps_shape=(3, 16, 16))
    assert adm.validate(r).startswith("malformed coil maps")
    r = _req(2, dcf=np.ones((4, 7), np.float32))
    assert adm.validate(r).startswith("malformed density weights")
    r = _req(3)
    r.niter = -1
    assert adm.validate(r).startswith("malformed request")
    assert adm.validate(_req(4)) is None


def test_known_trajectory_skips_the_coordinate_scan():
    coord = np.full((4, 8, 2), np.nan, np.float32)
    r = _req(0, coord=coord, kshape=(4, 8), traj="planned")
    assert _adm(known={"planned": None}).validate(r) is None
    assert _adm().validate(r).startswith("malformed coordinates")
