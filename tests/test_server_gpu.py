"""The request server (apo_server_*): continuous batching with admission by
free HBM.  Every request's result must be the same alone and in the mix,
whatever arrives while it runs."""
import time

import numpy as np
import pytest

from apocharmm_b200 import api
from apocharmm_b200.systems import batch_system, water_box, write_charmm_files

pytestmark = pytest.mark.gpu


def _systems(tmp_path):
    a = water_box(216, 19.0, seed=7)
    a.settings = dict(kappa=0.34, nfft=(20, 20, 20), order=4, ctofnb=8.0, ctonnb=7.0, cutnb=9.0)
    b = batch_system(11, 3000)
    c = water_box(400, 23.5, seed=3)
    c.settings = dict(kappa=0.30, nfft=(24, 24, 24), order=4, ctofnb=9.0, ctonnb=7.5, cutnb=10.5)
    systems = [a, b, c]
    bt = api.batch_from_systems(systems, str(tmp_path / "relax"))
    xs = api.relax_batch(bt, [api.water_indices(s) for s in systems], iterations=100)
    handles = []
    for k, s in enumerate(systems):
        p = write_charmm_files(s, str(tmp_path / f"s{k}"))
        handles.append((api.CharmmPsf(p["psf"]), api.CharmmParameters(p["prm"])))
    return systems, xs, handles


# (system, kind, steps, seed): MD segments of lengths that end inside a
# segment, and one energy/force request
REQUESTS = [(0, 0, 60, 11), (1, 0, 130, 12), (2, 1, 0, 13), (2, 0, 45, 14)]


def _submit(srv, systems, xs, handles, req):
    k, kind, steps, seed = req
    s = systems[k]
    return srv.submit(kind, handles[k][0], handles[k][1], s.box, s.settings, xs[k], seed, steps)


def _result(srv, rid, kind):
    assert srv.wait(rid, 300.0) == api.Server.DONE
    if kind == 0:
        return srv.coordinates(rid), srv.velocities(rid)
    return srv.forces(rid), srv.energies(rid)


def test_results_alone_equal_results_in_mix(tmp_path):
    systems, xs, handles = _systems(tmp_path)
    alone = []
    for req in REQUESTS:
        srv = api.Server(hbm_fraction=0.5, seed=99)
        rid = _submit(srv, systems, xs, handles, req)
        alone.append(_result(srv, rid, req[1]))
        srv.close()
    # all at once; then staggered, so the batch is re-formed while requests
    # run; then with an HBM share so small that one request runs at a time
    for pattern in ("together", "staggered", "one at a time"):
        srv = api.Server(hbm_fraction=1e-9 if pattern == "one at a time" else 0.5, seed=99)
        ids = []
        for req in REQUESTS:
            ids.append(_submit(srv, systems, xs, handles, req))
            if pattern == "staggered":
                time.sleep(0.05)
        for req, rid, ref in zip(REQUESTS, ids, alone):
            got = _result(srv, rid, req[1])
            if req[1] == 0:
                assert np.array_equal(got[0], ref[0]), (pattern, req)
                assert np.array_equal(got[1], ref[1]), (pattern, req)
                assert np.all(np.isfinite(got[0]))
            else:
                assert np.array_equal(got[0], ref[0]), (pattern, req)
                for t in ref[1]:
                    assert got[1][t] == pytest.approx(ref[1][t], rel=1e-12, abs=1e-9), (pattern, t)
            assert srv.latency(rid) > 0.0
        st = srv.stats()
        assert st["system_steps"] == sum(r[2] for r in REQUESTS if r[1] == 0)
        if pattern == "staggered":
            assert st["rebuilds"] >= 2
        srv.close()


def test_md_result_moves_and_stays_bound(tmp_path):
    systems, xs, handles = _systems(tmp_path)
    srv = api.Server(seed=5)
    rid = _submit(srv, systems, xs, handles, (1, 0, 200, 3))
    x, v = _result(srv, rid, 0)
    assert not np.array_equal(x, xs[1])
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(v))
    srv.release(rid)
    with pytest.raises(Exception):
        srv.poll(rid)
    srv.close()


def test_a_request_that_cannot_join_fails_alone(tmp_path):
    """A request whose coordinates are not finite cannot join the batch: it
    is answered with an error, while the request already running goes on
    and ends as it does alone."""
    systems, xs, handles = _systems(tmp_path)
    good_req = (1, 0, 20000, 12)
    alone = api.Server(hbm_fraction=0.5, seed=99)
    ref = _result(alone, _submit(alone, systems, xs, handles, good_req), 0)
    alone.close()
    srv = api.Server(hbm_fraction=0.5, seed=99)
    good = _submit(srv, systems, xs, handles, good_req)
    time.sleep(0.3)  # the good request is running by now
    bad_x = np.array(xs[0], copy=True)
    bad_x[5, 1] = np.nan
    s = systems[0]
    bad = srv.submit(0, handles[0][0], handles[0][1], s.box, s.settings, bad_x, 11, 60)
    assert srv.wait(bad, 300.0) == api.Server.FAILED
    got = _result(srv, good, 0)
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
    # the server still takes requests
    again = _submit(srv, systems, xs, handles, (0, 0, 60, 11))
    assert srv.wait(again, 300.0) == api.Server.DONE
    srv.close()
