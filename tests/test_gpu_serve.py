"""The serving loop on the GPU: jobs admitted by HBM footprint into slots
(streams), overlapping on the device, each result the same alone and in the
mix.  Jobs are whole small scenes and burst sub-ranges of them."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [dict(n_bursts=3, lines_per_burst=200, samples_per_burst=512, overlap_lines=20,
               dem_lines=192, dem_pixels=192, seed=51),
          dict(n_bursts=2, lines_per_burst=180, samples_per_burst=640, overlap_lines=18,
               dem_lines=192, dem_pixels=192, seed=52)]


@pytest.fixture(scope="module")
def scenes(T):
    return [T.Scene(**s) for s in SHAPES]


def _alone(T, S, b0, k):
    """The same job through a standalone plan (eager run)."""
    m = T.sub_swath(S.swath[0], b0, k)
    s = T.sub_swath(S.swath[1], b0, k)
    P = T.Pair(m, s, S.dem.shape)
    di = S.dem_info
    w = (T.DemWindow * k)(*[T.DemWindow(*S.dem_window(b0 + i)) for i in range(k)])
    P.set_dem(S.dem, di.lat0, di.lon0, di.dlat, di.dlon, w)
    L = S.cfg.lines_per_burst
    P.upload(np.ascontiguousarray(S.slc[0][b0 * L:(b0 + k) * L]),
             np.ascontiguousarray(S.slc[1][b0 * L:(b0 + k) * L]))
    P.run()
    out = P.download()
    P.close()
    return out


def _jobs():
    # (scene, first burst, bursts)
    return [(0, 0, 3), (1, 0, 2), (0, 1, 2), (1, 1, 1), (0, 0, 1), (0, 2, 1)]


def _check(out, ref, k):
    assert np.array_equal(out["reslave"], ref["reslave"])
    assert np.array_equal(out["reslave_esd"], ref["reslave_esd"])
    assert np.array_equal(out["coh"], ref["coh"])
    assert np.array_equal(out["cpm"], ref["cpm"])
    if k > 1:
        assert np.array_equal(out["shifts"][:k - 1], ref["shifts"][:k - 1])


def test_results_same_alone_and_in_the_mix(T, scenes):
    jobs = _jobs()
    refs = [_alone(T, scenes[i], b0, k) for i, b0, k in jobs]
    srv = T.Server(hbm_budget=3 << 30, slots=3)
    dems = [srv.add_dem(S.dem, S.dem_info.lat0, S.dem_info.lon0, S.dem_info.dlat,
                        S.dem_info.dlon) for S in scenes]
    outs, ids = {}, []
    for rep in range(2):                      # every job twice, all at once
        for (i, b0, k) in jobs:
            d, o = srv.job(scenes[i], dems[i], b0, k)
            jid = srv.submit(d, keep=o)
            outs[jid] = (o, refs[jobs.index((i, b0, k))], k)
            ids.append(jid)
    srv.drain()
    done = srv.poll()
    assert sorted(x.job_id for x in done) == sorted(ids)
    assert all(x.status == T.TOPS_OK for x in done)
    st = srv.stats()
    assert st.completed == len(ids) and st.running == 0 and st.queued == 0
    assert st.hbm_peak <= 3 << 30 and st.hbm_in_use == 0
    for x in done:
        o, ref, k = outs[x.job_id]
        _check(o, ref, k)
        assert x.arrival_s <= x.admit_s <= x.done_s
    srv.close()


def test_budget_admission_serialises_jobs(T, scenes):
    """A budget for about one job at a time: jobs run one after another, in
    arrival order, and the peak never exceeds the budget."""
    S = scenes[0]
    srv = T.Server(hbm_budget=1 << 30, slots=4)
    dem = srv.add_dem(S.dem, S.dem_info.lat0, S.dem_info.lon0, S.dem_info.dlat, S.dem_info.dlon)
    d0, _ = srv.job(S, dem, 0, 3)
    fp = T.lib.tops_server_job_footprint(d0)
    srv.close()
    srv = T.Server(hbm_budget=int(fp * 1.5), slots=4)
    dem = srv.add_dem(S.dem, S.dem_info.lat0, S.dem_info.lon0, S.dem_info.dlat, S.dem_info.dlon)
    keep = []
    for _ in range(4):
        d, o = srv.job(S, dem, 0, 3)
        keep.append(o)
        srv.submit(d, keep=o)
    srv.drain()
    done = sorted(srv.poll(), key=lambda x: x.job_id)
    assert len(done) == 4 and all(x.status == T.TOPS_OK for x in done)
    for a, b in zip(done, done[1:]):          # one at a time, in order
        assert b.admit_s >= a.done_s - 1e-3
    assert srv.stats().hbm_peak <= int(fp * 1.5)
    ref = _alone(T, S, 0, 3)
    for o in keep:
        _check(o, ref, 3)
    srv.close()


def test_job_larger_than_budget_is_rejected(T, scenes):
    S = scenes[0]
    srv = T.Server(hbm_budget=4 << 20, slots=2)
    dem = srv.add_dem(S.dem, S.dem_info.lat0, S.dem_info.lon0, S.dem_info.dlat, S.dem_info.dlon)
    d, o = srv.job(S, dem, 0, 3)
    assert T.lib.tops_server_job_footprint(d) > 4 << 20
    srv.submit(d, keep=o)
    srv.drain()
    done = srv.poll()
    assert len(done) == 1 and done[0].status == T.TOPS_E_BUDGET
    assert srv.stats().rejected == 1
    srv.close()
