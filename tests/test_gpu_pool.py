"""Admission by HBM footprint (serving.SweepServer with pool_bytes): the lanes
of every device length share one device-memory budget, a length whose
arrived requests outnumber its free member slots gets a new lane when the
lane's measured footprint fits, and an idle lane of a length with nothing
waiting is retired to make room.  Here the stream switches from one length to
the other part-way, under a budget that holds two lanes of the shorter length
beside one of the longer but not a second lane of the longer beside them
(footprints as the library counts its own device bytes): lanes move between the
lengths, the budget is never exceeded, and every result is bit-identical to
the same request solved alone."""
import numpy as np
import pytest

from voxphoton_b200 import geometry as geo
from voxphoton_b200 import serving as sv

pytestmark = pytest.mark.gpu


def small(periods):
    return geo.bragg(periods=periods, period=320e-9, len_abs=0.32e-6, res=40e-9, M=16)


def test_lanes_follow_the_mix_and_results_match_alone():
    band = (1500e-9, 1600e-9)
    fams = [sv.Family(k, small(k), band, nG=3, members=2) for k in (2, 4)]
    cfg = sv.ServeConfig(tol=1e-5, keep_x=True)
    srv = sv.SweepServer(fams, cfg, pool_bytes=1 << 60)
    srv.prepare_pool(1)  # one measured lane per length
    lb = srv.lane_bytes
    # room for two lanes of length 2 beside one of length 4, not for a second
    # lane of length 4 beside them
    srv.pool_bytes = 2 * lb[2] + lb[4] + lb[4] // 2
    lams = np.linspace(band[0], band[1], 8)
    reqs = ([sv.Request(i, 2, float(l), 0.0) for i, l in enumerate(lams)] +
            [sv.Request(100 + i, 4, float(l), 0.4) for i, l in enumerate(lams)])
    mix, _ = srv.serve(reqs, realtime=True)
    ev = srv.pool_events
    assert any(e[0] == "add" and e[1] == 2 for e in ev[2:]), ev   # grew for length 2
    assert any(e[0] == "retire" and e[1] == 2 for e in ev), ev    # gave way to length 4
    assert any(e[0] == "add" and e[1] == 4 for e in ev[2:]), ev   # grew for length 4
    assert srv.pool_peak() <= srv.pool_bytes
    srv.close_pool()
    # the same requests one at a time on a fresh lane per length
    for f in fams:
        f.add_slot()
    alone = {}
    for r in reqs:
        res, _ = sv.SweepServer(fams, cfg).serve([r], realtime=False)
        alone[r.rid] = res[0]
    assert len(mix) == len(reqs)
    for m in mix:
        a = alone[m.rid]
        assert m.flag == 0 and a.flag == 0 and m.relres <= 1e-5
        assert m.iters == a.iters
        assert np.array_equal(m.x, a.x)
    for f in fams:
        f.close()
