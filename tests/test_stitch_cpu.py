"""Debursting line selection (Stitch_OneSubswath / getLineIdxInMetaData,
Func.cpp:2766-2933): the product's tops_stitch_line_map and the oracle
against the reference's own getLineIdxInMetaData (tests/golden/ref_stitch.npz,
made by tests/golden/make_golden.py stitch).  No GPU."""
import os

import numpy as np
import pytest

from conftest import ROOT

G = np.load(os.path.join(ROOT, "tests", "golden", "ref_stitch.npz"))
NCASES = len([k for k in G.files if k.endswith("_map")])


def _case(ci):
    nb, L, b0, bN = (int(v) for v in G[f"case{ci}_params"])
    dt, flt = (float(v) for v in G[f"case{ci}_dt"])
    fv, lv = G[f"case{ci}_valid"]
    return nb, L, b0, bN, dt, flt, fv, lv, G[f"case{ci}_first"], G[f"case{ci}_last"], \
        G[f"case{ci}_map"]


def _info(T, nb, L, dt, flt, first, last):
    s = T.SwathInfo()
    s.n_bursts, s.lines_per_burst, s.samples_per_burst = nb, L, 4096
    s.dt, s.first_line_time = dt, flt
    for b in range(nb):
        s.burst_first_line_time[b] = first[b]
        s.burst_last_line_time[b] = last[b]
    return s


@pytest.mark.parametrize("ci", range(NCASES))
def test_line_map_matches_reference(T, O, ci):
    nb, L, b0, bN, dt, flt, fv, lv, first, last, ref = _case(ci)
    info = _info(T, nb, L, dt, flt, first, last)
    om = O.stitch_line_map(first, last, L, dt, flt, fv, lv, b0, bN)
    if (ref < 0).any():
        # a line no burst covers: the reference stops (Func.cpp:2866-2873)
        assert om is None
        with pytest.raises(T.TopsError):
            T.stitch_line_map(info, fv, lv, b0, bN)
        return
    assert np.array_equal(om, ref)
    assert np.array_equal(T.stitch_line_map(info, fv, lv, b0, bN), ref)


def test_line_map_shape(T):
    """Every row of the burst stack appears at most once, in increasing
    order, and each overlap switches bursts once."""
    nb, L, b0, bN, dt, flt, fv, lv, first, last, ref = _case(0)
    m = T.stitch_line_map(_info(T, nb, L, dt, flt, first, last), fv, lv, b0, bN)
    assert np.all(np.diff(m) > 0)
    jumps = np.flatnonzero(np.diff(m) > 1)
    assert len(jumps) == bN - b0
    assert m[0] == fv[b0]   # the first valid line of burst0


def test_line_map_argument_checks(T):
    nb, L, b0, bN, dt, flt, fv, lv, first, last, ref = _case(0)
    info = _info(T, nb, L, dt, flt, first, last)
    for a, b in ((-1, 3), (3, 2), (0, nb)):
        with pytest.raises(T.TopsError):
            T.stitch_line_map(info, fv, lv, a, b)
