"""The config.txt-driven run (tops_run_config): the reference's main program
on this library.  CPU tests check the refusals that come before any device
work; the GPU test checks every written raster against the device-resident
plan run directly on the same synthetic inputs, bit for bit."""
import numpy as np
import pytest

SMALL = dict(n_bursts=3, lines_per_burst=300, samples_per_burst=512, overlap_lines=30,
             dem_lines=192, dem_pixels=192, seed=11)


def _write_config(path, out_dir, **over):
    keys = dict(process_dir=str(out_dir), masterpath="(synthetic)", slavepath="(synthetic)",
                firstsubswath=1, lastsubswath=2, burst0=2, burstN=3, stitch=1, **SMALL)
    keys.update(over)
    path.write_text("".join(f"{k}={v}\n" for k, v in keys.items()))
    return path


def test_refuses_bad_configs(T, tmp_path):
    cfg = _write_config(tmp_path / "a.txt", tmp_path / "out", npoints=6)
    with pytest.raises(T.TopsError) as e:
        T.run_config(cfg)
    assert e.value.status == T.TOPS_E_CONFIG
    cfg = _write_config(tmp_path / "b.txt", tmp_path / "out", burst0=3, burstN=4)
    with pytest.raises(T.TopsError) as e:
        T.run_config(cfg)
    assert e.value.status == T.TOPS_E_INVALID
    (tmp_path / "c.txt").write_text("burst0\n")
    with pytest.raises(T.TopsError) as e:
        T.run_config(tmp_path / "c.txt")
    assert e.value.status == T.TOPS_E_CONFIG


@pytest.mark.gpu
def test_run_config_outputs_match_the_plan(T, tmp_path):
    out = tmp_path / "proc"
    st = T.run_config(_write_config(tmp_path / "config.txt", out))
    assert st.subswaths == 2 and st.burst_pairs == 4
    # the stage times the run overlaps: each positive, none above the sum
    assert min(st.load_seconds, st.process_seconds, st.write_seconds) > 0.0
    assert st.seconds > 0.0
    for nsub in (1, 2):
        S = T.Scene(**{**SMALL, "seed": SMALL["seed"] + 1000 * (nsub - 1)})
        m, s = T.sub_swath(S.swath[0], 1, 2), T.sub_swath(S.swath[1], 1, 2)
        P = T.Pair(m, s, S.dem.shape, T.pair_opts())
        di = S.dem_info
        w = (T.DemWindow * 2)(*[T.DemWindow(*S.dem_window(b)) for b in (1, 2)])
        P.set_dem(S.dem, di.lat0, di.lon0, di.dlat, di.dlon, w)
        L = S.cfg.lines_per_burst
        P.upload(np.ascontiguousarray(S.slc[0][L:3 * L]), np.ascontiguousarray(S.slc[1][L:3 * L]))
        P.run()
        ref = P.download()
        P.close()
        assert np.array_equal(T.tiff_read(out / f"ReSlave-{nsub}.tif"), ref["reslave"])
        assert np.array_equal(T.tiff_read(out / f"ReSlaveESD-{nsub}.tif"), ref["reslave_esd"])
        coh = T.tiff_read(out / f"Coh-{nsub}.tif")
        assert np.array_equal(coh, ref["coh"])
        mp = T.stitch_line_map(m, np.zeros(2, np.int32), np.full(2, L - 1, np.int32), 0, 1)
        assert np.array_equal(T.tiff_read(out / f"CohStitch-{nsub}.tif"), ref["coh"][mp])
    assert abs(st.shifts[0] - ref["shifts"][0]) == 0.0
