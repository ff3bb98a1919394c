"""The config.txt run on product files (tops_run_config with masterpath set).

A synthetic pair is written as the reference's inputs: a SAFE directory per
image (annotation/*-iw1-slc-vv-*.xml, measurement/ raster of the same name),
a precise-orbit file per image and a float32 GeoTIFF DEM.  The slave holds
only the scene's bursts 1 and 2, so burst matching has an offset to find.
The CPU tests check the refusals that come before any device work; the GPU
test runs the config and compares every written raster, bit for bit, with
the device-resident plan run directly on the inputs read back from the same
files (annotation, orbit, grid, burst matching, DEM windows of the burst
boxes plus 24 DEM pixels, the matched bursts' SLC rows).
"""
import math
import os

import numpy as np
import pytest

import s1_files as F

SMALL = dict(n_bursts=3, lines_per_burst=300, samples_per_burst=512, overlap_lines=30,
             dem_lines=192, dem_pixels=192, seed=11)
STEM = "s1a-iw1-slc-vv-20210601t135300-20210601t135325-038000-047c0f-004"


def _product(T, S, which, root, first_burst, n_bursts):
    info = T.sub_swath(S.swath[which], first_burst, n_bursts)
    info.first_line_time = info.burst_first_line_time[0]   # the product's own lines
    info.last_line_time = info.burst_last_line_time[n_bursts - 1]
    L, W = info.lines_per_burst, info.samples_per_burst
    safe = os.path.join(root, ("M" if which == 0 else "S") + ".SAFE")
    os.makedirs(os.path.join(safe, "annotation"), exist_ok=True)
    os.makedirs(os.path.join(safe, "measurement"), exist_ok=True)
    grid = F.grid_from_scene(S, info, first_burst=first_burst)
    F.write_annotation(os.path.join(safe, "annotation", STEM + ".xml"), info, grid)
    slc = np.ascontiguousarray(S.slc[which][first_burst * L:(first_burst + n_bursts) * L])
    T.tiff_write(os.path.join(safe, "measurement", STEM + ".tiff"), slc)
    n = info.n_sv
    t = np.array(info.sv_t[:n])
    xyz = np.array([info.sv_x[:n], info.sv_y[:n], info.sv_z[:n]]).T
    eof = os.path.join(root, ("m" if which == 0 else "s") + ".EOF")
    F.write_eof(eof, t, xyz, np.zeros_like(xyz))
    return safe, eof


@pytest.fixture(scope="module")
def products(T, tmp_path_factory):
    root = str(tmp_path_factory.mktemp("products"))
    S = T.Scene(**SMALL)
    m_safe, m_eof = _product(T, S, 0, root, 0, 3)
    s_safe, s_eof = _product(T, S, 1, root, 1, 2)
    di = S.dem_info
    dem = os.path.join(root, "dem.tif")
    T.tiff_write_georef(dem, np.ascontiguousarray(S.dem, np.float32),
                        [di.lon0, di.dlon, 0.0, di.lat0, 0.0, -di.dlat])
    S.close()
    return dict(root=root, masterpath=m_safe, slavepath=s_safe, preciseOrbitMaster=m_eof,
                preciseOrbitSlave=s_eof, SpecificDemPath=dem)


def _config(path, out_dir, products, **over):
    keys = dict(process_dir=str(out_dir), firstsubswath=1, lastsubswath=1, burst0=2, burstN=3,
                polarisation="vv", stitch=1,
                **{k: v for k, v in products.items() if k != "root"})
    keys.update(over)
    path.write_text("".join(f"{k}={v}\n" for k, v in keys.items()))
    return path


@pytest.mark.parametrize("over", [dict(polarisation="vh"), dict(lastsubswath=2),
                                  dict(masterpath="/nonexistent/M.SAFE"),
                                  dict(preciseOrbitSlave="/nonexistent/s.EOF")])
def test_refusals_before_device_work(T, tmp_path, products, over):
    """Missing annotation files (another polarisation, a sub-swath the
    product lacks, no product) and a missing orbit file are refused."""
    with pytest.raises(T.TopsError):
        T.run_config(_config(tmp_path / "c.txt", tmp_path / "out", products, **over))


def _dem_window(ann, b, gt):
    """The burst's DEM window as the driver forms it (RefDem::getData,
    DataTypes.cpp:236-262): its lat/lon box plus 24 DEM pixels."""
    lat_max, lon_min, dlat, dlon = gt[3], gt[0], abs(gt[5]), abs(gt[1])
    la0, la1 = ann.burst_lat_min[b] - 24 * dlat, ann.burst_lat_max[b] + 24 * dlat
    lo0, lo1 = ann.burst_lon_min[b] - 24 * dlon, ann.burst_lon_max[b] + 24 * dlon
    r0, c0 = math.floor((lat_max - la1) / dlat), math.floor((lo0 - lon_min) / dlon)
    r1, c1 = math.ceil((lat_max - la0) / dlat), math.ceil((lo1 - lon_min) / dlon)
    return int(r0), int(c0), int(r1 - r0 + 1), int(c1 - c0 + 1)


@pytest.mark.gpu
def test_product_run_matches_the_plan(T, tmp_path, products):
    out = tmp_path / "proc"
    st = T.run_config(_config(tmp_path / "config.txt", out, products))
    assert st.subswaths == 1 and st.burst_pairs == 2
    # the same inputs, read back from the files
    parsed = {}
    for tag, safe, eof in (("m", products["masterpath"], products["preciseOrbitMaster"]),
                           ("s", products["slavepath"], products["preciseOrbitSlave"])):
        xml = os.path.join(safe, "annotation", STEM + ".xml")
        info, ann = T.s1_annotation_read(xml)
        T.s1_orbit_read(eof, ann.first_line_utc.decode(), ann.last_line_utc.decode(), info)
        slc = T.tiff_read(os.path.join(safe, "measurement", STEM + ".tiff"))
        parsed[tag] = (info, ann, T.s1_geogrid_read(xml), slc)
    (mi, mann, mg, mslc), (si, _, sg, sslc) = parsed["m"], parsed["s"]
    mb0, mbN, sb0, sbN = T.s1_burst_overlap(2, 3, mi, mg, si, sg)
    assert (mb0, mbN, sb0, sbN) == (1, 2, 0, 1)
    k = mbN - mb0 + 1
    m, s = T.sub_swath(mi, mb0, k), T.sub_swath(si, sb0, k)
    dem = T.tiff_read(products["SpecificDemPath"])
    gt = T.tiff_georef(products["SpecificDemPath"])
    P = T.Pair(m, s, dem.shape, T.pair_opts())
    w = (T.DemWindow * k)(*[T.DemWindow(*_dem_window(mann, mb0 + i, gt)) for i in range(k)])
    P.set_dem(dem, gt[3], gt[0], abs(gt[5]), abs(gt[1]), w)
    L = mi.lines_per_burst
    P.upload(np.ascontiguousarray(mslc[mb0 * L:(mbN + 1) * L]),
             np.ascontiguousarray(sslc[sb0 * L:(sbN + 1) * L]))
    P.run()
    ref = P.download()
    P.close()
    assert np.array_equal(T.tiff_read(out / "ReSlave-1.tif"), ref["reslave"])
    assert np.array_equal(T.tiff_read(out / "ReSlaveESD-1.tif"), ref["reslave_esd"])
    assert np.array_equal(T.tiff_read(out / "Coh-1.tif"), ref["coh"])
    fv = np.array([mann.first_valid_line[mb0 + i] for i in range(k)], np.int32)
    lv = np.array([mann.last_valid_line[mb0 + i] for i in range(k)], np.int32)
    mp = T.stitch_line_map(m, fv, lv, 0, k - 1)
    assert np.array_equal(T.tiff_read(out / "CohStitch-1.tif"), ref["coh"][mp])
    assert st.shifts[0] == ref["shifts"][0]
    # the coherence of a matched pair is high where the scene is
    assert float(np.median(ref["coh"])) > 0.5
