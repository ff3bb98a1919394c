"""Sentinel-1 annotation and precise-orbit (EOF) files for the front-end tests.

Writes the elements the readers take (the reference's S1_Initialize,
ComputeDerampPara and S1_OrbitInitialize paths, Func.cpp:135-574,
695-819, 1868-2010) from a topsb200.SwathInfo and a geolocation grid, so a
reader test can compare what it parses with what was written.  Times are
seconds of the day on one date; doubles are written with 17 significant
digits, times with 9 decimals.
"""
import numpy as np

DATE = "2021-06-01"


def utc(t: float, date: str = DATE, decimals: int = 9) -> str:
    h = int(t // 3600)
    m = int((t - 3600 * h) // 60)
    s = t - 3600 * h - 60 * m
    w = 3 + decimals if decimals else 2
    return f"{date}T{h:02d}:{m:02d}:{s:0{w}.{decimals}f}"


def g17(x: float) -> str:
    return f"{x:.17g}"


def grid_from_scene(scene, info, points: int = 11, first_burst: int = 0) -> dict:
    """A geolocation grid with one row per burst start and one after the
    last burst: azimuth times of the burst first lines (and the last burst's
    last line), slant-range times across the swath, and latitude / longitude
    running across each burst's DEM-window box from its north-west to its
    south-east corner, so the per-burst boxes the reader derives cover the
    bursts (the reference uses the grid for those boxes and to seed its
    range-Doppler solution, Func.cpp:494-537, 1627-1640).  info may hold the
    scene's bursts from first_burst on."""
    nb = info.n_bursts
    di = scene.dem_info
    boxes = []
    for b in range(nb):
        r0, c0, nr, nc = scene.dem_window(min(first_burst + b, scene.cfg.n_bursts - 1), 0)
        boxes.append((di.lat0 - r0 * di.dlat, di.lat0 - (r0 + nr - 1) * di.dlat,
                      di.lon0 + c0 * di.dlon, di.lon0 + (c0 + nc - 1) * di.dlon))
    boxes.append(boxes[-1])
    az = [info.burst_first_line_time[b] for b in range(nb)] + [info.burst_last_line_time[nb - 1]]
    rg = info.slr_time + np.linspace(0.0, (info.samples_per_burst - 1) / (2.0 * info.rsr), points)
    lines = nb + 1
    u = np.linspace(0.0, 1.0, points)
    g = {"az_time": np.repeat(np.array(az)[:, None], points, axis=1),
         "slr_time": np.repeat(rg[None, :], lines, axis=0),
         "lat": np.array([b[0] + (b[1] - b[0]) * u for b in boxes]),
         "lon": np.array([b[2] + (b[3] - b[2]) * u for b in boxes]),
         "incidence": np.repeat(np.linspace(30.0, 46.0, points)[None, :], lines, axis=0),
         "line": np.repeat(np.arange(lines)[:, None] * info.lines_per_burst, points, axis=1)}
    return g


def write_annotation(path, info, grid, *, polarisation="VV", dc_method="Data Analysis",
                     fm_as_polynomial=True, first_valid=None, last_valid=None,
                     radar_frequency=None, date=DATE, range_bandwidth=5.6e7,
                     azimuth_pixel_spacing=13.9, heading=-167.0):
    """first_valid / last_valid: [n_bursts][lines_per_burst] ints (default:
    every line valid over the whole burst width)."""
    nb, L, W = info.n_bursts, info.lines_per_burst, info.samples_per_burst
    if first_valid is None:
        first_valid = np.zeros((nb, L), int)
    if last_valid is None:
        last_valid = np.full((nb, L), W - 1, int)
    if radar_frequency is None:
        radar_frequency = 299792458.0 / info.wavelength
    x = []
    x.append('<?xml version="1.0" encoding="UTF-8"?>')
    x.append("<product>")
    x.append(f"  <adsHeader><polarisation>{polarisation}</polarisation></adsHeader>")
    x.append("  <generalAnnotation>")
    x.append("    <productInformation>")
    x.append(f"      <radarFrequency>{g17(radar_frequency)}</radarFrequency>")
    x.append(f"      <rangeSamplingRate>{g17(info.rsr)}</rangeSamplingRate>")
    x.append(f"      <azimuthSteeringRate>{g17(info.steering_rate_deg)}</azimuthSteeringRate>")
    x.append(f"      <platformHeading>{g17(heading)}</platformHeading>")
    x.append("    </productInformation>")
    x.append(f'    <azimuthFmRateList count="{info.n_fm}">')
    for k in range(info.n_fm):
        f = info.fm_list[k]
        x.append("      <azimuthFmRate>")
        x.append(f"        <azimuthTime>{utc(f.aztime, date)}</azimuthTime>")
        x.append(f"        <t0>{g17(f.t0)}</t0>")
        if fm_as_polynomial:
            x.append(f'        <azimuthFmRatePolynomial count="3">{g17(f.c0)} {g17(f.c1)} '
                     f"{g17(f.c2)}</azimuthFmRatePolynomial>")
        else:
            x.append(f"        <c0>{g17(f.c0)}</c0><c1>{g17(f.c1)}</c1><c2>{g17(f.c2)}</c2>")
        x.append("      </azimuthFmRate>")
    x.append("    </azimuthFmRateList>")
    x.append("  </generalAnnotation>")
    x.append("  <imageAnnotation>")
    x.append("    <imageInformation>")
    x.append(f"      <productFirstLineUtcTime>{utc(info.first_line_time, date)}"
             "</productFirstLineUtcTime>")
    x.append(f"      <productLastLineUtcTime>{utc(info.last_line_time, date)}"
             "</productLastLineUtcTime>")
    x.append(f"      <ascendingNodeTime>{utc(info.first_line_time - 1200.0, date)}"
             "</ascendingNodeTime>")
    x.append(f"      <slantRangeTime>{g17(2.0 * info.slr_time)}</slantRangeTime>")
    x.append(f"      <rangePixelSpacing>{g17(info.range_spacing)}</rangePixelSpacing>")
    x.append(f"      <azimuthPixelSpacing>{g17(azimuth_pixel_spacing)}</azimuthPixelSpacing>")
    x.append(f"      <azimuthTimeInterval>{g17(info.dt)}</azimuthTimeInterval>")
    x.append(f"      <numberOfSamples>{W}</numberOfSamples>")
    x.append(f"      <numberOfLines>{nb * L}</numberOfLines>")
    x.append("    </imageInformation>")
    x.append("    <processingInformation>")
    x.append(f"      <dcMethod>{dc_method}</dcMethod>")
    x.append("      <swathProcParamsList count=\"1\"><swathProcParams>")
    x.append(f"        <rangeProcessing><processingBandwidth>{g17(range_bandwidth)}"
             "</processingBandwidth></rangeProcessing>")
    x.append(f"        <azimuthProcessing><processingBandwidth>{g17(info.az_bandwidth)}"
             "</processingBandwidth></azimuthProcessing>")
    x.append("      </swathProcParams></swathProcParamsList>")
    x.append("    </processingInformation>")
    x.append("  </imageAnnotation>")
    x.append("  <dopplerCentroid>")
    x.append(f'    <dcEstimateList count="{info.n_dc}">')
    for k in range(info.n_dc):
        d = info.dc_list[k]
        # the polynomial the reader must not take is offset, so a wrong
        # choice shows
        other = (d.c0 + 100.0, d.c1, d.c2)
        data, geom = ((d.c0, d.c1, d.c2), other) if dc_method == "Data Analysis" else \
            (other, (d.c0, d.c1, d.c2))
        x.append("      <dcEstimate>")
        x.append(f"        <azimuthTime>{utc(d.aztime, date)}</azimuthTime>")
        x.append(f"        <t0>{g17(d.t0)}</t0>")
        x.append('        <geometryDcPolynomial count="3">' + " ".join(g17(v) for v in geom) +
                 "</geometryDcPolynomial>")
        x.append('        <dataDcPolynomial count="3">' + " ".join(g17(v) for v in data) +
                 "</dataDcPolynomial>")
        x.append("      </dcEstimate>")
    x.append("    </dcEstimateList>")
    x.append("  </dopplerCentroid>")
    x.append("  <swathTiming>")
    x.append(f"    <linesPerBurst>{L}</linesPerBurst>")
    x.append(f"    <samplesPerBurst>{W}</samplesPerBurst>")
    x.append(f'    <burstList count="{nb}">')
    for b in range(nb):
        x.append("      <burst>")
        x.append(f"        <azimuthTime>{utc(info.burst_first_line_time[b], date)}</azimuthTime>")
        x.append(f'        <firstValidSample count="{L}">' +
                 " ".join(str(int(v)) for v in first_valid[b]) + "</firstValidSample>")
        x.append(f'        <lastValidSample count="{L}">' +
                 " ".join(str(int(v)) for v in last_valid[b]) + "</lastValidSample>")
        x.append("      </burst>")
    x.append("    </burstList>")
    x.append("  </swathTiming>")
    x.append("  <geolocationGrid>")
    n = grid["az_time"].size
    x.append(f'    <geolocationGridPointList count="{n}">')
    for i in range(grid["az_time"].shape[0]):
        for j in range(grid["az_time"].shape[1]):
            x.append("      <geolocationGridPoint>")
            x.append(f"        <azimuthTime>{utc(grid['az_time'][i, j], date)}</azimuthTime>")
            x.append(f"        <slantRangeTime>{g17(2.0 * grid['slr_time'][i, j])}"
                     "</slantRangeTime>")
            x.append(f"        <line>{int(grid['line'][i, j])}</line><pixel>{j}</pixel>")
            x.append(f"        <latitude>{g17(grid['lat'][i, j])}</latitude>")
            x.append(f"        <longitude>{g17(grid['lon'][i, j])}</longitude>")
            x.append("        <height>0</height>")
            x.append(f"        <incidenceAngle>{g17(grid['incidence'][i, j])}</incidenceAngle>")
            x.append("      </geolocationGridPoint>")
    x.append("    </geolocationGridPointList>")
    x.append("  </geolocationGrid>")
    x.append("</product>")
    with open(path, "w") as f:
        f.write("\n".join(x) + "\n")


def write_eof(path, t, xyz, vel, date=DATE):
    """A precise-orbit file: OSVs at times t (seconds of the day, whole
    seconds as in the real files), positions and velocities [n][3]."""
    x = ['<?xml version="1.0" ?>', "<Earth_Explorer_File>",
         "  <Earth_Explorer_Header><Fixed_Header><Mission>Sentinel-1A</Mission></Fixed_Header>"
         "</Earth_Explorer_Header>", "  <Data_Block type=\"xml\">",
         f'    <List_of_OSVs count="{len(t)}">']
    for i in range(len(t)):
        x.append("      <OSV>")
        x.append(f"        <TAI>TAI={utc(t[i] + 37.0, date, 6)}</TAI>")
        x.append(f"        <UTC>UTC={utc(t[i], date, 6)}</UTC>")
        x.append("        <Absolute_Orbit>+38000</Absolute_Orbit>")
        for k, ax in enumerate("XYZ"):
            x.append(f'        <{ax} unit="m">{xyz[i][k]:.6f}</{ax}>')
        for k, ax in enumerate(("VX", "VY", "VZ")):
            x.append(f'        <{ax} unit="m/s">{vel[i][k]:.6f}</{ax}>')
        x.append("        <Quality>NOMINAL</Quality>")
        x.append("      </OSV>")
    x += ["    </List_of_OSVs>", "  </Data_Block>", "</Earth_Explorer_File>"]
    with open(path, "w") as f:
        f.write("\n".join(x) + "\n")
