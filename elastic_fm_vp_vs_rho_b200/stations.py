"""Real-station geometry: latitude/longitude -> grid cells.

Restates LecturaEstacionesSismologicasProyecto/lecturaEstacionesSismologicasProyecto.py
(the DMS parsing and the flat-earth projection about a reference corner) and the driver's
use of its output (mainPropElastic3D_MT.py:2868-2878: positions stored on a 1 km grid,
rescaled to the model's spacing).  Host-side setup, no device work.
"""
from __future__ import annotations

import math
import re

import numpy as np

EARTH_DIAMETER_KM = 12756.320
REF_LAT = 6.0
REF_LON = -74.0

_DMS = re.compile(r"(\d+(?:\.\d*)?)\s*°\s*(\d+(?:\.\d*)?)\s*'\s*(\d+(?:\.\d*)?)\s*\"\s*([NSEW])")


def parse_dms(text: str) -> float:
    """One 'D° M' S.sss" H' coordinate -> decimal degrees (S and W negative)."""
    m = _DMS.search(text)
    if m is None:
        raise ValueError(f"not a D M S coordinate: {text!r}")
    d, mi, se, h = float(m.group(1)), float(m.group(2)), float(m.group(3)), m.group(4)
    v = d + mi / 60.0 + se / 3600.0
    return -v if h in "SW" else v


def parse_dms_list(block: str) -> np.ndarray:
    """Every D M S coordinate of a multi-line block, in order."""
    return np.array([parse_dms(line) for line in block.splitlines() if line.strip()], np.float64)


def latlon_to_grid(lat, lon, cell_km=1.0, ref_lat=REF_LAT, ref_lon=REF_LON,
                   earth_d_km=EARTH_DIAMETER_KM):
    """Grid (x, y, z) cells of stations: x east of ref_lon along the reference latitude's
    parallel, y north of ref_lat (the script's projection, truncated toward zero like
    numpy's astype(int)); z = 1."""
    lat = np.asarray(lat, np.float64)
    lon = np.asarray(lon, np.float64)
    x = ((lon - ref_lon) * earth_d_km * math.pi * np.cos(math.radians(ref_lat)) / 360.0) / cell_km
    y = ((lat - ref_lat) * earth_d_km * math.pi / 360.0) / cell_km
    return x.astype(int), y.astype(int), np.ones(len(x))


def rescale(pos, dx, stored_spacing_m=2e3):
    """Positions stored on one grid rescaled to spacing dx, as the driver loads them
    ((load(...) / (2e3 / dx)).astype(int), mainPropElastic3D_MT.py:2868-2875)."""
    return (np.asarray(pos) / (stored_spacing_m / dx)).astype(int)


def receivers_from_npy(path_x, path_y, dx, z=2, stored_spacing_m=2e3):
    """(nrec, 3) int32 receiver cells from the station .npy files, at depth index z."""
    x = rescale(np.load(path_x), dx, stored_spacing_m)
    y = rescale(np.load(path_y), dx, stored_spacing_m)
    return np.stack([x, y, np.full(len(x), z)], axis=1).astype(np.int32)


def subset_inside(rec, nx, ny, nz, lenpml):
    """Receivers that fall inside the non-absorbing part of an (ny, nz, nx) grid."""
    rec = np.asarray(rec)
    ok = ((rec[:, 0] >= lenpml) & (rec[:, 0] < nx - lenpml) & (rec[:, 1] >= lenpml)
          & (rec[:, 1] < ny - lenpml) & (rec[:, 2] >= 0) & (rec[:, 2] < nz))
    return rec[ok]
