"""Seeded synthetic inputs for the Tsunami-HySEA time stepper.

The reference ships no usable input grid (its only example bathymetry is
missing), so every workload here is synthetic and seeded:

* ``plain_small``   512 x 512 cells, 1 arc-min, linear eastern shelf, one
  Okada fault, 600 s (the reference's CPU-runnable case);
* ``single_large``  4096 x 4096 cells, Gaussian-random-field bathymetry with a
  shelf and coastline (~10 % dry), four contiguous subfaults, 3600 s;
* ``batch_uniform`` 64 scenarios sharing one 2048 x 2048 bathymetry, one
  random fault each, 1800 s;
* ``mixed``         32 scenarios with log-uniform sides in [256, 4096], own
  bathymetry and fault, 600-7200 s;
* ``serving``       a Poisson request stream (2 req/s) of ``mixed``-style
  scenarios.

A :class:`Problem` holds exactly what the reference's problem file
(src/Problema.cxx:176-343 grammar) and its GRD/points files carry, in the
same units: degrees, metres, seconds, the dimensionless scales L and H.
:func:`write_problem` writes the three files the reference's loader reads.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional, Sequence

import numpy as np

ARCMIN = 1.0 / 60.0
KM_PER_DEG = 111.19492664455873  # 6371.0088 km mean radius, only used to place faults


@dataclasses.dataclass
class Fault:
    """One Okada rectangular source, in the reference's problem-file order:
    time(s) lon lat depth(km, fault centroid) length(km) width(km) strike dip rake slip(m)."""

    time: float
    lon: float
    lat: float
    depth: float
    length: float
    width: float
    strike: float
    dip: float
    rake: float
    slip: float

    def as_row(self) -> List[float]:
        return [self.time, self.lon, self.lat, self.depth, self.length, self.width,
                self.strike, self.dip, self.rake, self.slip]


def centroid_depth(top_km: float, width_km: float, dip_deg: float) -> float:
    """Okada's reference depth here is the fault centroid (AW1=-W/2, AW2=+W/2);
    sources quoted by their top edge are converted with top + (W/2) sin(dip)."""
    return top_km + 0.5 * width_km * math.sin(math.radians(dip_deg))


@dataclasses.dataclass
class Problem:
    name: str
    lon: np.ndarray                 # (nx,) degrees, float64
    lat: np.ndarray                 # (ny,) degrees, float64
    z: np.ndarray                   # (ny, nx) topobathymetry, metres, positive up, float32
    faults: List[Fault] = dataclasses.field(default_factory=list)
    eta_init: Optional[np.ndarray] = None   # (ny, nx) initial sea surface (m) when not Okada
    crop_flag: int = 0
    crop_value: float = 0.0
    borders: Sequence[float] = (1.0, 1.0, 1.0, 1.0)   # upper, lower, left, right
    sim_time: float = 600.0
    save_time: float = -1.0
    points: Optional[np.ndarray] = None     # (n, 2) lon, lat
    series_time: float = -1.0
    cfl: float = 0.5
    eps_h: float = 5e-3
    hpos: float = 20.0
    stability: float = 0.2
    manning: float = 0.03
    vmax: float = 100.0
    L: float = 1e5
    H: float = 1e3
    dif_at: float = 1e-6

    @property
    def nx(self) -> int:
        return int(self.lon.shape[0])

    @property
    def ny(self) -> int:
        return int(self.lat.shape[0])

    @property
    def cells(self) -> int:
        return self.nx * self.ny

    def fault_array(self) -> np.ndarray:
        return np.asarray([f.as_row() for f in self.faults], dtype=np.float64).reshape(-1, 10)


# ---------------------------------------------------------------------------
# grids and bathymetry
# ---------------------------------------------------------------------------

def lonlat_grid(nx: int, ny: int, spacing_deg: float = ARCMIN, lon0: float = 0.0, lat_centre: float = 0.0):
    lon = lon0 + spacing_deg * np.arange(nx, dtype=np.float64)
    lat = lat_centre + spacing_deg * (np.arange(ny, dtype=np.float64) - 0.5 * (ny - 1))
    return lon, lat


def gaussian_random_field(nx: int, ny: int, corr_cells: float, rng: np.random.Generator) -> np.ndarray:
    """Unit-variance Gaussian random field with a Gaussian covariance of
    correlation length ``corr_cells`` (FFT filtering of white noise)."""
    noise = rng.standard_normal((ny, nx))
    kx = np.fft.rfftfreq(nx)
    ky = np.fft.fftfreq(ny)
    k2 = ky[:, None] ** 2 + kx[None, :] ** 2
    filt = np.exp(-2.0 * (math.pi * corr_cells) ** 2 * k2)
    field = np.fft.irfft2(np.fft.rfft2(noise) * filt, s=(ny, nx))
    field -= field.mean()
    std = field.std()
    return field / (std if std > 0 else 1.0)


def shelf_bathymetry(nx: int, ny: int, rng: np.random.Generator, dry_fraction: float = 0.10,
                     corr_cells: float = 50.0, mean: float = -3000.0, std: float = 800.0) -> np.ndarray:
    """Random-field ocean (mean, std, clipped to [-7000, -50] m) that rises over
    the eastern quarter to a coastline; the land height is tuned by bisection
    so that about ``dry_fraction`` of the cells are above sea level."""
    field = mean + std * gaussian_random_field(nx, ny, min(corr_cells, max(nx, ny) / 4.0), rng)
    field = np.clip(field, -7000.0, -50.0)
    s = np.clip((np.arange(nx) / max(nx - 1, 1) - 0.75) / 0.25, 0.0, 1.0)[None, :]
    lo, hi = 0.0, 20000.0
    z = field
    for _ in range(40):
        land = 0.5 * (lo + hi)
        z = field * (1.0 - s) + s * land
        frac = float((z > 0).mean())
        if frac < dry_fraction:
            lo = land
        else:
            hi = land
    return z.astype(np.float32)


# ---------------------------------------------------------------------------
# the benchmark workloads
# ---------------------------------------------------------------------------

def seeded_points(lon, lat, z, n: int, rng: np.random.Generator) -> np.ndarray:
    """n distinct time-series gauges at random ocean cell centres."""
    ocean = np.argwhere(z < -100.0)
    pick = ocean[rng.choice(len(ocean), size=min(n, len(ocean)), replace=False)]
    return np.stack([lon[pick[:, 1]], lat[pick[:, 0]]], axis=1)


def plain_small(nx: int = 512, ny: int = 512, seed: int = 1, sim_time: float = 600.0,
                save_time: float = 300.0, series_time: float = 60.0, npoints: int = 16) -> Problem:
    """Plain small problem: linear eastern shelf to +200 m land, -4000 m ocean, sigma 20 m
    noise, one Okada fault (100 x 50 km, 5 m slip, strike 0, dip 15, rake 90,
    top 10 km) centred at 30 % of the width."""
    rng = np.random.default_rng(seed)
    lon, lat = lonlat_grid(nx, ny)
    x = np.arange(nx)
    x0 = int(round(0.85 * nx))
    prof = np.full(nx, -4000.0)
    ramp = x >= x0
    prof[ramp] = -4000.0 + (x[ramp] - x0) * (4200.0 / max(nx - 1 - x0, 1))
    z = (prof[None, :] + rng.normal(0.0, 20.0, size=(ny, nx))).astype(np.float32)
    flt = Fault(0.0, float(lon[0] + 0.3 * (lon[-1] - lon[0])), float(0.5 * (lat[0] + lat[-1])),
                centroid_depth(10.0, 50.0, 15.0), 100.0, 50.0, 0.0, 15.0, 90.0, 5.0)
    pts = seeded_points(lon, lat, z, npoints, rng) if npoints > 0 else None
    return Problem(name="plain_small", lon=lon, lat=lat, z=z, faults=[flt], sim_time=sim_time,
                   save_time=save_time, points=pts, series_time=series_time if npoints > 0 else -1.0)


def single_large(n: int = 4096, seed: int = 2, sim_time: float = 3600.0, save_time: float = -1.0,
                 npoints: int = 0) -> Problem:
    """Single large scenario: random-field bathymetry with shelf and ~10 % dry cells; four
    contiguous 100 x 50 km subfaults along strike 0 (dip 15, rake 90, top
    10 km), slip U(2, 8) m."""
    rng = np.random.default_rng(seed)
    lon, lat = lonlat_grid(n, n)
    z = shelf_bathymetry(n, n, rng)
    lon_c = float(lon[0] + 0.45 * (lon[-1] - lon[0]))
    lat_mid = float(0.5 * (lat[0] + lat[-1]))
    faults = []
    for i in range(4):
        lat_c = lat_mid + (i - 1.5) * 100.0 / KM_PER_DEG
        faults.append(Fault(0.0, lon_c, lat_c, centroid_depth(10.0, 50.0, 15.0), 100.0, 50.0,
                            0.0, 15.0, 90.0, float(rng.uniform(2.0, 8.0))))
    pts = seeded_points(lon, lat, z, npoints, rng) if npoints > 0 else None
    return Problem(name="single_large", lon=lon, lat=lat, z=z, faults=faults, sim_time=sim_time,
                   save_time=save_time, points=pts, series_time=60.0 if npoints > 0 else -1.0)


def random_fault(lon, lat, z, rng: np.random.Generator, time: float = 0.0) -> Fault:
    """One fault as in the batched configs: L~U(50,300) km, W=L/2, slip U(1,10) m,
    strike U(0,360), dip U(10,30), top U(5,20) km, rake 90, centred on a
    random ocean cell."""
    L = float(rng.uniform(50.0, 300.0))
    W = 0.5 * L
    dip = float(rng.uniform(10.0, 30.0))
    top = float(rng.uniform(5.0, 20.0))
    ocean = np.argwhere(z < 0.0)
    j, i = ocean[rng.integers(len(ocean))]
    return Fault(time, float(lon[i]), float(lat[j]), centroid_depth(top, W, dip), L, W,
                 float(rng.uniform(0.0, 360.0)), dip, 90.0, float(rng.uniform(1.0, 10.0)))


def batch_uniform(count: int = 64, n: int = 2048, seed: int = 3, sim_time: float = 1800.0) -> List[Problem]:
    """Uniform batch: ``count`` scenarios on one shared random-field bathymetry."""
    rng = np.random.default_rng(seed)
    lon, lat = lonlat_grid(n, n)
    z = shelf_bathymetry(n, n, rng)
    out = []
    for k in range(count):
        out.append(Problem(name=f"batch_{k:03d}", lon=lon, lat=lat, z=z,
                           faults=[random_fault(lon, lat, z, rng)], sim_time=sim_time))
    return out


def mixed_scenario(rng: np.random.Generator, name: str, side_range=(256, 4096), time_range=(600.0, 7200.0)) -> Problem:
    side = int(round(math.exp(rng.uniform(math.log(side_range[0]), math.log(side_range[1])))))
    lon, lat = lonlat_grid(side, side)
    z = shelf_bathymetry(side, side, rng)
    return Problem(name=name, lon=lon, lat=lat, z=z, faults=[random_fault(lon, lat, z, rng)],
                   sim_time=float(rng.uniform(*time_range)))


def mixed(count: int = 32, seed: int = 4, side_range=(256, 4096), time_range=(600.0, 7200.0)) -> List[Problem]:
    """Mixed-size batch: log-uniform sides, own bathymetry, one fault, U(600, 7200) s."""
    rng = np.random.default_rng(seed)
    return [mixed_scenario(rng, f"mixed_{k:03d}", side_range, time_range) for k in range(count)]


def poisson_arrivals(rate: float = 2.0, duration: float = 600.0, seed: int = 5) -> np.ndarray:
    """Serving stream: arrival times (s) of a Poisson stream."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return np.asarray(out)
        out.append(t)


# ---------------------------------------------------------------------------
# files in the reference's formats
# ---------------------------------------------------------------------------

def write_grd(path: str, lon: np.ndarray, lat: np.ndarray, z: np.ndarray) -> None:
    """GRD input: dims lon/lat, double lon/lat variables and float z[lat][lon]
    (the layout src/GPU/netcdfTH.cu:13-83 reads)."""
    from scipy.io import netcdf_file

    with netcdf_file(path, "w", version=2) as f:
        f.createDimension("lon", lon.shape[0])
        f.createDimension("lat", lat.shape[0])
        vx = f.createVariable("lon", "d", ("lon",))
        vx[:] = lon
        vy = f.createVariable("lat", "d", ("lat",))
        vy[:] = lat
        vz = f.createVariable("z", "f", ("lat", "lon"))
        vz[:] = z.astype(np.float32)


def write_problem(p: Problem, directory: str, prefix: Optional[str] = None) -> str:
    """Writes <name>.grd, the points file and the problem .txt in the grammar
    of src/Problema.cxx:219-343 (one value per non-comment line).  The NetCDF
    output prefix is an absolute path inside ``directory`` unless given."""
    os.makedirs(directory, exist_ok=True)
    grd = f"{p.name}.grd"
    write_grd(os.path.join(directory, grd), p.lon, p.lat, p.z)
    lines = [f"{p.name}    # Problem name", f"{grd}    # Bathymetry file"]
    if p.faults:
        lines.append("1    # Initialization type (0: from file, 1: standard Okada)")
        lines.append(f"{len(p.faults)}    # Number of faults")
        for flt in p.faults:
            lines.append(" ".join(repr(float(v)) for v in flt.as_row()) +
                         "  # Time(s) Lon Lat Depth(km) Length(km) Width(km) Strike Dip Rake Slip(m)")
        lines.append(f"{p.crop_flag}    # Crop deformations")
        if p.crop_flag in (1, 2):
            lines.append(f"{p.crop_value!r}    # crop value")
    else:
        est = f"{p.name}_eta.grd"
        write_grd(os.path.join(directory, est), p.lon, p.lat,
                  np.zeros_like(p.z) if p.eta_init is None else p.eta_init)
        lines.append("0    # Initialization type (0: from file, 1: standard Okada)")
        lines.append(f"{est}    # Initial state file")
    out_prefix = prefix if prefix is not None else os.path.join(os.path.abspath(directory), p.name)
    lines.append(f"{out_prefix}    # NetCDF file prefix")
    lines.append("1    # Number of levels")
    b = list(p.borders)
    lines += [f"{b[0]!r}    # Upper border", f"{b[1]!r}    # Lower border",
              f"{b[2]!r}    # Left border", f"{b[3]!r}    # Right border"]
    lines.append(f"{p.sim_time!r}    # Simulation time (sec)")
    lines.append(f"{p.save_time!r}    # Saving time of NetCDF files (sec)")
    if p.points is not None and len(p.points) > 0:
        pts = f"{p.name}_points.txt"
        with open(os.path.join(directory, pts), "w") as fh:
            fh.write(f"{len(p.points)}\n")
            for lo, la in p.points:
                fh.write(f"{float(lo)!r} {float(la)!r}\n")
        lines.append("1    # Read points from file")
        lines.append(f"{pts}    # File with points")
        lines.append(f"{p.series_time!r}    # Saving time of time series (sec)")
    else:
        lines.append("0    # Read points from file")
    lines += [f"{p.cfl!r}    # CFL", f"{p.eps_h!r}    # Epsilon h (m)", f"{p.hpos!r}    # Threshold 2s+WAF (m)",
              f"{p.stability!r}    # Stability coefficient", f"{p.manning!r}    # Manning",
              f"{p.vmax!r}    # Maximum velocity", f"{p.L!r}    # L", f"{p.H!r}    # H",
              f"{p.dif_at!r}    # Threshold for arrival times (m)"]
    txt = os.path.join(directory, f"{p.name}.txt")
    with open(txt, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return txt
