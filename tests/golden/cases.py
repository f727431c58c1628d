"""The seeded problems behind the golden fixtures (small enough for the
FP64 oracle to finish in about a second each)."""
import numpy as np

from thysea import synth


def _plain():
    return synth.plain_small(nx=96, ny=80, sim_time=240.0, save_time=120.0, series_time=30.0, npoints=6)


def _shelf():
    p = synth.single_large(n=112, seed=21, sim_time=600.0, save_time=300.0, npoints=5)
    p.name = "shelf"
    return p


def _walls_crop():
    p = synth.single_large(n=96, seed=22, sim_time=400.0, save_time=200.0)
    p.name = "walls"
    p.borders = (-1.0, -1.0, -1.0, -1.0)
    p.crop_flag, p.crop_value = 1, 5e-3
    return p


def _periodic():
    p = synth.single_large(n=96, seed=23, sim_time=400.0, save_time=200.0)
    p.name = "periodic"
    p.borders = (1.0, -1.0, 2.0, 2.0)
    p.crop_flag, p.crop_value = 2, 0.05
    return p


def _two_faults():
    p = synth.plain_small(nx=90, ny=72, sim_time=300.0, save_time=100.0, npoints=3, series_time=50.0)
    p.name = "twofault"
    f0 = p.faults[0]
    p.faults = [synth.Fault(120.0, f0.lon + 0.2, f0.lat + 0.1, 12.0, 60.0, 30.0, 45.0, 20.0, 80.0, 3.0), f0]
    return p


def _from_file():
    p = synth.plain_small(nx=80, ny=64, sim_time=200.0, save_time=100.0, npoints=0)
    p.name = "fromfile"
    p.faults = []
    yy, xx = np.mgrid[0:64, 0:80]
    p.eta_init = (2.0 * np.exp(-((xx - 30) ** 2 + (yy - 30) ** 2) / 40.0)).astype(np.float32)
    return p


CASES = {
    "plain": _plain,
    "shelf": _shelf,
    "walls": _walls_crop,
    "periodic": _periodic,
    "twofault": _two_faults,
    "fromfile": _from_file,
}
