"""thy_apply_okada_noalloc: the Okada stage for callers that cannot allocate
device memory (their GPU memory belongs to a caching or budgeted allocator,
or a cudaMalloc's implicit device-wide synchronisation is not allowed where
they run).  It must give exactly what thy_apply_okada gives on the same
inputs, call after call, although its scratch is a fixed array inside the
library that keeps the previous call's contents.

This file is collected last on purpose: it also passes when run alone in a
fresh process.
"""
import ctypes

import numpy as np
import pytest

from thysea import _ffi

pytestmark = pytest.mark.gpu

TOL = 1e-12   # the Okada-stage tolerance of the other GPU tests (FP64)
MAX_CELLS = 1 << 20   # THY_OKADA_NOALLOC_MAX_CELLS


def _inputs(nx, ny, seed):
    rng = np.random.default_rng(seed)
    Hs = rng.uniform(0.5, 6.0, size=(ny, nx))
    h = np.maximum(Hs - 0.3, 0.0)
    return np.stack([h.ravel(), Hs.ravel()], axis=1)


def _call(fn, nx, ny, fault, crop_flag, crop_value, state, with_eta=True, stream=None):
    import torch

    dev = torch.from_numpy(state.copy()).cuda()
    eta = torch.zeros(nx * ny, dtype=torch.float64, device="cuda") if with_eta else None
    f = np.asarray(fault, np.float64)
    rc = fn(nx, ny, 9.0, 1.0 / 60.0, 3.5, 1.0 / 60.0, f.ctypes.data_as(_ffi.f64p), 1000.0, crop_flag, crop_value,
            ctypes.c_void_p(dev.data_ptr()), None if eta is None else ctypes.c_void_p(eta.data_ptr()), stream)
    torch.cuda.synchronize()
    return rc, dev.cpu().numpy(), (None if eta is None else eta.cpu().numpy())


# (fault, crop flag, crop value, seed, eta_initial passed): different faults
# one after the other, so that a call cannot pass on a stale deformation
# field or cropping maximum of the call before it
CASES = [
    ([0.0, 13.0, 7.0, 16.47, 100.0, 50.0, 33.0, 15.0, 90.0, 5.0], 1, 5e-3, 1, True),    # relative crop
    ([0.0, 12.6, 6.9, 9.0, 40.0, 20.0, 200.0, 60.0, 30.0, 0.5], 1, 2e-2, 2, True),      # relative crop
    ([0.0, 13.4, 7.4, 12.0, 80.0, 40.0, 120.0, 25.0, 70.0, 3.0], 0, 0.0, 3, True),      # no crop
    ([0.0, 12.9, 7.1, 20.0, 120.0, 60.0, 300.0, 20.0, 110.0, 8.0], 2, 1e-4, 4, True),   # absolute crop
    ([0.0, 13.1, 6.8, 15.0, 60.0, 30.0, 45.0, 35.0, 90.0, 2.0], 2, 5e-5, 5, False),     # no eta_initial
]


def test_noalloc_matches_allocating_entry_point_twice_in_a_row():
    L = _ffi.lib()
    nx, ny = 640, 480
    for rnd in range(2):
        for fault, cf, cv, seed, with_eta in CASES:
            st = _inputs(nx, ny, seed)
            rc_a, out_a, eta_a = _call(L.thy_apply_okada, nx, ny, fault, cf, cv, st, with_eta)
            rc_b, out_b, eta_b = _call(L.thy_apply_okada_noalloc, nx, ny, fault, cf, cv, st, with_eta)
            assert rc_a == 0 and rc_b == 0, (rnd, fault)
            assert np.abs(out_b - out_a).max() <= TOL
            assert np.abs(out_a[:, 1] - st[:, 1]).max() > 1e-4   # the bathymetry was deformed
            if with_eta:
                assert np.abs(eta_b - eta_a).max() <= TOL
                assert np.abs(eta_a).max() > 1e-4
            if cf:
                # cropping zeroed part of the deformation
                assert (np.abs(out_a[:, 1] - st[:, 1]) == 0).any()


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    L = _ffi.lib()
    nx = ny = 1025   # 1050625 cells > THY_OKADA_NOALLOC_MAX_CELLS
    assert nx * ny > MAX_CELLS
    # a real device buffer of the full grid's size, so that nothing could
    # write out of bounds of the state even if the size check were gone
    state = torch.zeros((nx * ny, 2), dtype=torch.float64, device="cuda")
    eta = torch.zeros(nx * ny, dtype=torch.float64, device="cuda")
    f = np.asarray([0.0, 10.0, 5.0, 10.0, 50.0, 25.0, 0.0, 15.0, 90.0, 1.0])
    rc = L.thy_apply_okada_noalloc(nx, ny, 9.0, 0.01, 3.5, 0.01, f.ctypes.data_as(_ffi.f64p), 1000.0, 0, 0.0,
                                   ctypes.c_void_p(state.data_ptr()), ctypes.c_void_p(eta.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == 9   # THY_ERR_TOO_LARGE, before touching any memory
    assert b"maximum" in L.thy_strerror(rc)
    assert float(state.abs().max()) == 0.0 and float(eta.abs().max()) == 0.0
