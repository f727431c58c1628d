"""thy_apply_okada (the Okada stage alone, on device memory in the
reference's double2 (h, H) layout) against the FP64 oracle's Okada."""
import ctypes

import numpy as np
import pytest

import oracle
from thysea import _ffi

pytestmark = pytest.mark.gpu

FAULTS = [
    [0.0, 10.3, 5.1, 16.47, 100.0, 50.0, 33.0, 15.0, 90.0, 5.0],
    [0.0, 10.6, 4.9, 12.0, 80.0, 40.0, 200.0, 60.0, 30.0, 2.0],
    [0.0, 10.0, 5.2, 8.0, 50.0, 25.0, 10.0, 90.0, 90.0, 2.0],
]


def okada_case(fault, crop_flag, crop_value, nx=300, ny=220):
    import torch

    lon0, lat0, d = 9.0, 3.5, 1.0 / 60.0
    rng = np.random.default_rng(4)
    Hs = rng.uniform(0.5, 6.0, size=(ny, nx))
    h = np.maximum(Hs - 0.3, 0.0)
    state = np.stack([h.ravel(), Hs.ravel()], axis=1)
    dev = torch.from_numpy(state.copy()).cuda()
    eta0 = torch.zeros(nx * ny, dtype=torch.float64, device="cuda")
    f = np.asarray(fault, np.float64)
    rc = _ffi.lib().thy_apply_okada(nx, ny, lon0, d, lat0, d, f.ctypes.data_as(_ffi.f64p), 1000.0, crop_flag,
                                    crop_value, ctypes.c_void_p(dev.data_ptr()), ctypes.c_void_p(eta0.data_ptr()),
                                    None)
    assert rc == 0
    torch.cuda.synchronize()
    jj, ii = np.mgrid[0:ny, 0:nx]
    U = oracle.oracle_okada_points((lon0 + ii * d).ravel(), (lat0 + jj * d).ravel(), f) / 1000.0
    if crop_flag == 1:
        thr = crop_value * float(np.abs(U).astype(np.float32).max())
        U = np.where(np.abs(U) < thr, 0.0, U)
    elif crop_flag == 2:
        U = np.where(np.abs(U) < crop_value, 0.0, U)
    out = dev.cpu().numpy()
    return out, eta0.cpu().numpy(), state, U


@pytest.mark.parametrize("k", range(len(FAULTS)))
@pytest.mark.parametrize("crop", [(0, 0.0), (1, 5e-3), (2, 1e-4)])
def test_apply_okada_matches_oracle(k, crop):
    out, eta, state, U = okada_case(FAULTS[k], *crop)
    assert np.array_equal(out[:, 0], state[:, 0])          # h unchanged
    assert np.abs(out[:, 1] - (state[:, 1] - U)).max() < 1e-12
    assert np.abs(eta - U).max() < 1e-12
    assert np.abs(U).max() > 1e-4                          # a real deformation
