"""Tile origin of a grid (kernels/kernels.h tile_origin) on the host.

Tile column tx starts at grid column x_org + 112 tx.  Tiles within two cells
of the left or right boundary (or reaching into a sponge layer) take the
general kernel, one warp per 28-column strip that holds a cell; the origin
shifts the tiling left by a multiple of 4 columns so that those tiles hold as
few strips as possible.  The deep kernels' boxes start at x0 - 4 and x0, so
the origin must keep x0 a multiple of 4."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "tsunami-hysea_b200", "csrc")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
TILE, STRIP = 112, 28


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("origin") / "origin_driver")
    cmd = ["g++", "-std=c++17", "-O1", "-I" + CSRC, "-I" + os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "native", "origin_driver.cpp"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _origins(exe, cases):
    args = [str(int(v)) for c in cases for v in c]
    r = subprocess.run([exe] + args, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    return [int(v) for v in r.stdout.split()]


def _cost(nx, org, spl, spr):
    """general-kernel strips of one row of tiles with tile 0 at column org"""
    need_l, need_r = max(2, spl), max(2, spr)
    tiles = (nx - org + TILE - 1) // TILE
    cost = 0
    for t in range(tiles):
        x0 = org + t * TILE
        if x0 >= need_l and x0 + TILE <= nx - need_r:
            continue
        cost += sum(1 for k in range(TILE // STRIP) if x0 + STRIP * (k + 1) > 0 and x0 + STRIP * k < nx)
    return cost


def test_known_grids(driver):
    # 4096 = 36 x 112 + 64: tile 0 holds 56 columns (2 strips), the last
    # tile 8 (1 strip): 3 general strips a row of tiles instead of 4 + 3
    assert _origins(driver, [(4096, 0, 0, 0)]) == [-56]
    assert _cost(4096, -56, 0, 0) == 3 and _cost(4096, 0, 0, 0) == 7
    # 2048 = 18 x 112 + 32: 28 + 4 columns, one strip each (6 with origin 0)
    assert _origins(driver, [(2048, 0, 0, 0)]) == [-84]
    assert _cost(2048, -84, 0, 0) == 2 and _cost(2048, 0, 0, 0) == 6
    # 1024 = 9 x 112 + 16: 12 + 4 columns
    assert _origins(driver, [(1024, 0, 0, 0)]) == [-100]
    assert _cost(1024, -100, 0, 0) == 2


def test_periodic_and_narrow_grids_keep_origin_zero(driver):
    assert _origins(driver, [(4096, 1, 0, 0), (2048, 1, 4, 4), (227, 0, 0, 0), (128, 0, 0, 0), (64, 0, 0, 0)]) == [0] * 5


@pytest.mark.parametrize("spl,spr", [(0, 0), (4, 4), (20, 0), (0, 60), (150, 3)])
def test_origin_is_the_first_minimiser(driver, spl, spr):
    sizes = list(range(228, 1200, 7)) + [2047, 2048, 3000, 4095, 4096, 4097, 8192]
    got = _origins(driver, [(nx, 0, spl, spr) for nx in sizes])
    for nx, org in zip(sizes, got):
        assert org % 4 == 0 and -TILE < org <= 0, (nx, org)
        costs = [_cost(nx, o, spl, spr) for o in range(0, -TILE, -4)]
        assert _cost(nx, org, spl, spr) == min(costs), (nx, org)
        assert org == -4 * costs.index(min(costs)), (nx, org)
        # tile 0 holds at least 4 columns of the grid; the tiles cover it
        tiles = (nx - org + TILE - 1) // TILE
        assert TILE + org >= 4 and org + tiles * TILE >= nx and org + (tiles - 1) * TILE < nx
