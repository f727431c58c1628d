"""Parity metrics between the GPU path and the oracles.

Tolerances (from the acceptance criteria of this port):
  * surface elevation: max |d eta| <= 1e-3 m over cells wet in both results;
  * maximum height: relative L2 <= 1e-4 over cells wet in both results.
Snapshots are only compared when their recorded times agree (a time-step
difference can move a snapshot by one whole step; the reference does not
truncate the last step to the save time).
"""
from __future__ import annotations

import numpy as np

ETA_TOL_M = 1e-3
MAXH_REL_L2 = 1e-4
FILL = -9999.0


def wet_both(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return (a != FILL) & (b != FILL)


def max_abs_eta(a: np.ndarray, b: np.ndarray) -> float:
    m = wet_both(a, b)
    if not m.any():
        return 0.0
    return float(np.abs(a[m].astype(np.float64) - b[m].astype(np.float64)).max())


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    m = wet_both(a, b)
    ref = b[m].astype(np.float64)
    den = float(np.sqrt((ref ** 2).sum()))
    num = float(np.sqrt(((a[m].astype(np.float64) - ref) ** 2).sum()))
    return num / den if den > 0 else num


def wet_mismatch(a: np.ndarray, b: np.ndarray) -> int:
    """cells wet in one result and dry in the other"""
    return int(((a == FILL) != (b == FILL)).sum())


def compare(gpu: dict, ref: dict, label: str = "") -> dict:
    """Returns the parity figures of a GPU run against an oracle run."""
    out = {
        "label": label,
        "maxh_rel_l2": rel_l2(gpu["max_height"], ref["max_height"]),
        "eta_final_max_abs": max_abs_eta(gpu["eta"], ref["eta"]),
        "wet_mismatch_final": wet_mismatch(gpu["eta"], ref["eta"]),
        "iterations": (int(gpu["iterations"]), int(ref["iterations"])),
        "final_time": (float(gpu["final_time"]), float(ref["final_time"])),
    }
    gs, rs = gpu.get("snapshots"), ref.get("snapshots")
    if gs is not None and rs is not None and len(gs["time"]) and len(rs["time"]):
        n = min(len(gs["time"]), len(rs["time"]))
        worst = 0.0
        for i in range(n):
            if abs(float(gs["time"][i]) - float(rs["time"][i])) > 1e-3:
                continue
            worst = max(worst, max_abs_eta(gs["eta"][i], rs["eta"][i]))
        out["eta_snap_max_abs"] = worst
        out["snap_times"] = (list(map(float, gs["time"][:n])), list(map(float, rs["time"][:n])))
    return out
