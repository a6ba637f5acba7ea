"""Helpers comparing the CUDA library's particle state with the oracle's,
matched by original particle index."""
from __future__ import annotations

import numpy as np

COMPARED = ("position", "velocity", "F", "B", "damage", "alpha", "psi_max", "stress", "volume", "FP", "pf_flux")


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return float(num / den) if den > 0 else float(num)


def errors(G, gpu, orc, x0: np.ndarray, fields=COMPARED, dx: float | None = None) -> dict:
    """Relative L2 error per field (positions as displacement from x0).  With
    dx given, also 'position_dx': the largest position difference in grid
    cells, which stays meaningful when displacements are tiny."""
    out = {}
    for f in fields:
        a = gpu.read(f, order=G.ORDER_ORIGINAL)
        b = orc.field_by_id(G.FIELD[f])
        if f == "position":
            if dx is not None:
                out["position_dx"] = float(np.abs(a - b).max() / dx)
            a, b = a - x0, b - x0
        out[f] = rel_l2(a, b)
    return out


def format_errors(e: dict) -> str:
    return " ".join(f"{k}={v:.2e}" for k, v in e.items())
