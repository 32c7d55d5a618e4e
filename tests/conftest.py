import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def gpu_present() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def load_golden(name: str):
    """Returns (params, fixture dict) of tests/golden/<name>.npz."""
    from capaz_b200.simulation import default_params
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    pd = json.loads(str(d.pop("params")))
    p = default_params()
    for k, v in pd.items():
        setattr(p, k, v)
    return p, d


GOLDEN_2PH = ["g2_default_15x15x1", "g2_3d_pd0_12x10x7", "g2_3d_pd_12x10x7", "g2_planar_17x13x1",
              "g2_min_3x3x3"]
GOLDEN_3PH = ["g3_column_1x15x1", "g3_3d_9x8x6"]
GOLDEN_BL = ["gbl_planar_20x15x1", "gbl_3d_gravity_12x10x6"]
GOLDEN_ENERGY = ["ge_column_1x15x1", "ge_9x8x6", "ge_11x7x1"]
ENERGY_STATE = ["P_w", "S_w", "S_n", "P_n", "P_g", "T"]


def interior(a: np.ndarray) -> np.ndarray:
    """Cells where the reference runs roS/Newton (cpu.cpp:621) on grids with
    nx, ny >= 3 (and the nx == 1 three-phase column)."""
    zs = slice(None) if a.shape[0] == 1 else slice(1, -1)
    xs = slice(None) if a.shape[2] == 1 else slice(1, -1)
    return a[zs, 1:-1, xs]


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """Normwise relative error max|a-b| / max|b| (0 for identical arrays)."""
    d = np.abs(np.asarray(a, dtype=np.float64) - np.asarray(b, dtype=np.float64)).max()
    s = np.abs(b).max()
    return float(d / s) if s > 0 else float(d)
