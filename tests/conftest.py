import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this container")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


# ----------------------------------------------------------------------
# comparison helpers (tolerances are the contract's: 1e-12 relative per site)
def site_rel_err(B, Bref, floor_frac=1e-3):
    """max_i |B_i - Bref_i| / max(|Bref_i|, floor_frac * max_j |Bref_j|)."""
    B = np.asarray(B).reshape(-1, 3)
    Bref = np.asarray(Bref).reshape(-1, 3)
    n = np.linalg.norm(Bref, axis=1)
    den = np.maximum(n, floor_frac * n.max() + 1e-300)
    return float((np.linalg.norm(B - Bref, axis=1) / den).max())


def scalar_rel_err(e, eref, floor_frac=1e-3):
    e = np.asarray(e).ravel()
    eref = np.asarray(eref).ravel()
    den = np.maximum(np.abs(eref), floor_frac * np.abs(eref).max() + 1e-300)
    return float((np.abs(e - eref) / den).max())
