import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def load_golden(name: str):
    d = np.load(os.path.join(GOLDEN, f"snap_{name}.npz"))
    r2 = 4.0 * d["hp"] ** 2
    r2 = np.where(d["u"] == 0.0, -r2, r2)
    return {k: d[k] for k in ("x", "y", "z", "am", "hp", "u", "grpot")} | {"range2": r2}


GOLDEN_CASES = ["collision_start2", "3stars_start1", "3stars_start2", "collision_start1"]


@pytest.fixture(scope="session")
def gpu_ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from starsmasher_b200 import Context
    ctx = Context(0)
    yield ctx
    ctx.close()


def rel_err_vec(ax, ay, az, bx, by, bz):
    """Per-particle |a - b| / |b|."""
    num = np.sqrt((ax - bx) ** 2 + (ay - by) ** 2 + (az - bz) ** 2)
    den = np.sqrt(bx ** 2 + by ** 2 + bz ** 2)
    return num / den


def err_report(ax, ay, az, pot, ox, oy, oz, opot):
    """max/RMS relative errors; particles with |a| < 1e-3 median |a| are
    reported separately (cancellation makes their relative error ill-conditioned)."""
    e = rel_err_vec(ax, ay, az, ox, oy, oz)
    amag = np.sqrt(ox ** 2 + oy ** 2 + oz ** 2)
    ill = amag < 1e-3 * np.median(amag)
    ep = np.abs(pot - opot) / np.abs(opot)
    good = ~ill
    return {
        "acc_max": float(e[good].max()) if good.any() else 0.0,
        "acc_rms": float(np.sqrt(np.mean(e[good] ** 2))) if good.any() else 0.0,
        "acc_max_ill": float(e[ill].max()) if ill.any() else 0.0,
        "n_ill": int(ill.sum()),
        "pot_max": float(ep.max()),
        "pot_rms": float(np.sqrt(np.mean(ep ** 2))),
    }
