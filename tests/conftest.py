import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name: str) -> dict:
    z = np.load(GOLDEN / f"{name}.npz")
    d = {k: z[k] for k in z.files}
    d["meta"] = json.loads(str(d["meta"]))
    return d


def golden_names():
    """The solve-path fixtures (the adjoint fixtures, adj*, hold only the two solves; the
    krylov* fixtures only the comparison solvers; the solve* fixtures only complete solves
    at the workload sizes)."""
    return sorted(p.stem for p in GOLDEN.glob("*.npz") if not p.stem.startswith(("adj", "krylov", "solve")))


def rel(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).reshape(-1)) / max(np.linalg.norm(b.reshape(-1)), 1e-300))
