"""Helpers shared by the tests: golden-fixture loading and error metrics."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from vidyut_b200.inputs import BoxCase
from vidyut_b200.mechanism import Mechanism

GOLDEN = Path(__file__).resolve().parent / "golden"
FIXTURES = sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_fixture(name: str):
    meta = json.loads((GOLDEN / f"{name}.json").read_text())
    mech = Mechanism.from_dict(meta["mech"])
    z = np.load(GOLDEN / f"{name}.npz")
    m = meta["meta"]
    case = BoxCase(mech=mech, dim=m["dim"], n=tuple(m["n"]), ghost=m["ghost"], dx=tuple(m["dx"]),
                   state=np.ascontiguousarray(z["state"]),
                   efield=[np.ascontiguousarray(z[f"efield{d}"]) for d in range(3)],
                   gradne=[np.ascontiguousarray(z[f"gradne{d}"]) for d in range(3)],
                   params=m["params"])
    outs = {k: z[k] for k in z.files if k not in ("state",) and not k.startswith(("efield", "gradne"))}
    return case, m, outs


def normwise_rel(a: np.ndarray, b: np.ndarray) -> float:
    """max|a-b| / max|b| (0 when both vanish)."""
    den = np.max(np.abs(b))
    num = np.max(np.abs(a - b))
    if den == 0.0:
        return float(num)
    return float(num / den)


def per_component_rel(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """normwise relative error of every leading-axis component."""
    return np.array([normwise_rel(a[c], b[c]) for c in range(a.shape[0])])


def max_elem_rel(a: np.ndarray, b: np.ndarray, floor: float = 0.0) -> float:
    den = np.maximum(np.abs(b), floor)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(den > 0, np.abs(a - b) / den, np.abs(a - b))
    return float(np.max(r))
