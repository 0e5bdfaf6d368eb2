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


def scaled_err(a: np.ndarray, b: np.ndarray, scale: np.ndarray) -> float:
    """max over cells of |a - b| / scale: the error relative to the gross magnitude
    of the terms summed into the value (cells with zero scale must agree exactly)."""
    d = np.abs(a - b)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(scale > 0, d / scale, np.where(d > 0, np.inf, 0.0))
    return float(np.max(r))


def update_scales(port, case, prm):
    """(rxn scale, dsdt scale, n_new scale) from the oracle, NS+1 components each."""
    ns = case.mech.ns
    g = case.gvec
    n_old = case.state[:ns + 1, g[2]:g[2] + case.n[2], g[1]:g[1] + case.n[1], g[0]:g[0] + case.n[0]]
    rs = port.rxn_scale(case, prm.Tg)
    ds = port.update_scale(case, prm)
    return rs, ds, np.abs(n_old) + prm.dt * ds
