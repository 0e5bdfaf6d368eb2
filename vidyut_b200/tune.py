"""Autotuner for the kernel variants of libvidyut_b200.

Each knob is a set of compiled variants of one kernel (vd_tune_set keys); the
tuner runs a representative workload through every value, times the kernel with
CUDA events on its launch stream (vd_profile_*), keeps the fastest, and records
the choice per GPU name in tuning.json beside this file.  ``apply()`` loads the
recorded choices into the library (api.mech_init calls it once per process).

    python -m vidyut_b200.tune            # tune on this GPU and write tuning.json
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import torch

from . import _abi as abi

TUNING_FILE = Path(__file__).resolve().parent / "tuning.json"

# knob -> values per dimension (the 3-D transport kernel runs 512-thread blocks)
TRANSPORT_MINBLOCKS = {1: [1, 2, 3, 4], 2: [1, 2, 3, 4], 3: [1, 2]}

_applied = False


def _gpu_key() -> str:
    return torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"


def kernel_ms(step, kernel: str, steps: int = 10, warmup: int = 3) -> float:
    """Average device time [ms] of `kernel` over `steps` calls of step()."""
    L = abi.lib()
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    L.vd_profile_enable(1)
    for _ in range(steps):
        step()
    torch.cuda.synchronize()
    prof = abi.profile_read()
    L.vd_profile_enable(0)
    n, ms = prof[kernel]
    return ms / n


def tune_transport(case, precisions=(abi.PREC_MIXED, abi.PREC_FP64), steps: int = 10) -> dict:
    """Fastest transport occupancy variant for case's dimension, per precision."""
    from . import api
    L = abi.lib()
    api.mech_init(case.mech)
    dc = api.upload(case)
    phi_new, _, _ = dc.new_outputs()
    out = {}
    for prec in precisions:
        pname = "mixed" if prec == abi.PREC_MIXED else "fp64"
        key = f"transport_minblocks_{case.dim}d_{pname}"
        prm = case.vd_params(precision=prec)
        times = {}
        for mb in TRANSPORT_MINBLOCKS[case.dim]:
            abi.check(L.vd_tune_set(key.encode(), mb), "vd_tune_set")
            times[mb] = kernel_ms(lambda: api.explicit_update_all(dc, prm, phi_new), "k_transport", steps)
        best = min(times, key=times.get)
        abi.check(L.vd_tune_set(key.encode(), best), "vd_tune_set")
        out[key] = {"best": best, "ms": {str(k): round(v, 5) for k, v in times.items()},
                    "workload": f"{case.mech.name} {case.dim}-D {'x'.join(map(str, case.n[:case.dim]))}"}
    return out


def save(results: dict, path: Path = TUNING_FILE) -> None:
    data = json.loads(path.read_text()) if path.exists() else {}
    data.setdefault(_gpu_key(), {}).update(results)
    path.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")


def apply(path: Path = TUNING_FILE, force: bool = False) -> dict:
    """Load the recorded choices for this GPU into the library (once per process)."""
    global _applied
    if _applied and not force:
        return {}
    _applied = True
    if not path.exists():
        return {}
    rec = json.loads(path.read_text()).get(_gpu_key(), {})
    L = abi.lib()
    for key, v in rec.items():
        L.vd_tune_set(key.encode(), int(v["best"]))
    return rec


def tune_batch(mech, cases, precisions=(abi.PREC_MIXED, abi.PREC_FP64), trials: int = 5) -> dict:
    """Fastest batched transport variant per dimension and precision on `cases`."""
    from . import api
    api.mech_init(mech)
    out = {}
    for prec in precisions:
        pname = "mixed" if prec == abi.PREC_MIXED else "fp64"
        need = sum(api.Batch.case_bytes(c, c.vd_params(precision=prec)) for c in cases)
        with api.Batch(prec, budget_bytes=int(need * 1.05) + (64 << 20), max_cases=len(cases)) as b:
            for c in cases:
                b.add(c, c.vd_params(precision=prec))
            b.step(1)
            ms = b.tune(trials=trials)
            st = b.stats()
        dims = sorted({d for d, _ in ms})
        for d in dims:
            times = {v: t for (dd, v), t in ms.items() if dd == d}
            out[f"batch_tile_{d}d_{pname}"] = {
                "best": int(st["tile_variant"][d]), "ms": {str(k): round(v, 5) for k, v in times.items()},
                "workload": f"{mech.name} batch of {len(cases)} {d}-D cases"}
    return out


def main() -> int:
    from . import inputs
    res = {}
    mech_b, cases_b = inputs.config_batched()
    one_d = inputs.build_case(mech_b, 1, (1000,), (1e-5,), inputs.BASE_SEED + 77, density="loguniform_smooth",
                              dens_range=(1e10, 1e18), te_range_ev=(0.3, 10.0), n_modes=4,
                              params=dict(inputs.MULTISTEP_PARAMS))
    for case in (max(cases_b, key=lambda c: c.ncell), one_d, inputs.config_precision3d()):
        r = tune_transport(case)
        res.update(r)
        for k, v in r.items():
            print(k, v, flush=True)
    r = tune_batch(mech_b, cases_b)
    res.update(r)
    for k, v in r.items():
        print(k, v, flush=True)
    save(res)
    print("wrote", TUNING_FILE)
    return 0


if __name__ == "__main__":
    sys.exit(main())
