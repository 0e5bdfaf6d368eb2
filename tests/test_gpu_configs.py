"""GPU parity at the workload configurations' full sizes, against the reference's
own hot-path code (oracle/_ref: Source/compute_explicit_flux.H, PlasmaChem.H and
the case headers compiled unmodified; the per-box loops of
Source/ScalarSolve.cpp:143-165,226-250 and Source/ElecEnergySource.cpp:65-171).

  config 1  2-D 256^2 argon box, plain FP64, one explicit step;
  config 2  3-D 128^3 box, 24 species / 150 reactions, FP64 and mixed, one step;
  config 3  a subset of the 64 batched 2-D cases (8 species / 40 reactions), 20
            steps in one batch against 20 steps of the reference code.

Tolerances as in test_gpu_parity.py: FP64 1e-12 relative to the gross magnitude
of the terms summed into each value (the generated chemistry adds and removes
the same rate, so last-bit differences of exp/pow move a net rate by eps times
the gross rate); mixed 1e-5 per species on the same scale.  The elementwise
relative errors (|gpu - ref| / |ref|) are printed per species for the record.
"""
import json
import os

import numpy as np
import pytest
import torch

import oracle
from tests._util import scaled_err
from vidyut_b200 import _abi as abi
from vidyut_b200 import api
from vidyut_b200 import inputs as vin

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_MIXED = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    abi.lib()
    abi.check_layout()


def _ref(case):
    if not oracle.RefLib.available(case.mech.name, case.dim):
        pytest.fail(f"reference build of {case.mech.name} ({case.dim}-D) missing: run oracle/build.py")
    return oracle.RefLib(case.mech.name, case.dim)


def _gpu_update(case, prm):
    api.mech_init(case.mech)
    dc = api.upload(case)
    phi_new, dsdt, rxn = dc.new_outputs()
    api.explicit_update_all(dc, prm, phi_new, dsdt, rxn)
    torch.cuda.synchronize()
    return {"phi_new": phi_new.cpu().numpy(), "dsdt": dsdt.cpu().numpy(), "rxn": rxn.cpu().numpy()}


def _elementwise(a, b):
    """per component max |a - b| / |b| over the cells where b != 0"""
    out = []
    for c in range(a.shape[0]):
        den = np.abs(b[c])
        m = den > 0
        out.append(float(np.max(np.abs(a[c] - b[c])[m] / den[m])) if m.any() else 0.0)
    return out


def _report(tag, rec):
    print(f"ELEMENTWISE {tag} " + json.dumps(rec))
    d = os.environ.get("VD_REPORT_DIR")
    if d:
        with open(os.path.join(d, f"elementwise_{tag}.json"), "w") as f:
            json.dump(rec, f)


def _check_one_step(case, prec, tol, tag):
    ns = case.mech.ns
    prm = case.vd_params(precision=prec)
    want = _ref(case).update_all(case, case.vd_params())  # the reference computes in FP64
    got = _gpu_update(case, prm)
    port = oracle.Port(case.mech)
    g = case.gvec
    n_old = case.state[:ns + 1, g[2]:g[2] + case.n[2], g[1]:g[1] + case.n[1], g[0]:g[0] + case.n[0]]
    rs = port.rxn_scale(case, prm.Tg)
    ds = port.update_scale(case, case.vd_params())
    ns_scale = np.abs(n_old) + prm.dt * ds
    rec = {"precision": "fp64" if prec == abi.PREC_FP64 else "mixed", "cells": case.ncell}
    worst = {}
    for key, scale in (("rxn", rs), ("dsdt", ds), ("phi_new", ns_scale)):
        a, b = got[key][:ns + 1], want[key][:ns + 1]
        per = [scaled_err(a[c], b[c], scale[c]) for c in range(ns + 1)]
        worst[key] = max(per)
        rec[f"{key}_scaled_per_species"] = per
        rec[f"{key}_elementwise_per_species"] = _elementwise(a, b)
    _report(tag, rec)
    for key, w in worst.items():
        if key == "rxn" and prec == abi.PREC_MIXED:
            continue  # mixed rates are FP32 (2e-7); the updated densities carry the bound
        assert w <= tol, f"{tag}: {key} error {w:.3e} > {tol}"
    return rec


def test_config1_argon_256x256_fp64_against_reference():
    case = vin.config_argon2d()
    rec = _check_one_step(case, abi.PREC_FP64, TOL64, "config1_argon256_fp64")
    # this mechanism has no production/loss cancellation: elementwise too
    assert max(rec["phi_new_elementwise_per_species"]) <= TOL64


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_config2_precision3d_128cubed_against_reference(prec):
    case = vin.config_precision3d()
    tol = TOL64 if prec == abi.PREC_FP64 else TOL_MIXED
    _check_one_step(case, prec, tol, f"config2_precision3d_{'fp64' if prec == abi.PREC_FP64 else 'mixed'}")


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_config3_batched_subset_20_steps_against_reference(prec):
    mech, cases = vin.config_batched()
    sub = sorted(cases, key=lambda c: c.ncell)[:3] + [max(cases, key=lambda c: c.ncell)]
    ref = oracle.RefLib(mech.name, 2)
    steps = 20
    api.mech_init(mech)
    H = 3
    with api.Batch(prec, budget_bytes=2 << 30, max_cases=8) as b:
        ids = [b.add(c, c.vd_params(precision=prec), nsteps=steps) for c in sub]
        b.step(steps)
        got = [b.read(i).numpy() for i in ids]
    ns = mech.ns
    comps = list(range(ns)) + [abi.EEN(ns), abi.ETEMP(ns)]
    worst = []
    for c, st in zip(sub, got):
        want = oracle.run_steps(ref, c, c.vd_params(), steps)
        w = api.trim_ghosts(c, want, H)
        sl = (comps, slice(None), slice(H, H + c.n[1]), slice(H, H + c.n[0]))
        e = _elementwise(st[sl], w[sl])
        worst.append(max(e))
    _report(f"config3_batched_subset_{'fp64' if prec == abi.PREC_FP64 else 'mixed'}",
            {"cases": [list(c.n[:2]) for c in sub], "steps": steps, "max_elementwise_per_case": worst})
    # 20 steps of a stiff explicit trajectory (the Te update near the density floor
    # amplifies last-bit differences): FP64 stays within 1e-9 elementwise, mixed 1e-5
    assert max(worst) <= (1e-9 if prec == abi.PREC_FP64 else TOL_MIXED), worst
