"""The verification headers with field-dependent transport and rates on the GPU.

streamer_2d (test/verification/Streamer/Chemistry.H): electron mobility and
diffusion as powers of |E|, the energy's 5/3 of both, and the field-driven
ionisation rate, which reads the reduced field REF.  he_rf_1d
(test/verification/He_RF_1d/Chemistry.H): the ions' |E|/N polynomial mobility,
the electrons' mean-energy fit over N, pressure-scaled diffusion and the elastic
loss at |E| = EN N 1e-21.  Golden outputs: the reference's own headers compiled
against the AMReX shim (tests/golden/make_golden.py).  Every path that evaluates
these models runs here: the mechanism-specialised and the table-driven chemistry,
FP64 and the mixed path, and the batched persistent launch.
"""
import numpy as np
import pytest
import torch

import oracle
from tests._util import load_fixture, scaled_err, update_scales
from vidyut_b200 import _abi as abi
from vidyut_b200 import api

pytestmark = pytest.mark.gpu

NAMES = ["streamer_2d", "he_rf_1d"]
TOLS = ((abi.PREC_FP64, 1e-12), (abi.PREC_MIXED, 1e-5))


def _check(case, outs, pn, rxn, tol, what):
    ns = case.mech.ns
    prm = case.vd_params()
    rs, _, nsc = update_scales(oracle.Port(case.mech), case, prm)
    if rxn is not None:
        assert scaled_err(rxn, outs["upd_rxn"], rs) <= tol, what
    per = [scaled_err(pn[s], outs["upd_phi_new"][s], nsc[s]) for s in range(ns + 1)]
    assert max(per) <= tol, (what, per)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("spec", [1, 0])
def test_update_both_chemistry_kernels_both_precisions(name, spec):
    case, meta, outs = load_fixture(name)
    L = abi.lib()
    try:
        L.vd_set_specialize(spec)
        api.mech_init(case.mech)
        assert L.vd_mech_specialized() == spec, L.vd_mech_specialize_status()
        dc = api.upload(case)
        for prec, tol in TOLS:
            phi_new, dsdt, rxn = dc.new_outputs()
            api.explicit_update_all(dc, case.vd_params(precision=prec), phi_new, dsdt, rxn)
            torch.cuda.synchronize()
            _check(case, outs, phi_new.cpu().numpy(), rxn.cpu().numpy(), tol, (spec, prec))
    finally:
        L.vd_set_specialize(1)
        api.mech_init(case.mech)


@pytest.mark.parametrize("name", NAMES)
def test_batched_step(name):
    """one step of the batched persistent launch (graph replay) equals the
    reference's update in the valid cells"""
    case, meta, outs = load_fixture(name)
    api.mech_init(case.mech)
    H = 3
    for prec, tol in TOLS:
        with api.Batch(prec, budget_bytes=1 << 28, max_cases=2) as b:
            i = b.add(case, case.vd_params(precision=prec))
            b.step(1)
            got = b.read(i).numpy()
        g = [H if d < case.dim else 0 for d in range(3)]
        v = got[:, g[2]:g[2] + case.n[2], g[1]:g[1] + case.n[1], g[0]:g[0] + case.n[0]]
        _check(case, outs, v, None, tol, ("batch", prec))
