"""Known answer for the flux path on the GPU: the reference's Advect
verification case (tests/_advect.py) through vd_explicit_update_all (hyp_order 5,
WENO-Z, the reference's user-velocity path), with the periodic ghost refill of
vd_fill_ghosts between Runge-Kutta stages.  The L2 error must fall at 5th order
on the smooth part of the range (20..160 cells), as the reference's plot shows.
"""
import numpy as np
import pytest
import torch

from tests._advect import SIZES, advect_case, l2_error, orders, rk4
from vidyut_b200 import _abi as abi
from vidyut_b200 import api

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    abi.lib()
    abi.check_layout()


def gpu_advect_error(n: int, weno: int = 3, precision=abi.PREC_FP64) -> float:
    case, x, nsteps, dt = advect_case(n, weno, precision)
    g = case.ghost
    api.mech_init(case.mech)
    dc = api.upload(case)
    phi_new, dsdt, _ = dc.new_outputs()
    prm = case.vd_params()
    stage = dc.state[1, 0, 0, g:g + n]

    def rate(u):
        stage.copy_(u)
        api.fill_ghosts(dc.state, case, g, [1], periodic=(1, 0, 0))
        api.explicit_update_all(dc, prm, phi_new, dsdt)
        return dsdt[1, 0, 0, :].clone()

    u = rk4(stage.clone(), rate, nsteps, dt)
    torch.cuda.synchronize()
    return l2_error(u.cpu().numpy(), x, nsteps * dt)


def test_wenoz_converges_at_fifth_order():
    errs = [gpu_advect_error(n) for n in SIZES]
    o = orders(errs)
    fit = np.polyfit(np.log(2.0 / np.array(SIZES[1:])), np.log(errs[1:]), 1)[0]  # slope of log error vs log dx
    print("Advect WENO-Z L2 errors", dict(zip(SIZES, errs)), "orders", o, "fit", fit)
    assert errs[-1] < 1e-7
    assert min(o[1:]) >= 4.5, o
    assert fit >= 4.5


def test_mixed_precision_tracks_fp64_on_advect():
    e64 = gpu_advect_error(40)
    emx = gpu_advect_error(40, precision=abi.PREC_MIXED)
    # FP32 reconstructions add rounding of ~1e-7 of the O(1) solution at most
    assert abs(emx - e64) < 5e-6
