"""The CPU oracle against the reference's known answer for the flux path: on the
Advect verification case (tests/_advect.py) the oracle's WENO-Z update converges
at 5th order on 20..160 cells, as the reference's own convergence plot shows
(test/verification/Advect/pic_adv_weno.gp:17-18)."""
import numpy as np

import oracle
from tests._advect import SIZES, advect_case, l2_error, orders, rk4
from vidyut_b200 import inputs as vin


def oracle_advect_error(n: int) -> float:
    case, x, nsteps, dt = advect_case(n)
    port = oracle.Port(case.mech)
    prm = case.vd_params()
    st, g = case.state, case.ghost

    def rate(u):
        st[1, 0, 0, g:g + n] = u
        vin.fill_ghosts(st, 1, g, periodic=(1, 0, 0))
        return port.update_all(case, prm)["dsdt"][1, 0, 0, :].copy()

    u = rk4(st[1, 0, 0, g:g + n].copy(), rate, nsteps, dt)
    return l2_error(u, x, nsteps * dt)


def test_oracle_wenoz_converges_at_fifth_order():
    errs = [oracle_advect_error(n) for n in SIZES]
    o = orders(errs)
    assert errs[-1] < 1e-7
    assert min(o[1:]) >= 4.5, o
    fit = np.polyfit(np.log(2.0 / np.array(SIZES[1:])), np.log(errs[1:]), 1)[0]
    assert fit >= 4.5
