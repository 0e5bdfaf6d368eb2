"""The CPU oracles of the potential and implicit species solves (oracle/poisson.py,
oracle/diffusion.py) and the C port's explicit update, stepped to steady state on
the reference's MMS case (tests/_mms.py): the errors against the manufactured
solution fall at 2nd order with hyp_order 5, as the reference's plots show
(test/verification/MMS/pic_conv_n.gp, pic_conv_phi.gp)."""
import numpy as np

import oracle
from oracle import diffusion as odif
from oracle import poisson as opois
from tests._mms import DT, ROBIN, SIZES, T_END, errors, mms_case, orders
from vidyut_b200 import _abi as abi
from vidyut_b200 import inputs as vin


def oracle_mms(n: int, hyp_order: int):
    case, x, src = mms_case(n, hyp_order)
    ns, g = case.mech.ns, case.ghost
    st = case.state
    prm = case.vd_params()
    port = oracle.Port(case.mech)
    for _ in range(int(round(T_END / DT))):
        nar = st[1, 0, 0, g:g + n].copy()
        phi = opois.solve(case, [True] * 3, [True] * 3, [0.0] * 3, [0.0] * 3, user_rhs=nar.reshape(1, 1, n))
        E = opois.cell_field(phi, 1, case.dx)
        st[abi.POT(ns), 0, 0, g:g + n] = phi[0, 0]
        st[abi.EFX(ns), 0, 0, g:g + n] = E[0][0, 0]
        vin.fill_ghosts(st, 1, g)
        dsdt = port.update_all(case, prm)["dsdt"][1] + src.reshape(1, 1, n)
        sol, _, _ = odif.solve(case, 1, st.copy(), dsdt, prm, port, robin=ROBIN)
        st[1, 0, 0, g:g + n] = sol[0, 0]
    return errors(st[1, 0, 0, g:g + n], phi[0, 0], x)


def test_oracle_mms_second_order_with_weno():
    errs = [oracle_mms(n, 5) for n in SIZES]
    on, op = orders([a for a, _ in errs]), orders([b for _, b in errs])
    assert min(on) >= 1.8, on
    assert min(op) >= 1.8, op
