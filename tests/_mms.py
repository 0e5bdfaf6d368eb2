"""The reference's method-of-manufactured-solutions case (test/verification/MMS),
shared by the CPU oracle test and the GPU test of the potential and implicit
species solves.

    dn/dt + d/dx(mu E n) = d/dx(D dn/dx) + 5 x^4/3 - x/6 - 2,   d2phi/dx2 = n,
    mu = -1, D = 1, E = -dphi/dx,  n(0) = 0, n(1) = 1,  phi(0) = phi(1) = 0,
    steady solution n = x^2, phi = (x^4 - x)/12                   (README:1-15)

The user functions of the case: the potential source add_user_potential_sources
(UserSources.H:63-75) adds n to the right-hand side; the species source
add_user_react_sources (UserSources.H:51) is added to dsdt before the implicit
solve; species_bc's Robin coefficients (UserFunctions.H:86-104) are a = 1, b = 0
with f = 0 low and 1 high; potential_bc's (UserFunctions.H:46-56) hold 0 at both
faces.  The reference plots the steady error against 1st and 2nd order slopes
(pic_conv_n.gp, pic_conv_phi.gp).
"""
from __future__ import annotations

import math

import numpy as np

from vidyut_b200 import _abi as abi
from vidyut_b200 import inputs as vin
from vidyut_b200 import mechanism as mm

SIZES = [8, 16, 32, 64]
DT = 0.01
T_END = 4.0
ROBIN = (((1.0,) * 3, (0.0,) * 3, (0.0,) * 3), ((1.0,) * 3, (0.0,) * 3, (1.0,) * 3))


def mms_mechanism() -> mm.Mechanism:
    """E and AR as the MMS case's Chemistry.H: specMob -1 for every species,
    specDiff 1 for AR (here D = 2 (Te/eV) |mu| at Te = 0.5 eV, which is exactly 1)."""
    return mm.Mechanism(name="mms", species=["E", "AR"], charge=[-1, 0], mw=[0.000549, 39.95], e_id=0,
                        mob_kind=[abi.MOB_CONST] * 3, mob_ref=[0] * 3, mob_p0=[-1.0] * 3, mob_p1=[0.0] * 3,
                        diff_kind=[abi.DIFF_ZERO, abi.DIFF_TE_ABSMOB, abi.DIFF_ZERO], diff_ref=[0, 1, 0],
                        diff_factor=[0.0, 2.0, 0.0], reactions=[], bg_species=[])


def mms_case(n: int, hyp_order: int):
    """(case, cell centres x, source S(x)) for n cells on [0, 1], densities zero."""
    mech = mms_mechanism()
    dx = 1.0 / n
    case = vin.build_case(mech, 1, (n,), (dx,), 3, density="loguniform", dens_range=(1.0, 2.0))
    case.state[:] = 0.0
    case.state[abi.ETEMP(mech.ns)] = 0.5 * vin.EV
    case.params.update(dict(elecenergy_solve=0, do_reactions=0, hyp_order=hyp_order, weno_scheme=3, dt=DT,
                            bc_lo=[[abi.BC_ROBIN] * 3] * 4, bc_hi=[[abi.BC_ROBIN] * 3] * 4))
    x = (np.arange(n) + 0.5) * dx
    return case, x, 5.0 * x ** 4 / 3.0 - x / 6.0 - 2.0


def errors(n_num, phi, x):
    return (math.sqrt(np.mean((n_num - x ** 2) ** 2)), math.sqrt(np.mean((phi - (x ** 4 - x) / 12.0) ** 2)))


def orders(e):
    return [math.log2(e[i] / e[i + 1]) for i in range(len(e) - 1)]
