"""The reference's Advect verification case (test/verification/Advect), shared by
the CPU oracle test and the GPU test of the WENO convergence order.

AR = sin(pi x - sin(pi x)/pi) is advected with the constant user velocity 1 on the
periodic domain [-1, 1] (Prob.H:71-72, inputs1d) to t = 0.1 on 10..160 cells
(postprocess.sh); the error is the L2 norm of the cell values against the
translated exact solution (get_error_1d.py:52-53), which the reference plots
against a 5th-order slope (pic_adv_weno.gp:17-18).  Time integration: the
classical 4-stage Runge-Kutta method from the update's dsdt at a Courant number
of 0.05, whose error stays far below the spatial one.
"""
from __future__ import annotations

import math

import numpy as np

from vidyut_b200 import _abi as abi
from vidyut_b200 import inputs as vin
from vidyut_b200 import mechanism as mm

T_END = 0.1
VEL = 1.0
CFL = 0.05
SIZES = [10, 20, 40, 80, 160]


def advect_mechanism() -> mm.Mechanism:
    """E and AR, as the Advect case's Chemistry.H (specMob -1, no reactions)."""
    return mm.Mechanism(name="advect", species=["E", "AR"], charge=[-1, 0], mw=[0.000549, 39.95], e_id=0,
                        mob_kind=[abi.MOB_CONST] * 3, mob_ref=[0] * 3, mob_p0=[-1.0] * 3, mob_p1=[0.0] * 3,
                        diff_kind=[0] * 3, diff_ref=[0] * 3, diff_factor=[1.0] * 3, reactions=[], bg_species=[])


def exact(x, t):
    y = x - VEL * t
    return np.sin(math.pi * y - np.sin(math.pi * y) / math.pi)


def advect_case(n: int, weno: int = 3, precision: int = abi.PREC_FP64):
    """(case, cell centres x, steps, dt): a 1-D periodic box of n cells holding the
    initial AR profile (ghosts filled), with the run parameters in case.params."""
    mech = advect_mechanism()
    dx = 2.0 / n
    case = vin.build_case(mech, 1, (n,), (dx,), 7, density="loguniform", dens_range=(1.0, 2.0),
                          periodic=(1, 0, 0))
    ns, g = mech.ns, case.ghost
    x = -1.0 + (np.arange(n) + 0.5) * dx
    st = case.state
    st[:] = 0.0
    st[1, 0, 0, g:g + n] = exact(x, 0.0)
    st[abi.ETEMP(ns), 0, 0, g:g + n] = 0.5 * vin.EV
    vin.fill_ghosts(st, 1, g, periodic=(1, 0, 0))
    nsteps = int(round(T_END / (CFL * dx)))
    dt = T_END / nsteps
    case.params.update(dict(user_defined_vel=1, vel_species=1, user_vel=(VEL, 0.0, 0.0), elecenergy_solve=0,
                            do_reactions=0, hyp_order=5, weno_scheme=weno, precision=precision,
                            bc_lo=[[abi.BC_PER] * 3] * 4, bc_hi=[[abi.BC_PER] * 3] * 4, dt=dt))
    return case, x, nsteps, dt


def rk4(u, rate, nsteps: int, dt: float):
    for _ in range(nsteps):
        k1 = rate(u)
        k2 = rate(u + 0.5 * dt * k1)
        k3 = rate(u + 0.5 * dt * k2)
        k4 = rate(u + dt * k3)
        u = u + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
    return u


def l2_error(u: np.ndarray, x: np.ndarray, t: float) -> float:
    return float(np.sqrt(np.mean((u - exact(x, t)) ** 2)))


def orders(errs):
    return [math.log2(errs[i] / errs[i + 1]) for i in range(len(errs) - 1)]
