"""The implicit diffusion oracle (oracle/diffusion.py) on the CPU: the discrete
problem conserves what it should.  With zero-gradient walls the solve changes the
total only by dt * sum(dsdt); with inhomogeneous-Neumann walls the change is
dt times the boundary fluxes D_face * g summed over the wall faces; across a
periodic direction nothing leaves."""
import numpy as np

import oracle
from oracle import diffusion as odf
from vidyut_b200 import _abi as abi
from vidyut_b200 import inputs
from vidyut_b200 import mechanism as mm


def _setup(bc, dt=1e-9, periodic=(0, 0, 0), bc_lo=None, bc_hi=None):
    m = mm.argon(10, 20261204)
    case = inputs.build_case(m, 2, (12, 8), (1e-5, 1e-5), 77, density="loguniform_smooth",
                             dens_range=(1e14, 1e16), te_range_ev=(0.5, 2.0), periodic=periodic)
    prm = case.vd_params(dt=dt, bc=bc, bound_specden=0, bc_lo=bc_lo, bc_hi=bc_hi)
    rng = np.random.default_rng(3)
    g = case.gvec
    v = case.state[:, g[2]:g[2] + 1, g[1]:g[1] + 8, g[0]:g[0] + 12]
    dsdt = 1e-3 * v[:m.ns + 1] / dt * rng.uniform(-1, 1, v[:m.ns + 1].shape)
    return m, case, prm, v, dsdt


def test_zero_gradient_walls_conserve():
    m, case, prm, v, dsdt = _setup(abi.BC_HNEU)
    for spec in (m.e_id, 3):
        sol, _, _ = odf.solve(case, spec, case.state, dsdt[spec], prm, oracle.Port(m))
        want = np.sum(v[spec]) + prm.dt * np.sum(dsdt[spec])
        assert abs(np.sum(sol) - want) <= 1e-12 * np.sum(np.abs(v[spec]))


def test_wall_flux_balance():
    m, case, prm, v, dsdt = _setup(abi.BC_IHNEU)
    spec = m.e_id
    sol, grads, _ = odf.solve(case, spec, case.state, dsdt[spec], prm, oracle.Port(m))
    D = odf.cell_diffusivity(case, spec, prm.Tg, oracle.Port(m))
    # the balance: a * sum(n) = sum(rhs) + sum over walls of (+-) b g / dx
    lhs = np.sum(sol) / prm.dt
    rhs = np.sum(v[spec]) / prm.dt + np.sum(dsdt[spec])
    walls = 0.0
    for d in range(2):
        G = grads[d]
        ax = 2 - d
        Dl, Dl1 = np.take(D, 0, axis=ax), np.take(D, 1, axis=ax)
        Dh, Dh1 = np.take(D, D.shape[ax] - 1, axis=ax), np.take(D, D.shape[ax] - 2, axis=ax)
        tr = tuple(s for i, s in enumerate([slice(None), slice(1, -1), slice(1, -1)]) if i != ax)
        bl = (2 * Dl * Dl1 / (Dl + Dl1))[tr]
        bh = (2 * Dh * Dh1 / (Dh + Dh1))[tr]
        walls += (np.sum(bh * np.take(G, G.shape[ax] - 1, axis=ax)) - np.sum(bl * np.take(G, 0, axis=ax))) / case.dx[d]
    assert abs(lhs - (rhs + walls)) <= 1e-10 * abs(rhs)


def test_periodic_directions_conserve():
    """periodic in x (and then in both directions) with zero-gradient walls
    elsewhere: the total changes by dt * sum(dsdt) only, and the electrons' face
    gradient on the periodic faces is the difference across the wrap"""
    for per in ((1, 0, 0), (1, 1, 0)):
        b = [[abi.BC_PER if per[d] else abi.BC_HNEU for d in range(3)] for _ in range(4)]
        m, case, prm, v, dsdt = _setup(abi.BC_HNEU, periodic=per, bc_lo=b, bc_hi=b)
        for spec in (m.e_id, 3, m.ns):
            sol, grads, _ = odf.solve(case, spec, case.state, dsdt[spec], prm, oracle.Port(m))
            want = np.sum(v[spec]) + prm.dt * np.sum(dsdt[spec])
            assert abs(np.sum(sol) - want) <= 1e-12 * np.sum(np.abs(v[spec]))
            if spec == m.e_id:
                G = grads[0]
                assert np.array_equal(G[..., 0], G[..., -1])
                assert np.allclose(G[..., 0], (sol[..., 0] - sol[..., -1]) / case.dx[0], rtol=0, atol=0)
