"""The CPU restatement of the potential step (oracle/poisson.py) against closed
forms: no charge between two electrodes gives the linear potential exactly, a
uniform charge the parabola, and the cell/face fields and reduced field follow."""
import numpy as np

from oracle import poisson
from vidyut_b200 import _abi as abi
from vidyut_b200 import inputs
from vidyut_b200.mechanism import synthetic


def _case(n, dim):
    mech = synthetic(8, 40, inputs.BASE_SEED + 21)
    return inputs.build_case(mech, dim, n, (1e-5,) * dim, 5, density="loguniform_smooth",
                             dens_range=(1e10, 1e18), n_modes=4)


def test_linear_potential_without_charge():
    c = _case((20, 7), 2)
    c.state[: c.mech.ns] = 0.0  # no charge
    V = 1234.5
    phi = poisson.solve(c, (1, 0, 0), (1, 0, 0), (V, 0, 0), (0.0, 0, 0))
    L = c.n[0] * c.dx[0]
    x = (np.arange(c.n[0]) + 0.5) * c.dx[0]
    np.testing.assert_allclose(phi[0], np.broadcast_to(V * (1 - x / L), phi[0].shape), rtol=1e-12, atol=1e-9)
    E = poisson.cell_field(phi, 2, c.dx)
    np.testing.assert_allclose(E[0], V / L, rtol=1e-9)
    np.testing.assert_allclose(E[1], 0.0, atol=1e-6)
    f = poisson.face_field(phi, 2, c.dx, 0, (1, 0, 0), (1, 0, 0), (V, 0, 0), (0.0, 0, 0))
    np.testing.assert_allclose(f, V / L, rtol=1e-9)


def test_uniform_charge_parabola():
    c = _case((40,), 1)
    ns = c.mech.ns
    g = c.gvec
    c.state[:ns] = 0.0
    ion = [s for s in range(ns) if c.mech.charge[s] == 1][0]
    n0 = 1e16
    c.state[ion, :, :, g[0]:g[0] + c.n[0]] = n0
    phi = poisson.solve(c, (1, 0, 0), (1, 0, 0), (0.0, 0, 0), (0.0, 0, 0))
    # -phi'' = e n0 / eps0 with phi = 0 at both faces: phi = e n0 / (2 eps0) x (L - x);
    # the face value enters through linear extrapolation to the ghost cell, which
    # is second-order accurate: the error is O((dx/L)^2), 6e-4 here
    L = c.n[0] * c.dx[0]
    x = (np.arange(c.n[0]) + 0.5) * c.dx[0]
    want = poisson.ECHARGE * n0 / (2 * poisson.EPS0) * x * (L - x)
    err = np.max(np.abs(phi[0, 0] - want)) / np.max(want)
    assert 1e-6 < err < 5e-3
    # second-order: twice the cells, a quarter of the error
    c2 = _case((80,), 1)
    c2.state[:ns] = 0.0
    c2.dx = (c.dx[0] / 2,)
    c2.state[ion, :, :, g[0]:g[0] + c2.n[0]] = n0
    phi2 = poisson.solve(c2, (1, 0, 0), (1, 0, 0), (0.0, 0, 0), (0.0, 0, 0))
    x2 = (np.arange(c2.n[0]) + 0.5) * c2.dx[0]
    want2 = poisson.ECHARGE * n0 / (2 * poisson.EPS0) * x2 * (L - x2)
    err2 = np.max(np.abs(phi2[0, 0] - want2)) / np.max(want2)
    assert 3.5 < err / err2 < 4.5
