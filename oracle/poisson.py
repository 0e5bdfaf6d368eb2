"""CPU oracle of the potential / electric-field step (TEST INFRASTRUCTURE).

Only tests/ use this module, as the checker of vd_poisson_solve.  The reference
solves the potential with AMReX's MLMG (Source/PotentialSolve.cpp:188-378), which
is not available here, so this oracle restates the discrete problem that MLMG
solves and solves it directly (scipy sparse LU): the cell-centred 2D+1-point
Laplacian with the charge right-hand side -(e/eps0) sum_k z_k n_k
(Source/PotentialSolve.cpp:199-215), Dirichlet faces holding the applied
potential at the face, zero-gradient faces elsewhere.  The cell field follows
get_efield_alongdir (Source/HelperFuncs.H:14-70), the reduced field
update_cc_efields (Source/PotentialSolve.cpp:419-424), the face field MLMG's
getGradSolution negated (Source/PotentialSolve.cpp:362-371).  Parity of the
multigrid itself against MLMG is unpinned (no AMReX); the discrete problem is.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

ECHARGE = 1.60217662e-19
EPS0 = 8.854187817e-12


def _lin(n, i, j, k):
    return i + n[0] * (j + n[1] * k)


def solve(case, dirichlet_lo, dirichlet_hi, v_lo, v_hi, user_rhs=None):
    """phi (nz, ny, nx) of the valid cells.  dirichlet_lo/hi[d]: bool per direction,
    v_lo/hi[d]: the face values; user_rhs (nz, ny, nx) is added to the right-hand
    side (the case's add_user_potential_sources, Source/PotentialSolve.cpp:220)."""
    dim, n, dx = case.dim, case.n, case.dx
    ns = case.mech.ns
    g = case.gvec
    valid = case.state[:, g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]
    rho = np.zeros((n[2], n[1], n[0]))
    for s in range(ns):
        if case.mech.charge[s] != 0:
            rho += case.mech.charge[s] * valid[s]
    rhs = (rho * (-ECHARGE / EPS0)).reshape(-1).copy()
    if user_rhs is not None:
        rhs += np.asarray(user_rhs, dtype=float).reshape(-1)
    N = n[0] * n[1] * n[2]
    rows, cols, vals = [], [], []
    diag = np.zeros(N)
    idx = np.arange(N)
    kk, jj, ii = np.unravel_index(idx, (n[2], n[1], n[0]))
    coords = [ii, jj, kk]
    for d in range(dim):
        w = 1.0 / (dx[d] * dx[d])
        c = coords[d]
        for side in (-1, 1):
            inside = (c + side >= 0) & (c + side < n[d])
            nb = idx + side * (1 if d == 0 else (n[0] if d == 1 else n[0] * n[1]))
            rows.append(idx[inside])
            cols.append(nb[inside])
            vals.append(np.full(inside.sum(), w))
            diag[inside] -= w
            edge = ~inside
            dirich = dirichlet_lo[d] if side < 0 else dirichlet_hi[d]
            val = v_lo[d] if side < 0 else v_hi[d]
            if dirich:
                diag[edge] -= 2.0 * w
                rhs[edge] -= 2.0 * w * val
    rows.append(idx)
    cols.append(idx)
    vals.append(diag)
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    phi = spla.spsolve(A.tocsc(), rhs)
    return phi.reshape(n[2], n[1], n[0])


def cell_field(phi, dim, dx):
    """E per direction (nz, ny, nx) by get_efield_alongdir's differences."""
    out = []
    for d in range(3):
        E = np.zeros_like(phi)
        if d < dim:
            ax = 2 - d
            n = phi.shape[ax]
            p = np.moveaxis(phi, ax, 0)
            e = np.moveaxis(E, ax, 0)
            if n > 2:
                e[1:-1] = -0.5 * (p[2:] - p[:-2]) / dx[d]
            if n - 1 > 2:
                e[0] = -0.5 * (-p[2] + 4.0 * p[1] - 3.0 * p[0]) / dx[d]
                e[-1] = -0.5 * (p[-3] - 4.0 * p[-2] + 3.0 * p[-1]) / dx[d]
            elif n > 1:
                e[0] = -(p[1] - p[0]) / dx[d]
                e[-1] = -(p[-1] - p[-2]) / dx[d]
        out.append(E)
    return out


def face_field(phi, dim, dx, d, dirichlet_lo, dirichlet_hi, v_lo, v_hi):
    """-dphi/dx_d on the face box of direction d (1, nz, ny, nx) with +1 along d."""
    ax = 2 - d
    p = np.moveaxis(phi, ax, 0)
    n = p.shape[0]
    f = np.zeros((n + 1,) + p.shape[1:])
    f[1:n] = -(p[1:] - p[:-1]) / dx[d]
    f[0] = -(p[0] - v_lo[d]) / (0.5 * dx[d]) if dirichlet_lo[d] else 0.0
    f[n] = -(v_hi[d] - p[n - 1]) / (0.5 * dx[d]) if dirichlet_hi[d] else 0.0
    return np.moveaxis(f, 0, ax)[None]


def reduced_field(case, E):
    n, g = case.n, case.gvec
    ns = case.mech.ns
    valid = case.state[:, g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]
    nd = valid[:ns].sum(axis=0)
    es = sum(E[d] * E[d] for d in range(case.dim))
    return (np.sqrt(es) / nd) / 1.0e-21


def time_scales(case, prm, port):
    """Vidyut::find_time_scales (Source/TimeStep.cpp:34-116) on the valid cells of
    case.state with the C port's specMob/specDiff."""
    import math
    from vidyut_b200 import _abi as abi
    ns, dim = case.mech.ns, case.dim
    n, g = case.n, case.gvec
    v = case.state[:, g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]
    te = v[abi.ETEMP(ns)].ravel()
    emag = np.sqrt(sum(v[abi.EFX(ns) + d] ** 2 for d in range(dim))).ravel()
    nd = v[:ns].sum(axis=0).ravel()
    ne = v[case.mech.e_id].ravel()
    mu = np.array([port.specmob(case.mech.e_id, te[q], nd[q], prm.Tg) for q in range(te.size)])
    dc = np.array([port.specdiff(case.mech.e_id, te[q], nd[q], prm.Tg) for q in range(te.size)])
    mdrift, mdiff, mmue = np.max(np.abs(mu) * emag), np.max(dc), np.max(np.abs(mu) * ne)
    big = 1.79769313486231570e308
    out = [big, big, big]
    for d in range(dim):
        if mdrift > 0:
            out[0] = min(out[0], case.dx[d] / mdrift)
        if mdiff > 0:
            out[1] = min(out[1], 0.5 * case.dx[d] * case.dx[d] / mdiff / dim)
    if mmue > 0:
        out[2] = EPS0 / ECHARGE / mmue
    return tuple(out)
