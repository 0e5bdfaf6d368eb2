"""CPU oracle of the implicit diffusion solve of one species (TEST INFRASTRUCTURE).

Only tests/ use this module, as the checker of vd_implicit_species_solve.  The
reference solves, per species, (1/dt) n - div(D grad n) = n_old/dt + dsdt_expl
with AMReX's MLABecLaplacian / MLMG (Vidyut::implicit_solve_scalar,
Source/ScalarSolve.cpp:289-680), which is not available here, so this oracle
restates the discrete problem MLMG solves on one box that is the whole domain and
solves it directly (scipy sparse LU):

- a = 1/dt, B = 1 (:323-325,438); rhs = n_old/dt + dsdt_expl (:455-457); the
  initial guess (unused by a direct solve) is the current state (:459-463).
- D at every cell of the box grown by one from specDiff(spec, Te, sum_s n_s, |E|,
  Tg) of the current state (:478-490), and on faces the harmonic mean of the two
  cells' values (average_cellcenter_to_face with harmonic averaging, :497-505).
- Domain faces (:508-558, Source/PlasmaChem.H:75-184): species_bc writes one value
  per boundary face into the ghost cell; VD_BC_DIRC uses it as the value at the
  face, VD_BC_IHNEU as the derivative along the coordinate direction there (the
  reference's "dc/dx = -flx/D"), VD_BC_HNEU and VD_BC_ROBIN (species_bc's default
  robin a = 0, b = 1, f = 0) give zero gradient.  Periodic directions are not
  covered.
- After the solve: densities floored when bound_specden (:590-617); for the
  electrons the face gradients (getGradSolution, :618-621); for the electron
  energy Te = (2/3)/kB eps / n_e(state), floored (:630-666).

The face gradient at a domain face is taken from the same face relation the
operator uses (half a cell to a Dirichlet value, the given derivative, or zero).
Parity of the multigrid against MLMG is unpinned (no AMReX); the discrete problem
is pinned by this direct solve.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

K_B = 1.380649e-23
PI = 3.14159265358979323846264338327950288
ME = 9.10938188e-31
M_AMU = 1.66054e-27
BC_PER, BC_DIRC, BC_HNEU, BC_IHNEU, BC_ROBIN = 0, 1, 2, 3, 4


def _valid(a, n, g):
    return a[..., g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]


def species_class(mech, s):
    if s == mech.ns:
        return 1  # energy
    if s == mech.e_id:
        return 0
    return 2 if mech.charge[s] != 0 else 3


def cell_diffusivity(case, spec, Tg, port):
    """specDiff at every cell of the box grown by one (Source/ScalarSolve.cpp:478-490):
    array (nz+2, ny+2, nx+2) below 3-D with the unused directions one thick."""
    from vidyut_b200 import _abi as abi
    ns, dim, n, g = case.mech.ns, case.dim, case.n, case.gvec
    lo = [g[d] - (1 if d < dim else 0) for d in range(3)]
    hi = [g[d] + n[d] + (1 if d < dim else 0) for d in range(3)]
    st = case.state[:, lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
    te = st[abi.ETEMP(ns)]
    nd = st[:ns].sum(axis=0)
    D = np.empty(te.shape)
    for idx in np.ndindex(te.shape):
        D[idx] = port.specdiff(spec, te[idx], nd[idx], Tg)
    return D


def boundary_value(case, spec, d, sgn, face_cell, Tg, port, mw):
    """species_bc (Source/PlasmaChem.H:75-184) for the domain face of direction d on
    side sgn (-1 low, +1 high) at the face's transverse position; face_cell is the
    face index as a (i, j, k) triple in valid-cell coordinates (low face: i = 0,
    high face: i = n)."""
    from vidyut_b200 import _abi as abi
    ns, g = case.mech.ns, case.gvec
    cint = list(face_cell)
    if sgn > 0:
        cint[d] -= 1
    s = case.state

    def at(comp, c):
        return s[comp, c[2] + g[2], c[1] + g[1], c[0] + g[0]]

    nd = sum(at(q, cint) for q in range(ns))
    te = at(abi.ETEMP(ns), cint)
    e_id = case.mech.e_id
    D = port.specdiff(spec, te, nd, Tg)
    if spec == e_id:
        cbar = math.sqrt(8.0 * K_B * te / PI / ME)
        flx = at(e_id, cint) * cbar / 4.0 * sgn
        return -flx / D
    if spec == ns:
        cbar = math.sqrt(8.0 * K_B * te / PI / ME)
        flx = (2.0 * K_B * te) * at(e_id, cint) * cbar / 4.0 * sgn
        return -flx / D
    if case.mech.charge[spec] != 0:
        mu = port.specmob(spec, te, nd, Tg)
        drift = mu * at(spec, cint) * at(abi.EFX(ns) + d, cint)
        return -drift / D if drift * sgn >= 0.0 else 0.0
    cbar = math.sqrt(8.0 * K_B * Tg / PI / (mw * M_AMU))
    # the reference reads the density at the face index itself (the ghost cell on
    # the high side)
    flx = at(spec, face_cell) * cbar / 4.0 * sgn
    return -flx / D


def solve(case, spec, state_old, dsdt, prm, port, robin=None):
    """Solution on the valid cells (nz, ny, nx), plus the electron face gradients
    (list per direction, (nz, ny, nx) with +1 along d) when spec is the electrons,
    and the Te that the energy solve writes (or None).  robin: the case's own
    species_bc coefficients ((a_lo, b_lo, f_lo), (a_hi, b_hi, f_hi)), one value
    per direction each: a n + b dn/dnu = f on the face (nu the outward normal),
    with the face value (n_c + n_g)/2 and dn/dnu = (n_g - n_c)/dx between the cell
    and its ghost, as MLMG's Robin faces; None: species_bc's values."""
    from vidyut_b200 import _abi as abi
    mech, dim, n, dx, g = case.mech, case.dim, case.n, case.dx, case.gvec
    ns = mech.ns
    dt, Tg = prm.dt, prm.Tg
    cls = species_class(mech, spec)
    bclo = [prm.bc_lo[cls][d] for d in range(3)]
    bchi = [prm.bc_hi[cls][d] for d in range(3)]
    per = [d < dim and bclo[d] == BC_PER for d in range(3)]
    if any((bclo[d] == BC_PER) != (bchi[d] == BC_PER) for d in range(dim)):
        raise ValueError("a periodic direction needs VD_BC_PER on both sides")
    mw = mech.mw[spec] if spec < ns else 0.0
    Dg = cell_diffusivity(case, spec, Tg, port)
    N = n[0] * n[1] * n[2]
    idx = np.arange(N).reshape(n[2], n[1], n[0])
    a = 1.0 / dt
    nold = _valid(state_old[spec], n, g)
    rhs = (nold * a + dsdt).reshape(-1).astype(float).copy()
    diag = np.full(N, a)
    rows, cols, vals = [], [], []
    off = [1 if dim > 0 else 0, 1 if dim > 1 else 0, 1 if dim > 2 else 0]
    bfaces = {}
    for d in range(dim):
        w = 1.0 / (dx[d] * dx[d])
        ax = 2 - d
        for c in np.ndindex(n[2], n[1], n[0]):
            k, j, i = c
            cell = (i, j, k)
            gc = (i + off[0], j + off[1], k + off[2])  # index into Dg
            for sgn in (-1, 1):
                nb = list(cell)
                nb[d] += sgn
                gnb = list(gc)
                gnb[d] += sgn
                Dc, Dn = Dg[gc[2], gc[1], gc[0]], Dg[gnb[2], gnb[1], gnb[0]]
                b = 2.0 * Dc * Dn / (Dc + Dn) if (Dc + Dn) != 0.0 else 0.0
                r = idx[k, j, i]
                if per[d] and not 0 <= nb[d] < n[d]:
                    # across the periodic direction: the cell on the other side,
                    # through the face whose D comes from the ghost cell (a periodic
                    # image of that cell)
                    nb[d] %= n[d]
                if 0 <= nb[d] < n[d]:
                    rows.append(r)
                    cols.append(idx[nb[2], nb[1], nb[0]])
                    vals.append(-b * w)
                    diag[r] += b * w
                    continue
                bc = bclo[d] if sgn < 0 else bchi[d]
                face = list(cell)
                if sgn > 0:
                    face[d] += 1
                if robin is not None:
                    ra, rb, rf = (robin[0] if sgn < 0 else robin[1])
                    den = 0.5 * ra[d] + rb[d] / dx[d]
                    # -b (n_g - n_c)/dx^2 with n_g - n_c = (f - a n_c)/den
                    diag[r] += b * w * ra[d] / den
                    rhs[r] += b * w * rf[d] / den
                    bfaces[(d, sgn, tuple(face))] = ("robin", (ra[d], rf[d], den), b)
                    continue
                val = boundary_value(case, spec, d, sgn, tuple(face), Tg, port, mw)
                bfaces[(d, sgn, tuple(face))] = (bc, val, b)
                if bc == BC_DIRC:
                    diag[r] += 2.0 * b * w
                    rhs[r] += 2.0 * b * w * val
                elif bc == BC_IHNEU:
                    # flux b * val through the face enters the divergence with the
                    # face's sign
                    rhs[r] += sgn * b * val / dx[d]
    A = sp.csr_matrix((np.concatenate([np.array(vals), diag]),
                       (np.concatenate([np.array(rows, dtype=int), np.arange(N)]),
                        np.concatenate([np.array(cols, dtype=int), np.arange(N)]))), shape=(N, N))
    sol = spla.spsolve(A.tocsc(), rhs).reshape(n[2], n[1], n[0])
    if prm.bound_specden and spec != ns:
        lo = prm.min_electron_density if spec == mech.e_id else prm.min_species_density
        sol = np.maximum(sol, lo)
    grads = None
    if spec == mech.e_id:
        grads = []
        for d in range(3):
            shape = [n[2], n[1], n[0]]
            shape[2 - d] += 1 if d < dim else 0
            G = np.zeros(shape)
            if d < dim:
                for c in np.ndindex(*shape):
                    k, j, i = c
                    f = [i, j, k]
                    if 0 < f[d] < n[d]:
                        m = list(f)
                        m[d] -= 1
                        G[c] = (sol[k, j, i] - sol[m[2], m[1], m[0]]) / dx[d]
                    elif per[d]:
                        first, last = list(f), list(f)
                        first[d], last[d] = 0, n[d] - 1
                        G[c] = (sol[first[2], first[1], first[0]] - sol[last[2], last[1], last[0]]) / dx[d]
                    else:
                        sgn = -1 if f[d] == 0 else 1
                        bc, val, b = bfaces[(d, sgn, tuple(f))]
                        inner = list(f)
                        if sgn > 0:
                            inner[d] -= 1
                        ni = sol[inner[2], inner[1], inner[0]]
                        if bc == BC_DIRC:
                            G[c] = (ni - val) / (0.5 * dx[d]) if sgn < 0 else (val - ni) / (0.5 * dx[d])
                        elif bc == BC_IHNEU:
                            G[c] = val
                        elif bc == "robin":
                            ra, rf, den = val
                            G[c] = sgn * (rf - ra * ni) / den / dx[d]
            grads.append(G)
    te = None
    if spec == ns:
        ne = _valid(case.state[mech.e_id], n, g)
        te = (2.0 / 3.0) / K_B * sol / ne
    return sol, grads, te
