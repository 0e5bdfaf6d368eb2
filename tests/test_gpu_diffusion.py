"""Implicit diffusion solve of one species (vd_implicit_species_solve) against the
direct solve of the same discrete problem (oracle/diffusion.py): the reference's
Vidyut::implicit_solve_scalar (Source/ScalarSolve.cpp:289-680) with species_bc
(Source/PlasmaChem.H:75-184) boundary values."""
import numpy as np
import pytest
import torch

import oracle
from oracle import diffusion as odf
from vidyut_b200 import _abi as abi
from vidyut_b200 import api, inputs
from vidyut_b200 import mechanism as mm

pytestmark = pytest.mark.gpu

K_B = 1.380649e-23


@pytest.fixture(scope="module")
def mech():
    m = mm.argon(10, 20261204)
    api.mech_init(m)
    return m


def make(mech, dim, n, seed, dt, bc_lo=None, bc_hi=None, bound=1, periodic=(0, 0, 0)):
    case = inputs.build_case(mech, dim, n, (1e-5,) * dim, seed, density="loguniform_smooth",
                             dens_range=(1e14, 1e18), te_range_ev=(0.5, 5.0), periodic=periodic)
    prm = case.vd_params(dt=dt, bc_lo=bc_lo, bc_hi=bc_hi, bound_specden=bound)
    rng = np.random.default_rng(seed + 1)
    ns = mech.ns
    old = case.state.copy()
    old[:ns + 1] *= 1.0 + 0.01 * rng.uniform(-1, 1, old[:ns + 1].shape)
    g = case.gvec
    v = case.state[:, g[2]:g[2] + case.n[2], g[1]:g[1] + case.n[1], g[0]:g[0] + case.n[0]]
    dsdt = 1e-3 * v[:ns + 1] / dt * rng.uniform(-1, 1, v[:ns + 1].shape)
    return case, prm, old, np.ascontiguousarray(dsdt)


def run(mech, case, prm, old, dsdt, spec, tol=1e-13, cycles=60):
    dc = api.upload(case)
    old_t = torch.from_numpy(old).cuda()
    ds_t = torch.from_numpy(dsdt).cuda()
    phi_new = dc.new_outputs()[0]
    grads = [api.face_tensor(case, d) for d in range(3)] if spec == mech.e_id else None
    nv, rr = api.implicit_species_solve(dc, spec, old_t, ds_t, phi_new, prm, gradne=grads, tol_rel=tol,
                                        max_vcycles=cycles)
    torch.cuda.synchronize()
    return phi_new.cpu().numpy(), ([t.cpu().numpy()[0] for t in grads] if grads else None), nv, rr


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("spec", [0, 1, 2, 3, 4], ids=["E", "AR", "ARm", "ARp", "energy"])
def test_2d_species_against_direct_solve(mech, spec):
    """Every species class and the electron energy, inhomogeneous-Neumann walls
    valued by species_bc (the wall loss of one step stays a few per cent of the
    wall cells' content at this dt)."""
    case, prm, old, dsdt = make(mech, 2, (20, 12), 910 + spec, dt=1e-12)
    got, grads, nv, rr = run(mech, case, prm, old, dsdt, spec)
    assert 0 < nv <= 60 and 0 <= rr <= 1e-13
    sol, ref_grads, te = odf.solve(case, spec, old, dsdt[spec], prm, oracle.Port(mech))
    assert rel(got[spec], sol) <= 1e-10
    if spec == mech.e_id:
        for d in range(2):
            assert rel(grads[d], ref_grads[d]) <= 1e-9
    if spec == mech.ns:
        ns = mech.ns
        ne_new = got[mech.e_id]
        te_ref = np.where(te < prm.min_electron_temp, prm.min_electron_temp, te)
        assert rel(got[abi.ETEMP(ns)], te_ref) <= 1e-10
        een_ref = np.where(te < prm.min_electron_temp, 1.5 * K_B * ne_new * prm.min_electron_temp, sol)
        assert rel(got[abi.EEN(ns)], een_ref) <= 1e-10


def test_mixed_boundary_kinds(mech):
    """Dirichlet, zero-gradient, Robin (species_bc's default) and inhomogeneous
    Neumann faces on one box, for the electrons (with their face gradients)."""
    E = abi.CLASS_ELECTRON
    lo = [[abi.BC_IHNEU] * 3 for _ in range(4)]
    hi = [[abi.BC_IHNEU] * 3 for _ in range(4)]
    lo[E][0], hi[E][0] = abi.BC_DIRC, abi.BC_ROBIN
    lo[E][1], hi[E][1] = abi.BC_HNEU, abi.BC_IHNEU
    case, prm, old, dsdt = make(mech, 2, (16, 16), 931, dt=1e-12, bc_lo=lo, bc_hi=hi)
    got, grads, _, _ = run(mech, case, prm, old, dsdt, mech.e_id)
    sol, ref_grads, _ = odf.solve(case, mech.e_id, old, dsdt[mech.e_id], prm, oracle.Port(mech))
    assert rel(got[mech.e_id], sol) <= 1e-10
    for d in range(2):
        assert rel(grads[d], ref_grads[d]) <= 1e-9


@pytest.mark.parametrize("dim,n", [(1, (64,)), (3, (8, 8, 6))])
def test_1d_and_3d(mech, dim, n):
    for spec in (mech.e_id, mech.ns):
        case, prm, old, dsdt = make(mech, dim, n, 950 + dim + spec, dt=1e-12)
        got, grads, _, _ = run(mech, case, prm, old, dsdt, spec)
        sol, ref_grads, _ = odf.solve(case, spec, old, dsdt[spec], prm, oracle.Port(mech))
        assert rel(got[spec], sol) <= 1e-10
        if grads is not None:
            for d in range(dim):
                assert rel(grads[d], ref_grads[d]) <= 1e-9


@pytest.mark.parametrize("dim,n", [(1, (64,)), (2, (32, 16))])
def test_diffusion_dominated_step(mech, dim, n):
    """Zero-gradient walls and a step long enough that D dt/dx^2 is of order one for
    the electrons and the energy, so the coarse levels carry the solve."""
    bc = [[abi.BC_HNEU] * 3 for _ in range(4)]
    for spec in (mech.e_id, mech.ns):
        case, prm, old, dsdt = make(mech, dim, n, 990 + dim + spec, dt=1e-8, bc_lo=bc, bc_hi=bc)
        got, grads, nv, rr = run(mech, case, prm, old, dsdt, spec)
        assert nv >= 1 and rr <= 1e-13
        sol, ref_grads, _ = odf.solve(case, spec, old, dsdt[spec], prm, oracle.Port(mech))
        assert rel(got[spec], sol) <= 1e-10
        if grads is not None:
            for d in range(dim):
                assert rel(grads[d], ref_grads[d]) <= 1e-9


@pytest.mark.parametrize("dim,n,per", [(1, (64,), (1, 0, 0)), (2, (32, 16), (1, 0, 0)), (2, (16, 16), (1, 1, 0)),
                                       (3, (8, 8, 6), (0, 1, 1))])
def test_periodic_directions(mech, dim, n, per):
    """Periodic directions (the state's ghosts filled periodically, as FillPatch
    does) against the direct solve, with zero-gradient walls elsewhere; a long
    step so that the wrap carries diffusion across the coarse levels."""
    b = [[abi.BC_PER if per[d] else abi.BC_HNEU for d in range(3)] for _ in range(4)]
    for spec in (mech.e_id, mech.ns, 3):
        case, prm, old, dsdt = make(mech, dim, n, 1010 + dim + spec, dt=1e-9, bc_lo=b, bc_hi=b, periodic=per)
        got, grads, nv, rr = run(mech, case, prm, old, dsdt, spec)
        assert nv >= 1 and rr <= 1e-13
        sol, ref_grads, _ = odf.solve(case, spec, old, dsdt[spec], prm, oracle.Port(mech))
        assert rel(got[spec], sol) <= 1e-10
        if grads is not None:
            for d in range(dim):
                assert rel(grads[d], ref_grads[d]) <= 1e-9


def test_fixed_cycles_and_refusals(mech):
    case, prm, old, dsdt = make(mech, 2, (16, 8), 970, dt=1e-12)
    _, _, nv, rr = run(mech, case, prm, old, dsdt, 3, tol=0.0, cycles=3)
    assert nv == 3 and rr == -1.0
    # periodic on one side only; an odd number of cells in a periodic direction
    lo = [[abi.BC_PER] * 3 for _ in range(4)]
    hi = [[abi.BC_HNEU] * 3 for _ in range(4)]
    case, prm, old, dsdt = make(mech, 2, (16, 8), 971, dt=1e-12, bc_lo=lo, bc_hi=hi)
    with pytest.raises(abi.VidyutError) as e:
        run(mech, case, prm, old, dsdt, 3)
    assert e.value.status == abi.ERR_ARG
    case, prm, old, dsdt = make(mech, 2, (15, 8), 972, dt=1e-12, bc_lo=lo, bc_hi=lo, periodic=(1, 1, 0))
    with pytest.raises(abi.VidyutError) as e:
        run(mech, case, prm, old, dsdt, 3)
    assert e.value.status == abi.ERR_ARG
