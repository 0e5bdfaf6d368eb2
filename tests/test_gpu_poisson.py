"""The potential step on the GPU (vd_poisson_solve) against the direct solve of the
same discrete problem (oracle/poisson.py): potential, cell field, face field,
reduced field, ghost refill, convergence and argument checks."""
import numpy as np
import pytest
import torch

from oracle import poisson
from vidyut_b200 import _abi as abi
from vidyut_b200 import api, inputs
from vidyut_b200.mechanism import synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mech():
    m = synthetic(8, 40, inputs.BASE_SEED + 21)
    api.mech_init(m)
    return m


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


# (15, 9): odd extents, so the hierarchy is the finest grid alone (its cycles are
# the one-CTA bottom solve and the correction is added by its own pass)
@pytest.mark.parametrize("n", [(64,), (40, 24), (16, 16, 12), (15, 9)])
def test_poisson_matches_direct_solve(mech, n):
    dim = len(n)
    # a strongly charged case: 1e16-1e18 ions over a 1e14 electron floor
    c = inputs.build_case(mech, dim, n, (1e-5,) * dim, 11, density="loguniform_smooth", dens_range=(1e14, 1e18),
                          n_modes=4)
    V = 1500.0
    dc = api.upload(c)
    prm = c.vd_params()
    pp = api.poisson_params(dim, V, 0.0, max_vcycles=60, tol_rel=1e-11)
    ncyc, rr = api.poisson_solve(dc, prm, pp)
    torch.cuda.synchronize()
    assert 1 <= ncyc < 60 and 0 <= rr <= 1e-11, (ncyc, rr)
    print(f"{n}: {ncyc} V-cycles, relative residual {rr:.2e}")
    ns = mech.ns
    g = c.gvec
    st = dc.state.cpu().numpy()
    v = (slice(g[2], g[2] + n[2] if dim > 2 else 1), slice(g[1], g[1] + (n[1] if dim > 1 else 1)),
         slice(g[0], g[0] + n[0]))
    dl, dh, vl, vh = (1, 0, 0), (1, 0, 0), (V, 0, 0), (0.0, 0, 0)
    phi = poisson.solve(c, dl, dh, vl, vh)
    assert rel(st[abi.POT(ns)][v], phi) <= 1e-9
    E = poisson.cell_field(phi, dim, c.dx)
    for d in range(3):
        got = st[abi.EFX(ns) + d][v]
        if d < dim:
            assert rel(got, E[d]) <= 1e-7, d
        else:
            assert np.all(got == 0.0)
    assert rel(st[abi.REF(ns)][v], poisson.reduced_field(c, E)) <= 1e-7
    for d in range(dim):
        f = poisson.face_field(phi, dim, c.dx, d, dl, dh, vl, vh)
        assert rel(dc.efield[d].cpu().numpy(), f) <= 1e-7, d
    # ghosts of the potential refilled by first-order extrapolation (x ghosts, valid rows)
    gx = st[abi.POT(ns)][v[0], v[1], :g[0]]
    assert np.all(gx == st[abi.POT(ns)][v[0], v[1], g[0]:g[0] + 1])


def test_fixed_cycles_and_errors(mech):
    c = inputs.build_case(mech, 2, (32, 16), (1e-5, 1e-5), 12, density="loguniform_smooth", n_modes=4)
    dc = api.upload(c)
    prm = c.vd_params()
    ncyc, rr = api.poisson_solve(dc, prm, api.poisson_params(2, 800.0, 0.0, max_vcycles=3, tol_rel=0.0))
    assert ncyc == 3 and rr == -1.0
    # the whole domain is required
    bad = c.vd_params()
    bad.domhi[0] = 100
    with pytest.raises(abi.VidyutError) as e:
        api.poisson_solve(dc, bad, api.poisson_params(2, 800.0))
    assert e.value.status == abi.ERR_ARG
    # at least one Dirichlet face
    pp = api.poisson_params(2, 800.0)
    pp.bc_lo[0] = pp.bc_hi[0] = abi.BC_HNEU
    with pytest.raises(abi.VidyutError) as e:
        api.poisson_solve(dc, prm, pp)
    assert e.value.status == abi.ERR_ARG


def test_warm_start_converges_faster(mech):
    c = inputs.build_case(mech, 3, (32, 32, 32), (1e-5,) * 3, 13, density="loguniform_smooth",
                          dens_range=(1e14, 1e18), n_modes=4)
    dc = api.upload(c)
    prm = c.vd_params()
    n1, _ = api.poisson_solve(dc, prm, api.poisson_params(3, 1000.0, max_vcycles=60, tol_rel=1e-11))
    n2, _ = api.poisson_solve(dc, prm, api.poisson_params(3, 1000.0, max_vcycles=60, tol_rel=1e-11))
    assert n2 < n1


def test_time_scales_match_reference_formula(mech):
    import oracle
    c = inputs.build_case(mech, 2, (30, 20), (1e-5, 2e-5), 14, density="loguniform_smooth", n_modes=4)
    dc = api.upload(c)
    prm = c.vd_params()
    got = api.time_scales(dc, prm)
    want = poisson.time_scales(c, prm, oracle.Port(mech))
    for g_, w_ in zip(got, want):
        assert abs(g_ - w_) <= 1e-12 * abs(w_), (got, want)
    assert all(0 < x < 1.0 for x in got)
