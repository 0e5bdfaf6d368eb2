"""GPU parity: every C-ABI entry point against the CPU oracle (and the golden
fixtures written by the reference's own code).

Tolerances:
  FP64 path   relative error <= 1e-12.  Fluxes and the Joule term: normwise,
              max|gpu - ref| / max|ref|.  rxn, dsdt and n + dt*dsdt: relative to the
              gross magnitude of the terms summed into each value (oracle
              update_scale: |face fluxes| counted as the magnitude of the stencil
              values they are reconstructed from): the generated chemistry adds and removes the same
              rate (wdot[E] -= q; wdot[E] += q), so a last-bit difference between
              CUDA's and glibc's exp/pow moves a net rate by eps times the gross
              rate, which can be 1e8 times the net one.  Mechanisms without that
              cancellation (argon, Ar_DC_1d) also pass normwise.
  mixed path  n + dt*dsdt within 1e-5 of the FP64 oracle relative to the same
              gross scale for every species and the electron energy; on spatially
              smooth inputs also elementwise, max|gpu - ref|/|ref| <= 1e-5.
"""
import numpy as np
import pytest
import torch

import oracle
from tests._util import (FIXTURES, load_fixture, normwise_rel, per_component_rel, max_elem_rel,
                         scaled_err, update_scales)
from vidyut_b200 import _abi as abi
from vidyut_b200 import api
from vidyut_b200 import inputs as vin
from vidyut_b200 import mechanism as mm

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_MIXED = 1e-5
SCHEMES = [(1, 3), (2, 3), (5, 1), (5, 2), (5, 3)]


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    abi.lib()
    abi.check_layout()


def seeded_cases():
    S = vin.BASE_SEED
    return {
        "argon2d": vin.build_case(mm.argon(10, S + 1), 2, (70, 45), (1e-5, 1e-5), S + 201, density="blob"),
        "synth24_3d": vin.build_case(mm.synthetic(24, 150, S + 11), 3, (19, 13, 11), (1e-5,) * 3, S + 202,
                                     density="loguniform", dens_range=(1e8, 1e22), te_range_ev=(0.3, 10.0)),
        "synth8_1d": vin.build_case(mm.synthetic(8, 40, S + 21), 1, (300,), (1e-5,), S + 203,
                                    density="loguniform", dens_range=(1e10, 1e18)),
        "synth8_2d": vin.build_case(mm.synthetic(8, 40, S + 21), 2, (45, 33), (1e-5, 2e-5), S + 204,
                                    density="loguniform", dens_range=(1e10, 1e18)),
        "synth24_3d_smooth": vin.build_case(mm.synthetic(24, 150, S + 11), 3, (48, 40, 36), (1e-5,) * 3, S + 205,
                                            density="loguniform_smooth", dens_range=(1e8, 1e22),
                                            te_range_ev=(0.3, 10.0)),
    }


CASES = seeded_cases()


def _gpu_flux(dc, d, s, h, w, **kw):
    fx = api.face_tensor(dc.case, d)
    api.compute_explicit_flux(dc, d, s, fx, hyp_order=h, weno=w, **kw)
    torch.cuda.synchronize()
    return fx.cpu().numpy()


# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", FIXTURES)
def test_golden_fixtures_on_gpu(name):
    """GPU entry points reproduce the reference's own outputs (golden fixtures)."""
    case, meta, outs = load_fixture(name)
    api.mech_init(case.mech)
    dc = api.upload(case)
    udv = 1 if "uvel" in meta else 0
    kw = dict(udv=udv, uvel=tuple(meta.get("uvel", (0, 0, 0))), vel_species=meta.get("vel_species", 0))
    if udv:
        kw.update(bclo=(0, 0, 0), bchi=(0, 0, 0))
    for key, want in outs.items():
        if key.startswith("flux_"):
            _, s, d, h, w = key.split("_")
            got = _gpu_flux(dc, int(d[1:]), int(s[1:]), int(h[1:]), int(w[1:]), **kw)
            assert normwise_rel(got, want) <= TOL64, key
    # Janev / F-fit rates (co2fits): their sums are ill-conditioned, see make_golden.py
    rtol = meta.get("rate_tol", TOL64)
    if "rxn" in outs or "upd_phi_new" in outs:
        prm = case.vd_params()
        rs, ds, nsc = update_scales(oracle.Port(case.mech), case, prm)
    if "rxn" in outs:
        _, _, rxn = dc.new_outputs()
        api.reaction_source(dc, rxn)
        assert scaled_err(rxn.cpu().numpy(), outs["rxn"], rs) <= rtol
    if "upd_phi_new" in outs:
        phi_new, dsdt, rxn = dc.new_outputs()
        api.explicit_update_all(dc, prm, phi_new, dsdt, rxn)
        torch.cuda.synchronize()
        ns = case.mech.ns
        assert scaled_err(dsdt.cpu().numpy(), outs["upd_dsdt"], ds) <= rtol
        assert scaled_err(rxn.cpu().numpy(), outs["upd_rxn"], rs) <= rtol
        pn, want = phi_new.cpu().numpy(), outs["upd_phi_new"]
        assert scaled_err(pn[:ns + 1], want[:ns + 1], nsc) <= rtol
        # diagnostics EJH / EIH and the untouched components
        assert per_component_rel(pn[ns + 1:], want[ns + 1:]).max() <= TOL64


@pytest.mark.parametrize("name", sorted(CASES))
def test_reaction_source_fp64(name):
    case = CASES[name]
    api.mech_init(case.mech)
    dc = api.upload(case)
    _, _, rxn = dc.new_outputs()
    api.reaction_source(dc, rxn)
    port = oracle.Port(case.mech)
    want = port.reaction_source(case)
    got = rxn.cpu().numpy()
    assert scaled_err(got, want, port.rxn_scale(case)) <= TOL64
    if case.mech.name.startswith("argon"):
        assert per_component_rel(got, want).max() <= TOL64


@pytest.mark.parametrize("name", sorted(CASES))
def test_explicit_flux_all_schemes(name):
    case = CASES[name]
    api.mech_init(case.mech)
    dc = api.upload(case)
    port = oracle.Port(case.mech)
    m = case.mech
    ion = next(s for s in range(m.ns) if m.charge[s] > 0)
    for s in (m.e_id, ion, m.ns):
        for d in range(case.dim):
            for h, w in SCHEMES:
                got = _gpu_flux(dc, d, s, h, w)
                want = port.flux(case, d, s, hyp_order=h, weno=w)
                assert normwise_rel(got, want) <= TOL64, (s, d, h, w)


def test_ihneubc_zero_flux_and_periodic_faces():
    """IHNEUBC forces zero flux on the domain faces (compute_explicit_flux.H:318-325);
    other codes leave them computed."""
    case = CASES["argon2d"]
    api.mech_init(case.mech)
    dc = api.upload(case)
    for d in range(2):
        z = _gpu_flux(dc, d, 0, 5, 3, bclo=(3, 3, 3), bchi=(3, 3, 3))
        nz = _gpu_flux(dc, d, 0, 5, 3, bclo=(2, 2, 2), bchi=(1, 1, 1))
        sl_lo = [slice(None)] * 4
        sl_hi = [slice(None)] * 4
        sl_lo[3 - d] = 0
        sl_hi[3 - d] = -1
        assert np.all(z[tuple(sl_lo)] == 0.0) and np.all(z[tuple(sl_hi)] == 0.0)
        assert np.any(nz[tuple(sl_lo)] != 0.0)


def test_dsdt_and_joule():
    case = CASES["synth8_2d"]
    m = case.mech
    api.mech_init(m)
    dc = api.upload(case)
    port = oracle.Port(m)
    rxn_np = port.reaction_source(case)
    rxn = torch.from_numpy(rxn_np).cuda()
    for s in (m.e_id, m.ns):
        fl_np = [port.flux(case, d, s) for d in range(2)]
        fl = [torch.from_numpy(f).cuda() for f in fl_np]
        out = torch.zeros((1, 1, case.n[1], case.n[0]), dtype=torch.float64, device="cuda")
        api.compute_dsdt(dc, s, fl, rxn, out)
        want = port.dsdt(case, s, fl_np, rxn_np)
        assert normwise_rel(out.cpu().numpy(), want) <= 1e-14
    prm = case.vd_params()
    de_want, pn_want = port.elecenergy(case, rxn_np, prm)
    de = torch.zeros((1, 1, case.n[1], case.n[0]), dtype=torch.float64, device="cuda")
    phi_new, _, _ = dc.new_outputs()
    api.compute_elecenergy_source(dc, rxn, de, phi_new, prm)
    torch.cuda.synchronize()
    assert normwise_rel(de.cpu().numpy(), de_want) <= TOL64
    ns = m.ns
    assert normwise_rel(phi_new.cpu().numpy()[abi.EJH(ns)], pn_want[abi.EJH(ns)]) <= TOL64
    assert np.array_equal(phi_new.cpu().numpy()[abi.EIH(ns)], pn_want[abi.EIH(ns)])


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("hw", [(5, 3), (5, 1), (2, 3), (1, 3)])
def test_update_all_fp64(name, hw):
    case = CASES[name]
    api.mech_init(case.mech)
    dc = api.upload(case)
    prm = case.vd_params(hyp_order=hw[0], weno_scheme=hw[1])
    phi_new, dsdt, rxn = dc.new_outputs()
    api.explicit_update_all(dc, prm, phi_new, dsdt, rxn)
    torch.cuda.synchronize()
    port = oracle.Port(case.mech)
    want = port.update_all(case, prm)
    rs, ds, nsc = update_scales(port, case, prm)
    ns = case.mech.ns
    assert scaled_err(rxn.cpu().numpy(), want["rxn"], rs) <= TOL64
    assert scaled_err(dsdt.cpu().numpy(), want["dsdt"], ds) <= TOL64
    pn = phi_new.cpu().numpy()
    assert scaled_err(pn[:ns + 1], want["phi_new"][:ns + 1], nsc) <= TOL64
    assert per_component_rel(pn[ns + 1:], want["phi_new"][ns + 1:]).max() <= TOL64


@pytest.mark.parametrize("name", sorted(CASES))
def test_update_all_mixed_precision(name):
    """FP32 WENO / rates / fluxes with FP64 accumulation: every updated density and
    the electron energy within 1e-5 of the FP64 oracle (elementwise)."""
    case = CASES[name]
    api.mech_init(case.mech)
    dc = api.upload(case)
    prm = case.vd_params(precision=abi.PREC_MIXED)
    phi_new, dsdt, rxn = dc.new_outputs()
    api.explicit_update_all(dc, prm, phi_new, dsdt, rxn)
    torch.cuda.synchronize()
    port = oracle.Port(case.mech)
    want = port.update_all(case, case.vd_params())
    _, _, nsc = update_scales(port, case, case.vd_params())
    ns = case.mech.ns
    pn = phi_new.cpu().numpy()
    per_species = [scaled_err(pn[s], want["phi_new"][s], nsc[s]) for s in range(ns + 1)]
    assert max(per_species) <= TOL_MIXED, per_species
    if "smooth" in name or name.startswith("argon"):
        elem = [max_elem_rel(pn[s], want["phi_new"][s]) for s in range(ns + 1)]
        assert max(elem) <= TOL_MIXED, elem


def test_checksums_charge_conservation():
    case = CASES["synth24_3d"]
    api.mech_init(case.mech)
    dc = api.upload(case)
    phi_new, dsdt, rxn = dc.new_outputs()
    api.explicit_update_all(dc, case.vd_params(), phi_new, dsdt, rxn)
    cs = api.box_checksums(dc, rxn, phi_new)
    assert abs(cs[0]) <= 1e-12 * cs[1]
    want = oracle.Port(case.mech).update_all(case, case.vd_params())
    assert abs(cs[3] - want["phi_new"][:case.mech.ns].sum()) <= 1e-12 * abs(cs[3])


def test_status_codes_without_launch():
    """Invalid calls return the reference's abort conditions as status codes and
    launch nothing."""
    case = CASES["argon2d"]
    api.mech_init(case.mech)
    dc = api.upload(case)
    fx = api.face_tensor(case, 0)
    with pytest.raises(abi.VidyutError) as e:
        api.compute_explicit_flux(dc, 0, 0, fx, hyp_order=3)
    assert e.value.status == abi.ERR_SCHEME
    with pytest.raises(abi.VidyutError) as e:
        api.compute_explicit_flux(dc, 0, 0, fx, hyp_order=5, weno=7)
    assert e.value.status == abi.ERR_SCHEME
    # a state with only one ghost layer cannot feed WENO-5
    small = vin.build_case(case.mech, 2, (16, 12), (1e-5, 1e-5), 7, density="blob", ghost=1)
    ds = api.upload(small)
    fx = api.face_tensor(small, 0)
    with pytest.raises(abi.VidyutError) as e:
        api.compute_explicit_flux(ds, 0, 0, fx, hyp_order=5)
    assert e.value.status == abi.ERR_GHOST
    api.compute_explicit_flux(ds, 0, 0, fx, hyp_order=1)  # one ghost suffices for upwind
    phi_new, dsdt, rxn = dc.new_outputs()
    with pytest.raises(abi.VidyutError) as e:
        api.explicit_update_all(dc, case.vd_params(dim=3), phi_new, dsdt, rxn)
    assert e.value.status == abi.ERR_DIM


@pytest.mark.parametrize("name", ["synth24_3d_smooth", "argon2d"])
def test_specialised_and_table_chemistry_agree(name):
    """vd_mech_init compiles chemistry specialised to the mechanism (NVRTC); the
    table-driven kernel (vd_set_specialize(0)) must give the same update."""
    case = CASES[name]
    L = abi.lib()
    outs = {}
    try:
        for spec in (1, 0):
            L.vd_set_specialize(spec)
            api.mech_init(case.mech)
            assert L.vd_mech_specialized() == spec, L.vd_mech_specialize_status()
            dc = api.upload(case)
            for prec in (abi.PREC_FP64, abi.PREC_MIXED):
                phi_new, dsdt, rxn = dc.new_outputs()
                api.explicit_update_all(dc, case.vd_params(precision=prec), phi_new, dsdt, rxn)
                torch.cuda.synchronize()
                outs[(spec, prec)] = (phi_new.cpu().numpy(), rxn.cpu().numpy())
    finally:
        L.vd_set_specialize(1)
        api.mech_init(case.mech)
    port = oracle.Port(case.mech)
    rs, _, nsc = update_scales(port, case, case.vd_params())
    ns = case.mech.ns
    for prec, tol in ((abi.PREC_FP64, TOL64), (abi.PREC_MIXED, 1e-6)):
        a, b = outs[(1, prec)], outs[(0, prec)]
        assert scaled_err(a[1], b[1], rs) <= tol
        assert scaled_err(a[0][:ns + 1], b[0][:ns + 1], nsc) <= tol


def test_fit_rates_table_and_specialised_kernels_agree():
    """The Janev / F-fit rates of the CO2 reactor header (golden fixture co2fits_2d)
    through the mechanism-specialised kernels and the table-driven ones agree, and
    the mixed-precision rates and updates stay within the mixed tolerance of FP64.
    The mixed path's rate coefficients are FP32 values: a fit that falls below
    FP32's range (k < 2^-126 at a low Te, where the polynomial in ln Te runs to
    large negative exponents) is zero there, so the rates are compared on the
    gross scale floored at 1e-20 of each component's largest over the box."""
    case, meta, outs = load_fixture("co2fits_2d")
    port = oracle.Port(case.mech)
    rs = port.rxn_scale(case)
    rs_floor = np.maximum(rs, 1e-20 * rs.reshape(rs.shape[0], -1).max(axis=1).reshape((-1,) + (1,) * (rs.ndim - 1)))
    prm = case.vd_params()
    _, _, nsc = update_scales(port, case, prm)
    ns = case.mech.ns
    got, pn = {}, {}
    for spec in (1, 0):
        abi.lib().vd_set_specialize(spec)
        try:
            api.mech_init(case.mech)
            assert abi.lib().vd_mech_specialized() == spec
            dc = api.upload(case)
            for prec in (abi.PREC_FP64, abi.PREC_MIXED):
                phi_new, dsdt, rxn = dc.new_outputs()
                api.explicit_update_all(dc, case.vd_params(precision=prec), phi_new, dsdt, rxn)
                torch.cuda.synchronize()
                got[(spec, prec)] = rxn.cpu().numpy()
                pn[(spec, prec)] = phi_new.cpu().numpy()
        finally:
            abi.lib().vd_set_specialize(1)
    api.mech_init(case.mech)
    assert scaled_err(got[(1, abi.PREC_FP64)], got[(0, abi.PREC_FP64)], rs) <= 1e-12
    assert scaled_err(got[(1, abi.PREC_FP64)], outs["upd_rxn"], rs) <= meta["rate_tol"]
    for spec in (1, 0):
        er = scaled_err(got[(spec, abi.PREC_MIXED)], got[(1, abi.PREC_FP64)], rs_floor)
        en = max(scaled_err(pn[(spec, abi.PREC_MIXED)][s], pn[(1, abi.PREC_FP64)][s], nsc[s]) for s in range(ns + 1))
        print(f"co2fits mixed vs FP64 (specialised {spec}): rates {er:.3e}, updates {en:.3e}")
        assert er <= TOL_MIXED and en <= TOL_MIXED
