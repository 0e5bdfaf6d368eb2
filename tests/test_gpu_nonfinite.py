"""Non-finite inputs and invalid scalars on the GPU entry points.

The reference aborts the run when it meets an invalid scheme or box
(Source/compute_explicit_flux.H:100,315); this library returns a status instead.
NaN and infinity are injected on the host, into the input arrays before they are
uploaded (no kernel is made to fault): with vd_params.check_finite the per-box
update reports VD_ERR_NONFINITE, a batch marks the case and stops stepping it,
and the server fails that request alone.  Tg <= 0 and a non-finite dt are refused
before anything is launched.
"""
import dataclasses

import numpy as np
import pytest
import torch

from vidyut_b200 import _abi as abi
from vidyut_b200 import api
from vidyut_b200 import inputs as vin
from vidyut_b200 import mechanism as mm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    abi.lib()
    abi.check_layout()


def _argon(n=(40, 32)):
    return vin.config_argon2d(n=n)


def _poisoned(case, comp, value, cell=(5, 7, 0)):
    """a copy of case with state component comp of one valid cell set to value"""
    st = case.state.copy()
    g = case.gvec
    st[comp, g[2] + cell[2], g[1] + cell[1], g[0] + cell[0]] = value
    return dataclasses.replace(case, state=st)


def _update(case, **over):
    api.mech_init(case.mech)
    dc = api.upload(case)
    phi_new, dsdt, rxn = dc.new_outputs()
    api.explicit_update_all(dc, case.vd_params(**over), phi_new, dsdt, rxn)
    torch.cuda.synchronize()
    return phi_new


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_clean_input_passes_the_check(prec):
    case = _argon()
    a = _update(case, precision=prec, check_finite=1).cpu().numpy()
    b = _update(case, precision=prec, check_finite=0).cpu().numpy()
    assert np.array_equal(a, b)  # the check changes no result


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
@pytest.mark.parametrize("what", ["electrons", "ion", "energy", "te", "efield_cell", "efield_face"])
def test_nan_or_inf_is_reported(prec, what):
    case = _argon()
    ns = case.mech.ns
    if what == "electrons":
        bad = _poisoned(case, case.mech.e_id, np.nan)
    elif what == "ion":
        bad = _poisoned(case, 1, np.inf)
    elif what == "energy":
        bad = _poisoned(case, abi.EEN(ns), -np.inf)
    elif what == "te":
        bad = _poisoned(case, abi.ETEMP(ns), np.nan)
    elif what == "efield_cell":
        bad = _poisoned(case, abi.EFX(ns), np.inf)
    else:
        ef = [a.copy() for a in case.efield]
        ef[1][0, 0, 9, 4] = np.nan
        bad = dataclasses.replace(case, efield=ef)
    with pytest.raises(abi.VidyutError) as e:
        _update(bad, precision=prec, check_finite=1)
    assert e.value.status == abi.ERR_NONFINITE
    # without the check the call returns normally (and does not synchronise)
    _update(bad, precision=prec, check_finite=0)


def test_invalid_scalars_are_refused_before_launch():
    case = _argon()
    api.mech_init(case.mech)
    dc = api.upload(case)
    phi_new, _, _ = dc.new_outputs()
    n0 = abi.lib().vd_launch_count()
    for over in (dict(Tg=0.0), dict(Tg=-300.0), dict(Tg=float("nan")), dict(dt=float("nan")),
                 dict(dt=float("inf")), dict(dt=-1e-12)):
        with pytest.raises(abi.VidyutError) as e:
            api.explicit_update_all(dc, case.vd_params(**over), phi_new)
        assert e.value.status == abi.ERR_ARG
        with pytest.raises(abi.VidyutError) as e:
            api.explicit_update_all_noalloc(dc, case.vd_params(**over), phi_new)
        assert e.value.status == abi.ERR_ARG
    assert abi.lib().vd_launch_count() == n0


def _multistep(n, seed):
    m = mm.synthetic(8, 40, vin.BASE_SEED + 21)
    return vin.build_case(m, 2, n, (1e-5, 1e-5), seed, density="loguniform_smooth", dens_range=(1e10, 1e18),
                          te_range_ev=(0.3, 10.0), params=dict(vin.MULTISTEP_PARAMS), n_modes=4)


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_batch_marks_the_case_and_stops_stepping_it(prec):
    good = _multistep((48, 40), 11)
    bad = _poisoned(_multistep((40, 33), 12), 0, np.nan, cell=(20, 16, 0))
    api.mech_init(good.mech)
    with api.Batch(prec, budget_bytes=1 << 30, max_cases=8) as b:
        ig = b.add(good, good.vd_params(precision=prec), nsteps=10)
        ib = b.add(bad, bad.vd_params(precision=prec), nsteps=10)
        b.step(3)
        assert b.nonfinite(ib) and not b.nonfinite(ig)
        b.step(3)
        assert b.info(ib)[0] == 3          # no further steps for the failed case
        assert b.info(ig)[0] == 6
        # loading a clean state clears the mark
        clean = _multistep((40, 33), 12)
        b.load(ib, api.trim_ghosts(clean, clean.state, 3), nsteps=2)
        b.step(2)
        assert not b.nonfinite(ib) and b.info(ib)[0] == 2


def test_server_fails_only_the_poisoned_request():
    good = _multistep((48, 40), 21)
    bad = _poisoned(_multistep((44, 30), 22), abi.ETEMP(8), np.inf, cell=(3, 4, 0))
    api.mech_init(good.mech)
    with api.Server(abi.PREC_MIXED, budget_bytes=1 << 30, max_cases=8, quantum_steps=5) as s:
        rg = s.submit(good, good.vd_params(precision=abi.PREC_MIXED), 12)
        rb = s.submit(bad, bad.vd_params(precision=abi.PREC_MIXED), 12)
        with pytest.raises(abi.VidyutError) as e:
            s.wait(rb, timeout_s=120.0)
        assert e.value.status == abi.ERR_NONFINITE
        out, lat = s.wait(rg, timeout_s=120.0)
        assert np.all(np.isfinite(out)) and lat > 0.0
        st = s.stats()
    assert st["failed"] == 1 and st["completed"] == 1
