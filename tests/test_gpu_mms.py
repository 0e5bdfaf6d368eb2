"""Known answer for the potential solve and the implicit species solve on the GPU:
the reference's MMS case (tests/_mms.py) through the C ABI.  Each step:
vd_poisson_solve with the case's potential source as vd_poisson_params.user_rhs,
vd_fill_ghosts, the explicit drift update (vd_explicit_update_all's dsdt), the
case's species source added to dsdt, then vd_implicit_species_solve with the
case's Robin coefficients (vd_diffusion_params.user_robin), as Source/Evolve.cpp
orders them; run to steady state on 8..64 cells.  With hyp_order 5 both n and phi
converge at 2nd order, with hyp_order 1 n converges at 1st order, as the
reference's plots show (pic_conv_n.gp, pic_conv_phi.gp)."""
import pytest
import torch

from tests._mms import DT, ROBIN, SIZES, T_END, errors, mms_case, orders
from vidyut_b200 import _abi as abi
from vidyut_b200 import api

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    abi.lib()
    abi.check_layout()


def gpu_mms(n: int, hyp_order: int):
    case, x, src_np = mms_case(n, hyp_order)
    ns, g = case.mech.ns, case.ghost
    prm = case.vd_params()
    api.mech_init(case.mech)
    dc = api.upload(case)
    phi_new, dsdt, _ = dc.new_outputs()
    src = torch.from_numpy(src_np).cuda()
    nar = dc.state[1, 0, 0, g:g + n]
    user_rhs = torch.zeros((1, 1, 1, n), dtype=torch.float64, device="cuda")
    pp = api.poisson_params(1, 0.0, 0.0, max_vcycles=6, tol_rel=0.0)
    api.set_poisson_user_rhs(pp, user_rhs)
    state_old = dc.state.clone()
    for _ in range(int(round(T_END / DT))):
        user_rhs[0, 0, 0].copy_(nar)                    # d2phi/dx2 = n
        api.poisson_solve(dc, prm, pp)
        api.fill_ghosts(dc.state, case, g, [0, 1])
        api.explicit_update_all(dc, prm, phi_new, dsdt)
        dsdt[1, 0, 0].add_(src)                         # add_user_react_sources
        state_old.copy_(dc.state)
        api.implicit_species_solve(dc, 1, state_old, dsdt, phi_new, prm, tol_rel=0.0, max_vcycles=4,
                                   robin=ROBIN)
        nar.copy_(phi_new[1, 0, 0])
    torch.cuda.synchronize()
    return errors(nar.cpu().numpy(), dc.state[abi.POT(ns), 0, 0, g:g + n].cpu().numpy(), x)


def test_mms_weno_converges_at_second_order():
    errs = [gpu_mms(n, 5) for n in SIZES]
    on, op = orders([a for a, _ in errs]), orders([b for _, b in errs])
    print("MMS hyp_order 5 errors", errs, "orders n", on, "orders phi", op)
    assert min(on) >= 1.8, on
    assert min(op) >= 1.8, op


def test_mms_upwind_converges_at_first_order():
    errs = [gpu_mms(n, 1) for n in SIZES]
    on = orders([a for a, _ in errs])
    print("MMS hyp_order 1 errors", errs, "orders n", on)
    assert on[-1] >= 0.7, on
    assert errs[-1][0] < errs[0][0] / 3.0
