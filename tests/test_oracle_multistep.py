"""Multi-step oracle (CPU): the C restatement stepped several times agrees bit for
bit with the reference's own code compiled here, on the batched workload's
mechanism, with the evolving-state flags (gradne from the state, Te update,
density floors) on; and the ghost refill matches the reference's foextrap."""
import numpy as np
import pytest

import oracle
from vidyut_b200 import _abi as abi
from vidyut_b200 import inputs
from vidyut_b200.mechanism import synthetic

REF = "synth8x40_s20261224"


def small_cases():
    mech = synthetic(8, 40, inputs.BASE_SEED + 21)
    out = []
    for i, (n, dim) in enumerate([((24, 13), 2), ((40,), 1)]):
        c = inputs.build_case(mech, dim, n, (1e-5,) * dim, 777 + i, density="loguniform_smooth",
                              dens_range=(1e10, 1e18), te_range_ev=(0.3, 10.0),
                              params=dict(inputs.MULTISTEP_PARAMS))
        out.append(c)
    return mech, out


@pytest.mark.parametrize("idx", [0, 1])
def test_port_matches_reference_over_steps(idx):
    mech, cases = small_cases()
    case = cases[idx]
    if not oracle.RefLib.available(REF, case.dim):
        pytest.skip("reference build not present")
    prm = case.vd_params()
    a = oracle.run_steps(oracle.Port(mech), case, prm, 4)
    b = oracle.run_steps(oracle.RefLib(REF, case.dim), case, prm, 4)
    g = case.gvec
    v = (slice(None), slice(g[2], g[2] + case.n[2]), slice(g[1], g[1] + case.n[1]), slice(g[0], g[0] + case.n[0]))
    assert np.array_equal(a[v], b[v])
    # the state moved
    assert not np.array_equal(a[v][:mech.ns], case.state[v][:mech.ns])


def test_gradne_from_state_equals_given_face_difference():
    """gradne_from_state = the face difference of ne, the way the inputs build gradne_fc."""
    mech, cases = small_cases()
    case = cases[0]
    port = oracle.Port(mech)
    p1 = case.vd_params(gradne_from_state=1)
    p0 = case.vd_params(gradne_from_state=0)
    assert np.array_equal(port.update_all(case, p1)["phi_new"], port.update_all(case, p0)["phi_new"])
    gr = inputs.face_gradients(case, case.state)
    for d in range(case.dim):
        assert np.array_equal(gr[d], case.gradne[d])


def test_fill_ghosts_periodic_wrap():
    # 1-D: 4 valid cells and 3 ghosts on each side
    st = np.zeros((2, 1, 1, 10))
    st[:, 0, 0, 3:7] = [[1, 2, 3, 4], [5, 6, 7, 8]]
    inputs.fill_ghosts(st, 1, 3, periodic=(1, 0, 0))
    assert list(st[0, 0, 0]) == [2, 3, 4, 1, 2, 3, 4, 1, 2, 3]
    st2 = np.zeros((2, 1, 1, 10))
    st2[:, 0, 0, 3:7] = [[1, 2, 3, 4], [5, 6, 7, 8]]
    inputs.fill_ghosts(st2, 1, 3)
    assert list(st2[1, 0, 0]) == [5, 5, 5, 5, 6, 7, 8, 8, 8, 8]
