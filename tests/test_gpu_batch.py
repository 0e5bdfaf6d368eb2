"""Batched cases on the GPU (vd_batch_*): parity with the multi-step oracle, with
the per-box entry points stepped case by case, independence of each case from the
rest of the batch, step limits, budget admission, graph replay, the tile tuner."""
import numpy as np
import pytest
import torch

import oracle
from vidyut_b200 import _abi as abi
from vidyut_b200 import api, inputs
from vidyut_b200.mechanism import synthetic

from _util import max_elem_rel, scaled_err, update_scales

pytestmark = pytest.mark.gpu

SEED = inputs.BASE_SEED


@pytest.fixture(scope="module")
def mech():
    m = synthetic(8, 40, SEED + 21)
    api.mech_init(m)
    return m


def make_cases(mech, shapes, seed=4242, **over):
    out = []
    for i, n in enumerate(shapes):
        dim = len(n)
        prm = dict(inputs.MULTISTEP_PARAMS)
        prm.update(over)
        out.append(inputs.build_case(mech, dim, n, (1e-5,) * dim, seed + i, density="loguniform_smooth",
                                     dens_range=(1e10, 1e18), te_range_ev=(0.3, 10.0), params=prm))
    return out


def valid(case, st):
    g = case.gvec
    st = st.numpy() if isinstance(st, torch.Tensor) else st
    return st[:, g[2]:g[2] + case.n[2], g[1]:g[1] + case.n[1], g[0]:g[0] + case.n[0]]


def ghost_trim(case, st, H):
    """case-shaped state -> the batch layout (H ghosts)"""
    return api.trim_ghosts(case, st, H)


def run_batch(cases, precision, nsteps, *, graph=True, per_call=None, limits=None, variant=None):
    out = []
    with api.Batch(precision, budget_bytes=1 << 30, max_cases=64) as b:
        b.set_graph(graph)
        if variant is not None:
            for d in (1, 2, 3):
                if variant < api.batch_tile_shape(d, 0)[1]:
                    b.set_tile_variant(d, variant)
        ids = []
        for i, c in enumerate(cases):
            prm = c.vd_params(precision=precision)
            ids.append(b.add(c, prm, nsteps=(limits[i] if limits else -1)))
        left = nsteps
        while left > 0:
            k = min(left, per_call or left)
            b.step(k)
            left -= k
        for i in ids:
            out.append(b.read(i).numpy().copy())
        st = b.stats()
    return out, st


def oracle_steps(mech, case, nsteps):
    return oracle.run_steps(oracle.Port(mech), case, case.vd_params(), nsteps)


def compare_valid(case, got_trim, ref_full, ns):
    H = 3
    ref = ghost_trim(case, ref_full, H)
    comps = list(range(ns)) + [abi.EEN(ns), abi.ETEMP(ns)]
    g = tuple(H if d < case.dim else 0 for d in range(3))
    v = (comps, slice(g[2], g[2] + case.n[2]), slice(g[1], g[1] + case.n[1]), slice(g[0], g[0] + case.n[0]))
    return got_trim[v], ref[v]


def test_batch_fp64_matches_multistep_oracle(mech):
    """Every step of the batch equals the oracle's step from the same state (FP64,
    error relative to the gross magnitude of the step's summed terms <= 1e-12),
    and the whole trajectory stays within 1e-9 elementwise of the oracle's own.
    The trajectory bound is looser than one step's because this synthetic
    workload is stiff for an explicit update: cells whose electrons fall to the
    density floor get Te = 2/3 EEN/(kB ne) spikes of 1e12 K, and rates evaluated
    there amplify last-bit differences of earlier steps (about 1e-11 seen)."""
    from dataclasses import replace
    n = 5
    ns = mech.ns
    cases = make_cases(mech, [(24, 13), (40, 9), (64,), (17, 31)])
    port = oracle.Port(mech)
    with api.Batch(abi.PREC_FP64, budget_bytes=1 << 28, max_cases=8) as b:
        ids = [b.add(c, c.vd_params(precision=abi.PREC_FP64)) for c in cases]
        st = b.stats()
        assert st["ncases_dim"][1] == 1 and st["ncases_dim"][2] == 3
        prev = [c.state.copy() for c in cases]
        for k in range(n):
            b.step(1)
            for i, c in enumerate(cases):
                got = b.read(ids[i]).numpy().copy()
                ck = replace(c, state=prev[i], gradne=inputs.face_gradients(c, prev[i]))
                want = oracle.run_steps(port, ck, ck.vd_params(), 1)
                _, _, nsc = update_scales(port, ck, ck.vd_params())
                a, w = valid_trim(c, got), valid_trim(c, want)
                es = scaled_err(a[:ns + 1], w[:ns + 1], nsc)
                assert es <= 1e-12, (k, c.n, es)
                prev[i] = got
    for c, g in zip(cases, prev):
        a, w = compare_valid(c, g, oracle_steps(mech, c, n), ns)
        ee = np.array([max_elem_rel(a[q], w[q]) for q in range(a.shape[0])])
        print(f"fp64 batch vs oracle {c.n}, {n} steps, elementwise per component: {ee}")
        assert ee.max() <= 1e-9


def test_batch_mixed_within_1e5_of_oracle(mech):
    """the mixed-precision bound: <= 1e-5 max relative error in every species density
    (and the energy, Te) after 20 mixed-precision steps"""
    cases = make_cases(mech, [(48, 40), (33, 57), (128,)], seed=99)
    got, _ = run_batch(cases, abi.PREC_MIXED, 20)
    for c, g in zip(cases, got):
        a, b = compare_valid(c, g, oracle_steps(mech, c, 20), mech.ns)
        errs = np.array([max_elem_rel(a[q], b[q]) for q in range(a.shape[0])])
        print(f"mixed batch vs oracle {c.n}, 20 steps, per component: {errs}")
        assert errs.max() <= 1e-5, errs


def per_box_steps(case, prm, nsteps):
    """the plain per-box path: vd_explicit_update_all + vd_fill_ghosts per step"""
    ns = case.mech.ns
    dc = api.upload(case)
    g = case.gvec
    v = (slice(None), slice(g[2], g[2] + case.n[2]), slice(g[1], g[1] + case.n[1]), slice(g[0], g[0] + case.n[0]))
    comps = list(range(ns)) + [abi.EEN(ns), abi.ETEMP(ns)]
    for _ in range(nsteps):
        phi_new, _, _ = dc.new_outputs()
        api.explicit_update_all(dc, prm, phi_new)
        dc.state[v] = phi_new
        api.fill_ghosts(dc.state, case, case.ghost, comps, case.periodic)
    torch.cuda.synchronize()
    return dc.state.cpu().numpy()


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_batch_equals_per_box_path(mech, precision):
    """the batched launch equals the per-box path stepped case by case (the tiles
    differ in shape, not a face's arithmetic): bit for bit in both precisions"""
    cases = make_cases(mech, [(32, 16), (45, 21)], seed=7)
    got, _ = run_batch(cases, precision, 4, variant=0)
    for c, g in zip(cases, got):
        ref = per_box_steps(c, c.vd_params(precision=precision), 4)
        a, b = compare_valid(c, g, ref, mech.ns)
        assert np.array_equal(a, b), max_elem_rel(a, b)


def test_case_alone_equals_case_in_mix(mech):
    """each result is the same alone and in a mixed batch (bit for bit)"""
    cases = make_cases(mech, [(40, 24), (64, 64), (100,), (23, 77)], seed=31)
    mix, _ = run_batch(cases, abi.PREC_MIXED, 6)
    for i, c in enumerate(cases):
        alone, _ = run_batch([c], abi.PREC_MIXED, 6)
        assert np.array_equal(valid_trim(c, alone[0]), valid_trim(c, mix[i]))


def valid_trim(case, st):
    g = tuple(3 if d < case.dim else 0 for d in range(3))
    return st[:, g[2]:g[2] + case.n[2], g[1]:g[1] + case.n[1], g[0]:g[0] + case.n[0]]


def test_step_limits_and_split_calls(mech):
    cases = make_cases(mech, [(30, 20), (20, 30), (50,)], seed=5)
    # case 0 stops after 3 steps, case 1 after 7, case 2 runs all 8; calls of 3 steps
    got, st = run_batch(cases, abi.PREC_FP64, 8, per_call=3, limits=[3, 7, -1])
    for c, g, n in zip(cases, got, [3, 7, 8]):
        ref, _ = run_batch([c], abi.PREC_FP64, n)
        assert np.array_equal(valid_trim(c, g), valid_trim(c, ref[0]))
    assert st["steps_run"] == 3 + 7 + 8


def test_graph_and_direct_launches_agree(mech):
    cases = make_cases(mech, [(36, 12), (70,)], seed=3)
    a, sa = run_batch(cases, abi.PREC_MIXED, 5, graph=True)
    b, sb = run_batch(cases, abi.PREC_MIXED, 5, graph=False)
    for c, x, y in zip(cases, a, b):
        assert np.array_equal(valid_trim(c, x), valid_trim(c, y))
    assert sa["graph_builds"] >= 1 and sb["graph_builds"] == 0


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 6, 7])
def test_tile_variants_agree(mech, variant):
    cases = make_cases(mech, [(37, 29), (90,)], seed=11)
    a, _ = run_batch(cases, abi.PREC_FP64, 3, variant=0)
    b, _ = run_batch(cases, abi.PREC_FP64, 3, variant=variant)
    for c, x, y in zip(cases, a, b):
        assert max_elem_rel(valid_trim(c, x), valid_trim(c, y)) <= 1e-13


@pytest.mark.parametrize("variant", [3, 5, 7])
def test_mixed_tile_variants_agree(mech, variant):
    """Tile shape, residency and species grouping change which thread computes a
    face, not its arithmetic: the mixed path gives the same bits for every variant."""
    cases = make_cases(mech, [(37, 29), (90,)], seed=12)
    a, _ = run_batch(cases, abi.PREC_MIXED, 3, variant=0)
    b, _ = run_batch(cases, abi.PREC_MIXED, 3, variant=variant)
    for c, x, y in zip(cases, a, b):
        assert np.array_equal(valid_trim(c, x), valid_trim(c, y))


def test_budget_admission_and_reuse(mech):
    cases = make_cases(mech, [(64, 64), (64, 64), (64, 64)], seed=13)
    prm = cases[0].vd_params(precision=abi.PREC_MIXED)
    need = api.Batch.case_bytes(cases[0], prm)
    assert need > 0
    with api.Batch(abi.PREC_MIXED, budget_bytes=2 * need + 4096, max_cases=8) as b:
        i0 = b.add(cases[0], prm)
        i1 = b.add(cases[1], prm)
        with pytest.raises(abi.VidyutError) as e:
            b.add(cases[2], prm)
        assert e.value.status == abi.ERR_BUDGET
        assert b.stats()["ncases"] == 2
        b.step(2)
        b.remove(i0)
        i2 = b.add(cases[2], prm)  # the freed region is reused
        b.step(2)
        assert b.info(i1)[0] == 4 and b.info(i2)[0] == 2
        s = b.stats()
        assert s["bytes_used"] <= s["bytes_budget"]


def test_tuner_does_not_advance_state(mech):
    cases = make_cases(mech, [(80, 40), (256,)], seed=17)
    with api.Batch(abi.PREC_MIXED, budget_bytes=1 << 28, max_cases=8) as b:
        ids = [b.add(c, c.vd_params(precision=abi.PREC_MIXED)) for c in cases]
        b.step(1)
        before = [b.read(i).numpy().copy() for i in ids]
        ms = b.tune(trials=2)
        assert (2, 0) in ms and (1, 0) in ms and all(v > 0 for v in ms.values())
        after = [b.read(i).numpy().copy() for i in ids]
        for c, x, y in zip(cases, before, after):
            assert np.array_equal(valid_trim(c, x), valid_trim(c, y))
        b.step(1)
        assert b.info(ids[0])[0] == 2


def test_fill_ghosts_matches_host_foextrap(mech):
    c = make_cases(mech, [(19, 11)], seed=23)[0]
    ns = mech.ns
    st = c.state.copy()
    g = c.gvec
    st[:, g[2]:g[2] + c.n[2], g[1]:g[1] + c.n[1], g[0]:g[0] + c.n[0]] *= 1.5
    dev = torch.from_numpy(st).cuda()
    comps = list(range(ns)) + [abi.EEN(ns)]
    for periodic in [(0, 0, 0), (1, 1, 0)]:
        d = dev.clone()
        api.fill_ghosts(d, c, 3, comps, periodic)
        ref = st.copy()
        sub = np.ascontiguousarray(ref[comps])
        inputs.fill_ghosts(sub, c.dim, 3, periodic)
        ref[comps] = sub
        got = d.cpu().numpy()
        # face-adjacent ghosts (x ghosts on valid rows, y ghosts on valid columns)
        x = (comps, slice(g[2], g[2] + 1), slice(g[1], g[1] + c.n[1]), slice(None))
        y = (comps, slice(g[2], g[2] + 1), slice(None), slice(g[0], g[0] + c.n[0]))
        assert np.array_equal(got[x], ref[x])
        assert np.array_equal(got[y], ref[y])


def test_batch_rejects_bad_input(mech):
    c = make_cases(mech, [(16, 16)], seed=29)[0]
    with api.Batch(abi.PREC_MIXED, budget_bytes=1 << 26, max_cases=2) as b:
        with pytest.raises(abi.VidyutError) as e:
            b.add(c, c.vd_params(precision=abi.PREC_FP64))  # precision differs from the batch's
        assert e.value.status == abi.ERR_ARG
        with pytest.raises(abi.VidyutError) as e:
            b.add(c, c.vd_params(precision=abi.PREC_MIXED, weno_scheme=7))
        assert e.value.status == abi.ERR_SCHEME
        with pytest.raises(abi.VidyutError):
            b.remove(12345)
        b.add(c, c.vd_params(precision=abi.PREC_MIXED))
        b.add(c, c.vd_params(precision=abi.PREC_MIXED))
        with pytest.raises(abi.VidyutError) as e:
            b.add(c, c.vd_params(precision=abi.PREC_MIXED))  # max_cases reached
        assert e.value.status == abi.ERR_BUDGET
