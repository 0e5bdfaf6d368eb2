"""Serving loop on the GPU (vd_server_*): a request's result is the same alone and
in a mix of concurrently resident requests, admission respects the HBM budget,
oversized requests are refused, bounded waits time out on the host, statistics."""
import time

import numpy as np
import pytest

from vidyut_b200 import _abi as abi
from vidyut_b200 import api, inputs
from vidyut_b200.mechanism import synthetic

pytestmark = pytest.mark.gpu

SEED = inputs.BASE_SEED


@pytest.fixture(scope="module")
def mech():
    m = synthetic(8, 40, SEED + 21)
    api.mech_init(m)
    return m


def make(mech, n, seed, volt=1000.0, p_bar=1.0):
    dim = len(n)
    return inputs.build_case(mech, dim, n, (1e-5,) * dim, seed, density="loguniform_smooth",
                             dens_range=(1e10, 1e18), te_range_ev=(0.3, 10.0), voltage=volt,
                             bg_density=2.4e25 * p_bar, params=dict(inputs.MULTISTEP_PARAMS), n_modes=4)


def valid(case, st):
    g = tuple(3 if d < case.dim else 0 for d in range(3))
    return st[:, g[2]:g[2] + case.n[2], g[1]:g[1] + case.n[1], g[0]:g[0] + case.n[0]]


def serve(reqs, precision=abi.PREC_MIXED, budget=1 << 30, quantum=7, stagger_s=0.0):
    out = []
    with api.Server(precision, budget_bytes=budget, max_cases=64, quantum_steps=quantum) as s:
        ids = []
        for c, n in reqs:
            ids.append(s.submit(c, c.vd_params(precision=precision), n))
            if stagger_s:
                time.sleep(stagger_s)
        for i in ids:
            out.append(s.wait(i, timeout_s=120.0))
        st = s.stats()
    return out, st


def test_result_alone_equals_result_in_mix(mech):
    reqs = [(make(mech, (40, 24), 1, 800.0, 0.3), 23), (make(mech, (300,), 2, 4000.0, 5.0), 40),
            (make(mech, (64, 33), 3, 2500.0, 1.0), 9), (make(mech, (128,), 4, 600.0, 0.1), 31),
            (make(mech, (17, 50), 5, 1500.0, 8.0), 16)]
    mix, st = serve(reqs, stagger_s=0.002)
    assert st["completed"] == len(reqs) and st["failed"] == 0
    for (c, n), (got, lat) in zip(reqs, mix):
        alone, _ = serve([(c, n)])
        assert np.array_equal(valid(c, got), valid(c, alone[0][0]))
        assert lat > 0.0
        # the state moved
        assert not np.array_equal(valid(c, got)[:c.mech.ns], valid(c, c.state)[:c.mech.ns])


def test_server_equals_batch(mech):
    c = make(mech, (48, 20), 7)
    (got, _), = serve([(c, 12)], precision=abi.PREC_FP64, quantum=5)[0]
    with api.Batch(abi.PREC_FP64, budget_bytes=1 << 28, max_cases=4) as b:
        i = b.add(c, c.vd_params(precision=abi.PREC_FP64))
        b.step(12)
        ref = b.read(i).numpy()
    assert np.array_equal(valid(c, got), valid(c, ref))


def test_admission_keeps_to_the_budget(mech):
    reqs = [(make(mech, (96, 96), 10 + i), 15) for i in range(5)]
    need = api.Batch.case_bytes(reqs[0][0], reqs[0][0].vd_params(precision=abi.PREC_MIXED))
    budget = 2 * need + 8192  # room for two at a time
    res, st = serve(reqs, budget=budget, quantum=4)
    assert st["completed"] == 5 and st["failed"] == 0
    assert 0 < st["peak_bytes_used"] <= budget
    assert st["peak_bytes_used"] >= 2 * need  # two were resident together
    assert st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["solves_per_s"] > 0 and st["cell_updates_per_s"] > 0
    # requests that queued behind the budget waited longer than the first ones
    lats = [lat for _, lat in res]
    assert max(lats[2:]) > min(lats[:2])


def test_oversized_request_refused_and_timeout(mech):
    big = make(mech, (256, 256), 20)
    with api.Server(abi.PREC_MIXED, budget_bytes=16 << 20, max_cases=4, quantum_steps=10) as s:
        with pytest.raises(abi.VidyutError) as e:
            s.submit(big, big.vd_params(precision=abi.PREC_MIXED), 10)
        assert e.value.status == abi.ERR_BUDGET
        small = make(mech, (64,), 21)
        rid = s.submit(small, small.vd_params(precision=abi.PREC_MIXED), 400)
        with pytest.raises(abi.VidyutError) as e:
            s.wait(rid, timeout_s=0.0)  # a host-side bounded wait: nothing waits on the GPU
        assert e.value.status == abi.ERR_TIMEOUT
        st, lat = s.wait(rid, timeout_s=120.0)
        assert np.all(np.isfinite(valid(small, st)))
        with pytest.raises(abi.VidyutError):
            s.wait(rid, timeout_s=1.0)  # already collected
        with pytest.raises(abi.VidyutError) as e:
            s.submit(small, small.vd_params(precision=abi.PREC_FP64), 5)  # precision differs
        assert e.value.status == abi.ERR_ARG
