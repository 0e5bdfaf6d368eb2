"""One box split into slabs over two or three ranks (vidyut_b200/slab.py), on the CPU with
the gloo backend: after the halo exchange each rank's slab holds exactly the
cells of the single box, the explicit update of each slab (the C oracle, with the
global domain passed in its parameters) equals the single-box update of those
cells bit for bit, and the common time step is the minimum over ranks."""
import dataclasses
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from vidyut_b200 import _abi as abi
from vidyut_b200.slab import Slab, split_extent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _make_case(dim, periodic):
    from vidyut_b200 import inputs
    from vidyut_b200 import mechanism as mm
    m = mm.argon(10, 20261204)
    n = (24, 17) if dim == 2 else (10, 8, 9)
    per = tuple(1 if (periodic and d == dim - 1) else 0 for d in range(3))
    return inputs.build_case(m, dim, n, (1e-5,) * dim, 61, density="blob", periodic=per)


def _params(case, periodic):
    if not periodic:
        return case.vd_params()
    ax = case.dim - 1
    lo = [[abi.BC_IHNEU if d != ax else abi.BC_PER for d in range(3)] for _ in range(4)]
    return case.vd_params(bc_lo=lo, bc_hi=lo)


def _worker(rank, world, port, dim, periodic):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import oracle
        case = _make_case(dim, periodic)
        port_ = oracle.Port(case.mech)
        want = port_.update_all(case, _params(case, periodic))["phi_new"]
        sl = Slab(case.n, dim, case.ghost, rank, world, periodic=periodic)
        ax = 3 - sl.axis
        win = [slice(None)] * 4
        win[ax] = sl.window(sl.axis)
        ref = np.ascontiguousarray(case.state[tuple(win)])
        local = torch.from_numpy(ref.copy())
        g = case.ghost
        below, above = sl.neighbours()
        if below is not None:
            local.narrow(ax, 0, g).fill_(float("nan"))
        if above is not None:
            local.narrow(ax, local.shape[ax] - g, g).fill_(float("nan"))
        sl.exchange(local)
        assert np.array_equal(local.numpy(), ref)
        # the slab's own explicit update, with its face arrays and the global domain
        lo, hi = sl.extent

        def faces(arrs):
            out = []
            for d, a in enumerate(arrs):
                w = [slice(None)] * 4
                w[ax] = slice(lo, hi + 1 + (1 if d == sl.axis else 0))
                out.append(np.ascontiguousarray(a[tuple(w)]))
            return out
        sc = dataclasses.replace(case, n=sl.n_local, state=local.numpy(), efield=faces(case.efield),
                                 gradne=faces(case.gradne))
        prm = _params(sc, periodic)
        domlo, domhi = sl.domain_in_slab()
        for d in range(3):
            prm.domlo[d], prm.domhi[d] = domlo[d], domhi[d]
        got = port_.update_all(sc, prm)["phi_new"]
        w = [slice(None)] * 4
        w[ax] = slice(lo, hi + 1)
        assert np.array_equal(got, want[tuple(w)])
        assert Slab.common_dt(1e-12 * (rank + 2)) == 2e-12
    finally:
        dist.destroy_process_group()


def test_split_extent():
    assert [split_extent(17, 2, r) for r in range(2)] == [(0, 8), (9, 16)]
    assert [split_extent(10, 3, r) for r in range(3)] == [(0, 3), (4, 6), (7, 9)]
    with pytest.raises(ValueError):
        split_extent(2, 3, 0)


@pytest.mark.parametrize("dim,periodic", [(2, False), (2, True), (3, False)])
def test_two_rank_slabs_match_single_box(dim, periodic):
    mp.spawn(_worker, args=(2, _free_port(), dim, periodic), nprocs=2, join=True)


@pytest.mark.parametrize("periodic", [False, True])
def test_three_rank_slabs_match_single_box(periodic):
    """A middle rank exchanges with both neighbours; uneven slabs (17 = 6 + 6 + 5)."""
    mp.spawn(_worker, args=(3, _free_port(), 2, periodic), nprocs=3, join=True)


def test_single_rank_periodic_wrap():
    case = _make_case(2, True)
    sl = Slab(case.n, 2, case.ghost, 0, 1, periodic=True)
    local = torch.from_numpy(case.state.copy())
    local.narrow(2, 0, case.ghost).fill_(float("nan"))
    local.narrow(2, local.shape[2] - case.ghost, case.ghost).fill_(float("nan"))
    sl.exchange(local)
    assert np.array_equal(local.numpy(), case.state)


def test_thin_slab_is_refused_on_one_rank_too():
    """A slab with fewer valid planes than ghost planes cannot fill its ghosts from
    its own cells: the periodic one-rank wrap refuses it like the exchange does."""
    s = Slab(n_global=(4, 2, 1), dim=2, ghost=3, rank=0, world=1, periodic=True)
    state = torch.zeros((1, 1, 2 + 6, 4 + 6), dtype=torch.float64)
    with pytest.raises(ValueError, match="thinner"):
        s.exchange(state)
