"""One box split into slabs (vidyut_b200/slab.py), each slab updated on the GPU by
the per-box C-ABI entry point with the global domain in its parameters.

The halo exchange itself runs between processes (tests/test_slab_gloo.py); here
the slabs are cut from the single box with their ghost planes already holding the
neighbours' cells (what the exchange delivers), so the GPU side of the slab path
is checked on one GPU with no kernels waiting on each other: every slab's update
must equal the single box's update of the same cells bit for bit, in both
precisions: the slabs' tiles lie differently from the box's, but a face's
arithmetic does not depend on the tile that computes it.
"""
import dataclasses

import numpy as np
import pytest
import torch

from tests._util import max_elem_rel
from vidyut_b200 import _abi as abi
from vidyut_b200 import api, inputs
from vidyut_b200 import mechanism as mm
from vidyut_b200.slab import Slab

pytestmark = pytest.mark.gpu


def _case(dim, periodic):
    m = mm.argon(10, 20261204)
    n = (40, 27) if dim == 2 else (20, 14, 17)
    per = tuple(1 if (periodic and d == dim - 1) else 0 for d in range(3))
    return inputs.build_case(m, dim, n, (1e-5,) * dim, 71, density="blob", periodic=per)


def _params(case, periodic, prec):
    if not periodic:
        return case.vd_params(precision=prec)
    ax = case.dim - 1
    lo = [[abi.BC_IHNEU if d != ax else abi.BC_PER for d in range(3)] for _ in range(4)]
    return case.vd_params(bc_lo=lo, bc_hi=lo, precision=prec)


def _update(case, prm):
    dc = api.upload(case)
    phi_new, dsdt, rxn = dc.new_outputs()
    api.explicit_update_all(dc, prm, phi_new, dsdt, rxn)
    torch.cuda.synchronize()
    return phi_new.cpu().numpy()


@pytest.mark.parametrize("dim,periodic,world", [(2, False, 2), (2, True, 3), (3, False, 2), (3, True, 3)])
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_slab_updates_equal_single_box(dim, periodic, world, prec):
    case = _case(dim, periodic)
    api.mech_init(case.mech)
    whole = _update(case, _params(case, periodic, prec))
    ns = case.mech.ns
    g = case.ghost
    for rank in range(world):
        sl = Slab(case.n, dim, g, rank, world, periodic=periodic)
        ax = 3 - sl.axis
        lo, hi = sl.extent
        # the slab's state with its ghost planes as the exchange fills them: the
        # neighbouring slabs' cells, or across a periodic direction the far side
        idx = np.arange(lo - g, hi + 1 + g)
        if periodic:
            idx = np.mod(idx, case.n[sl.axis])
        idx = idx + g
        win = [slice(None)] * 4
        win[ax] = slice(lo, hi + 1 + 2 * g)
        st = np.ascontiguousarray(np.take(case.state, idx, axis=ax)) if periodic else \
            np.ascontiguousarray(case.state[tuple(win)])

        def faces(arrs):
            out = []
            for d, a in enumerate(arrs):
                w = [slice(None)] * 4
                w[ax] = slice(lo, hi + 1 + (1 if d == sl.axis else 0))
                out.append(np.ascontiguousarray(a[tuple(w)]))
            return out
        sc = dataclasses.replace(case, n=sl.n_local, state=st, efield=faces(case.efield), gradne=faces(case.gradne))
        prm = _params(sc, periodic, prec)
        domlo, domhi = sl.domain_in_slab()
        for d in range(3):
            prm.domlo[d], prm.domhi[d] = domlo[d], domhi[d]
        got = _update(sc, prm)
        w = [slice(None)] * 4
        w[ax] = slice(lo, hi + 1)
        want = whole[tuple(w)]
        assert np.array_equal(got, want), (rank, max_elem_rel(got[:ns + 1], want[:ns + 1]))
