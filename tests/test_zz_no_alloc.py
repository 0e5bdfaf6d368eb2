"""The allocation-free explicit update, checked against the regular entry point.

Hosts that cannot let the library allocate device memory while they step (an
AMReX application's memory arena typically owns most of the GPU; other callers
allow no allocation inside the time-step loop) call
vd_explicit_update_all_noalloc, whose scratch is a fixed array inside the
library.  Its results must equal those of vd_explicit_update_all within the
FP64 parity tolerance of the other GPU tests (1e-12), on consecutive calls that
reuse the same array, and a box whose scratch does not fit must be refused.  The
array is reserved when the device is set up (vd_mech_init); after that the entry
point must not take any device memory, which a fresh process checks with the
device's free-memory count.
This file is collected last so that a run stopping at the first failure has run
everything else first; it also passes on its own in a fresh process.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from tests._util import normwise_rel, per_component_rel
from vidyut_b200 import _abi as abi
from vidyut_b200 import api
from vidyut_b200 import inputs as vin
from vidyut_b200 import mechanism as mm

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _regular(dc, prm):
    phi_new, dsdt, rxn = dc.new_outputs()
    api.explicit_update_all(dc, prm, phi_new, dsdt, rxn)
    torch.cuda.synchronize()
    return phi_new.cpu().numpy(), dsdt.cpu().numpy(), rxn.cpu().numpy()


def _noalloc(dc, prm, keep_rxn):
    phi_new, dsdt, rxn = dc.new_outputs()
    api.explicit_update_all_noalloc(dc, prm, phi_new, dsdt, rxn if keep_rxn else None)
    torch.cuda.synchronize()
    return phi_new.cpu().numpy(), dsdt.cpu().numpy(), (rxn.cpu().numpy() if keep_rxn else None)


def _same(a, b):
    return max(per_component_rel(a, b).max(), normwise_rel(a, b)) <= TOL


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    abi.lib()
    abi.check_layout()


def test_noalloc_matches_regular_entry_point_on_consecutive_calls():
    case = vin.config_argon2d(n=(96, 80))
    api.mech_init(case.mech)
    dc = api.upload(case)
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        prm = case.vd_params(precision=prec)
        want = _regular(dc, prm)
        # two calls in a row through the shared array: the reaction source lives in
        # the array (rxn not kept) on the first, the caller's rxn on the second
        for keep_rxn in (False, True):
            got = _noalloc(dc, prm, keep_rxn)
            assert _same(got[0], want[0]) and _same(got[1], want[1])
            if keep_rxn:
                assert _same(got[2], want[2])


def test_noalloc_second_mechanism_reuses_array():
    """a different mechanism and dimension right after: nothing stale leaks in"""
    case = vin.build_case(mm.synthetic(8, 40, vin.BASE_SEED + 21), 3, (20, 18, 16), (1e-5,) * 3,
                          vin.BASE_SEED + 77, density="loguniform_smooth", dens_range=(1e10, 1e18))
    api.mech_init(case.mech)
    dc = api.upload(case)
    prm = case.vd_params()
    want = _regular(dc, prm)
    for _ in range(2):
        got = _noalloc(dc, prm, keep_rxn=False)
        assert _same(got[0], want[0]) and _same(got[1], want[1])


def test_noalloc_refuses_boxes_beyond_the_fixed_scratch():
    # 24 species on 72^3 cells: (78^3 + 25 * 72^3) doubles > 64 MiB
    case = vin.build_case(mm.synthetic(24, 150, vin.BASE_SEED + 11), 3, (72, 72, 72), (1e-5,) * 3,
                          vin.BASE_SEED + 78, density="loguniform_smooth")
    api.mech_init(case.mech)
    dc = api.upload(case)
    phi_new, _, _ = dc.new_outputs()
    with pytest.raises(abi.VidyutError) as e:
        api.explicit_update_all_noalloc(dc, case.vd_params(), phi_new)
    assert e.value.status == abi.ERR_NOMEM
    assert "scratch" in str(e.value)
    assert abi.NOALLOC_SCRATCH_BYTES == 64 << 20


_NO_ALLOC_PROBE = r"""
import json, torch
from vidyut_b200 import api, inputs as vin
torch.cuda.set_device(0)
big = vin.config_argon2d(n=(96, 80))
small = vin.config_argon2d(n=(12, 10))
torch.zeros(1, device="cuda")
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
api.mech_init(big.mech)                 # device set-up: the fixed array is reserved here
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
dcs, dcb = api.upload(small), api.upload(big)
outs, outb = dcs.new_outputs(), dcb.new_outputs()
prms = [big.vd_params(precision=p, check_finite=c) for p in (0, 1) for c in (0, 1)]
api.explicit_update_all_noalloc(dcs, small.vd_params(), outs[0])   # first launch of each kernel
torch.cuda.synchronize()
free2 = torch.cuda.mem_get_info()[0]
for prm in prms:
    for keep in (False, True):
        api.explicit_update_all_noalloc(dcb, prm, outb[0], outb[1], outb[2] if keep else None)
torch.cuda.synchronize()
free3 = torch.cuda.mem_get_info()[0]
print(json.dumps({"reserved_at_setup": free0 - free1, "taken_by_calls": free2 - free3}))
"""


def test_noalloc_calls_take_no_device_memory():
    """In a fresh process: after set-up and one first call (which loads the
    kernels' code), eight allocation-free calls on a larger box, both
    precisions, with and without the non-finite check and the caller's rxn,
    leave the device's free memory exactly as it was."""
    root = Path(__file__).resolve().parents[1]
    env = dict(os.environ, CUDA_MODULE_LOADING="LAZY", PYTHONPATH=str(root))
    r = subprocess.run([sys.executable, "-c", _NO_ALLOC_PROBE], cwd=root, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = json.loads(r.stdout.strip().splitlines()[-1])
    assert got["taken_by_calls"] == 0, got
    assert got["reserved_at_setup"] >= abi.NOALLOC_SCRATCH_BYTES, got
