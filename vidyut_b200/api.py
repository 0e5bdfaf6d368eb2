"""Host-side driver of the C ABI, mirroring the reference's per-box calls.

Function names follow the reference:
    mech_init                  plasmachem::init + the case Chemistry.H
    compute_explicit_flux      ParallelFor(convert(bx, dir)) { compute_flux(...) }
    compute_dsdt               Vidyut::compute_dsdt
    reaction_source            the rxnsrc lambda of update_rxnsrc_at_all_levels
    compute_elecenergy_source  Vidyut::compute_elecenergy_source
    explicit_update_all        one explicit step of the whole path (fused)

Device memory and streams come from PyTorch (plumbing only); every computation
runs in libvidyut_b200.so.  A failed call raises VidyutError with the library's
status and message; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi as abi
from .inputs import BoxCase
from .mechanism import Mechanism

_loaded_mech = None


def mech_init(mech: Mechanism) -> None:
    global _loaded_mech
    L = abi.lib()
    from . import tune
    tune.apply()
    cm = mech.to_c()
    abi.check(L.vd_mech_init(C.byref(cm)), "vd_mech_init")
    _loaded_mech = mech


def _stream(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def t_a4(t: torch.Tensor, begin) -> abi.VdArray4:
    """Array4 over a contiguous float64 tensor of shape (ncomp, nz, ny, nx)."""
    assert t.dtype == torch.float64 and t.is_contiguous() and t.dim() == 4
    return abi.make_array4(t.data_ptr(), tuple(t.shape), begin)


@dataclass
class DeviceCase:
    """A BoxCase resident on the GPU."""
    case: BoxCase
    state: torch.Tensor
    efield: list
    gradne: list

    @property
    def ns(self):
        return self.case.mech.ns

    def sb(self) -> abi.VdArray4:
        return t_a4(self.state, self.case.state_begin())

    def box(self) -> abi.VdBox:
        return abi.make_box(self.case.lo, self.case.hi, self.case.dim)

    def face_a4s(self, which):
        arrs = self.efield if which == "efield" else self.gradne
        return (abi.VdArray4 * 3)(*[t_a4(arrs[d], (0, 0, 0)) for d in range(3)])

    def new_outputs(self):
        """phi_new initialised with the valid-region state (components the update does
        not write keep their values), zeroed dsdt and rxn (NS+1 components)."""
        c = self.case
        g = c.gvec
        valid = self.state[:, g[2]:g[2] + c.n[2], g[1]:g[1] + c.n[1], g[0]:g[0] + c.n[0]]
        phi_new = valid.contiguous().clone()
        shp = (self.ns + 1, c.n[2], c.n[1], c.n[0])
        return (phi_new, torch.zeros(shp, dtype=torch.float64, device=self.state.device),
                torch.zeros(shp, dtype=torch.float64, device=self.state.device))


def upload(case: BoxCase, device="cuda") -> DeviceCase:
    st = torch.from_numpy(case.state).to(device)
    ef = [torch.from_numpy(a).to(device) for a in case.efield]
    gn = [torch.from_numpy(a).to(device) for a in case.gradne]
    return DeviceCase(case, st, ef, gn)


def face_tensor(case: BoxCase, d: int, device="cuda") -> torch.Tensor:
    n = list(case.n)
    n[d] += 1
    return torch.zeros((1, n[2], n[1], n[0]), dtype=torch.float64, device=device)


def compute_explicit_flux(dc: DeviceCase, d: int, specid: int, fx: torch.Tensor, *, hyp_order=5, weno=3,
                          bclo=(3, 3, 3), bchi=(3, 3, 3), Tg=300.0, dt=1e-12, udv=0, uvel=(0.0, 0.0, 0.0),
                          vel_species=0, stream=None) -> None:
    L = abi.lib()
    c = dc.case
    i3 = lambda v: (C.c_int32 * 3)(*[int(x) for x in v])  # noqa: E731
    d3 = lambda v: (C.c_double * 3)(*[float(x) for x in v])  # noqa: E731
    rc = L.vd_compute_explicit_flux(C.byref(dc.box()), d, specid, dc.sb(), i3(bclo), i3(bchi), i3((0, 0, 0)),
                                    i3([c.n[q] - 1 for q in range(3)]), t_a4(fx, (0, 0, 0)), Tg, 0.0, 0.0,
                                    d3(c.dx), dt, hyp_order, udv, weno, d3(uvel), vel_species, _stream(stream))
    abi.check(rc, "vd_compute_explicit_flux")


def compute_dsdt(dc: DeviceCase, specid: int, flux: list, rxn: torch.Tensor, dsdt: torch.Tensor,
                 stream=None) -> None:
    L = abi.lib()
    fl = (abi.VdArray4 * 3)(*[t_a4(flux[d] if d < len(flux) else flux[0], (0, 0, 0)) for d in range(3)])
    d3 = (C.c_double * 3)(*dc.case.dx)
    rc = L.vd_compute_dsdt(C.byref(dc.box()), specid, fl, t_a4(rxn, (0, 0, 0)), t_a4(dsdt, (0, 0, 0)), d3,
                           _stream(stream))
    abi.check(rc, "vd_compute_dsdt")


def reaction_source(dc: DeviceCase, rxn: torch.Tensor, Tg=300.0, stream=None) -> None:
    L = abi.lib()
    rc = L.vd_reaction_source(C.byref(dc.box()), dc.sb(), t_a4(rxn, (0, 0, 0)), Tg, 0.0, 0.0, _stream(stream))
    abi.check(rc, "vd_reaction_source")


def compute_elecenergy_source(dc: DeviceCase, rxn: torch.Tensor, dsdt_energy: torch.Tensor,
                              phi_new: torch.Tensor, prm: abi.VdParams, stream=None) -> None:
    L = abi.lib()
    rc = L.vd_elecenergy_source(C.byref(dc.box()), dc.sb(), t_a4(rxn, (0, 0, 0)), dc.face_a4s("efield"),
                                dc.face_a4s("gradne"), t_a4(dsdt_energy, (0, 0, 0)), t_a4(phi_new, (0, 0, 0)),
                                C.byref(prm), _stream(stream))
    abi.check(rc, "vd_elecenergy_source")


def explicit_update_all(dc: DeviceCase, prm: abi.VdParams, phi_new: torch.Tensor, dsdt: torch.Tensor | None = None,
                        rxn: torch.Tensor | None = None, stream=None) -> None:
    L = abi.lib()
    rc = L.vd_explicit_update_all(C.byref(dc.box()), dc.sb(), dc.face_a4s("efield"), dc.face_a4s("gradne"),
                                  t_a4(phi_new, (0, 0, 0)),
                                  t_a4(dsdt, (0, 0, 0)) if dsdt is not None else abi.null_array4(),
                                  t_a4(rxn, (0, 0, 0)) if rxn is not None else abi.null_array4(),
                                  C.byref(prm), _stream(stream))
    abi.check(rc, "vd_explicit_update_all")


def box_checksums(dc: DeviceCase, rxn: torch.Tensor, phi_new: torch.Tensor, stream=None) -> np.ndarray:
    L = abi.lib()
    out = torch.zeros(4, dtype=torch.float64, device=rxn.device)
    rc = L.vd_box_checksums(C.byref(dc.box()), t_a4(rxn, (0, 0, 0)), t_a4(phi_new, (0, 0, 0)), out.data_ptr(),
                            _stream(stream))
    abi.check(rc, "vd_box_checksums")
    return out.cpu().numpy()


def explicit_update_all_noalloc(dc: DeviceCase, prm: abi.VdParams, phi_new: torch.Tensor,
                                dsdt: torch.Tensor | None = None, rxn: torch.Tensor | None = None,
                                stream=None) -> None:
    """explicit_update_all for callers that must not have the library allocate
    device memory during a step (for example a host whose memory arena owns the
    GPU): its scratch comes from a fixed VD_NOALLOC_SCRATCH_BYTES array in the
    library.  Boxes whose scratch would not fit raise VidyutError(ERR_NOMEM)."""
    L = abi.lib()
    rc = L.vd_explicit_update_all_noalloc(C.byref(dc.box()), dc.sb(), dc.face_a4s("efield"),
                                          dc.face_a4s("gradne"), t_a4(phi_new, (0, 0, 0)),
                                          t_a4(dsdt, (0, 0, 0)) if dsdt is not None else abi.null_array4(),
                                          t_a4(rxn, (0, 0, 0)) if rxn is not None else abi.null_array4(),
                                          C.byref(prm), _stream(stream))
    abi.check(rc, "vd_explicit_update_all_noalloc")
