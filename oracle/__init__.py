"""CPU oracle for the explicit species / electron-energy update (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
package, and only as the checker (or the timed CPU baseline); the product path in
vidyut_b200 never does.

  Port(mech)          the plain-C restatement (vd_oracle.c) driven by the runtime
                      mechanism table, any mechanism and dimension
  RefLib(name, dim)   the reference's own headers compiled against the AMReX shim
                      for one case (oracle/_ref/libvdref_<name>_<dim>d.so)

Both expose the same numpy interface: reaction_source, flux, dsdt, elecenergy,
update_all.  Arrays follow vidyut_b200.inputs.BoxCase: state (NVAR, nz+2g, ny+2g,
nx+2g), outputs on the valid box.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from vidyut_b200 import _abi as abi  # noqa: E402
from vidyut_b200.inputs import BoxCase  # noqa: E402

from .build import ORACLE_LIB, ref_lib_path  # noqa: E402

A4 = abi.VdArray4
A4P = C.POINTER(A4)
BOXP = C.POINTER(abi.VdBox)
MECHP = C.POINTER(abi.VdMech)
PRMP = C.POINTER(abi.VdParams)
I32P = C.POINTER(C.c_int32)
DP = C.POINTER(C.c_double)


def np_a4(arr: np.ndarray, begin) -> A4:
    assert arr.dtype == np.float64 and arr.flags.c_contiguous and arr.ndim == 4
    return abi.make_array4(arr.ctypes.data, arr.shape, begin)


def _i3(v):
    return (C.c_int32 * 3)(*[int(x) for x in v])


def _d3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


def face_shape(case: BoxCase, d: int):
    n = list(case.n)
    n[d] += 1
    return (1, n[2], n[1], n[0])


class _Base:
    """numpy-level driver shared by the port and the reference build.  lo/hi select a
    sub-box of the case (default: the whole box); outputs cover that sub-box."""

    def _box(self, case: BoxCase, lo=None, hi=None):
        return abi.make_box(lo or case.lo, hi or case.hi, case.dim)

    def _sb(self, case):
        return np_a4(case.state, case.state_begin())

    def new_outputs(self, case: BoxCase, lo=None, hi=None):
        lo = lo or case.lo
        hi = hi or case.hi
        ns = case.mech.ns
        g = case.gvec
        valid = case.state[:, g[2] + lo[2]:g[2] + hi[2] + 1, g[1] + lo[1]:g[1] + hi[1] + 1,
                           g[0] + lo[0]:g[0] + hi[0] + 1]
        phi_new = np.ascontiguousarray(valid.copy())
        shp = (ns + 1,) + phi_new.shape[1:]
        return phi_new, np.zeros(shp), np.zeros(shp)

    def flux_ws(self, case, lo=None, hi=None):
        lo = lo or case.lo
        hi = hi or case.hi
        ws = []
        for d in range(3):
            n = [hi[q] - lo[q] + 1 for q in range(3)]
            n[d] += 1
            ws.append(np.zeros((1, n[2], n[1], n[0])))
        return ws, (A4 * 3)(*[np_a4(w, lo) for w in ws])

class Port(_Base):
    """The C restatement, loaded once per process."""

    _lib = None

    def __init__(self, mech):
        if Port._lib is None:
            if not ORACLE_LIB.exists():
                raise RuntimeError(f"{ORACLE_LIB} missing: run `python oracle/build.py`")
            L = C.CDLL(str(ORACLE_LIB))
            L.orc_reaction_source.argtypes = [MECHP, BOXP, A4P, A4P, C.c_double]
            L.orc_compute_explicit_flux.argtypes = [MECHP, BOXP, C.c_int, C.c_int, A4P, I32P, I32P, I32P, I32P,
                                                    A4P, C.c_double, DP, C.c_double, C.c_int, C.c_int, C.c_int,
                                                    DP, C.c_int]
            L.orc_compute_dsdt.argtypes = [BOXP, C.c_int, A4P, A4P, A4P, DP]
            L.orc_elecenergy_source.argtypes = [MECHP, BOXP, A4P, A4P, A4P, A4P, A4P, A4P, PRMP]
            L.orc_explicit_update_all.argtypes = [MECHP, BOXP, A4P, A4P, A4P, A4P, A4P, A4P, A4P, PRMP]
            L.orc_update_scale.argtypes = [MECHP, BOXP, A4P, A4P, A4P, A4P, A4P, PRMP]
            L.orc_fill_ghosts.argtypes = [BOXP, A4P, C.c_int, I32P]
            L.orc_fill_ghosts.restype = None
            L.orc_specmob.argtypes = [MECHP, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]
            L.orc_specmob.restype = C.c_double
            L.orc_specdiff.argtypes = [MECHP, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]
            L.orc_specdiff.restype = C.c_double
            L.orc_weno.argtypes = [C.c_double] * 5 + [C.c_int]
            L.orc_weno.restype = C.c_double
            Port._lib = L
        self.L = Port._lib
        self.mech = mech
        self.cm = mech.to_c()

    def reaction_source(self, case: BoxCase, Tg=300.0):
        _, _, rxn = self.new_outputs(case)
        self.L.orc_reaction_source(C.byref(self.cm), C.byref(self._box(case)), C.byref(self._sb(case)),
                                   C.byref(np_a4(rxn, (0, 0, 0))), Tg)
        return rxn

    def flux(self, case: BoxCase, d: int, specid: int, hyp_order=5, weno=3, bclo=(3, 3, 3), bchi=(3, 3, 3),
             Tg=300.0, dt=1e-12, udv=0, uvel=(0, 0, 0), vel_species=0):
        fx = np.zeros(face_shape(case, d))
        domhi = [case.n[q] - 1 for q in range(3)]
        self.L.orc_compute_explicit_flux(C.byref(self.cm), C.byref(self._box(case)), d, specid,
                                         C.byref(self._sb(case)), _i3(bclo), _i3(bchi), _i3((0, 0, 0)),
                                         _i3(domhi), C.byref(np_a4(fx, (0, 0, 0))), Tg, _d3(case.dx), dt,
                                         hyp_order, udv, weno, _d3(uvel), vel_species)
        return fx

    def update_all(self, case: BoxCase, prm: abi.VdParams, lo=None, hi=None):
        lo = lo or case.lo
        phi_new, dsdt, rxn = self.new_outputs(case, lo, hi)
        ws, wsa = self.flux_ws(case, lo, hi)
        ef = (A4 * 3)(*[np_a4(case.efield[d], (0, 0, 0)) for d in range(3)])
        gn = (A4 * 3)(*[np_a4(case.gradne[d], (0, 0, 0)) for d in range(3)])
        self.L.orc_explicit_update_all(C.byref(self.cm), C.byref(self._box(case, lo, hi)), C.byref(self._sb(case)),
                                       ef, gn, C.byref(np_a4(phi_new, lo)), C.byref(np_a4(dsdt, lo)),
                                       C.byref(np_a4(rxn, lo)), wsa, C.byref(prm))
        return dict(phi_new=phi_new, dsdt=dsdt, rxn=rxn)

    def elecenergy(self, case: BoxCase, rxn: np.ndarray, prm: abi.VdParams):
        """Joule term alone: returns (dsdt_energy starting from 0, phi_new)."""
        phi_new, _, _ = self.new_outputs(case)
        de = np.zeros((1, case.n[2], case.n[1], case.n[0]))
        ef = (A4 * 3)(*[np_a4(case.efield[d], (0, 0, 0)) for d in range(3)])
        gn = (A4 * 3)(*[np_a4(case.gradne[d], (0, 0, 0)) for d in range(3)])
        self.L.orc_elecenergy_source(C.byref(self.cm), C.byref(self._box(case)), C.byref(self._sb(case)),
                                     C.byref(np_a4(np.ascontiguousarray(rxn), (0, 0, 0))), ef, gn,
                                     C.byref(np_a4(de, (0, 0, 0))), C.byref(np_a4(phi_new, (0, 0, 0))),
                                     C.byref(prm))
        return de, phi_new

    def dsdt(self, case: BoxCase, specid: int, fluxes: list, rxn: np.ndarray):
        out = np.zeros((1, case.n[2], case.n[1], case.n[0]))
        fl = (A4 * 3)(*[np_a4(fluxes[d] if d < len(fluxes) else fluxes[0], (0, 0, 0)) for d in range(3)])
        self.L.orc_compute_dsdt(C.byref(self._box(case)), specid, fl,
                                C.byref(np_a4(np.ascontiguousarray(rxn), (0, 0, 0))),
                                C.byref(np_a4(out, (0, 0, 0))), _d3(case.dx))
        return out

    def update_scale(self, case: BoxCase, prm: abi.VdParams):
        """Per cell and component (NS+1): the gross magnitude of the terms summed into
        dsdt (sum of |face fluxes|/dx, of |chemistry terms| and of |Joule terms|).
        rxn errors are measured against the chemistry part, dsdt errors against the
        whole, and n + dt*dsdt errors against |n| + dt*scale."""
        _, scale, _ = self.new_outputs(case)
        ws, wsa = self.flux_ws(case)
        ef = (A4 * 3)(*[np_a4(case.efield[d], (0, 0, 0)) for d in range(3)])
        gn = (A4 * 3)(*[np_a4(case.gradne[d], (0, 0, 0)) for d in range(3)])
        self.L.orc_update_scale(C.byref(self.cm), C.byref(self._box(case)), C.byref(self._sb(case)), ef, gn,
                                C.byref(np_a4(scale, (0, 0, 0))), wsa, C.byref(prm))
        return scale

    def rxn_scale(self, case: BoxCase, Tg=300.0):
        """gross magnitude of the chemistry terms only (transport switched off)"""
        return self.update_scale(case, case.vd_params(do_transport=0, elecenergy_solve=0, Tg=Tg))

    def specmob(self, s, Te, N, Tg=300.0):
        return self.L.orc_specmob(C.byref(self.cm), s, Te, N, 0.0, Tg)

    def specdiff(self, s, Te, N, Tg=300.0):
        return self.L.orc_specdiff(C.byref(self.cm), s, Te, N, 0.0, Tg)

    def weno(self, a, b, c, d, e, scheme=3):
        return self.L.orc_weno(a, b, c, d, e, scheme)


class RefLib(_Base):
    """The reference's own hot-path code for one (case, dimension)."""

    _cache: dict = {}

    def __init__(self, name: str, dim: int):
        key = (name, dim)
        if key not in RefLib._cache:
            p = ref_lib_path(name, dim)
            if not p.exists():
                raise FileNotFoundError(f"{p} missing: run `python oracle/build.py` where the reference tree exists")
            L = C.CDLL(str(p))
            L.ref_reaction_source.argtypes = [BOXP, A4, A4, C.c_double, C.c_double, C.c_double]
            L.ref_compute_explicit_flux.argtypes = [BOXP, C.c_int, C.c_int, A4, I32P, I32P, I32P, I32P, A4,
                                                    C.c_double, C.c_double, C.c_double, DP, C.c_double, C.c_int,
                                                    C.c_int, C.c_int, DP, C.c_int]
            L.ref_compute_dsdt.argtypes = [BOXP, C.c_int, A4P, A4, A4, DP]
            L.ref_elecenergy_source.argtypes = [BOXP, A4, A4, A4P, A4P, A4, A4, PRMP]
            L.ref_explicit_update_all.argtypes = [BOXP, A4, A4P, A4P, A4, A4, A4, A4P, PRMP]
            L.ref_init()
            RefLib._cache[key] = L
        self.L = RefLib._cache[key]
        self.ns = self.L.ref_nspecies()
        self.dim = self.L.ref_dim()

    @staticmethod
    def available(name: str, dim: int) -> bool:
        return ref_lib_path(name, dim).exists()

    def reaction_source(self, case: BoxCase, Tg=300.0):
        _, _, rxn = self.new_outputs(case)
        self.L.ref_reaction_source(C.byref(self._box(case)), self._sb(case), np_a4(rxn, (0, 0, 0)), Tg, 0.0, 0.0)
        return rxn

    def flux(self, case: BoxCase, d: int, specid: int, hyp_order=5, weno=3, bclo=(3, 3, 3), bchi=(3, 3, 3),
             Tg=300.0, dt=1e-12, udv=0, uvel=(0, 0, 0), vel_species=0):
        fx = np.zeros(face_shape(case, d))
        domhi = [case.n[q] - 1 for q in range(3)]
        rc = self.L.ref_compute_explicit_flux(C.byref(self._box(case)), d, specid, self._sb(case), _i3(bclo),
                                              _i3(bchi), _i3((0, 0, 0)), _i3(domhi), np_a4(fx, (0, 0, 0)), Tg,
                                              0.0, 0.0, _d3(case.dx), dt, hyp_order, udv, weno, _d3(uvel),
                                              vel_species)
        if rc:
            raise RuntimeError(f"reference compute_flux aborted (status {rc})")
        return fx

    def update_all(self, case: BoxCase, prm: abi.VdParams, lo=None, hi=None):
        lo = lo or case.lo
        phi_new, dsdt, rxn = self.new_outputs(case, lo, hi)
        ws, wsa = self.flux_ws(case, lo, hi)
        ef = (A4 * 3)(*[np_a4(case.efield[d], (0, 0, 0)) for d in range(3)])
        gn = (A4 * 3)(*[np_a4(case.gradne[d], (0, 0, 0)) for d in range(3)])
        rc = self.L.ref_explicit_update_all(C.byref(self._box(case, lo, hi)), self._sb(case), ef, gn,
                                            np_a4(phi_new, lo), np_a4(dsdt, lo), np_a4(rxn, lo), wsa,
                                            C.byref(prm))
        if rc:
            raise RuntimeError(f"reference update aborted (status {rc})")
        return dict(phi_new=phi_new, dsdt=dsdt, rxn=rxn)


def run_steps(backend, case: BoxCase, prm: abi.VdParams, nsteps: int) -> np.ndarray:
    """nsteps explicit steps of one case on the CPU (backend: Port or RefLib).  Each
    step is the reference's per-box update (update_all) on the current state,
    followed by the ghost refill of the new state's species, EEN and ETEMP
    (first-order extrapolation, or periodic wrap; FillPatch before the next step,
    Source/Vidyut.cpp:90-101).  With prm.gradne_from_state the Joule term's
    gradne_fc is the face difference of the current electron density.  Returns the
    final state, laid out like case.state."""
    from dataclasses import replace
    from vidyut_b200.inputs import face_gradients, fill_ghosts
    ns = case.mech.ns
    g = case.gvec
    comps = list(range(ns)) + [abi.EEN(ns), abi.ETEMP(ns)]
    valid = (slice(None), slice(g[2], g[2] + case.n[2]), slice(g[1], g[1] + case.n[1]),
             slice(g[0], g[0] + case.n[0]))
    st = case.state.copy()
    for _ in range(nsteps):
        gradne = face_gradients(case, st) if prm.gradne_from_state else case.gradne
        c = replace(case, state=st, gradne=gradne)
        out = backend.update_all(c, prm)
        new = st.copy()
        new[valid] = out["phi_new"]
        sub = np.ascontiguousarray(new[comps])
        fill_ghosts(sub, case.dim, case.ghost, case.periodic)
        new[comps] = sub
        st = new
    return st
