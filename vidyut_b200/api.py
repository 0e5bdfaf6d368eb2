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


def fill_ghosts(state: torch.Tensor, case: BoxCase, ghost: int, comps, periodic=(0, 0, 0), stream=None) -> None:
    """Ghost refill of a device state laid out like case.state (FillPatch with
    first-order extrapolation / periodic wrap on face-adjacent ghosts)."""
    L = abi.lib()
    cl = (C.c_int32 * max(1, len(comps)))(*[int(c) for c in comps])
    per = (C.c_int32 * 3)(*[int(p) for p in periodic])
    rc = L.vd_fill_ghosts(C.byref(abi.make_box(case.lo, case.hi, case.dim)), t_a4(state, case.state_begin()),
                          int(ghost), cl, len(comps), per, _stream(stream))
    abi.check(rc, "vd_fill_ghosts")


def stencil_halo(hyp_order: int) -> int:
    return 3 if hyp_order == 5 else int(hyp_order)


def trim_ghosts(case: BoxCase, state: np.ndarray, H: int) -> np.ndarray:
    """The state restricted to the box grown by H ghosts (H <= case.ghost)."""
    g = case.gvec
    sl = [slice(None)]
    for d in (2, 1, 0):
        h = H if d < case.dim else 0
        sl.append(slice(g[d] - h, g[d] + case.n[d] + h))
    return np.ascontiguousarray(state[tuple(sl)])


class Batch:
    """Many independent cases resident in one HBM arena and stepped together
    (vd_batch_* of the C ABI): per step one persistent launch each of the prep
    (density sums + chemistry), transport (per dimension present) and ghost-refill
    kernels over a work list of all cases, replayed from a captured CUDA graph."""

    def __init__(self, precision=abi.PREC_MIXED, budget_bytes: int = 4 << 30, max_cases: int = 1024):
        L = abi.lib()
        self._h = C.c_void_p()
        abi.check(L.vd_batch_create(C.byref(self._h), int(precision), int(budget_bytes), int(max_cases)),
                  "vd_batch_create")
        self.precision = int(precision)
        self.cases = {}

    def close(self) -> None:
        if self._h:
            abi.lib().vd_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass

    @staticmethod
    def case_bytes(case: BoxCase, prm: abi.VdParams) -> int:
        return int(abi.lib().vd_batch_case_bytes(C.byref(abi.make_box(case.lo, case.hi, case.dim)), C.byref(prm)))

    def add(self, case: BoxCase, prm: abi.VdParams, nsteps: int = -1, stream=None) -> int:
        """Copy the case into the arena; raises VidyutError(ERR_BUDGET) when it does
        not fit.  Returns the case id."""
        L = abi.lib()
        H = stencil_halo(prm.hyp_order)
        st = trim_ghosts(case, case.state, H)
        ef = [np.ascontiguousarray(case.efield[d]) for d in range(3)]
        gn = [np.ascontiguousarray(case.gradne[d]) for d in range(3)]
        efp = (C.c_void_p * 3)(*[a.ctypes.data for a in ef])
        gnp = (C.c_void_p * 3)(*[a.ctypes.data for a in gn])
        per = (C.c_int32 * 3)(*[int(p) for p in case.periodic])
        cid = C.c_int32()
        rc = L.vd_batch_add_case(self._h, C.byref(abi.make_box(case.lo, case.hi, case.dim)), st.ctypes.data,
                                 efp, gnp, C.byref(prm), per, int(nsteps), _stream(stream), C.byref(cid))
        abi.check(rc, "vd_batch_add_case")
        self.cases[cid.value] = (case, H)
        return cid.value

    def remove(self, cid: int) -> None:
        abi.check(abi.lib().vd_batch_remove_case(self._h, int(cid)), "vd_batch_remove_case")
        self.cases.pop(cid, None)

    def step(self, nsteps: int, stream=None) -> None:
        abi.check(abi.lib().vd_batch_step(self._h, int(nsteps), _stream(stream)), "vd_batch_step")

    def nonfinite(self, cid: int) -> bool:
        """True when a step of case cid met a NaN or infinity (it then takes no
        further steps); waits for the batch's queued work."""
        f = C.c_int32()
        abi.check(abi.lib().vd_batch_case_status(self._h, int(cid), C.byref(f)), "vd_batch_case_status")
        return bool(f.value)

    def info(self, cid: int):
        done, left = C.c_int64(), C.c_int64()
        abi.check(abi.lib().vd_batch_case_info(self._h, int(cid), C.byref(done), C.byref(left)),
                  "vd_batch_case_info")
        return done.value, left.value

    def read(self, cid: int, stream=None, out: torch.Tensor | None = None) -> torch.Tensor:
        """The case's current state (ghost-grown box, NVAR components).  Into a
        device tensor when out is given (asynchronous), else a host array."""
        case, H = self.cases[cid]
        ns = case.mech.ns
        shp = [abi.NVAR(ns)]
        for d in (2, 1, 0):
            shp.append(case.n[d] + (2 * H if d < case.dim else 0))
        if out is None:
            host = torch.empty(shp, dtype=torch.float64, pin_memory=True)
            abi.check(abi.lib().vd_batch_read_case(self._h, int(cid), host.data_ptr(), _stream(stream)),
                      "vd_batch_read_case")
            (stream or torch.cuda.current_stream()).synchronize()
            return host
        assert tuple(out.shape) == tuple(shp) and out.dtype == torch.float64 and out.is_contiguous()
        abi.check(abi.lib().vd_batch_read_case(self._h, int(cid), out.data_ptr(), _stream(stream)),
                  "vd_batch_read_case")
        return out

    def load(self, cid: int, state, nsteps: int = -1, stream=None) -> None:
        """Replace the case's state (a device tensor or host array in the batch
        layout, see read) and restart its step count."""
        src = state if isinstance(state, torch.Tensor) else np.ascontiguousarray(state)
        ptr = src.data_ptr() if isinstance(src, torch.Tensor) else src.ctypes.data
        abi.check(abi.lib().vd_batch_load_case(self._h, int(cid), ptr, int(nsteps), _stream(stream)),
                  "vd_batch_load_case")

    def tune(self, trials: int = 5, stream=None) -> dict:
        ms = (C.c_double * 32)()
        abi.check(abi.lib().vd_batch_tune(self._h, int(trials), _stream(stream), ms), "vd_batch_tune")
        return {(d, v): ms[d * 8 + v] for d in range(1, 4) for v in range(8) if ms[d * 8 + v] >= 0}

    def set_tile_variant(self, dim: int, variant: int) -> None:
        abi.check(abi.lib().vd_batch_set_tile_variant(self._h, int(dim), int(variant)), "vd_batch_set_tile_variant")

    def set_graph(self, on: bool) -> None:
        abi.check(abi.lib().vd_batch_set_graph(self._h, int(bool(on))), "vd_batch_set_graph")

    def stats(self) -> dict:
        s = abi.VdBatchStats()
        abi.check(abi.lib().vd_batch_get_stats(self._h, C.byref(s)), "vd_batch_get_stats")
        return dict(ncases=s.ncases, ncases_dim=list(s.ncases_dim), cells=s.cells, bytes_used=s.bytes_used,
                    bytes_budget=s.bytes_budget, steps_run=s.steps_run, graph_builds=s.graph_builds,
                    tile_variant=list(s.tile_variant), launches_per_step=s.launches_per_step)


def batch_tile_shape(dim: int, variant: int):
    """(tile shape, number of variants of dim, target resident CTAs per SM)"""
    t = (C.c_int32 * 3)()
    mb = C.c_int32()
    n = abi.lib().vd_batch_tile_shape(int(dim), int(variant), t, C.byref(mb))
    if n < 0:
        abi.check(n, "vd_batch_tile_shape")
    return tuple(t), n, mb.value


class Server:
    """Continuous-batching request loop on one GPU (vd_server_* of the C ABI).
    submit() queues a case and returns at once; the library's worker thread admits
    it when the HBM budget has room, steps it together with every other resident
    case and brings its final state back; wait() blocks for it."""

    def __init__(self, precision=abi.PREC_MIXED, budget_bytes: int = 4 << 30, max_cases: int = 1024,
                 quantum_steps: int = 25):
        self._h = C.c_void_p()
        abi.check(abi.lib().vd_server_create(C.byref(self._h), int(precision), int(budget_bytes), int(max_cases),
                                             int(quantum_steps)), "vd_server_create")
        self.precision = int(precision)
        self.requests = {}

    def close(self) -> None:
        if self._h:
            abi.lib().vd_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass

    def submit(self, case: BoxCase, prm: abi.VdParams, nsteps: int) -> int:
        H = stencil_halo(prm.hyp_order)
        st = trim_ghosts(case, case.state, H)
        ef = [np.ascontiguousarray(case.efield[d]) for d in range(3)]
        gn = [np.ascontiguousarray(case.gradne[d]) for d in range(3)]
        efp = (C.c_void_p * 3)(*[a.ctypes.data for a in ef])
        gnp = (C.c_void_p * 3)(*[a.ctypes.data for a in gn])
        per = (C.c_int32 * 3)(*[int(p) for p in case.periodic])
        rid = C.c_int64()
        rc = abi.lib().vd_server_submit(self._h, C.byref(abi.make_box(case.lo, case.hi, case.dim)), st.ctypes.data,
                                        efp, gnp, C.byref(prm), per, int(nsteps), C.byref(rid))
        abi.check(rc, "vd_server_submit")
        self.requests[rid.value] = st.shape
        return rid.value

    def wait(self, rid: int, timeout_s: float = -1.0):
        """(final state in the ghost-grown layout, latency in ms)"""
        shape = self.requests.get(rid)
        out = np.empty(shape, dtype=np.float64) if shape is not None else None
        lat = C.c_double()
        rc = abi.lib().vd_server_wait(self._h, int(rid), out.ctypes.data if out is not None else None,
                                      float(timeout_s), C.byref(lat))
        abi.check(rc, "vd_server_wait")
        del self.requests[rid]
        return out, lat.value

    def stats(self) -> dict:
        s = abi.VdServerStats()
        abi.check(abi.lib().vd_server_get_stats(self._h, C.byref(s)), "vd_server_get_stats")
        return {k: getattr(s, k) for k, _ in abi.VdServerStats._fields_}


def poisson_params(dim: int, v_lo: float, v_hi: float = 0.0, max_vcycles: int = 30, tol_rel: float = 1e-12,
                   dirichlet_dir: int = 0) -> abi.VdPoissonParams:
    """Applied potential v_lo at the low face and v_hi at the high face of
    direction dirichlet_dir (the electrodes), zero normal gradient elsewhere."""
    pp = abi.VdPoissonParams()
    for d in range(3):
        pp.bc_lo[d] = abi.BC_DIRC if d == dirichlet_dir else abi.BC_HNEU
        pp.bc_hi[d] = abi.BC_DIRC if d == dirichlet_dir else abi.BC_HNEU
    pp.value_lo[dirichlet_dir] = v_lo
    pp.value_hi[dirichlet_dir] = v_hi
    pp.max_vcycles = max_vcycles
    pp.tol_rel = tol_rel
    return pp


def set_poisson_user_rhs(pp: abi.VdPoissonParams, rhs: torch.Tensor | None) -> None:
    """Add rhs (one component over the valid cells, (1, nz, ny, nx)) to the
    potential's right-hand side (the case's add_user_potential_sources); None
    removes it.  pp keeps a pointer: rhs must stay alive while pp is used."""
    pp.user_rhs = t_a4(rhs, (0, 0, 0)) if rhs is not None else abi.null_array4()


def poisson_solve(dc: DeviceCase, prm: abi.VdParams, pp: abi.VdPoissonParams, state: torch.Tensor | None = None,
                  stream=None):
    """Potential and fields of dc (or of `state`, laid out like dc.state): writes
    POT, EFX..EFZ, REF into the state and the face fields into dc.efield.
    Returns (V-cycles done, relative residual or -1 when not checked)."""
    st = state if state is not None else dc.state
    nv = C.c_int32()
    rr = C.c_double()
    rc = abi.lib().vd_poisson_solve(C.byref(dc.box()), t_a4(st, dc.case.state_begin()), dc.face_a4s("efield"),
                                    C.byref(prm), C.byref(pp), C.byref(nv), C.byref(rr), _stream(stream))
    abi.check(rc, "vd_poisson_solve")
    return nv.value, rr.value


def implicit_species_solve(dc: DeviceCase, spec: int, state_old: torch.Tensor, dsdt: torch.Tensor,
                           phi_new: torch.Tensor, prm: abi.VdParams, *, dsdt_comp: int | None = None,
                           gradne: list | None = None, tol_rel: float = 1e-12, max_vcycles: int = 50,
                           robin=None, stream=None):
    """Implicit diffusion solve of species `spec` (NS: the electron energy) of dc
    (Vidyut::implicit_solve_scalar): state_old laid out like dc.state, dsdt and
    phi_new over the valid cells (phi_new with NVAR components).  gradne: three
    face tensors that receive the electron face gradients.  robin: the case's own
    species_bc coefficients, ((a_lo, b_lo, f_lo), (a_hi, b_hi, f_hi)) with one
    value per direction each (a n + b dn/dnu = f, nu outward), else species_bc's
    defaults.  Returns (V-cycles done, relative residual or -1 when not checked)."""
    dp = abi.VdDiffusionParams()
    dp.spec = spec
    dp.dsdt_comp = spec if dsdt_comp is None else dsdt_comp
    dp.max_vcycles = max_vcycles
    dp.tol_rel = tol_rel
    if robin is not None:
        dp.user_robin = 1
        for side in range(2):
            a, b, f = robin[side]
            for d in range(3):
                dp.robin_a[side][d], dp.robin_b[side][d], dp.robin_f[side][d] = a[d], b[d], f[d]
    nv = C.c_int32()
    rr = C.c_double()
    g = None
    if gradne is not None:
        g = (abi.VdArray4 * 3)(*[t_a4(gradne[d], (0, 0, 0)) for d in range(3)])
    rc = abi.lib().vd_implicit_species_solve(C.byref(dc.box()), dc.sb(), t_a4(state_old, dc.case.state_begin()),
                                             t_a4(dsdt, (0, 0, 0)), t_a4(phi_new, (0, 0, 0)), g, C.byref(prm),
                                             C.byref(dp), C.byref(nv), C.byref(rr), _stream(stream))
    abi.check(rc, "vd_implicit_species_solve")
    return nv.value, rr.value


# Source/Vidyut.cpp:32-42: the names of the state components after the species
PLASMA_VAR_NAMES = ("Electron_energy", "Electron_Temp", "Potential", "Efieldx", "Efieldy", "Efieldz",
                    "Electron_Jheat", "Electron_inelasticHeat", "Electron_elasticHeat", "ReducedEF")


def plot_var_names(mech: Mechanism) -> list:
    """The reference's plotfile variable names (allvarnames, Source/Vidyut.cpp:44-52)."""
    return list(mech.species) + list(PLASMA_VAR_NAMES)


def write_plotfile(path, case: BoxCase, valid_state, *, time: float = 0.0, step: int = 0,
                   prob_lo=(0.0, 0.0, 0.0), names=None) -> None:
    """Writes a plotfile of the case's valid cells: valid_state is a host (numpy) or
    device (torch) array (NVAR, nz, ny, nx), e.g. the phi_new of an update."""
    if isinstance(valid_state, torch.Tensor):
        valid_state = valid_state.detach().cpu().numpy()
    a = np.ascontiguousarray(valid_state, dtype=np.float64)
    names = list(names) if names is not None else plot_var_names(case.mech)
    if len(names) != a.shape[0]:
        raise ValueError(f"{len(names)} names for {a.shape[0]} components")
    cn = (C.c_char_p * len(names))(*[n.encode() for n in names])
    lo = (C.c_double * 3)(*prob_lo)
    dx = (C.c_double * 3)(*case.dx)
    rc = abi.lib().vd_write_plotfile(str(path).encode(), C.byref(case_box(case)),
                                     a.ctypes.data_as(C.POINTER(C.c_double)), a.shape[0], cn, lo, dx, float(time),
                                     int(step))
    abi.check(rc, "vd_write_plotfile")


def write_checkpoint(path, case: BoxCase, valid_state, *, istep: int = 0, dt: float = 0.0,
                     time: float = 0.0) -> None:
    """Checkpoint of the case's valid cells (Vidyut::WriteCheckpointFile)."""
    if isinstance(valid_state, torch.Tensor):
        valid_state = valid_state.detach().cpu().numpy()
    a = np.ascontiguousarray(valid_state, dtype=np.float64)
    rc = abi.lib().vd_write_checkpoint(str(path).encode(), C.byref(case_box(case)),
                                       a.ctypes.data_as(C.POINTER(C.c_double)), a.shape[0], int(istep), float(dt),
                                       float(time))
    abi.check(rc, "vd_write_checkpoint")


def read_checkpoint(path):
    """(state (ncomp, nz, ny, nx), box lo, box hi, dim, istep, dt, time) of a
    checkpoint (Vidyut::ReadCheckpointFile)."""
    L = abi.lib()
    bx = abi.VdBox()
    nc, st = C.c_int(), C.c_int()
    dt, tm = C.c_double(), C.c_double()
    abi.check(L.vd_read_checkpoint(str(path).encode(), C.byref(bx), None, 0, C.byref(nc), C.byref(st), C.byref(dt),
                                   C.byref(tm)), "vd_read_checkpoint")
    n = [bx.hi[d] - bx.lo[d] + 1 for d in range(3)]
    out = np.empty((nc.value, n[2], n[1], n[0]), dtype=np.float64)
    abi.check(L.vd_read_checkpoint(str(path).encode(), C.byref(bx), out.ctypes.data_as(C.POINTER(C.c_double)),
                                   out.size, C.byref(nc), C.byref(st), C.byref(dt), C.byref(tm)),
              "vd_read_checkpoint")
    return out, tuple(bx.lo), tuple(bx.hi), bx.dim, st.value, dt.value, tm.value


def case_box(case: BoxCase) -> abi.VdBox:
    return abi.make_box(case.lo, case.hi, case.dim)


def time_scales(dc: DeviceCase, prm: abi.VdParams, stream=None):
    """(dt_edrift, dt_ediff, dt_diel_relax) of the case's current state
    (Vidyut::find_time_scales)."""
    out = (C.c_double * 3)()
    abi.check(abi.lib().vd_time_scales(C.byref(dc.box()), dc.sb(), C.byref(prm), out, _stream(stream)),
              "vd_time_scales")
    return tuple(out)
