"""ctypes mirror of include/vidyut_b200.h and the loader of libvidyut_b200.so.

The structs below repeat the C layouts field for field; ``check_layout`` compares
their sizes with ``vd_sizeof`` from the library so a header change that is not
mirrored here fails loudly.  No CPU fallback exists: ``lib()`` raises when the
CUDA library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

MAX_SPECIES = 64
MAX_REACTIONS = 448
MAX_FITS = 48
MAX_REACTANTS = 3
MAX_TERMS = 6

OK = 0
ERR_ARG, ERR_SCHEME, ERR_GHOST, ERR_DIM, ERR_MECH, ERR_CUDA = -1, -2, -3, -4, -5, -6
ERR_TIMEOUT, ERR_NOMEM, ERR_NONFINITE, ERR_BUDGET, ERR_STATE = -7, -8, -9, -10, -11

BC_PER, BC_DIRC, BC_HNEU, BC_IHNEU, BC_ROBIN = 0, 1, 2, 3, 4
CLASS_ELECTRON, CLASS_ENERGY, CLASS_ION, CLASS_NEUTRAL = 0, 1, 2, 3

RATE_ARRHENIUS_TE, RATE_CONST, RATE_ARRHENIUS_TG = 0, 1, 2
RATE_JANEV, RATE_FFIT, RATE_JANEV_FFIT, RATE_TOWNSEND = 3, 4, 5, 6
RXN_NONE, RXN_EXCITATION, RXN_IONIZATION, RXN_RECOMB, RXN_ELASTIC = 0, 1, 2, 3, 5
RXN_ATTACH, RXN_DETACH = 4, 7
MOB_ZERO, MOB_ELECTRON, MOB_ION_TG, MOB_SCALED, MOB_CONST_N, MOB_CONST = 0, 1, 2, 3, 4, 5
MOB_POW_EMAG, MOB_EN_POLY, MOB_EXP_MEANE = 6, 7, 8
DIFF_ZERO, DIFF_TE_ABSMOB, DIFF_TG_MOB, DIFF_CONST = 0, 1, 2, 3
DIFF_POW_EMAG, DIFF_PRES, DIFF_TE_PRES, DIFF_SCALED = 4, 5, 6, 7
PREC_FP64, PREC_MIXED = 0, 1
NOALLOC_SCRATCH_BYTES = 64 << 20


def EEN(ns): return ns
def ETEMP(ns): return ns + 1
def POT(ns): return ns + 2
def EFX(ns): return ns + 3
def EFY(ns): return ns + 4
def EFZ(ns): return ns + 5
def EJH(ns): return ns + 6
def EIH(ns): return ns + 7
def EEH(ns): return ns + 8
def REF(ns): return ns + 9
def NVAR(ns): return ns + 10


class VdArray4(C.Structure):
    _fields_ = [("p", C.c_void_p), ("jstride", C.c_int64), ("kstride", C.c_int64),
                ("nstride", C.c_int64), ("begin", C.c_int32 * 3), ("end", C.c_int32 * 3),
                ("ncomp", C.c_int32)]


class VdBox(C.Structure):
    _fields_ = [("lo", C.c_int32 * 3), ("hi", C.c_int32 * 3), ("itype", C.c_int32 * 3),
                ("dim", C.c_int32)]


class VdReaction(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nreac", C.c_int32), ("reac", C.c_int32 * MAX_REACTANTS),
                ("rxntype", C.c_int32), ("elidx", C.c_int32), ("nterms", C.c_int32),
                ("term_sp", C.c_int32 * MAX_TERMS), ("term_coef", C.c_double * MAX_TERMS),
                ("A", C.c_double), ("b", C.c_double), ("C", C.c_double), ("eexci", C.c_double),
                ("fit", C.c_int32), ("pad0", C.c_int32)]


class VdRateFit(C.Structure):
    _fields_ = [("jA", C.c_double), ("jc", C.c_double * 9), ("fA", C.c_double), ("fc", C.c_double * 4),
                ("switch_ev", C.c_double)]


class VdMech(C.Structure):
    _fields_ = [("nspecies", C.c_int32), ("nreactions", C.c_int32), ("e_id", C.c_int32),
                ("charge", C.c_int32 * MAX_SPECIES), ("mw", C.c_double * MAX_SPECIES),
                ("mob_kind", C.c_int32 * (MAX_SPECIES + 1)), ("mob_ref", C.c_int32 * (MAX_SPECIES + 1)),
                ("mob_p0", C.c_double * (MAX_SPECIES + 1)), ("mob_p1", C.c_double * (MAX_SPECIES + 1)),
                ("diff_kind", C.c_int32 * (MAX_SPECIES + 1)), ("diff_ref", C.c_int32 * (MAX_SPECIES + 1)),
                ("diff_factor", C.c_double * (MAX_SPECIES + 1)), ("diff_p1", C.c_double * (MAX_SPECIES + 1)),
                ("elastic_loss", C.c_int32), ("pad0", C.c_int32), ("elastic_mass", C.c_double),
                ("rxn", VdReaction * MAX_REACTIONS), ("nfits", C.c_int32), ("pad1", C.c_int32),
                ("fits", VdRateFit * MAX_FITS)]


class VdParams(C.Structure):
    _fields_ = [("dim", C.c_int32), ("hyp_order", C.c_int32), ("weno_scheme", C.c_int32),
                ("user_defined_vel", C.c_int32), ("vel_species", C.c_int32), ("precision", C.c_int32),
                ("user_vel", C.c_double * 3), ("Tg", C.c_double), ("Pg", C.c_double),
                ("time", C.c_double), ("dt", C.c_double), ("dx", C.c_double * 3),
                ("domlo", C.c_int32 * 3), ("domhi", C.c_int32 * 3),
                ("bc_lo", (C.c_int32 * 3) * 4), ("bc_hi", (C.c_int32 * 3) * 4),
                ("elecenergy_solve", C.c_int32), ("do_reactions", C.c_int32),
                ("do_transport", C.c_int32), ("do_bg_reactions", C.c_int32),
                ("floor_jh", C.c_int32), ("const_ele_trans", C.c_int32), ("cs_technique", C.c_int32),
                ("bound_specden", C.c_int32), ("ele_mob", C.c_double), ("ele_diff", C.c_double),
                ("min_species_density", C.c_double), ("min_electron_density", C.c_double),
                ("min_electron_temp", C.c_double), ("bg_mask", C.c_uint64), ("update_te", C.c_int32),
                ("gradne_from_state", C.c_int32), ("check_finite", C.c_int32), ("pad1", C.c_int32)]


STRUCTS = [VdArray4, VdBox, VdReaction, VdMech, VdParams]

# exported symbols and their prototypes (restype, argtypes)
A4 = VdArray4
A4P = C.POINTER(VdArray4)
BOXP = C.POINTER(VdBox)
I32P = C.POINTER(C.c_int32)
DP = C.POINTER(C.c_double)
PRMP = C.POINTER(VdParams)

PROTOTYPES = {
    "vd_abi_version": (C.c_int, []),
    "vd_sizeof": (C.c_size_t, [C.c_int]),
    "vd_last_error": (C.c_char_p, []),
    "vd_status_string": (C.c_char_p, [C.c_int]),
    "vd_mech_init": (C.c_int, [C.POINTER(VdMech)]),
    "vd_compute_explicit_flux": (C.c_int, [BOXP, C.c_int, C.c_int, A4, I32P, I32P, I32P, I32P, A4,
                                           C.c_double, C.c_double, C.c_double, DP, C.c_double, C.c_int,
                                           C.c_int, C.c_int, DP, C.c_int, C.c_void_p]),
    "vd_compute_dsdt": (C.c_int, [BOXP, C.c_int, A4P, A4, A4, DP, C.c_void_p]),
    "vd_reaction_source": (C.c_int, [BOXP, A4, A4, C.c_double, C.c_double, C.c_double, C.c_void_p]),
    "vd_elecenergy_source": (C.c_int, [BOXP, A4, A4, A4P, A4P, A4, A4, PRMP, C.c_void_p]),
    "vd_explicit_update_all": (C.c_int, [BOXP, A4, A4P, A4P, A4, A4, A4, PRMP, C.c_void_p]),
    "vd_box_checksums": (C.c_int, [BOXP, A4, A4, C.c_void_p, C.c_void_p]),
    "vd_explicit_update_all_noalloc": (C.c_int, [BOXP, A4, A4P, A4P, A4, A4, A4, PRMP, C.c_void_p]),
    "vd_launch_count": (C.c_int64, []),
    "vd_mech_specialized": (C.c_int, []),
    "vd_mech_specialize_status": (C.c_char_p, []),
    "vd_set_specialize": (C.c_int, [C.c_int]),
    "vd_mech_specialize_check": (C.c_int, [C.POINTER(VdMech), C.POINTER(C.c_size_t)]),
    "vd_profile_enable": (C.c_int, [C.c_int]),
    "vd_profile_read": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_double), C.c_int]),
}


def profile_read(max_kernels: int = 32) -> dict:
    """{kernel name: (launches, total device ms)} recorded since vd_profile_enable(1)."""
    L = lib()
    names = C.create_string_buffer(4096)
    cnt = (C.c_int64 * max_kernels)()
    ms = (C.c_double * max_kernels)()
    n = L.vd_profile_read(names, 4096, cnt, ms, max_kernels)
    if n < 0:
        check(n, "vd_profile_read")
    keys = names.raw.split(b"\0")
    return {keys[i].decode(): (int(cnt[i]), float(ms[i])) for i in range(n)}

LIB_PATH = Path(__file__).resolve().parent / "libvidyut_b200.so"
_lib = None


class VidyutError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


def lib() -> C.CDLL:
    """Load the CUDA library (built in-tree by vidyut_b200.build)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m vidyut_b200.build` "
                               "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_LOCAL)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check_layout(L=None) -> None:
    L = L or lib()
    structs = STRUCTS + [VdPoissonParams, VdDiffusionParams, VdBatchStats, VdServerStats]
    for i, S in enumerate(structs):
        n = L.vd_sizeof(i)
        if n != C.sizeof(S):
            raise RuntimeError(f"ABI layout mismatch for {S.__name__}: C {n} vs ctypes {C.sizeof(S)}")


def check(status: int, where: str) -> None:
    if status != OK:
        msg = lib().vd_last_error().decode(errors="replace")
        raise VidyutError(status, where, msg)


def make_box(lo, hi, dim: int) -> VdBox:
    b = VdBox()
    for d in range(3):
        b.lo[d] = int(lo[d]) if d < len(lo) else 0
        b.hi[d] = int(hi[d]) if d < len(hi) else 0
        b.itype[d] = 0
    b.dim = dim
    return b


def make_array4(ptr: int, shape, begin, ncomp: int | None = None) -> VdArray4:
    """Array4 over a C-ordered buffer of shape (ncomp, nz, ny, nx) whose element
    [n, 0, 0, 0] is cell (begin[0], begin[1], begin[2])."""
    nc, nz, ny, nx = shape
    a = VdArray4()
    a.p = ptr
    a.jstride = nx
    a.kstride = nx * ny
    a.nstride = nx * ny * nz
    for d in range(3):
        a.begin[d] = int(begin[d])
    a.end[0] = begin[0] + nx
    a.end[1] = begin[1] + ny
    a.end[2] = begin[2] + nz
    a.ncomp = nc if ncomp is None else ncomp
    return a


def null_array4() -> VdArray4:
    return VdArray4()


PROTOTYPES.update({
    "vd_tune_set": (C.c_int, [C.c_char_p, C.c_int]),
    "vd_tune_get": (C.c_int, [C.c_char_p]),
})


class VdBatchStats(C.Structure):
    _fields_ = [("ncases", C.c_int32), ("ncases_dim", C.c_int32 * 4), ("cells", C.c_int64),
                ("bytes_used", C.c_uint64), ("bytes_budget", C.c_uint64), ("steps_run", C.c_int64),
                ("graph_builds", C.c_int64), ("tile_variant", C.c_int32 * 4), ("launches_per_step", C.c_int32)]


DPP = C.POINTER(C.c_void_p)  # const double* const[3]
PROTOTYPES.update({
    "vd_fill_ghosts": (C.c_int, [BOXP, A4, C.c_int, I32P, C.c_int, I32P, C.c_void_p]),
    "vd_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_uint64, C.c_int]),
    "vd_batch_destroy": (C.c_int, [C.c_void_p]),
    "vd_batch_case_bytes": (C.c_uint64, [BOXP, PRMP]),
    "vd_batch_add_case": (C.c_int, [C.c_void_p, BOXP, C.c_void_p, DPP, DPP, PRMP, I32P, C.c_int64, C.c_void_p,
                                    I32P]),
    "vd_batch_remove_case": (C.c_int, [C.c_void_p, C.c_int32]),
    "vd_batch_step": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "vd_batch_case_info": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "vd_batch_case_status": (C.c_int, [C.c_void_p, C.c_int32, I32P]),
    "vd_batch_read_case": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "vd_batch_load_case": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p]),
    "vd_batch_tune": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, DP]),
    "vd_batch_set_tile_variant": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "vd_batch_tile_shape": (C.c_int, [C.c_int, C.c_int, I32P, I32P]),
    "vd_batch_set_graph": (C.c_int, [C.c_void_p, C.c_int]),
    "vd_batch_get_stats": (C.c_int, [C.c_void_p, C.POINTER(VdBatchStats)]),
})


class VdServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64), ("queued", C.c_int64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double), ("span_s", C.c_double),
                ("solves_per_s", C.c_double), ("cell_updates_per_s", C.c_double), ("bytes_budget", C.c_uint64),
                ("peak_bytes_used", C.c_uint64), ("quanta", C.c_int64), ("graph_builds", C.c_int64)]


PROTOTYPES.update({
    "vd_server_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_uint64, C.c_int, C.c_int]),
    "vd_server_destroy": (C.c_int, [C.c_void_p]),
    "vd_server_submit": (C.c_int, [C.c_void_p, BOXP, C.c_void_p, DPP, DPP, PRMP, I32P, C.c_int64,
                                   C.POINTER(C.c_int64)]),
    "vd_server_wait": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_double, C.POINTER(C.c_double)]),
    "vd_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(VdServerStats)]),
})


class VdPoissonParams(C.Structure):
    _fields_ = [("bc_lo", C.c_int32 * 3), ("bc_hi", C.c_int32 * 3), ("value_lo", C.c_double * 3),
                ("value_hi", C.c_double * 3), ("max_vcycles", C.c_int32), ("pad0", C.c_int32),
                ("tol_rel", C.c_double), ("user_rhs", VdArray4)]


PROTOTYPES.update({
    "vd_poisson_solve": (C.c_int, [BOXP, A4, A4P, PRMP, C.POINTER(VdPoissonParams), I32P, DP, C.c_void_p]),
})

PROTOTYPES.update({
    "vd_time_scales": (C.c_int, [BOXP, A4, PRMP, DP, C.c_void_p]),
})


PROTOTYPES.update({
    "vd_write_plotfile": (C.c_int, [C.c_char_p, BOXP, DP, C.c_int, C.POINTER(C.c_char_p), DP, DP, C.c_double,
                                    C.c_int]),
    "vd_write_checkpoint": (C.c_int, [C.c_char_p, BOXP, DP, C.c_int, C.c_int, C.c_double, C.c_double]),
    "vd_read_checkpoint": (C.c_int, [C.c_char_p, BOXP, DP, C.c_int64, C.POINTER(C.c_int), C.POINTER(C.c_int), DP,
                                     DP]),
})


class VdDiffusionParams(C.Structure):
    _fields_ = [("spec", C.c_int32), ("dsdt_comp", C.c_int32), ("max_vcycles", C.c_int32), ("pad0", C.c_int32),
                ("tol_rel", C.c_double), ("user_robin", C.c_int32), ("pad1", C.c_int32),
                ("robin_a", (C.c_double * 3) * 2), ("robin_b", (C.c_double * 3) * 2),
                ("robin_f", (C.c_double * 3) * 2)]


PROTOTYPES.update({
    "vd_implicit_species_solve": (C.c_int, [BOXP, A4, A4, A4, A4, A4P, PRMP, C.POINTER(VdDiffusionParams), I32P,
                                            DP, C.c_void_p]),
})
