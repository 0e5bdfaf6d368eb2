"""C-ABI checks that need no GPU: the library loads, exports every function that
include/vidyut_b200.h declares, and its struct layouts match the ctypes mirror."""
import ctypes as C
import re
from pathlib import Path

import pytest

from vidyut_b200 import _abi as abi
from vidyut_b200 import build as vbuild
from vidyut_b200 import mechanism as mm

HEADER = Path(__file__).resolve().parents[1] / "include" / "vidyut_b200.h"


@pytest.fixture(scope="module")
def lib():
    if not abi.LIB_PATH.exists():
        vbuild.build()
    return abi.lib()


def declared_functions():
    txt = HEADER.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(vd_\w+)\s*\(", txt)))


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), f"{n} declared in the header but not exported"
    assert set(abi.PROTOTYPES) <= set(names)


def test_struct_layouts(lib):
    abi.check_layout(lib)
    assert lib.vd_abi_version() == 2
    # vd_array4 has amrex::Array4<Real>'s layout: pointer, 3 strides, begin/end Dim3, ncomp
    assert C.sizeof(abi.VdArray4) == 64


def test_status_strings(lib):
    assert lib.vd_status_string(abi.ERR_GHOST) == b"too few ghost cells"
    assert lib.vd_status_string(0) == b"ok"


def test_mechanism_validation_rejects_bad_tables(lib):
    """vd_mech_init checks the table before touching the device."""
    m = mm.argon(10, 1).to_c()
    m.nspecies = 0
    assert lib.vd_mech_init(C.byref(m)) == abi.ERR_MECH
    m = mm.argon(10, 1).to_c()
    m.rxn[3].reac[0] = 17
    assert lib.vd_mech_init(C.byref(m)) == abi.ERR_MECH
    assert b"reactant" in lib.vd_last_error()
    m = mm.argon(10, 1).to_c()
    m.mob_kind[4] = abi.MOB_SCALED
    m.mob_ref[4] = 4
    assert lib.vd_mech_init(C.byref(m)) == abi.ERR_MECH
    m = mm.argon(10, 1).to_c()
    m.rxn[0].A = -1.0
    assert lib.vd_mech_init(C.byref(m)) == abi.ERR_MECH
    # field-dependent models: the coefficient fit must exist, kinds must be known,
    # the temperature scale of the pressure-scaled diffusion nonzero
    m = mm.argon(10, 1).to_c()
    m.mob_kind[0], m.mob_ref[0] = abi.MOB_EXP_MEANE, 0
    assert lib.vd_mech_init(C.byref(m)) == abi.ERR_MECH
    assert b"fit index" in lib.vd_last_error()
    m = mm.argon(10, 1).to_c()
    m.diff_kind[0] = 8
    assert lib.vd_mech_init(C.byref(m)) == abi.ERR_MECH
    m = mm.argon(10, 1).to_c()
    m.diff_kind[0], m.diff_p1[0] = abi.DIFF_TE_PRES, 0.0
    assert lib.vd_mech_init(C.byref(m)) == abi.ERR_MECH
    m = mm.argon(10, 1).to_c()
    m.rxn[0].kind, m.rxn[0].fit = abi.RATE_TOWNSEND, 0
    assert lib.vd_mech_init(C.byref(m)) == abi.ERR_MECH


def test_calls_before_mech_init_fail_cleanly(lib):
    """Without a loaded mechanism (or without a GPU) nothing is launched."""
    b = abi.make_box((0, 0, 0), (3, 3, 0), 2)
    z = abi.null_array4()
    rc = lib.vd_reaction_source(C.byref(b), z, z, 300.0, 0.0, 0.0, None)
    assert rc in (abi.ERR_MECH, abi.ERR_CUDA, abi.ERR_ARG)
    # the implicit species solve checks its argument blocks before anything else
    prm = abi.VdParams()
    rc = lib.vd_implicit_species_solve(C.byref(b), z, z, z, z, None, C.byref(prm), None, None, None, None)
    assert rc == abi.ERR_ARG and b"null" in lib.vd_last_error()
    dp = abi.VdDiffusionParams()
    rc = lib.vd_implicit_species_solve(C.byref(b), z, z, z, z, None, C.byref(prm), C.byref(dp), None, None, None)
    assert rc in (abi.ERR_MECH, abi.ERR_CUDA, abi.ERR_ARG, abi.ERR_DIM)


def _fixture_mech(name):
    from tests._util import load_fixture
    return load_fixture(name)[0].mech


@pytest.mark.parametrize("mech", [mm.argon(10, 20261204), mm.synthetic(8, 40, 20261224),
                                  mm.synthetic(24, 150, 20261214), _fixture_mech("co2fits_2d"),
                                  _fixture_mech("streamer_2d"), _fixture_mech("he_rf_1d")], ids=lambda m: m.name)
def test_specialised_chemistry_compiles_for_sm100a(lib, mech):
    """vd_mech_init compiles the mechanism-specialised chemistry with NVRTC; the same
    source must compile here (no GPU needed) without local-memory spills of note."""
    lib.vd_mech_specialize_check.argtypes = [C.POINTER(abi.VdMech), C.POINTER(C.c_size_t)]
    cm = mech.to_c()
    n = C.c_size_t(0)
    rc = lib.vd_mech_specialize_check(C.byref(cm), C.byref(n))
    assert rc == abi.OK, lib.vd_last_error().decode()
    assert n.value > 0
    log = lib.vd_last_error().decode()
    assert "vd_spec_prep_fp64" in log and "vd_spec_prep_mixed" in log
