"""Build the CPU oracle (TEST INFRASTRUCTURE ONLY).

  oracle/_build/libvdoracle.so   the C restatement (vd_oracle.c), gcc -O2, no FP
                                 contraction, OpenMP
  oracle/_ref/libvdref_<case>_<dim>d.so
                                 the reference's own hot-path headers compiled
                                 unmodified against oracle/refshim, one library
                                 per (case, dimension) as the reference builds
                                 one executable per case.  Needs the reference
                                 tree ($VIDYUT_REFERENCE, or a checkout named
                                 "reference" beside this repository); skipped (not
                                 an error) when it is absent, in which case
                                 previously built libraries are used.

    python oracle/build.py            # oracle + every reference case
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
BUILD = HERE / "_build"
REF_OUT = HERE / "_ref"
# The reference tree: $VIDYUT_REFERENCE, else a checkout named "reference" beside
# this repository's directory.
REF_TREE = Path(os.environ["VIDYUT_REFERENCE"]) if os.environ.get("VIDYUT_REFERENCE") else ROOT.parent / "reference"

ORACLE_LIB = BUILD / "libvdoracle.so"

CFLAGS = ["-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math"]


def build_oracle(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    src = HERE / "vd_oracle.c"
    hdr = ROOT / "include" / "vidyut_b200.h"
    if force or not ORACLE_LIB.exists() or max(src.stat().st_mtime, hdr.stat().st_mtime) > ORACLE_LIB.stat().st_mtime:
        cmd = ["gcc", "-std=c11", *CFLAGS, str(src), "-lm", "-o", str(ORACLE_LIB)]
        subprocess.run(cmd, check=True)
    return ORACLE_LIB


def _ref_cases():
    """(name, case directory, dims, extra defines, mechanism or None).  Generated
    cases (mechanism given) are written to _ref/gen/<name>/ first."""
    sys.path.insert(0, str(ROOT))
    from vidyut_b200 import mechanism as mm
    from vidyut_b200.inputs import BASE_SEED
    t = REF_TREE / "test"
    cases = [
        ("ar_dc_1d", t / "models" / "Ar_DC_1d", (2,), [], None),
        ("axisym_ar", t / "models" / "Axisymmetric_streamer_Ar", (2,), [], None),
        ("ionelec", t / "models" / "ionelec_DC_1d", (1, 2), [], None),
        ("advect", t / "verification" / "Advect", (2, 3), ["-DVD_PROBPARM_HAS_VEL"], None),
        ("streamer", t / "verification" / "Streamer", (2,), [], None),
        ("he_rf", t / "verification" / "He_RF_1d", (1,), [], None),
    ]
    gen = [
        (mm.argon(10, BASE_SEED + 1), (1, 2, 3)),            # argon 2-D workload mechanism
        (mm.synthetic(24, 150, BASE_SEED + 11), (3,)),       # 3-D precision workload mechanism
        (mm.synthetic(8, 40, BASE_SEED + 21), (1, 2, 3)),    # batched / serving mechanism
        (mm.synthetic(12, 60, BASE_SEED + 31), (3,)),        # large-case mechanism
    ]
    co2 = t / "Reactor" / "CO2_H2_Ar_mechanism_reduced" / "Chemistry.H"
    if co2.exists():  # its Janev / F-fit reactions, in that header's code form
        from headers import fit_submechanism
        gen.append((fit_submechanism(co2, "co2fits"), (2,)))
    for m, dims in gen:
        cases.append((m.name, REF_OUT / "gen" / m.name, dims, [], m))
    return cases


def ref_lib_path(name: str, dim: int) -> Path:
    return REF_OUT / f"libvdref_{name}_{dim}d.so"


def build_ref(force: bool = False, only: str | None = None) -> list[Path]:
    if not (REF_TREE / "Source" / "compute_explicit_flux.H").exists():
        return sorted(REF_OUT.glob("libvdref_*.so"))
    sys.path.insert(0, str(HERE))
    from gen_case import write_case
    REF_OUT.mkdir(exist_ok=True)
    drv = HERE / "refdriver" / "vd_ref_driver.cpp"
    shim = HERE / "refshim"
    out = []
    for name, cdir, dims, defs, mech in _ref_cases():
        if only and name != only:
            continue
        if mech is not None:
            write_case(mech, cdir)
        deps = [drv, ROOT / "include" / "vidyut_b200.h", *shim.glob("*.H"), *Path(cdir).glob("*.H")]
        for dim in dims:
            lib = ref_lib_path(name, dim)
            if not force and lib.exists() and all(d.stat().st_mtime <= lib.stat().st_mtime for d in deps):
                out.append(lib)
                continue
            cmd = ["g++", "-std=c++17", "-O3", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
                   f"-DAMREX_SPACEDIM={dim}", *defs, f"-I{shim}", f"-I{cdir}", f"-I{REF_TREE / 'Source'}",
                   str(drv), "-o", str(lib)]
            subprocess.run(cmd, check=True)
            out.append(lib)
    return out


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_ref(force)


if __name__ == "__main__":
    build_all(force="-f" in sys.argv)
    print(ORACLE_LIB)
    for p in sorted(REF_OUT.glob("libvdref_*.so")):
        print(p)
