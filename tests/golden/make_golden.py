"""Generate the golden fixtures of tests/golden/ from the reference's own code.

Run here, where the reference tree and oracle/_ref/ exist:

    python tests/golden/make_golden.py [fixture ...]   # all, or only the named ones

1. Parses the reference's test/models/Ar_DC_1d/Chemistry.H (species, charges,
   molecular weights, the specMob constants, every productionRate block) into a
   runtime mechanism table -> ar_dc_1d_mech.json.
2. Runs the reference's hot-path code compiled against the AMReX shim
   (oracle/_ref/libvdref_<case>_<dim>d.so) on small seeded boxes and stores
   inputs and outputs as <fixture>.npz, together with the mechanism JSON.

The reference ships no function-level golden vectors for this path, so these
files (outputs of the reference's own compute_flux / CKWC / Joule code) are what
pins the oracle when the reference tree is not mounted.
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from vidyut_b200 import _abi as abi  # noqa: E402
from vidyut_b200 import mechanism as mm  # noqa: E402
from vidyut_b200.inputs import build_case, BASE_SEED  # noqa: E402
import oracle  # noqa: E402
from oracle.build import REF_TREE, build_ref  # noqa: E402
from oracle.headers import fit_submechanism, he_rf_header, parse_case_header, streamer_header  # noqa: E402

FLUX_VARIANTS = [(1, 3), (2, 3), (5, 1), (5, 2), (5, 3)]


def parse_argon_header(path: Path) -> mm.Mechanism:
    """Mechanism table of the Ar_DC_1d case header."""
    return parse_case_header(path, "ar_dc_1d", ["AR"])


def advect_mechanism() -> mm.Mechanism:
    """The two-species Advect verification case (test/verification/Advect): the
    flux uses the user's constant velocity for AR; specMob returns -1."""
    ns = 2
    return mm.Mechanism(name="advect", species=["E", "AR"], charge=[-1, 0], mw=[0.000549, 39.95], e_id=0,
                        mob_kind=[abi.MOB_CONST] * 3, mob_ref=[0] * 3, mob_p0=[-1.0] * 3, mob_p1=[0.0] * 3,
                        diff_kind=[0] * 3, diff_ref=[0] * 3, diff_factor=[1.0] * 3, reactions=[],
                        bg_species=[])


ONLY: set = set()   # fixture names to write (empty: all)


def _save(name: str, case, mech: mm.Mechanism, out: dict, meta: dict):
    if ONLY and name not in ONLY:
        return
    arrays = {"state": case.state}
    for d in range(3):
        arrays[f"efield{d}"] = case.efield[d]
        arrays[f"gradne{d}"] = case.gradne[d]
    arrays.update(out)
    np.savez_compressed(HERE / f"{name}.npz", **arrays)
    meta = dict(meta, dim=case.dim, n=list(case.n), dx=list(case.dx), ghost=case.ghost, params=case.params)
    (HERE / f"{name}.json").write_text(json.dumps({"meta": meta, "mech": mech.to_dict()}, indent=1, default=float))


def flux_outputs(lib, case, species):
    out = {}
    for s in species:
        for d in range(case.dim):
            for h, w in FLUX_VARIANTS:
                out[f"flux_s{s}_d{d}_h{h}_w{w}"] = lib.flux(case, d, s, hyp_order=h, weno=w)
    return out


def main():
    build_ref()
    # 1. the reference's own Ar_DC_1d mechanism header
    mech = parse_argon_header(REF_TREE / "test" / "models" / "Ar_DC_1d" / "Chemistry.H")
    case = build_case(mech, 2, (12, 10), (1e-5, 1e-5), BASE_SEED + 101, density="blob", te_range_ev=(0.5, 5.0))
    ref = oracle.RefLib("ar_dc_1d", 2)
    out = {"rxn": ref.reaction_source(case)}
    out.update(flux_outputs(ref, case, range(mech.ns + 1)))
    upd = ref.update_all(case, case.vd_params())
    out.update({f"upd_{k}": v for k, v in upd.items()})
    _save("ar_dc_1d_2d", case, mech, out, {"ref": "ar_dc_1d", "header": "test/models/Ar_DC_1d/Chemistry.H"})

    # 1b. the reference's other model headers: Axisymmetric_streamer_Ar (the argon
    # form) and ionelec_DC_1d (constant mobilities and diffusion coefficients)
    models = [("axisym_ar", "Axisymmetric_streamer_Ar", ["AR"], [2]), ("ionelec", "ionelec_DC_1d", ["HE"], [1, 2])]
    for name, sub, bg, dims in models:
        hdr = REF_TREE / "test" / "models" / sub / "Chemistry.H"
        m = parse_case_header(hdr, name, bg)
        for dim in dims:
            n = (12, 10) if dim == 2 else (48,)
            case = build_case(m, dim, n, (1e-5,) * dim, BASE_SEED + 110 + dim, density="blob",
                              te_range_ev=(0.5, 5.0))
            ref = oracle.RefLib(name, dim)
            out = {"rxn": ref.reaction_source(case)}
            out.update(flux_outputs(ref, case, range(m.ns + 1)))
            upd = ref.update_all(case, case.vd_params())
            out.update({f"upd_{k}": v for k, v in upd.items()})
            # ionelec_DC_1d writes k = A exp(-C/Te) N_A: the table holds A N_A (rounding apart)
            _save(f"{name}_{dim}d", case, m, out, {"ref": name, "header": f"test/models/{sub}/Chemistry.H",
                                                   "exact": name != "ionelec"})

    # 1c. the verification headers with field-dependent transport: Streamer (power
    # laws in |E|, the field-driven ionisation rate, which reads the reduced field
    # REF) and He_RF_1d (|E|/N and mean-energy mobility fits, pressure-scaled
    # diffusion, the elastic loss at |E| = EN N 1e-21)
    vmodels = [("streamer", "Streamer", streamer_header, ["N2"], 2, 1),
               ("he_rf", "He_RF_1d", he_rf_header, ["HE"], 1, 1)]
    for name, sub, parse, bg, dim, een in vmodels:
        m = parse(REF_TREE / "test" / "verification" / sub / "Chemistry.H", name, bg)
        n = (12, 10) if dim == 2 else (48,)
        case = build_case(m, dim, n, (1e-5,) * dim, BASE_SEED + 130 + dim, density="blob", te_range_ev=(0.5, 5.0),
                          params=dict(elecenergy_solve=een))
        ref = oracle.RefLib(name, dim)
        out = {"rxn": ref.reaction_source(case)}
        out.update(flux_outputs(ref, case, range(m.ns + 1)))
        upd = ref.update_all(case, case.vd_params())
        out.update({f"upd_{k}": v for k, v in upd.items()})
        _save(f"{name}_{dim}d", case, m, out, {"ref": name, "header": f"test/verification/{sub}/Chemistry.H"})

    # 2. the Advect verification case: constant user velocity (udv=1) for AR
    am = advect_mechanism()
    case = build_case(am, 2, (16, 6), (0.1, 0.1), BASE_SEED + 102, density="loguniform", dens_range=(1.0, 2.0))
    ref = oracle.RefLib("advect", 2)
    out = {}
    for d in range(2):
        for h, w in FLUX_VARIANTS:
            out[f"flux_s1_d{d}_h{h}_w{w}"] = ref.flux(case, d, 1, hyp_order=h, weno=w, udv=1, uvel=(1.0, 0.5, 0.0),
                                                      bclo=(0, 0, 0), bchi=(0, 0, 0))
    _save("advect_2d", case, am, out, {"ref": "advect", "uvel": [1.0, 0.5, 0.0], "vel_species": 1})

    # 2b. the Janev / F-fit electron-impact reactions of the CO2 reactor header
    # (test/Reactor/CO2_H2_Ar_mechanism_reduced/Chemistry.H:940-1030) in that header's
    # code form; Te over 0.3-20 eV so that both branches of the piecewise fits run
    fm = fit_submechanism(REF_TREE / "test" / "Reactor" / "CO2_H2_Ar_mechanism_reduced" / "Chemistry.H", "co2fits")
    case = build_case(fm, 2, (11, 9), (1e-5, 1e-5), BASE_SEED + 120, density="loguniform", te_range_ev=(0.3, 20.0),
                      dens_range=(1e10, 1e20))
    ref = oracle.RefLib("co2fits", 2)
    out = {"rxn": ref.reaction_source(case)}
    upd = ref.update_all(case, case.vd_params())
    out.update({f"upd_{k}": v for k, v in upd.items()})
    # rate_tol: the fit sums cancel terms up to ~1e5 times larger than the result, so
    # a difference of a few ulp in pow() or in the summation moves a rate by up to
    # ~1e-9 relative (the reference's own result carries the same spread)
    _save("co2fits_2d", case, fm, out, {"ref": "co2fits", "rate_tol": 2e-9,
                                        "header": "test/Reactor/CO2_H2_Ar_mechanism_reduced/Chemistry.H"})

    # 3. generated-header mechanisms of the workloads, one small box each
    gens = [
        (mm.argon(10, BASE_SEED + 1), 2, (20, 14), "blob", (0.5, 5.0), (1e8, 1e22)),
        (mm.synthetic(24, 150, BASE_SEED + 11), 3, (7, 6, 5), "loguniform", (0.3, 10.0), (1e8, 1e22)),
        (mm.synthetic(8, 40, BASE_SEED + 21), 1, (40, 1, 1), "loguniform", (0.5, 5.0), (1e10, 1e18)),
        (mm.synthetic(8, 40, BASE_SEED + 21), 2, (11, 9), "loguniform", (0.5, 5.0), (1e10, 1e18)),
    ]
    for m, dim, n, dens, te, dr in gens:
        dxs = (1e-5,) * dim
        case = build_case(m, dim, n, dxs, BASE_SEED + 103 + dim, density=dens, te_range_ev=te, dens_range=dr)
        ref = oracle.RefLib(m.name, dim)
        out = {"rxn": ref.reaction_source(case)}
        out.update(flux_outputs(ref, case, [m.e_id, m.ns]))
        upd = ref.update_all(case, case.vd_params())
        out.update({f"upd_{k}": v for k, v in upd.items()})
        _save(f"{m.name}_{dim}d", case, m, out, {"ref": m.name})
    print("fixtures written to", HERE)


if __name__ == "__main__":
    ONLY.update(sys.argv[1:])
    main()
