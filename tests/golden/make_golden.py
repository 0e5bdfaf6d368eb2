"""Generate the golden fixtures of tests/golden/ from the reference's own code.

Run here, where the reference tree and oracle/_ref/ exist:

    python tests/golden/make_golden.py

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

FLUX_VARIANTS = [(1, 3), (2, 3), (5, 1), (5, 2), (5, 3)]


def parse_argon_header(path: Path) -> mm.Mechanism:
    """Mechanism table of a generated argon case header (the Ar_DC_1d form)."""
    txt = path.read_text()
    species = {}
    for name, idx in re.findall(r"#define\s+(\w+)_ID\s+(\d+)", txt):
        if name not in ("NUM",):
            species[int(idx)] = name
    ns = int(re.search(r"#define\s+NUM_SPECIES\s+(\d+)", txt).group(1))
    names = [species[i] for i in range(ns)]
    charge = [0] * ns
    for i, z in re.findall(r"kcharge\[(\d+)\]\s*=\s*(-?\d+)", txt):
        charge[int(i)] = int(z)
    mwb = re.search(r"get_mw\(amrex::Real \*mw_new\)\s*\{(.*?)\}", txt, re.S).group(1)
    mw = [0.0] * ns
    for i, v in re.findall(r"mw_new\[(\d+)\]\s*=\s*([0-9.eE+-]+)", mwb):
        mw[int(i)] = float(v)
    e_cs = float(re.search(r"E_cs\s*=\s*([0-9.eE+-]+)", txt).group(1))
    ion_cs = float(re.search(r"Arp_cs\s*=\s*([0-9.eE+-]+)", txt).group(1))
    ion_amu = float(re.search(r"nu_Arp=std::sqrt\(8\.0\*K_B\*T/PI/\(([0-9.]+)\*M_AMU\)\)", txt).group(1))
    el_amu = float(re.search(r"\(2\.0\*ME/\(([0-9.]+)\*M_AMU\)\)", txt).group(1))
    e_id = names.index("E")
    ion = names.index("ARp")
    body = re.search(r"productionRate\(amrex::Real\* wdot.*?\n\}\n", txt, re.S).group(0)
    blocks = re.findall(r"\{\s*//\s*reaction\s+\d+:\s*([^\n]*)\n(.*?)\n\s*\}", body, re.S)
    rx = []
    for label, blk in blocks:
        b1 = " ".join(blk.split())
        mk = re.search(r"k_f = ([0-9.eE+-]+)\*std::pow\(Te,([0-9.eE+-]+)\)\*std::exp\((-?[0-9.eE+-]+)/Te\)", b1)
        if mk:
            A, b, C = float(mk.group(1)), float(mk.group(2)), -float(mk.group(3))
            kind = abi.RATE_ARRHENIUS_TE
        else:
            A = float(re.search(r"k_f = ([0-9.eE+-]+)\s*;", b1).group(1))
            b = C = 0.0
            kind = abi.RATE_CONST
        reac = [int(s) for s in re.findall(r"sc\[(\d+)\]", re.search(r"qf = k_f \* \((.*?)\);", b1).group(1))]
        terms = []
        for s, op, coef in re.findall(r"wdot\[(\d+)\] ([+-])= (?:([0-9.]+) \* )?qdot;", b1):
            c = float(coef) if coef else 1.0
            terms.append((int(s), c if op == "+" else -c))
        mt = re.search(r"int rxntype = (\d+);", b1)
        rxntype = int(mt.group(1)) if mt else abi.RXN_NONE
        me = re.search(r"eexci = (-?[0-9.eE+-]+);", b1)
        ml = re.search(r"int elidx = (\d+);", b1)
        rx.append(mm.Reaction(reac, [], A, b, C, kind, rxntype, float(me.group(1)) if me else 0.0,
                              int(ml.group(1)) if ml else 0, terms=terms, label=label.strip()))
    tr = mm._ar_like_transport(ns, e_id, {ion: (ion_cs, ion_amu * mm.M_AMU)}, ion, e_cs=e_cs)
    return mm.Mechanism(name="ar_dc_1d", species=names, charge=charge, mw=mw, e_id=e_id, reactions=rx,
                        elastic_loss=1, elastic_mass=el_amu * mm.M_AMU, bg_species=[names.index("AR")], **tr)


def advect_mechanism() -> mm.Mechanism:
    """The two-species Advect verification case (test/verification/Advect): the
    flux uses the user's constant velocity for AR; specMob returns -1."""
    ns = 2
    return mm.Mechanism(name="advect", species=["E", "AR"], charge=[-1, 0], mw=[0.000549, 39.95], e_id=0,
                        mob_kind=[abi.MOB_CONST] * 3, mob_ref=[0] * 3, mob_p0=[-1.0] * 3, mob_p1=[0.0] * 3,
                        diff_kind=[0] * 3, diff_ref=[0] * 3, diff_factor=[1.0] * 3, reactions=[],
                        bg_species=[])


def _save(name: str, case, mech: mm.Mechanism, out: dict, meta: dict):
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
    main()
