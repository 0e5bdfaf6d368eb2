"""Readers of the reference's generated case headers (TEST INFRASTRUCTURE).

Only tests/golden/make_golden.py and oracle/build.py use this module, to turn a
case's Chemistry.H into the runtime mechanism table that the oracle and the CUDA
library take, so that both can be run on the same inputs as the header compiled
unmodified in oracle/_ref.  Forms read:

  test/models/Ar_DC_1d, Axisymmetric_streamer_Ar   Arrhenius / constant rates,
      argon transport (electron and ion cross sections, Chemistry.H:177-239)
  test/models/ionelec_DC_1d                        A exp(-C/Te) N_A rates, constant
      mobilities and diffusion coefficients (Chemistry.H:167-209)
  test/Reactor/CO2_H2_Ar_mechanism_reduced         its Janev / F-fit electron-impact
      reactions (Chemistry.H:940-1030) as a sub-mechanism (fit_submechanism)
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from vidyut_b200 import _abi as abi  # noqa: E402
from vidyut_b200 import mechanism as mm  # noqa: E402

NUM = r"([0-9.]+(?:[eE][+-]?[0-9]+)?)"


def header_species(txt: str):
    """(names, charges, molecular weights) of a generated header"""
    species = {}
    for name, idx in re.findall(r"#define\s+(\w+)_ID\s+(\d+)", txt):
        if name != "NUM":
            species[int(idx)] = name
    m = re.search(r"#define\s+NUM_SPECIES\s+(\d+)", txt) or re.search(r"#define\s+NUM_GAS_SPECIES\s+(\d+)", txt)
    ns = int(m.group(1))
    names = [species[i] for i in range(ns)]
    charge = [0] * ns
    for i, z in re.findall(r"kcharge\[(\d+)\]\s*=\s*(-?\d+)", txt):
        charge[int(i)] = int(z)
    mwb = re.search(r"get_mw\(amrex::Real \*mw_new\)\s*\{(.*?)\}", txt, re.S).group(1)
    mw = [0.0] * ns
    for i, v in re.findall(r"mw_new\[(\d+)\]\s*=\s*([0-9.eE+-]+)", mwb):
        mw[int(i)] = float(v)
    return names, charge, mw


def production_rate_body(txt: str) -> str:
    """the body of productionRate, by matching braces"""
    start = re.search(r"productionRate\(amrex::Real\s*\*\s*wdot", txt).start()
    i = txt.index("{", start)
    depth, j = 0, i
    while True:
        depth += {"{": 1, "}": -1}.get(txt[j], 0)
        j += 1
        if depth == 0:
            return txt[i:j]


def reaction_blocks(body: str):
    """(label, block text) of every '{ // reaction k: ...' block, by matching braces"""
    out = []
    for m in re.finditer(r"\{\s*//\s*reaction\s+\d+:\s*([^\n]*)\n", body):
        i, depth, j = m.start(), 0, m.start()
        while True:
            depth += {"{": 1, "}": -1}.get(body[j], 0)
            j += 1
            if depth == 0:
                break
        out.append((m.group(1).strip(), body[m.end():j - 1]))
    return out


def _species_index(tok: str, names: list) -> int:
    tok = tok.strip()
    if tok.isdigit():
        return int(tok)
    return names.index(tok[:-3] if tok.endswith("_ID") else tok)


def _reactants_terms(b1: str, names: list):
    reac = [_species_index(s, names)
            for s in re.findall(r"sc\[(\w+)\]", re.search(r"qf = k_f \* \((.*?)\);", b1).group(1))]
    terms = []
    for s, op, coef in re.findall(r"wdot\[(\w+)\] ([+-])= (?:([0-9.]+) \* )?qdot;", b1):
        c = float(coef) if coef else 1.0
        terms.append((_species_index(s, names), c if op == "+" else -c))
    mt = re.search(r"int rxntype = (\d+);", b1)
    me = re.search(r"eexci = (-?[0-9.eE+-]+);", b1)
    ml = re.search(r"int elidx = (\d+);", b1)
    return reac, terms, int(mt.group(1)) if mt else abi.RXN_NONE, float(me.group(1)) if me else 0.0, \
        int(ml.group(1)) if ml else 0


def header_reactions(txt: str, names: list):
    """the productionRate blocks of an Ar_DC_1d / Axisymmetric_streamer_Ar /
    ionelec_DC_1d-form header as table reactions"""
    rx = []
    for label, blk in reaction_blocks(production_rate_body(txt)):
        b1 = " ".join(blk.split())
        mk = re.search(r"k_f = " + NUM + r"\*std::pow\(Te,(-?[0-9.eE+-]+)\)\*std::exp\((-?[0-9.eE+-]+)/Te\)", b1)
        mk2 = re.search(r"k_f = " + NUM + r"\*std::exp\((-?[0-9.eE+-]+)/Te\)\*" + NUM + r"\s*;", b1)
        if mk:
            A, b, C = float(mk.group(1)), float(mk.group(2)), -float(mk.group(3))
            kind = abi.RATE_ARRHENIUS_TE
        elif mk2:  # A exp(-C/Te) times Avogadro's number (ionelec_DC_1d)
            A, b, C = float(mk2.group(1)) * float(mk2.group(3)), 0.0, -float(mk2.group(2))
            kind = abi.RATE_ARRHENIUS_TE
        else:
            A = float(re.search(r"k_f = " + NUM + r"\s*;", b1).group(1))
            b = C = 0.0
            kind = abi.RATE_CONST
        reac, terms, rxntype, eexci, elidx = _reactants_terms(b1, names)
        rx.append(mm.Reaction(reac, [], A, b, C, kind, rxntype, eexci, elidx, terms=terms, label=label))
    return rx


def parse_case_header(path: Path, name: str, bg: list) -> mm.Mechanism:
    """Mechanism table of a generated case header.  Transport: the argon form
    (electron and ion cross sections, test/models/Ar_DC_1d/Chemistry.H:177-239) or
    the constant form (test/models/ionelec_DC_1d/Chemistry.H:167-209: constant
    mobilities and diffusion coefficients, the energy's 5/3 of the electrons')."""
    txt = Path(path).read_text()
    names, charge, mw = header_species(txt)
    ns = len(names)
    e_id = names.index("E")
    rx = header_reactions(txt, names)
    el_amu = float(re.search(r"\(2\.0\*ME/\(([0-9.]+)\*M_AMU\)\)", txt).group(1))
    if "E_cs" in txt:
        e_cs = float(re.search(r"E_cs\s*=\s*([0-9.eE+-]+)", txt).group(1))
        ion_cs = float(re.search(r"Arp_cs\s*=\s*([0-9.eE+-]+)", txt).group(1))
        ion_amu = float(re.search(r"nu_Arp=std::sqrt\(8\.0\*K_B\*T/PI/\(([0-9.]+)\*M_AMU\)\)", txt).group(1))
        ion = names.index("ARp")
        tr = mm._ar_like_transport(ns, e_id, {ion: (ion_cs, ion_amu * mm.M_AMU)}, ion, e_cs=e_cs)
    else:
        mob = re.search(r"specMob\(.*?\n\}", txt, re.S).group(0)
        dif = re.search(r"specDiff\(.*?\n\}", txt, re.S).group(0)
        emob = float(re.search(r"elecmob\s*=\s*(-?[0-9.eE+-]+);", mob).group(1))
        ediff = float(re.search(r"elecdcoeff\s*=\s*(-?[0-9.eE+-]+);", dif).group(1))
        tr = dict(mob_kind=[abi.MOB_ZERO] * (ns + 1), mob_ref=[0] * (ns + 1), mob_p0=[0.0] * (ns + 1),
                  mob_p1=[0.0] * (ns + 1), diff_kind=[abi.DIFF_ZERO] * (ns + 1), diff_ref=[0] * (ns + 1),
                  diff_factor=[0.0] * (ns + 1))
        for sp, v in re.findall(r"if\(specid==(\w+)_ID\)\s*\{\s*mob=(-?[0-9.eE+-]+);", mob):
            s = names.index(sp)
            tr["mob_kind"][s], tr["mob_p0"][s] = abi.MOB_CONST, float(v)
        for sp, v in re.findall(r"if\(specid==(\w+)_ID\)\s*\{\s*dcoeff=(-?[0-9.eE+-]+);", dif):
            s = names.index(sp)
            tr["diff_kind"][s], tr["diff_factor"][s] = abi.DIFF_CONST, float(v)
        tr["mob_kind"][e_id], tr["mob_p0"][e_id] = abi.MOB_CONST, emob
        tr["diff_kind"][e_id], tr["diff_factor"][e_id] = abi.DIFF_CONST, ediff
        tr["mob_kind"][ns], tr["mob_ref"][ns], tr["mob_p0"][ns] = abi.MOB_SCALED, e_id, 5.0 / 3.0
        tr["diff_kind"][ns], tr["diff_factor"][ns] = abi.DIFF_CONST, (5.0 / 3.0) * ediff
    return mm.Mechanism(name=name, species=names, charge=charge, mw=mw, e_id=e_id, reactions=rx,
                        elastic_loss=1, elastic_mass=el_amu * mm.M_AMU, bg_species=[names.index(b) for b in bg],
                        **tr)


def fit_submechanism(path: Path, name: str) -> mm.Mechanism:
    """The Janev / F-fit electron-impact reactions of the CO2 reactor header
    (test/Reactor/CO2_H2_Ar_mechanism_reduced/Chemistry.H:940-1030 and the like) as a
    mechanism of their own: the electrons and every species these reactions touch
    (electrons first, then in header order), each reaction with its reactants,
    wdot updates, rxntype, eexci and fit coefficients as the header writes them.
    Transport: the argon form, the first ion as the reference ion (the
    sub-mechanism's header is generated from this table, so any consistent
    transport serves)."""
    txt = Path(path).read_text()
    names, charge, mw = header_species(txt)
    blocks = []
    for label, blk in reaction_blocks(production_rate_body(txt)):
        if "Janev_sum = 0.0" not in blk or "qf = k_f" not in blk:
            continue
        b1 = " ".join(blk.split())
        if "Corr" in b1 or "qr = 0.0" not in b1:
            continue  # third-body or reversible forms stay out
        fit = {"jA": 0.0, "jc": [0.0] * 9, "fA": 0.0, "fc": [0.0] * 4, "switch_ev": 0.0}
        mj = re.search(r"Jfit_coefs = \{([^}]*)\}; double Jfit_A = ([0-9.eE+-]+);", b1)
        mf = re.search(r"Ffit_coefs = \{([^}]*)\}; double Ffit_A = ([0-9.eE+-]+);", b1)
        ms = re.search(r"if\(TeeV < ([0-9.eE+-]+)\)", b1)
        if mj:
            fit["jc"] = [float(v) for v in mj.group(1).split(",")]
            fit["jA"] = float(mj.group(2))
        if mf:
            fit["fc"] = [float(v) for v in mf.group(1).split(",")]
            fit["fA"] = float(mf.group(2))
        if mj and mf:
            kind = abi.RATE_JANEV_FFIT
            fit["switch_ev"] = float(ms.group(1))
        else:
            kind = abi.RATE_JANEV if mj else abi.RATE_FFIT
        reac, terms, rxntype, eexci, elidx = _reactants_terms(b1, names)
        blocks.append((label, reac, terms, rxntype, eexci, elidx, kind, fit))
    used = sorted({names.index("E")} | {s for b in blocks for s in b[1] + [t for t, _ in b[2]]})
    e_old = names.index("E")
    order = [e_old] + [s for s in used if s != e_old]
    new = {s: i for i, s in enumerate(order)}
    rx = []
    for label, reac, terms, rxntype, eexci, elidx, kind, fit in blocks:
        rx.append(mm.Reaction([new[s] for s in reac], [], 0.0, 0.0, 0.0, kind, rxntype, eexci,
                              new.get(elidx, 0), terms=[(new[s], c) for s, c in terms], label=label, fit=fit))
    sub_names = [names[s] for s in order]
    sub_charge = [charge[s] for s in order]
    ns = len(order)
    ion = next(i for i, z in enumerate(sub_charge) if z > 0)
    tr = mm._ar_like_transport(ns, 0, {ion: (120e-20, mw[order[ion]] * mm.M_AMU)}, ion)
    return mm.Mechanism(name=name, species=[n.replace("+", "p") for n in sub_names], charge=sub_charge,
                        mw=[mw[s] for s in order], e_id=0, reactions=rx, elastic_loss=0, elastic_mass=0.0,
                        bg_species=[], **tr)
