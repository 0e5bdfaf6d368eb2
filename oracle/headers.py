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
  test/verification/Streamer                       the field-driven ionisation rate and
      power laws in |E| for the electron mobility and diffusion (Chemistry.H:164-282)
  test/verification/He_RF_1d                       E/N-polynomial ion mobility, mean-energy
      fit electron mobility, pressure-scaled diffusion, elastic loss with
      |E| = EN N 1e-21 (Chemistry.H:217-299,603-625)
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
        # A Te^b alone (He_RF_1d): A Te^b exp(-0/Te) is the same number
        mk3 = re.search(r"k_f = " + NUM + r"\*std::pow\(Te,(-?[0-9.eE+-]+)\)\s*;", b1)
        if mk:
            A, b, C = float(mk.group(1)), float(mk.group(2)), -float(mk.group(3))
            kind = abi.RATE_ARRHENIUS_TE
        elif mk3:
            A, b, C = float(mk3.group(1)), float(mk3.group(2)), 0.0
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


def _num(pat: str, txt: str, group: int = 1) -> float:
    return float(re.search(pat, txt, re.S).group(group))


def _transport_table(ns: int) -> dict:
    return dict(mob_kind=[abi.MOB_ZERO] * (ns + 1), mob_ref=[0] * (ns + 1), mob_p0=[0.0] * (ns + 1),
                mob_p1=[0.0] * (ns + 1), diff_kind=[abi.DIFF_ZERO] * (ns + 1), diff_ref=[0] * (ns + 1),
                diff_factor=[0.0] * (ns + 1), diff_p1=[0.0] * (ns + 1))


def streamer_header(path: Path, name: str, bg: list) -> mm.Mechanism:
    """Mechanism table of the Streamer verification header
    (test/verification/Streamer/Chemistry.H): electron mobility p0 |E|^p1 and
    diffusion f |E|^q, the energy's 5/3 of both, an immobile ion, and the one
    field-driven ionisation reaction (alpha - eta) mu_e |E| of :260-281, first
    order in the electrons, with wdot updates E +1, N2 -1, N2p +1."""
    txt = Path(path).read_text()
    names, charge, mw = header_species(txt)
    ns = len(names)
    e_id = names.index("E")
    mob = re.search(r"specMob\(.*?\n\}", txt, re.S).group(0)
    dif = re.search(r"specDiff\(.*?\n\}", txt, re.S).group(0)
    tr = _transport_table(ns)
    m = re.search(r"elecmob\s*=\s*(-?[0-9.eE+-]+)\*std::pow\(emag,(-?[0-9.eE+-]+)\)", mob)
    tr["mob_kind"][e_id], tr["mob_p0"][e_id], tr["mob_p1"][e_id] = abi.MOB_POW_EMAG, float(m.group(1)), float(m.group(2))
    m = re.search(r"elecdcoeff\s*=\s*(-?[0-9.eE+-]+)\s*\*\s*std::pow\(emag,(-?[0-9.eE+-]+)\)", dif)
    tr["diff_kind"][e_id], tr["diff_factor"][e_id], tr["diff_p1"][e_id] = \
        abi.DIFF_POW_EMAG, float(m.group(1)), float(m.group(2))
    assert re.search(r"mob=\(5\.0/3\.0\)\*elecmob", mob) and re.search(r"dcoeff=\(5\.0/3\.0\)\*elecdcoeff", dif)
    tr["mob_kind"][ns], tr["mob_ref"][ns], tr["mob_p0"][ns] = abi.MOB_SCALED, e_id, 5.0 / 3.0
    tr["diff_kind"][ns], tr["diff_ref"][ns], tr["diff_factor"][ns] = abi.DIFF_SCALED, e_id, 5.0 / 3.0
    body = " ".join(production_rate_body(txt).split())
    c = [_num(r"alpha = \(" + NUM + r" \+", body), _num(r"\+ " + NUM + r"/std::pow\(efield_mag,3\.0\)", body),
         _num(r"std::exp\(-" + NUM + r"/efield_mag\)", body), _num(r"eta = " + NUM + r";", body)]
    m = re.search(r"mu_e = " + NUM + r" \* std::pow\(efield_mag,(-?[0-9.eE+-]+)\)", body)
    c += [float(m.group(1)), float(m.group(2))]
    terms = [(_species_index(sp, names), 1.0 if op == "+" else -1.0)
             for sp, op in re.findall(r"wdot\[(\w+)\] ([+-])= k_f\*sc\[E_ID\];", body)]
    rx = [mm.Reaction([e_id], [], 0.0, kind=abi.RATE_TOWNSEND, terms=terms, label="N2 + E => E + N2p + E",
                      fit={"jc": c + [0.0] * 3})]
    return mm.Mechanism(name=name, species=names, charge=charge, mw=mw, e_id=e_id, reactions=rx,
                        elastic_loss=0, elastic_mass=0.0, bg_species=[names.index(b) for b in bg], **tr)


def he_rf_header(path: Path, name: str, bg: list) -> mm.Mechanism:
    """Mechanism table of the He_RF_1d verification header
    (test/verification/He_RF_1d/Chemistry.H): the ions' mobility
    p0 (1 + c0 (|E|/N)^2 + c1 (|E|/N)^4)^p, the electrons' exp(mean-energy fit)/N,
    pressure-scaled diffusion (the electrons' also times Te / T0), the energy's
    5/3 of the electrons' mobility and diffusion, Arrhenius / constant rates and
    the elastic loss of CKWC (:603-625) with a 4 amu partner."""
    txt = Path(path).read_text()
    names, charge, mw = header_species(txt)
    ns = len(names)
    e_id = names.index("E")
    mob = re.search(r"specMob\(.*?\n\}", txt, re.S).group(0)
    dif = re.search(r"specDiff\(.*?\n\}", txt, re.S).group(0)
    tr = _transport_table(ns)
    mob_coef = {}
    m = re.search(r"(\w+)mob=" + NUM + r"\*std::pow\(\(1\.0\+" + NUM + r"\*std::pow\(EbyN,2\.0\)\+" + NUM
                  + r"\*std::pow\(EbyN,4\.0\)\),(-?[0-9.eE+-]+)\);", mob)
    ion_var, p0, c0, c1, pw = m.group(1), float(m.group(2)), float(m.group(3)), float(m.group(4)), float(m.group(5))
    same = {ion_var} | set(re.findall(r"(\w+)mob=" + ion_var + r"mob;", mob))
    for sp, var in re.findall(r"if\(specid==(\w+)_ID\)\s*\{(?:\s*//[^\n]*)*\s*mob=(\w+);", mob):
        if var in {v + "mob" for v in same}:
            s = names.index(sp)
            tr["mob_kind"][s], tr["mob_p0"][s], tr["mob_p1"][s] = abi.MOB_EN_POLY, p0, pw
            mob_coef[str(s)] = [c0, c1]
    m = re.search(r"elecmob = \((-?[0-9.]+)\)\*std::exp\(" + NUM + r" \+ " + NUM + r"\*std::log\(meanE\) \+ "
                  + NUM + r"/meanE\s*-" + NUM + r"/std::pow\(meanE,2\.0\) \+ \(" + NUM
                  + r"\)/std::pow\(meanE,3\.0\)\) / ndens;", mob)
    tr["mob_kind"][e_id], tr["mob_p0"][e_id] = abi.MOB_EXP_MEANE, float(m.group(1))
    mob_coef[str(e_id)] = [float(m.group(2)), float(m.group(3)), float(m.group(4)), -float(m.group(5)),
                           float(m.group(6))]
    tr["mob_kind"][ns], tr["mob_ref"][ns], tr["mob_p0"][ns] = abi.MOB_SCALED, e_id, 5.0 / 3.0
    m = re.search(r"elecdcoeff=" + NUM + r"\*\(Te/" + NUM + r"\)\*Pres_ratio;", dif)
    tr["diff_kind"][e_id], tr["diff_factor"][e_id], tr["diff_p1"][e_id] = \
        abi.DIFF_TE_PRES, float(m.group(1)), float(m.group(2))
    for sp, v in re.findall(r"if\(specid==(\w+)_ID\)\s*\{(?:\s*//[^\n]*)*\s*dcoeff=" + NUM + r"\*Pres_ratio;", dif):
        s = names.index(sp)
        tr["diff_kind"][s], tr["diff_factor"][s] = abi.DIFF_PRES, float(v)
    tr["diff_kind"][ns], tr["diff_ref"][ns], tr["diff_factor"][ns] = abi.DIFF_SCALED, e_id, 5.0 / 3.0
    rx = header_reactions(txt, names)
    el_amu = float(re.search(r"\(2\.0\*ME/\(([0-9.]+)\*M_AMU\)\)", txt).group(1))
    return mm.Mechanism(name=name, species=names, charge=charge, mw=mw, e_id=e_id, reactions=rx,
                        elastic_loss=1, elastic_mass=el_amu * mm.M_AMU, bg_species=[names.index(b) for b in bg],
                        mob_coef=mob_coef, **tr)
