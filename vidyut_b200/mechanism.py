"""Runtime plasma-chemistry mechanisms (the reference compiles them in as Chemistry.H).

A ``Mechanism`` carries what the reference's generated case header provides
(test/models/Ar_DC_1d/Chemistry.H): species with charges (CKCHRG) and molecular
weights (get_mw), the mobility / diffusion models (specMob, specDiff), and the
reaction list of productionRate with its energy-exchange types (comp_ener_exch).
``to_c()`` packs it into the ``vd_mech`` table that ``vd_mech_init`` loads.

Reaction updates keep the generated header's order: ``terms`` lists the
``wdot[sp] += coef * qdot`` updates in the order they are applied, so a
species on both sides (``E + AR => E + ARm``) gets a separate -1 and +1 term, as
the header writes ``wdot[0] -= qdot; wdot[0] += qdot;``.

Generators (seeded, all parameters drawn with numpy's PCG64):
  argon(n_reactions, seed)          E, AR, ARm, ARp with Arrhenius-Te rates
  synthetic(n_species, n_reactions, seed)   charge-conserving random mechanism
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field, asdict

import numpy as np

from . import _abi as abi

# Source/UnivConstants.H:4-18
N_A = 6.02214076e23
K_B = 1.380649e-23
ECHARGE = 1.60217662e-19
EV = ECHARGE / K_B          # kelvin per eV
ME = 9.10938188e-31
M_AMU = 1.66054e-27
PI = 3.14159265358979323846264338327950288

# three-body rates: pseudo-two-body rate at this density lies in the stated range
THREE_BODY_NREF = 2.4e25


@dataclass
class Reaction:
    reactants: list            # species indices, q = k * prod(sc[r]) in this order
    products: list
    A: float                   # table units: (m^3/mol)^(n-1)/s, k = A Te^b exp(-C/Te), Te in K
    b: float = 0.0
    C: float = 0.0             # kelvin
    kind: int = abi.RATE_ARRHENIUS_TE
    rxntype: int = abi.RXN_NONE
    eexci: float = 0.0         # eV
    elidx: int = 0
    terms: list = field(default_factory=list)   # [(species, coef)] update order
    label: str = ""
    # fit rate kinds (RATE_JANEV, RATE_FFIT, RATE_JANEV_FFIT): {"jA", "jc" (9), "fA",
    # "fc" (4), "switch_ev"} as the CO2 reactor header writes them
    fit: dict | None = None

    def fill_terms(self) -> "Reaction":
        """Default update order: species ascending; reactant loss then product gain."""
        if not self.terms:
            sp = sorted(set(self.reactants) | set(self.products))
            t = []
            for s in sp:
                nr = self.reactants.count(s)
                npd = self.products.count(s)
                if nr:
                    t.append((s, -float(nr)))
                if npd:
                    t.append((s, float(npd)))
            self.terms = t
        return self


@dataclass
class Mechanism:
    name: str
    species: list
    charge: list
    mw: list                   # g/mol
    e_id: int
    mob_kind: list             # length NS+1 (last entry: electron energy)
    mob_ref: list
    mob_p0: list
    mob_p1: list
    diff_kind: list
    diff_ref: list
    diff_factor: list
    reactions: list
    elastic_loss: int = 0
    elastic_mass: float = 0.0  # kg
    bg_species: list = field(default_factory=list)
    diff_p1: list | None = None   # DIFF_POW_EMAG exponent / DIFF_TE_PRES scale (default 0)
    # MOB_EN_POLY / MOB_EXP_MEANE coefficients c per species ({str(s): [c0, ...]});
    # to_c stores them as fits and points mob_ref at them
    mob_coef: dict = field(default_factory=dict)

    @property
    def ns(self) -> int:
        return len(self.species)

    @property
    def nvar(self) -> int:
        return self.ns + 10

    def to_c(self) -> abi.VdMech:
        if self.ns > abi.MAX_SPECIES or len(self.reactions) > abi.MAX_REACTIONS:
            raise ValueError("mechanism exceeds the table limits")
        m = abi.VdMech()
        m.nspecies = self.ns
        m.nreactions = len(self.reactions)
        m.e_id = self.e_id
        for s in range(self.ns):
            m.charge[s] = int(self.charge[s])
            m.mw[s] = float(self.mw[s])
        for s in range(self.ns + 1):
            m.mob_kind[s] = int(self.mob_kind[s])
            m.mob_ref[s] = int(self.mob_ref[s])
            m.mob_p0[s] = float(self.mob_p0[s])
            m.mob_p1[s] = float(self.mob_p1[s])
            m.diff_kind[s] = int(self.diff_kind[s])
            m.diff_ref[s] = int(self.diff_ref[s])
            m.diff_factor[s] = float(self.diff_factor[s])
            m.diff_p1[s] = float(self.diff_p1[s]) if self.diff_p1 is not None else 0.0
        m.elastic_loss = int(self.elastic_loss)
        m.elastic_mass = float(self.elastic_mass)
        nfits = 0
        for i, r in enumerate(self.reactions):
            r.fill_terms()
            if len(r.terms) > abi.MAX_TERMS or len(r.reactants) > abi.MAX_REACTANTS:
                raise ValueError(f"reaction {i} too large")
            c = m.rxn[i]
            c.kind = r.kind
            c.nreac = len(r.reactants)
            for t, s in enumerate(r.reactants):
                c.reac[t] = s
            c.rxntype = r.rxntype
            c.elidx = r.elidx
            c.nterms = len(r.terms)
            for t, (s, coef) in enumerate(r.terms):
                c.term_sp[t] = s
                c.term_coef[t] = coef
            c.A, c.b, c.C, c.eexci = float(r.A), float(r.b), float(r.C), float(r.eexci)
            if r.kind >= abi.RATE_JANEV:  # the Townsend kind keeps its c in jc
                if nfits >= abi.MAX_FITS:
                    raise ValueError("too many fit rates")
                f = m.fits[nfits]
                f.jA, f.fA = float(r.fit.get("jA", 0.0)), float(r.fit.get("fA", 0.0))
                for j, v in enumerate(r.fit.get("jc", [0.0] * 9)):
                    f.jc[j] = float(v)
                for j, v in enumerate(r.fit.get("fc", [0.0] * 4)):
                    f.fc[j] = float(v)
                f.switch_ev = float(r.fit.get("switch_ev", 0.0))
                c.fit = nfits
                nfits += 1
        for s in range(self.ns + 1):
            if self.mob_kind[s] in (abi.MOB_EN_POLY, abi.MOB_EXP_MEANE):
                if nfits >= abi.MAX_FITS:
                    raise ValueError("too many fits")
                coef = self.mob_coef[str(s)]
                for j, v in enumerate(coef):
                    m.fits[nfits].jc[j] = float(v)
                m.mob_ref[s] = nfits
                nfits += 1
        m.nfits = nfits
        return m

    def to_dict(self) -> dict:
        d = asdict(self)
        return d

    @staticmethod
    def from_dict(d: dict) -> "Mechanism":
        d = dict(d)
        rx = [Reaction(**{**r, "terms": [tuple(t) for t in r.get("terms", [])]}) for r in d.pop("reactions")]
        return Mechanism(reactions=rx, **d)

    def to_json(self) -> str:
        return json.dumps(self.to_dict(), indent=1)

    @staticmethod
    def from_json(s: str) -> "Mechanism":
        return Mechanism.from_dict(json.loads(s))

    def bg_mask(self) -> int:
        m = 0
        for s in self.bg_species:
            m |= 1 << s
        return m

    def charge_balance_ok(self) -> bool:
        for r in self.reactions:
            zr = sum(self.charge[s] for s in r.reactants)
            zp = sum(self.charge[s] for s in r.products)
            if zr != zp:
                return False
        return True


# ---------------------------------------------------------------------------
def _ar_like_transport(ns: int, e_id: int, ions: dict, neutral_ref: int | None, e_cs=40e-20):
    """Mobility/diffusion tables in the form of the argon case header
    (test/models/Ar_DC_1d/Chemistry.H:177-239): electrons collide with the gas
    (cross section e_cs), ions with the gas at Tg, neutrals do not drift, the
    electron energy drifts with 5/3 of the electron mobility; D_e = Te[eV] |mu_e|,
    D_ion = Tg[eV] mu_ion, neutral diffusion borrows the reference ion's mobility.
    ions: {species: (cross section, mass kg)}."""
    mob_kind = [abi.MOB_ZERO] * (ns + 1)
    mob_ref = [0] * (ns + 1)
    mob_p0 = [0.0] * (ns + 1)
    mob_p1 = [0.0] * (ns + 1)
    diff_kind = [abi.DIFF_ZERO] * (ns + 1)
    diff_ref = [0] * (ns + 1)
    diff_factor = [1.0] * (ns + 1)
    mob_kind[e_id] = abi.MOB_ELECTRON
    mob_p0[e_id] = e_cs
    diff_kind[e_id] = abi.DIFF_TE_ABSMOB
    diff_ref[e_id] = e_id
    for s, (cs, mass) in ions.items():
        mob_kind[s] = abi.MOB_ION_TG
        mob_p0[s] = cs
        mob_p1[s] = mass
        diff_kind[s] = abi.DIFF_TG_MOB
        diff_ref[s] = s
    for s in range(ns):
        if mob_kind[s] == abi.MOB_ZERO and s != e_id and neutral_ref is not None:
            diff_kind[s] = abi.DIFF_TG_MOB
            diff_ref[s] = neutral_ref
    mob_kind[ns] = abi.MOB_SCALED
    mob_ref[ns] = e_id
    mob_p0[ns] = 5.0 / 3.0
    diff_kind[ns] = abi.DIFF_TE_ABSMOB
    diff_ref[ns] = e_id
    diff_factor[ns] = 5.0 / 3.0
    return dict(mob_kind=mob_kind, mob_ref=mob_ref, mob_p0=mob_p0, mob_p1=mob_p1,
                diff_kind=diff_kind, diff_ref=diff_ref, diff_factor=diff_factor)


def _draw_rate(rng, nreac: int, a_lo=1e-20, a_hi=1e-14, b_lo=-1.0, b_hi=1.0, c_lo=0.0, c_hi=20.0):
    """A log-uniform [m^3/s] (the rate at Te = 1 eV), b uniform, C uniform [eV].
    Stored in the reference's form k = A Te^b exp(-C/Te) with Te in kelvin and
    concentrations in mol/m^3: A_table = A N_A^(n-1) (eV in K)^(-b), C_table = C EV."""
    A = 10.0 ** rng.uniform(math.log10(a_lo), math.log10(a_hi))
    if nreac == 3:
        A /= THREE_BODY_NREF
    b = float(rng.uniform(b_lo, b_hi))
    c = float(rng.uniform(c_lo, c_hi))
    A_tab = A * N_A ** (nreac - 1) * EV ** (-b)
    return A_tab, b, c * EV


def argon(n_reactions: int = 10, seed: int = 20261203) -> Mechanism:
    """Argon discharge mechanism on the species of test/models/Ar_DC_1d
    (E, AR, ARm, ARp; AR is the background gas) with seeded Arrhenius-Te rates."""
    rng = np.random.default_rng(seed)
    E, AR, ARm, ARp = 0, 1, 2, 3
    templates = [
        ([E, AR], [E, E, ARp], abi.RXN_IONIZATION, 15.76, 0, "E + AR => E + E + ARp"),
        ([E, ARm], [E, E, ARp], abi.RXN_IONIZATION, 4.21, 0, "E + ARm => E + E + ARp"),
        ([E, AR], [E, ARm], abi.RXN_EXCITATION, 11.55, 0, "E + AR => E + ARm"),
        ([E, ARm], [E, AR], abi.RXN_EXCITATION, -11.55, 0, "E + ARm => E + AR"),
        ([ARm, ARm], [E, AR, ARp], abi.RXN_IONIZATION, -7.0, 0, "ARm + ARm => E + AR + ARp"),
        ([E, ARp], [ARm], abi.RXN_RECOMB, 0.0, 0, "E + ARp => ARm"),
        ([E, E, ARp], [E, ARm], abi.RXN_RECOMB, 0.0, 0, "E + E + ARp => E + ARm"),
        ([AR, ARm], [AR, AR], abi.RXN_NONE, 0.0, 0, "AR + ARm => AR + AR"),
        ([E, AR], [E, AR], abi.RXN_ELASTIC, 0.0, AR, "E + AR => E + AR"),
        ([E, ARp, AR], [ARm, AR], abi.RXN_RECOMB, 0.0, 0, "E + ARp + AR => ARm + AR"),
    ]
    rx = []
    for i in range(n_reactions):
        reac, prod, rt, ee, el, lab = templates[i % len(templates)]
        A, b, C = _draw_rate(rng, len(reac))
        rx.append(Reaction(list(reac), list(prod), A, b, C, abi.RATE_ARRHENIUS_TE, rt, ee, el,
                           label=lab).fill_terms())
    m_ar = 39.948 * M_AMU
    tr = _ar_like_transport(4, E, {ARp: (120e-20, m_ar)}, ARp)
    return Mechanism(name=f"argon{n_reactions}_s{seed}", species=["E", "AR", "ARm", "ARp"],
                     charge=[-1, 0, 0, 1], mw=[0.000549, 39.95, 39.95, 39.949451], e_id=E,
                     reactions=rx, elastic_loss=1, elastic_mass=m_ar, bg_species=[AR], **tr)


def synthetic(n_species: int, n_reactions: int, seed: int = 20261203) -> Mechanism:
    """Charge-conserving random mechanism: species 0 electrons, 1 background gas M,
    then neutral/ion pairs (X_k, X_k+) and, for an odd remainder, one excited
    neutral.  Reaction templates: ionization, excitation / de-excitation, elastic
    momentum transfer, two- and three-body recombination, charge exchange, Penning
    ionization, neutral exchange and three-body association; 2-3 reactants each."""
    if n_species < 4:
        raise ValueError("synthetic mechanisms need >= 4 species")
    rng = np.random.default_rng(seed)
    names = ["E", "M"]
    charge = [-1, 0]
    mw = [0.000549, 39.948]
    neutrals = [1]
    ions = []
    parent = {}
    npair = (n_species - 2) // 2
    for k in range(npair):
        m = float(np.round(rng.uniform(4.0, 100.0), 3))
        names += [f"X{k}", f"X{k}+"]
        charge += [0, 1]
        mw += [m, m - 0.000549]
        neutrals.append(len(names) - 2)
        ions.append(len(names) - 1)
        parent[len(names) - 1] = len(names) - 2
    if (n_species - 2) % 2:
        names.append("Xs")
        charge.append(0)
        mw.append(float(np.round(rng.uniform(4.0, 100.0), 3)))
        neutrals.append(len(names) - 1)
    ns = len(names)
    E, M = 0, 1
    ion_of = {v: k for k, v in parent.items()}
    ionizable = [n for n in neutrals if n in ion_of] + [M]

    def pick(lst):
        return int(lst[rng.integers(len(lst))])

    kinds = ["ion", "exc", "dexc", "ela", "rec2", "rec3", "cx", "penning", "nn", "assoc3"]
    weights = np.array([3, 3, 2, 2, 2, 1, 2, 1, 2, 1], dtype=float)
    weights /= weights.sum()
    rx = []
    while len(rx) < n_reactions:
        kind = kinds[rng.choice(len(kinds), p=weights)]
        rt, ee, el = abi.RXN_NONE, 0.0, 0
        if kind == "ion":
            n = pick([x for x in ionizable if x in ion_of] or [neutrals[1]])
            if n not in ion_of:
                continue
            reac, prod = [E, n], [E, E, ion_of[n]]
            rt, ee = abi.RXN_IONIZATION, float(rng.uniform(8.0, 25.0))
        elif kind in ("exc", "dexc"):
            a, b_ = pick(neutrals), pick(neutrals)
            if a == b_:
                continue
            reac, prod = [E, a], [E, b_]
            rt = abi.RXN_EXCITATION
            ee = float(rng.uniform(1.0, 12.0)) * (1 if kind == "exc" else -1)
        elif kind == "ela":
            n = pick(neutrals)
            reac, prod = [E, n], [E, n]
            rt, el = abi.RXN_ELASTIC, n
        elif kind == "rec2":
            if not ions:
                continue
            i = pick(ions)
            reac, prod, rt = [E, i], [parent[i]], abi.RXN_RECOMB
        elif kind == "rec3":
            if not ions:
                continue
            i = pick(ions)
            reac, prod, rt = [E, i, M], [parent[i], M], abi.RXN_RECOMB
        elif kind == "cx":
            if not ions:
                continue
            i = pick(ions)
            n = pick([x for x in neutrals if x in ion_of and x != parent[i]] or [parent[i]])
            if n == parent[i]:
                continue
            reac, prod = [i, n], [parent[i], ion_of[n]]
        elif kind == "penning":
            a, b_ = pick(neutrals), pick(neutrals)
            tgt = pick([x for x in neutrals if x in ion_of] or [-1])
            if tgt < 0 or tgt in (a, b_):
                continue
            reac, prod = [a, b_], [E, ion_of[tgt], a]
            rt, ee = abi.RXN_IONIZATION, -float(rng.uniform(1.0, 5.0))
        elif kind == "nn":
            a, b_, c, d = pick(neutrals), pick(neutrals), pick(neutrals), pick(neutrals)
            reac, prod = [a, b_], [c, d]
        else:  # assoc3
            a, b_, c = pick(neutrals), pick(neutrals), pick(neutrals)
            reac, prod = [a, b_, M], [c, M]
        if len(set(reac)) + len(set(prod)) > abi.MAX_TERMS:
            continue
        A, b, C = _draw_rate(rng, len(reac))
        lab = " + ".join(names[s] for s in reac) + " => " + " + ".join(names[s] for s in prod)
        rx.append(Reaction(reac, prod, A, b, C, abi.RATE_ARRHENIUS_TE, rt, ee, el, label=lab).fill_terms())
    m_M = 39.948 * M_AMU
    tr = _ar_like_transport(ns, E, {i: (120e-20, mw[i] * M_AMU) for i in ions},
                            ions[0] if ions else None)
    mech = Mechanism(name=f"synth{ns}x{n_reactions}_s{seed}", species=names, charge=charge, mw=mw,
                     e_id=E, reactions=rx, elastic_loss=1, elastic_mass=m_M, bg_species=[M], **tr)
    assert mech.charge_balance_ok()
    return mech
