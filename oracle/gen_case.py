"""Emit a case directory (Chemistry.H, UserFunctions.H, ProbParm.H) for a runtime
mechanism, in the form of the reference's generated case headers
(test/models/Ar_DC_1d/Chemistry.H, UserFunctions.H, ProbParm.H), so that the
reference's own Source/compute_explicit_flux.H and Source/PlasmaChem.H compile
against it unchanged (TEST INFRASTRUCTURE ONLY; output goes to oracle/_ref/gen/).

Every number is printed with repr() so the header and the runtime table hold the
same doubles; expressions keep the operand order of the argon header
(k_f = A*std::pow(Te,b)*std::exp(-C/Te), qf = k_f * (sc[a] * sc[b]), ...).
"""
from __future__ import annotations

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from vidyut_b200 import _abi as abi  # noqa: E402
from vidyut_b200.mechanism import Mechanism  # noqa: E402


def _r(x: float) -> str:
    s = repr(float(x))
    if s in ("inf", "-inf", "nan"):
        raise ValueError("non-finite constant")
    return s


def _mob_expr(m: Mechanism, s: int) -> str:
    k = m.mob_kind[s]
    if k == abi.MOB_ELECTRON:
        return (f"{{ amrex::Real nu = std::sqrt(8.0*K_B*Te/PI/ME)*ndens*{_r(m.mob_p0[s])};"
                f" mob = -ECHARGE/ME/nu; }}")
    if k == abi.MOB_ION_TG:
        M = _r(m.mob_p1[s])
        return (f"{{ amrex::Real nu = std::sqrt(8.0*K_B*T/PI/({M}))*ndens*{_r(m.mob_p0[s])};"
                f" mob = ECHARGE/({M})/nu; }}")
    if k == abi.MOB_SCALED:
        return f"{{ mob = {_r(m.mob_p0[s])}*specMob({m.mob_ref[s]},Te,ndens,emag,T); }}"
    if k == abi.MOB_CONST_N:
        return f"{{ mob = {_r(m.mob_p0[s])}/ndens; }}"
    if k == abi.MOB_CONST:
        return f"{{ mob = {_r(m.mob_p0[s])}; }}"
    if k != abi.MOB_ZERO:  # the |E| forms are pinned on the reference's own headers
        raise ValueError(f"mobility kind {k} is not generated")
    return "{ mob = 0.0; }"


def _diff_expr(m: Mechanism, s: int) -> str:
    k = m.diff_kind[s]
    if k == abi.DIFF_TE_ABSMOB:
        return (f"{{ amrex::Real mb = specMob({m.diff_ref[s]},Te,ndens,emag,T); amrex::Real Te_in_ev = Te/eV;"
                f" dcoeff = {_r(m.diff_factor[s])}*Te_in_ev*amrex::Math::abs(mb); }}")
    if k == abi.DIFF_TG_MOB:
        return (f"{{ amrex::Real mb = specMob({m.diff_ref[s]},Te,ndens,emag,T); amrex::Real Tg_in_ev = T/eV;"
                f" dcoeff = {_r(m.diff_factor[s])}*Tg_in_ev*mb; }}")
    if k == abi.DIFF_CONST:
        return f"{{ dcoeff = {_r(m.diff_factor[s])}; }}"
    if k != abi.DIFF_ZERO:
        raise ValueError(f"diffusion kind {k} is not generated")
    return "{ dcoeff = 0.0; }"


def chemistry_h(m: Mechanism) -> str:
    ns = m.ns
    L = []
    w = L.append
    w("/* generated for a runtime mechanism in the reference's Chemistry.H form (test infrastructure) */")
    w("#ifndef MECHANISM_H\n#define MECHANISM_H\n#include <AMReX_Gpu.H>\n#include <AMReX_REAL.H>")
    w("#include <UnivConstants.H>\n#include <VarDefines.H>\n#include <vector>\n")
    w(f"#define E_ID {m.e_id}")
    w(f"#define NUM_SPECIES {ns}\n#define NUM_REACTIONS {len(m.reactions)}\n")
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void get_mw(amrex::Real *mw_new) {")
    for s in range(ns):
        w(f"  mw_new[{s}] = {_r(m.mw[s])};")
    w("}")
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE amrex::Real mw(const int n) {")
    w(f"  const amrex::Real t[{ns}] = {{{', '.join(_r(x) for x in m.mw)}}};\n  return t[n];\n}}")
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKCHRG(int kcharge[]) {")
    for s in range(ns):
        w(f"  kcharge[{s}] = {int(m.charge[s])};")
    w("}")
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE amrex::Real\n"
      "specMob(const int specid, const amrex::Real Te, const amrex::Real ndens, const amrex::Real emag, const amrex::Real T)\n{")
    w("  amrex::Real mob = 0.0;")
    for s in range(ns + 1):
        w(f"  if (specid == {s}) {_mob_expr(m, s)}")
    w("  return mob;\n}")
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE amrex::Real\n"
      "specDiff(const int specid, const amrex::Real Te, const amrex::Real ndens, const amrex::Real emag, const amrex::Real T)\n{")
    w("  amrex::Real dcoeff = 0.0;")
    for s in range(ns + 1):
        w(f"  if (specid == {s}) {_diff_expr(m, s)}")
    w("  return dcoeff;\n}")
    # comp_ener_exch: the argon header's body
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void comp_ener_exch(amrex::Real qf, amrex::Real qr, "
      "const amrex::Real * sc, amrex::Real kf, int rxntype, amrex::Real eexci, int elidx, "
      "amrex::Real * enerExch, amrex::Real Ue, amrex::Real T, const amrex::Real Te)\n{")
    w("  amrex::Real eV2J = 1.602176620800000e-19;\n  amrex::Real NA = 6.02214085774e23;\n"
      "  amrex::Real kB = 1.380649e-23;\n  amrex::Real ne = sc[E_ID] * NA;\n  amrex::Real mee = Ue / ne;")
    w(f"  amrex::Real wt[NUM_SPECIES];\n  get_mw(wt);")
    w("  amrex::Real sefact = (tanh((Te - T) / 0.5) + 1.0) / 2.0 ;")
    w("  if(rxntype == 1 || rxntype == 2){ *enerExch -= (eexci*eV2J)*NA*(qf - qr) * sefact; }")
    w("  if(rxntype == 3){ *enerExch -= mee*NA*(qf - qr); }")
    w("  if(rxntype == 4){ *enerExch -= mee*NA*(qf - qr); }")
    w("  if(rxntype == 7){ *enerExch += mee*NA*(qf - qr); }")
    w("  if(rxntype == 5){ amrex::Real qq = sc[E_ID] * sc[elidx] * kf;"
      " *enerExch -= 3.0 * kB * (wt[E_ID] / wt[elidx]) * (Te - T) * qq * NA; }")
    w("}")
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void\n"
      "productionRate(amrex::Real* wdot, const amrex::Real* sc, const amrex::Real T, const amrex::Real Te, "
      "amrex::Real * enerExch)\n{")
    w(f"  for (int i = 0; i < {ns}; ++i) wdot[i] = 0.0;")
    w("  amrex::Real ne = sc[E_ID] * 6.02214085774e23;\n  amrex::Real Ue = 1.5 * Te * ne * 1.380649e-23;")
    if any(r.kind >= abi.RATE_JANEV for r in m.reactions):
        # the fit-rate preamble of the CO2 reactor header
        # (test/Reactor/CO2_H2_Ar_mechanism_reduced/Chemistry.H:943-955)
        w("  double Janev_sum;\n  double TeeV = Te / 11595.0;\n  double logTe = log(TeeV);")
        w("  double invTeeV = (Te == 0) ? 1.0:1.0 / (TeeV);")
        w("  double Te_pow[] = {" + ", ".join(f"pow(logTe, {j})" for j in range(9)) + "};")
        w("  double invTe_pow[] = {" + ", ".join(f"pow(invTeeV, {j})" for j in range(1, 5)) + "};")
        w("  std::vector<double> Jfit_coefs = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};")
        w("  std::vector<double> Ffit_coefs = {0.0, 0.0, 0.0, 0.0};")

    def fit_block(f, janev, ind):
        if janev:
            w(f"{ind}Jfit_coefs = {{{', '.join(_r(c) for c in f['jc'])}}};")
            w(f"{ind}double Jfit_A = {_r(f['jA'])};")
            w(f"{ind}for(int j = 0; j<9; j++) Janev_sum += Jfit_coefs[j] * Te_pow[j];")
            w(f"{ind}k_f = Jfit_A * exp(Janev_sum) * 6.02214085774e23;")
        else:
            w(f"{ind}Ffit_coefs = {{{', '.join(_r(c) for c in f['fc'])}}};")
            w(f"{ind}double Ffit_A = {_r(f['fA'])};")
            w(f"{ind}for(int j = 0; j<4; j++) Janev_sum += Ffit_coefs[j] * invTe_pow[j];")
            w(f"{ind}k_f = Ffit_A * exp(Janev_sum) * 6.02214085774e23;")

    for i, r in enumerate(m.reactions):
        r.fill_terms()
        w(f"  {{\n    // reaction {i}: {r.label}")
        if r.kind == abi.RATE_TOWNSEND:
            raise ValueError("the field-driven rate is pinned on the Streamer header, not generated")
        if r.kind >= abi.RATE_JANEV:
            w("    Janev_sum = 0.0;\n    amrex::Real k_f;")
            if r.kind == abi.RATE_JANEV_FFIT:
                w(f"    if(TeeV < {_r(r.fit['switch_ev'])}){{")
                fit_block(r.fit, True, "        ")
                w("    } else {")
                fit_block(r.fit, False, "        ")
                w("    }")
            else:
                fit_block(r.fit, r.kind == abi.RATE_JANEV, "    ")
        elif r.kind == abi.RATE_ARRHENIUS_TE:
            w(f"    const amrex::Real k_f = {_r(r.A)}*std::pow(Te,{_r(r.b)})*std::exp(-{_r(r.C)}/Te);")
        elif r.kind == abi.RATE_ARRHENIUS_TG:
            w(f"    const amrex::Real k_f = {_r(r.A)}*std::pow(T,{_r(r.b)})*std::exp(-{_r(r.C)}/T);")
        else:
            w(f"    const amrex::Real k_f = {_r(r.A)};")
        prod = " * ".join(f"sc[{s}]" for s in r.reactants)
        w(f"    const amrex::Real qf = k_f * ({prod});")
        w("    const amrex::Real qr = 0.0;\n    const amrex::Real qdot = qf - qr;")
        for s, c in r.terms:
            w(f"    wdot[{s}] += ({_r(c)}) * qdot;")
        if r.rxntype != abi.RXN_NONE:
            w(f"    comp_ener_exch(qf, qr, sc, k_f, {r.rxntype}, {_r(r.eexci)}, {r.elidx}, enerExch, Ue, T, Te);")
        w("  }")
    if m.elastic_loss:
        w("  amrex::Real emag = 0.0;\n  amrex::Real ndens = 0.0;")
        w("  for(int sp=0; sp<NUM_SPECIES; sp++) ndens += sc[sp]*N_A;")
        w("  amrex::Real mu = specMob(E_ID,Te,ndens,emag,T);\n  amrex::Real nu = -ECHARGE/ME/mu;")
        w(f"  amrex::Real elec_elastic_coll_term= 3.0/2.0 * K_B * sc[E_ID] * N_A * (Te-T) * nu * "
          f"(2.0*ME/({_r(m.elastic_mass)}));")
        w("  *enerExch -= elec_elastic_coll_term;")
    w("}")
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void\n"
      "CKWC(const amrex::Real T, amrex::Real C[], amrex::Real wdot[], const amrex::Real Te, "
      "const amrex::Real EN, amrex::Real * ener_exch)\n{")
    w(f"  for (int id = 0; id < {ns}; ++id) C[id] *= 1.0e6;")
    w("  productionRate(wdot, C, T, Te, ener_exch);")
    w(f"  for (int id = 0; id < {ns}; ++id) {{ C[id] *= 1.0e-6; wdot[id] *= 1.0e-6; }}")
    w("}\n#endif")
    return "\n".join(L) + "\n"


USERFUNCTIONS_H = """/* generated (test infrastructure): user_transport as in the reference cases */
#ifndef _TRANSPORT_H_
#define _TRANSPORT_H_
#include <Chemistry.H>
using namespace amrex;
namespace user_transport
{
    AMREX_GPU_DEVICE AMREX_INLINE
    amrex::Real compute_vel(IntVect cellid, int dir, int specid, Array4<Real> const& phi,
                            GpuArray<Real, AMREX_SPACEDIM> dx, const Real time,
                            ProbParm const& prob_parm, amrex::Real Tg, amrex::Real Pg)
    {
        amrex::Real vel[3] = {prob_parm.velx, prob_parm.vely, prob_parm.velz};
        return (specid == prob_parm.vel_species) ? vel[dir] : 0.0;
    }
}
#endif
"""

PROBPARM_H = """/* generated (test infrastructure) */
#ifndef CNS_PROB_PARM_H_
#define CNS_PROB_PARM_H_
#include <AMReX_REAL.H>
#include <UnivConstants.H>
struct ProbParm
{
    amrex::Real velx = 0.0;
    amrex::Real vely = 0.0;
    amrex::Real velz = 0.0;
    int vel_species = 0;
};
#define VD_PROBPARM_HAS_VEL 1
#define VD_PROBPARM_HAS_VEL_SPECIES 1
#endif
"""


def write_case(m: Mechanism, outdir: Path) -> Path:
    outdir.mkdir(parents=True, exist_ok=True)
    files = {"Chemistry.H": chemistry_h(m), "UserFunctions.H": USERFUNCTIONS_H, "ProbParm.H": PROBPARM_H}
    for name, text in files.items():
        p = outdir / name
        if not p.exists() or p.read_text() != text:
            p.write_text(text)
    return outdir
