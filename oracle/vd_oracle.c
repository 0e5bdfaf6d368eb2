/*
 * vd_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * A plain-C restatement of the reference's explicit species / electron-energy update,
 * driven by the same runtime mechanism table (vd_mech) as the CUDA library.  Only the
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the
 * product path never does.  Arithmetic follows the reference expression by
 * expression (same operand order, no contraction: build with -ffp-contract=off) so
 * that it reproduces the reference build bit for bit; it is pinned against the
 * reference's own headers compiled unmodified (oracle/refdriver) in tests/.
 *
 * Reference files (paths within hsitaram/vidyut3d):
 *   Source/compute_explicit_flux.H   gk, weno, weno_reconstruct, MINBEE, WAF, upwind, compute_flux
 *   Source/PlasmaChem.H:187-206      plasmachem_transport::compute_vel
 *   Source/ScalarSolve.cpp:17-55     compute_dsdt
 *   Source/ScalarSolve.cpp:143-165   rxnsrc lambda (CKWC driver)
 *   Source/ElecEnergySource.cpp:65-171  Joule heating lambda
 *   Source/Evolve.cpp:278-284        background-species update
 *   Source/ScalarSolve.cpp:659-666   electron temperature update and floor
 *   test/models/Ar_DC_1d/Chemistry.H:177-506  specMob, specDiff, comp_ener_exch,
 *                                    productionRate, CKWC (the generated-header form)
 */
#include <math.h>
#include <string.h>
#include <stdlib.h>
#include "../include/vidyut_b200.h"

/* Source/UnivConstants.H:4-18 (physical constants; values must be identical) */
#define N_A 6.02214076e23
#define K_B 1.380649e-23
#define PI 3.14159265358979323846264338327950288
#define ECHARGE 1.60217662e-19
#define eV (ECHARGE / K_B)
#define ME 9.10938188e-31
#define P_NTP 101325.0
#define fivebythree (5.0 / 3.0)
#define twothird (2.0 / 3.0)

/* ------------------------------------------------------------------------- */
static inline double *A4P(const vd_array4 *a, int i, int j, int k, int n)
{
    return a->p + ((int64_t)(i - a->begin[0]) + (int64_t)(j - a->begin[1]) * a->jstride +
                   (int64_t)(k - a->begin[2]) * a->kstride + (int64_t)n * a->nstride);
}
#define A4(a, i, j, k, n) (*A4P((a), (i), (j), (k), (n)))

/* ------------------------------------------------------------------------- */
/* specMob (test/models/Ar_DC_1d/Chemistry.H:177-202), table-driven; the power
 * law in |E| of test/verification/Streamer/Chemistry.H:165-183.                 */
double orc_specmob(const vd_mech *m, int specid, double Te, double ndens, double emag, double T)
{
    int kind = m->mob_kind[specid];
    double mob = 0.0;
    if (kind == VD_MOB_ELECTRON) {
        double cs = m->mob_p0[specid];
        double nu_elec = sqrt(8.0 * K_B * Te / PI / ME) * ndens * cs;
        mob = -ECHARGE / ME / nu_elec;
    } else if (kind == VD_MOB_ION_TG) {
        double cs = m->mob_p0[specid];
        double M = m->mob_p1[specid];
        double nu_i = sqrt(8.0 * K_B * T / PI / (M)) * ndens * cs;
        mob = ECHARGE / (M) / nu_i;
    } else if (kind == VD_MOB_SCALED) {
        mob = m->mob_p0[specid] * orc_specmob(m, m->mob_ref[specid], Te, ndens, emag, T);
    } else if (kind == VD_MOB_CONST_N) {
        mob = m->mob_p0[specid] / ndens;
    } else if (kind == VD_MOB_CONST) {
        mob = m->mob_p0[specid];
    } else if (kind == VD_MOB_POW_EMAG) {
        mob = m->mob_p0[specid] * pow(emag, m->mob_p1[specid]);
    } else if (kind == VD_MOB_EN_POLY) {
        /* test/verification/He_RF_1d/Chemistry.H:231-238 (the ions) */
        const double *c = m->fits[m->mob_ref[specid]].jc;
        double EbyN = emag / ndens;
        mob = m->mob_p0[specid] * pow((1.0 + c[0] * pow(EbyN, 2.0) + c[1] * pow(EbyN, 4.0)), m->mob_p1[specid]);
    } else if (kind == VD_MOB_EXP_MEANE) {
        /* test/verification/He_RF_1d/Chemistry.H:232,242-243 (the electrons) */
        const double *c = m->fits[m->mob_ref[specid]].jc;
        double meanE = 1.5 * Te / eV;
        mob = m->mob_p0[specid] * exp(c[0] + c[1] * log(meanE) + c[2] / meanE + c[3] / pow(meanE, 2.0) +
                                      c[4] / pow(meanE, 3.0)) / ndens;
    }
    return mob;
}

/* specDiff (test/models/Ar_DC_1d/Chemistry.H:204-239), table-driven.          */
double orc_specdiff(const vd_mech *m, int specid, double Te, double ndens, double emag, double T)
{
    int kind = m->diff_kind[specid];
    double dcoeff = 0.0;
    if (kind == VD_DIFF_TE_ABSMOB) {
        double mob = orc_specmob(m, m->diff_ref[specid], Te, ndens, emag, T);
        double Te_in_ev = Te / eV;
        dcoeff = m->diff_factor[specid] * Te_in_ev * fabs(mob);
    } else if (kind == VD_DIFF_TG_MOB) {
        double mob = orc_specmob(m, m->diff_ref[specid], Te, ndens, emag, T);
        double Tg_in_ev = T / eV;
        dcoeff = m->diff_factor[specid] * Tg_in_ev * mob;
    } else if (kind == VD_DIFF_CONST) {
        /* a constant coefficient (test/models/ionelec_DC_1d/Chemistry.H:190-209) */
        dcoeff = m->diff_factor[specid];
    } else if (kind == VD_DIFF_POW_EMAG) {
        /* test/verification/Streamer/Chemistry.H:185-204 */
        dcoeff = m->diff_factor[specid] * pow(emag, m->diff_p1[specid]);
    } else if (kind == VD_DIFF_PRES || kind == VD_DIFF_TE_PRES) {
        /* test/verification/He_RF_1d/Chemistry.H:270-296 */
        double Pg = ndens * K_B * T;
        double Pres_ratio = (P_NTP / Pg);
        if (kind == VD_DIFF_PRES)
            dcoeff = m->diff_factor[specid] * Pres_ratio;
        else
            dcoeff = m->diff_factor[specid] * (Te / m->diff_p1[specid]) * Pres_ratio;
    } else if (kind == VD_DIFF_SCALED) {
        /* the energy's 5/3 of the electrons' coefficient (Streamer/Chemistry.H:199-202) */
        dcoeff = m->diff_factor[specid] * orc_specdiff(m, m->diff_ref[specid], Te, ndens, emag, T);
    }
    return dcoeff;
}

/* comp_ener_exch (test/models/Ar_DC_1d/Chemistry.H:315-359).                   */
static void orc_comp_ener_exch(const vd_mech *m, double qf, double qr, const double *sc, double kf,
                               int rxntype, double eexci, int elidx, double *enerExch, double Ue,
                               double T, double Te)
{
    double eV2J = 1.602176620800000e-19;
    double NA = 6.02214085774e23;
    double kB = 1.380649e-23;
    double ne = sc[m->e_id] * NA;
    double mee = Ue / ne;
    double sefact = (tanh((Te - T) / 0.5) + 1.0) / 2.0;
    if (rxntype == 1 || rxntype == 2) {
        *enerExch -= (eexci * eV2J) * NA * (qf - qr) * sefact;
    }
    if (rxntype == 3) {
        *enerExch -= mee * NA * (qf - qr);
    }
    /* attachment and detachment, as the CO2 reactor header's comp_ener_exch
     * (test/Reactor/CO2_H2_Ar_mechanism_reduced/Chemistry.H:872-881)        */
    if (rxntype == 4) {
        *enerExch -= mee * NA * (qf - qr);
    }
    if (rxntype == 7) {
        *enerExch += mee * NA * (qf - qr);
    }
    if (rxntype == 5) {
        double qq = sc[m->e_id] * sc[elidx] * kf;
        *enerExch -= 3.0 * kB * (m->mw[m->e_id] / m->mw[elidx]) * (Te - T) * qq * NA;
    }
}

/* Janev / F-fit electron-impact rates as the CO2 reactor header evaluates them
 * (test/Reactor/CO2_H2_Ar_mechanism_reduced/Chemistry.H:945-964,1013-1030):
 * Te_eV = Te/11595, the powers of ln(Te_eV) and 1/Te_eV by pow(), the sum
 * accumulated in order, k = A exp(sum) * 6.02214085774e23.                    */
static double orc_fit_rate(const vd_mech *m, const vd_reaction *r, double Te)
{
    const vd_rate_fit *F = &m->fits[r->fit];
    double TeeV = Te / 11595.0;
    double logTe = log(TeeV);
    double invTeeV = (Te == 0) ? 1.0 : 1.0 / (TeeV);
    double Te_pow[9], invTe_pow[4];
    for (int j = 0; j < 9; j++) Te_pow[j] = pow(logTe, j);
    for (int j = 0; j < 4; j++) invTe_pow[j] = pow(invTeeV, j + 1);
    double Janev_sum = 0.0;
    int janev = r->kind == VD_RATE_JANEV || (r->kind == VD_RATE_JANEV_FFIT && TeeV < F->switch_ev);
    if (janev) {
        for (int j = 0; j < 9; j++) Janev_sum += F->jc[j] * Te_pow[j];
        return F->jA * exp(Janev_sum) * 6.02214085774e23;
    }
    for (int j = 0; j < 4; j++) Janev_sum += F->fc[j] * invTe_pow[j];
    return F->fA * exp(Janev_sum) * 6.02214085774e23;
}

/* Field-driven ionisation (test/verification/Streamer/Chemistry.H:266-280) at the
 * field magnitude efm, coefficients c = fits[fit].jc in the header's order.   */
static double orc_townsend_rate(const double *c, double efm)
{
    double alpha = (c[0] + c[1] / pow(efm, 3.0)) * exp(-c[2] / efm);
    double eta = c[3];
    double alpha_bar = alpha - eta;
    double mu_e = c[4] * pow(efm, c[5]);
    return alpha_bar * mu_e * efm;
}

/* k_f of one reaction (productionRate, e.g. Ar_DC_1d/Chemistry.H:392); efm is
 * the field magnitude EN * N * 1e-21 of the field-driven kinds. */
static double orc_rate(const vd_mech *m, const vd_reaction *r, double T, double Te, double efm)
{
    if (r->kind == VD_RATE_TOWNSEND) return orc_townsend_rate(m->fits[r->fit].jc, efm);
    if (r->kind == VD_RATE_ARRHENIUS_TE) return r->A * pow(Te, r->b) * exp(-r->C / Te);
    if (r->kind == VD_RATE_ARRHENIUS_TG) return r->A * pow(T, r->b) * exp(-r->C / T);
    if (r->kind >= VD_RATE_JANEV) return orc_fit_rate(m, r, Te);
    return r->A;
}

/* productionRate (test/models/Ar_DC_1d/Chemistry.H:361-487).  The gibbs() evaluation
 * of the generated header has no effect on irreversible reactions and is omitted. */
void orc_production_rate(const vd_mech *m, double *wdot, const double *sc, double T, double Te,
                         double EN, double *enerExch)
{
    int ns = m->nspecies;
    for (int i = 0; i < ns; ++i) wdot[i] = 0.0;
    /* E/N [Td] to |E| (test/verification/Streamer/Chemistry.H:256-264) */
    double mixture = 0.0;
    for (int i = 0; i < ns; ++i) mixture += sc[i];
    double efm = EN * (mixture * 6.02214076e23) * 1e-21;
    double ne = sc[m->e_id] * 6.02214085774e23;
    double Ue = 1.5 * Te * ne * 1.380649e-23;
    for (int ir = 0; ir < m->nreactions; ++ir) {
        const vd_reaction *r = &m->rxn[ir];
        double k_f = orc_rate(m, r, T, Te, efm);
        double prod = sc[r->reac[0]];
        for (int t = 1; t < r->nreac; ++t) prod = prod * sc[r->reac[t]];
        double qf = k_f * prod;
        double qr = 0.0;
        double qdot = qf - qr;
        for (int t = 0; t < r->nterms; ++t) wdot[r->term_sp[t]] += r->term_coef[t] * qdot;
        if (r->rxntype != VD_RXN_NONE)
            orc_comp_ener_exch(m, qf, qr, sc, k_f, r->rxntype, r->eexci, r->elidx, enerExch, Ue, T,
                               Te);
    }
    if (m->elastic_loss) {
        /* Ar_DC_1d/Chemistry.H:479-486; |E| = EN N 1e-21 as the He_RF_1d header
         * passes it (its mobility reads it; the argon ones pass 0 and do not) */
        double ndens = 0.0;
        for (int sp = 0; sp < ns; sp++) ndens += sc[sp] * N_A;
        double emag = EN * ndens * 1.0e-21;
        double mu = orc_specmob(m, m->e_id, Te, ndens, emag, T);
        double nu = -ECHARGE / ME / mu;
        double term = 3.0 / 2.0 * K_B * sc[m->e_id] * N_A * (Te - T) * nu *
                      (2.0 * ME / m->elastic_mass);
        *enerExch -= term;
    }
}

/* CKWC (test/models/Ar_DC_1d/Chemistry.H:490-506). */
void orc_ckwc(const vd_mech *m, double T, double *C, double *wdot, double Te, double EN,
              double *ener_exch)
{
    int ns = m->nspecies;
    for (int id = 0; id < ns; ++id) C[id] *= 1.0e6;
    orc_production_rate(m, wdot, C, T, Te, EN, ener_exch);
    for (int id = 0; id < ns; ++id) {
        C[id] *= 1.0e-6;
        wdot[id] *= 1.0e-6;
    }
}

/* rxnsrc lambda (Source/ScalarSolve.cpp:143-165) over one box. */
int orc_reaction_source(const vd_mech *m, const vd_box *bx, const vd_array4 *sb, const vd_array4 *rxn,
                        double Tg)
{
    int ns = m->nspecies;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
        for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
            for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                double spec_C[VD_MAX_SPECIES];
                double spec_wdot[VD_MAX_SPECIES];
                double Te = A4(sb, i, j, k, VD_ETEMP(ns));
                double EN = A4(sb, i, j, k, VD_REF(ns));
                double ener_exch = 0.0;
                for (int sp = 0; sp < ns; sp++) spec_C[sp] = A4(sb, i, j, k, sp) * 1.0e-6 / N_A;
                orc_ckwc(m, Tg, spec_C, spec_wdot, Te, EN, &ener_exch);
                for (int sp = 0; sp < ns; sp++) A4(rxn, i, j, k, sp) = spec_wdot[sp] * N_A * 1.0e6;
                A4(rxn, i, j, k, ns) = ener_exch;
            }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* gk, weno (Source/compute_explicit_flux.H:16-112).                           */
static double orc_gk(double wk, double gama_k)
{
    return wk * (gama_k + gama_k * gama_k - 3.0 * gama_k * wk + wk * wk) /
           (gama_k * gama_k + wk * (1 - 2.0 * gama_k));
}

static double sq(double x) { return x * x; } /* std::pow(x, 2.0) is exactly x*x */

double orc_weno(double phi_im2, double phi_im1, double phi_i, double phi_ip1, double phi_ip2,
                int scheme)
{
    double eps = 1e-20;
    double phi_iphalf_1 = (1.0 / 3.0) * phi_im2 - (7.0 / 6.0) * phi_im1 + (11.0 / 6.0) * phi_i;
    double phi_iphalf_2 = -(1.0 / 6.0) * phi_im1 + (5.0 / 6.0) * phi_i + (1.0 / 3.0) * phi_ip1;
    double phi_iphalf_3 = (1.0 / 3.0) * phi_i + (5.0 / 6.0) * phi_ip1 - (1.0 / 6.0) * phi_ip2;

    double beta_1 = (13.0 / 12.0) * sq((phi_im2 - 2.0 * phi_im1 + phi_i)) +
                    (1.0 / 4.0) * sq((phi_im2 - 4.0 * phi_im1 + 3.0 * phi_i));
    double beta_2 = (13.0 / 12.0) * sq((phi_im1 - 2.0 * phi_i + phi_ip1)) +
                    (1.0 / 4.0) * sq((phi_im1 - phi_ip1));
    double beta_3 = (13.0 / 12.0) * sq((phi_i - 2.0 * phi_ip1 + phi_ip2)) +
                    (1.0 / 4.0) * sq((3.0 * phi_i - 4.0 * phi_ip1 + phi_ip2));

    double gama_1 = (1.0 / 10.0), gama_2 = (6.0 / 10.0), gama_3 = (3.0 / 10.0);
    double w1, w2, w3, alpha_1, alpha_2, alpha_3;
    if (scheme == 1) {
        alpha_1 = gama_1 / sq((beta_1 + eps));
        alpha_2 = gama_2 / sq((beta_2 + eps));
        alpha_3 = gama_3 / sq((beta_3 + eps));
    } else if (scheme == 2) {
        alpha_1 = gama_1 / sq((beta_1 + eps));
        alpha_2 = gama_2 / sq((beta_2 + eps));
        alpha_3 = gama_3 / sq((beta_3 + eps));
        double sum_alpha = (alpha_1 + alpha_2 + alpha_3);
        w1 = alpha_1 / sum_alpha;
        w2 = alpha_2 / sum_alpha;
        w3 = alpha_3 / sum_alpha;
        alpha_1 = orc_gk(w1, gama_1);
        alpha_2 = orc_gk(w2, gama_2);
        alpha_3 = orc_gk(w3, gama_3);
    } else {
        double tau = fabs(beta_1 - beta_3);
        alpha_1 = gama_1 * (1.0 + sq(tau / (beta_1 + eps)));
        alpha_2 = gama_2 * (1.0 + sq(tau / (beta_2 + eps)));
        alpha_3 = gama_3 * (1.0 + sq(tau / (beta_3 + eps)));
    }
    double sum_alpha = (alpha_1 + alpha_2 + alpha_3);
    w1 = alpha_1 / sum_alpha;
    w2 = alpha_2 / sum_alpha;
    w3 = alpha_3 / sum_alpha;
    return w1 * phi_iphalf_1 + w2 * phi_iphalf_2 + w3 * phi_iphalf_3;
}

/* MINBEE limiter, WAF and upwind fluxes (Source/compute_explicit_flux.H:130-198). */
#define heps 1.0e-30
static double orc_slope_lim(double c, double dl, double dm, double dr)
{
    double r = (c >= 0.0) ? dl / (dm + heps) : dr / (dm + heps);
    double lim;
    if (r <= 0.0) lim = 1.0;
    else if (r > 0.0 && r <= 1.0) lim = 1.0 - (1.0 - fabs(c)) * r;
    else lim = fabs(c);
    return lim;
}
static double orc_waf(double vL, double vR, double pLm1, double pL, double pR, double pRp1, double dx,
                      double dt)
{
    double dl = pL - pLm1, dm = pR - pL, dr = pRp1 - pR;
    double vmid = 0.5 * (vL + vR);
    double vsgn = copysign(1.0, vmid);
    double c = vmid * dt / dx;
    double fL = pL * vL, fR = pR * vR;
    double lim = orc_slope_lim(c, dl, dm, dr);
    return 0.5 * (fL + fR) - 0.5 * vsgn * lim * (fR - fL);
}
static double orc_upwind(double vL, double vR, double pL, double pR)
{
    double fL = pL * vL, fR = pR * vR;
    double vmid = 0.5 * (vL + vR);
    double vsgn = copysign(1.0, vmid);
    return fL * 0.5 * (1.0 + vsgn) + fR * 0.5 * (1.0 - vsgn);
}

/* plasmachem_transport::compute_vel (Source/PlasmaChem.H:187-206) or the constant
 * user velocity of test/verification/Advect/UserFunctions.H:50-66.              */
static double orc_vel(const vd_mech *m, const vd_array4 *phi, int c[3], int dir, int specid,
                      double Tg, int udv, const double *uvel, int vel_species)
{
    int ns = m->nspecies;
    if (udv) return (specid == vel_species) ? uvel[dir] : 0.0;
    double ex = A4(phi, c[0], c[1], c[2], VD_EFX(ns));
    double ey = A4(phi, c[0], c[1], c[2], VD_EFY(ns));
    double ez = A4(phi, c[0], c[1], c[2], VD_EFZ(ns));
    double efieldmag = sqrt(sq(ex) + sq(ey) + sq(ez));
    double ndens = 0.0;
    for (int sp = 0; sp < ns; sp++) ndens += A4(phi, c[0], c[1], c[2], sp);
    double mu = orc_specmob(m, specid, A4(phi, c[0], c[1], c[2], VD_ETEMP(ns)), ndens, efieldmag, Tg);
    return mu * A4(phi, c[0], c[1], c[2], VD_EFX(ns) + dir);
}

/* compute_flux at one face (Source/compute_explicit_flux.H:200-326). */
static double orc_face_flux(const vd_mech *m, int i, int j, int k, int sweepdir, int specid,
                            const vd_array4 *phi, const int32_t *bclo, const int32_t *bchi,
                            const int32_t *domlo, const int32_t *domhi, double Tg, const double *dx,
                            double dt, int hyp_order, int udv, int weno_scheme, const double *uvel,
                            int vel_species, int dim)
{
    int face[3] = {i, j, k}, left[3] = {i, j, k}, right[3] = {i, j, k};
    left[sweepdir] -= 1;
    double phi_L = A4(phi, left[0], left[1], left[2], specid);
    double phi_R = A4(phi, right[0], right[1], right[2], specid);
    double vel_L = orc_vel(m, phi, left, sweepdir, specid, Tg, udv, uvel, vel_species);
    double vel_R = orc_vel(m, phi, right, sweepdir, specid, Tg, udv, uvel, vel_species);
    double fx;
    if (hyp_order == 1) {
        fx = orc_upwind(vel_L, vel_R, phi_L, phi_R);
    } else if (hyp_order == 2) {
        int l1[3] = {i, j, k}, r1[3] = {i, j, k};
        l1[sweepdir] -= 2;
        r1[sweepdir] += 1;
        double pLm1 = A4(phi, l1[0], l1[1], l1[2], specid);
        double pRp1 = A4(phi, r1[0], r1[1], r1[2], specid);
        double dxmin = dx[0];
        for (int d = 1; d < dim; d++) dxmin = (dx[d] < dxmin) ? dx[d] : dxmin;
        fx = orc_waf(vel_L, vel_R, pLm1, phi_L, phi_R, pRp1, dxmin, dt);
    } else {
        int l1[3] = {i, j, k}, r1[3] = {i, j, k}, l2[3] = {i, j, k}, r2[3] = {i, j, k};
        l1[sweepdir] -= 2;
        r1[sweepdir] += 1;
        l2[sweepdir] -= 3;
        r2[sweepdir] += 2;
        double vel_Lm1 = orc_vel(m, phi, l1, sweepdir, specid, Tg, udv, uvel, vel_species);
        double vel_Lm2 = orc_vel(m, phi, l2, sweepdir, specid, Tg, udv, uvel, vel_species);
        double vel_Rp1 = orc_vel(m, phi, r1, sweepdir, specid, Tg, udv, uvel, vel_species);
        double vel_Rp2 = orc_vel(m, phi, r2, sweepdir, specid, Tg, udv, uvel, vel_species);
        double ulm2 = A4(phi, l2[0], l2[1], l2[2], specid);
        double ulm1 = A4(phi, l1[0], l1[1], l1[2], specid);
        double ul = phi_L, ur = phi_R;
        double urp1 = A4(phi, r1[0], r1[1], r1[2], specid);
        double urp2 = A4(phi, r2[0], r2[1], r2[2], specid);
        double flm2 = ulm2 * vel_Lm2, flm1 = ulm1 * vel_Lm1, fl = ul * vel_L, fr = ur * vel_R;
        double frp1 = urp1 * vel_Rp1, frp2 = urp2 * vel_Rp2;
        double lambda_max = fabs(0.5 * (vel_L + vel_R));
        double fphalf = orc_weno(flm2, flm1, fl, fr, frp1, weno_scheme);
        double fmhalf = orc_weno(frp2, frp1, fr, fl, flm1, weno_scheme);
        double uphalf = orc_weno(ulm2, ulm1, ul, ur, urp1, weno_scheme);
        double umhalf = orc_weno(urp2, urp1, ur, ul, ulm1, weno_scheme);
        fx = 0.5 * (fphalf + lambda_max * uphalf) + 0.5 * (fmhalf - lambda_max * umhalf);
    }
    if ((face[sweepdir] == domlo[sweepdir]) && (bclo[sweepdir] == VD_BC_IHNEU)) fx = 0.0;
    if ((face[sweepdir] == (domhi[sweepdir] + 1)) && (bchi[sweepdir] == VD_BC_IHNEU)) fx = 0.0;
    return fx;
}

/* Magnitude of the values one face flux is built from (test error scale): for
 * WENO, 10/3 (the largest sum of |candidate-polynomial coefficients|) times
 * max|f| + lambda*max|u| over the six stencil cells; for the first/second-order
 * fluxes |f_L| + |f_R| (+ the WAF limiter's |f_R - f_L|).                      */
static double orc_face_scale(const vd_mech *m, int i, int j, int k, int sweepdir, int specid,
                             const vd_array4 *phi, double Tg, int hyp_order, int udv, const double *uvel,
                             int vel_species)
{
    int H = (hyp_order == 5) ? 3 : hyp_order;
    double fmax = 0.0, umax = 0.0, vL = 0.0, vR = 0.0, fL = 0.0, fR = 0.0;
    for (int q = -H; q < H; q++) {
        int c[3] = {i, j, k};
        c[sweepdir] += q;
        double u = A4(phi, c[0], c[1], c[2], specid);
        double v = orc_vel(m, phi, c, sweepdir, specid, Tg, udv, uvel, vel_species);
        if (fabs(u * v) > fmax) fmax = fabs(u * v);
        if (fabs(u) > umax) umax = fabs(u);
        if (q == -1) { vL = v; fL = u * v; }
        if (q == 0) { vR = v; fR = u * v; }
    }
    if (hyp_order == 5) return (10.0 / 3.0) * (fmax + fabs(0.5 * (vL + vR)) * umax);
    return 2.0 * (fabs(fL) + fabs(fR));
}

/* The ParallelFor over convert(bx, dir) (Source/ScalarSolve.cpp:208-250). */
int orc_compute_explicit_flux(const vd_mech *m, const vd_box *bx, int dir, int specid,
                              const vd_array4 *phi, const int32_t *bclo, const int32_t *bchi,
                              const int32_t *domlo, const int32_t *domhi, const vd_array4 *fx,
                              double Tg, const double *dx, double dt, int hyp_order, int udv,
                              int weno_scheme, const double *uvel, int vel_species)
{
    int hi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
    hi[dir] += 1;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = bx->lo[2]; k <= hi[2]; ++k)
        for (int j = bx->lo[1]; j <= hi[1]; ++j)
            for (int i = bx->lo[0]; i <= hi[0]; ++i)
                A4(fx, i, j, k, 0) =
                    orc_face_flux(m, i, j, k, dir, specid, phi, bclo, bchi, domlo, domhi, Tg, dx, dt,
                                  hyp_order, udv, weno_scheme, uvel, vel_species, bx->dim);
    return 0;
}

/* compute_dsdt (Source/ScalarSolve.cpp:44-53). dsdt is a 1-component view. */
int orc_compute_dsdt(const vd_box *bx, int specid, const vd_array4 *flux, const vd_array4 *rxn,
                     const vd_array4 *dsdt, const double *dx)
{
    int dim = bx->dim;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
        for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
            for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                double *d = A4P(dsdt, i, j, k, 0);
                *d = (A4(&flux[0], i, j, k, 0) - A4(&flux[0], i + 1, j, k, 0)) / dx[0] +
                     A4(rxn, i, j, k, specid);
                if (dim > 1) *d += (A4(&flux[1], i, j, k, 0) - A4(&flux[1], i, j + 1, k, 0)) / dx[1];
                if (dim == 3) *d += (A4(&flux[2], i, j, k, 0) - A4(&flux[2], i, j, k + 1, 0)) / dx[2];
            }
    return 0;
}

/* Joule heating lambda (Source/ElecEnergySource.cpp:65-171).  dsdt: 1 component. */
int orc_elecenergy_source(const vd_mech *m, const vd_box *bx, const vd_array4 *sb,
                          const vd_array4 *rxn, const vd_array4 *ef, const vd_array4 *gne,
                          const vd_array4 *dsdt, const vd_array4 *phi_new, const vd_params *p)
{
    int ns = m->nspecies, dim = bx->dim, eidx = m->e_id;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
        for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
            for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                double charge = (double)m->charge[eidx] * ECHARGE;
                double elec_jheat = 0.0;
                for (int idim = 0; idim < dim; idim++) {
                    for (int f = 0; f < 2; f++) {
                        int face[3] = {i, j, k};
                        face[idim] += f;
                        if (face[idim] == p->domlo[idim]) face[idim] += 1;
                        if (face[idim] == (p->domhi[idim] + 1)) face[idim] -= 1;
                        int l[3] = {face[0], face[1], face[2]}, r[3] = {face[0], face[1], face[2]};
                        l[idim] -= 1;
                        double etemp = 0.5 * (A4(sb, l[0], l[1], l[2], VD_ETEMP(ns)) +
                                              A4(sb, r[0], r[1], r[2], VD_ETEMP(ns)));
                        double Esum = 0.0, evf[3];
                        for (int d = 0; d < dim; d++) {
                            evf[d] = 0.5 * (A4(sb, l[0], l[1], l[2], VD_EFX(ns) + d) +
                                            A4(sb, r[0], r[1], r[2], VD_EFX(ns) + d));
                            Esum += sq(evf[d]);
                        }
                        double efield_mag = sqrt(Esum);
                        double ne = 0.5 * (A4(sb, l[0], l[1], l[2], eidx) + A4(sb, r[0], r[1], r[2], eidx));
                        double efield_face = p->cs_technique ? evf[idim]
                                                             : A4(&ef[idim], face[0], face[1], face[2], 0);
                        /* gradne_fc is the face difference of ne (the electron solve's
                         * gradient); gradne_from_state forms it from the step's state */
                        double gradne_face =
                            p->gradne_from_state
                                ? (A4(sb, r[0], r[1], r[2], eidx) - A4(sb, l[0], l[1], l[2], eidx)) / p->dx[idim]
                                : A4(&gne[idim], face[0], face[1], face[2], 0);
                        double ndens = 0.0;
                        for (int sp = 0; sp < ns; sp++)
                            ndens += 0.5 * (A4(sb, l[0], l[1], l[2], sp) + A4(sb, r[0], r[1], r[2], sp));
                        double mu = p->const_ele_trans ? p->ele_mob / ndens
                                                       : orc_specmob(m, eidx, etemp, ndens, efield_mag, p->Tg);
                        double dcoeff = p->const_ele_trans ? p->ele_diff / ndens
                                                           : orc_specdiff(m, eidx, etemp, ndens, efield_mag, p->Tg);
                        double current_density = charge * (mu * ne * efield_face - dcoeff * gradne_face);
                        elec_jheat += current_density * efield_face;
                    }
                }
                elec_jheat *= 0.5;
                if (p->floor_jh && elec_jheat < 0.0) elec_jheat = 0.0;
                A4(dsdt, i, j, k, 0) += elec_jheat;
                A4(phi_new, i, j, k, VD_EJH(ns)) = elec_jheat;
                A4(phi_new, i, j, k, VD_EIH(ns)) = A4(rxn, i, j, k, ns);
            }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* species class for boundary codes (Source/Evolve.cpp:208-288) */
static int orc_class(const vd_mech *m, int s)
{
    if (s == m->nspecies) return VD_CLASS_ENERGY;
    if (s == m->e_id) return VD_CLASS_ELECTRON;
    return m->charge[s] != 0 ? VD_CLASS_ION : VD_CLASS_NEUTRAL;
}

static vd_array4 orc_comp_view(const vd_array4 *a, int n)
{
    vd_array4 v = *a;
    v.p = a->p + (int64_t)n * a->nstride;
    v.ncomp = 1;
    return v;
}

/* One explicit step over one box: rxnsrc, flux + dsdt of every transported species
 * and the electron energy (+ Joule), n_new = n + dt*dsdt, background species
 * n += dt*rxn (Source/Evolve.cpp:278-284), and the Te update when requested.
 * flux_ws: 3 face arrays large enough for convert(bx, d) (1 component each).
 * dsdt_out / rxn_out must be valid arrays (NS+1 components) covering bx.         */
int orc_explicit_update_all(const vd_mech *m, const vd_box *bx, const vd_array4 *sb,
                            const vd_array4 *ef, const vd_array4 *gne, const vd_array4 *phi_new,
                            const vd_array4 *dsdt_out, const vd_array4 *rxn_out,
                            const vd_array4 *flux_ws, const vd_params *p)
{
    int ns = m->nspecies, dim = bx->dim;
    if (p->do_reactions) {
        orc_reaction_source(m, bx, sb, rxn_out, p->Tg);
    } else {
        for (int n = 0; n <= ns; n++)
            for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
                for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
                    for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) A4(rxn_out, i, j, k, n) = 0.0;
    }
    for (int s = 0; s <= ns; s++) {
        int is_energy = (s == ns);
        if (is_energy && !p->elecenergy_solve) continue;
        int is_bg = (!is_energy) && ((p->bg_mask >> s) & 1ull);
        vd_array4 dv = orc_comp_view(dsdt_out, s);
        if (is_bg) {
            for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
                for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
                    for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                        double v = A4(sb, i, j, k, s);
                        if (p->do_bg_reactions) {
                            v += A4(rxn_out, i, j, k, s) * p->dt;
                            if (v < p->min_species_density && p->bound_specden) v = p->min_species_density;
                        }
                        A4(phi_new, i, j, k, s) = v;
                        A4(&dv, i, j, k, 0) = A4(rxn_out, i, j, k, s);
                    }
            continue;
        }
        int cls = orc_class(m, s);
        for (int d = 0; d < dim; d++) {
            vd_box fb = *bx;
            if (p->do_transport) {
                orc_compute_explicit_flux(m, bx, d, s, sb, p->bc_lo[cls], p->bc_hi[cls], p->domlo,
                                          p->domhi, &flux_ws[d], p->Tg, p->dx, p->dt, p->hyp_order,
                                          p->user_defined_vel, p->weno_scheme, p->user_vel,
                                          p->vel_species);
            } else {
                fb.hi[d] += 1;
                for (int k = fb.lo[2]; k <= fb.hi[2]; ++k)
                    for (int j = fb.lo[1]; j <= fb.hi[1]; ++j)
                        for (int i = fb.lo[0]; i <= fb.hi[0]; ++i) A4(&flux_ws[d], i, j, k, 0) = 0.0;
            }
        }
        orc_compute_dsdt(bx, s, flux_ws, rxn_out, &dv, p->dx);
        if (is_energy) orc_elecenergy_source(m, bx, sb, rxn_out, ef, gne, &dv, phi_new, p);
        for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
            for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
                for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                    double v = A4(sb, i, j, k, s) + p->dt * A4(&dv, i, j, k, 0);
                    if (p->bound_specden && !is_energy) {
                        /* solution clipping of the species solve (Source/ScalarSolve.cpp:599-625) */
                        double lo = (s == m->e_id) ? p->min_electron_density : p->min_species_density;
                        if (v < lo) v = lo;
                    }
                    A4(phi_new, i, j, k, s) = v;
                }
    }
    if (p->update_te && p->elecenergy_solve) {
        /* Source/ScalarSolve.cpp:659-666: Te from the new energy and the step's input ne */
        int eidx = m->e_id;
        for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
            for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
                for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                    double te = twothird / K_B * A4(phi_new, i, j, k, VD_EEN(ns)) / A4(sb, i, j, k, eidx);
                    if (te < p->min_electron_temp) {
                        te = p->min_electron_temp;
                        A4(phi_new, i, j, k, VD_EEN(ns)) = 1.5 * K_B * A4(phi_new, i, j, k, eidx) * te;
                    }
                    A4(phi_new, i, j, k, VD_ETEMP(ns)) = te;
                }
    }
    return 0;
}

/* foextrap / periodic ghost fill of every component (Source/Vidyut.cpp:90-101 sets
 * foextrap on non-periodic faces; FillPatch wraps periodic directions).  ng ghosts. */
void orc_fill_ghosts(const vd_box *bx, const vd_array4 *a, int ng, const int *periodic)
{
    int dim = bx->dim;
    for (int d = 0; d < dim; d++) {
        int lo[3], hi[3];
        for (int e = 0; e < 3; e++) {
            lo[e] = (e < d || e >= dim) ? bx->lo[e] - ((e < dim) ? ng : 0) : bx->lo[e];
            hi[e] = (e < d || e >= dim) ? bx->hi[e] + ((e < dim) ? ng : 0) : bx->hi[e];
        }
        /* directions already filled (e < d) include their ghosts so corners get values */
        int n = bx->hi[d] - bx->lo[d] + 1;
        for (int c = 0; c < a->ncomp; c++)
            for (int g = 1; g <= ng; g++)
                for (int k = lo[2]; k <= hi[2]; k++)
                    for (int j = lo[1]; j <= hi[1]; j++)
                        for (int i = lo[0]; i <= hi[0]; i++) {
                            int idx[3] = {i, j, k};
                            int gl[3] = {i, j, k}, gh[3] = {i, j, k}, sl[3] = {i, j, k}, sh[3] = {i, j, k};
                            if (idx[d] != bx->lo[d]) continue;
                            gl[d] = bx->lo[d] - g;
                            gh[d] = bx->hi[d] + g;
                            if (periodic[d]) {
                                sl[d] = bx->hi[d] - ((g - 1) % n);
                                sh[d] = bx->lo[d] + ((g - 1) % n);
                            } else {
                                sl[d] = bx->lo[d];
                                sh[d] = bx->hi[d];
                            }
                            A4(a, gl[0], gl[1], gl[2], c) = A4(a, sl[0], sl[1], sl[2], c);
                            A4(a, gh[0], gh[1], gh[2], c) = A4(a, sh[0], sh[1], sh[2], c);
                        }
    }
}

/* ------------------------------------------------------------------------- */
/* Error scales (test infrastructure).  Every output of the update is a sum of
 * terms; a last-bit change of any term (for instance exp/pow of one library
 * against another) moves the sum by about eps times the sum of the absolute
 * terms, not eps times the sum.  These functions return that gross magnitude per
 * cell so that tests measure errors relative to it.                            */

/* gross magnitude of productionRate: gw[s] = sum |coef*qdot|, *ge = sum of the
 * absolute energy-exchange terms (same order and units as orc_production_rate). */
static void orc_production_gross(const vd_mech *m, double *gw, const double *sc, double T, double Te,
                                 double EN, double *ge)
{
    int ns = m->nspecies;
    for (int i = 0; i < ns; ++i) gw[i] = 0.0;
    *ge = 0.0;
    double mixture = 0.0;
    for (int i = 0; i < ns; ++i) mixture += sc[i];
    double efm = EN * (mixture * 6.02214076e23) * 1e-21;
    double ne = sc[m->e_id] * 6.02214085774e23;
    double Ue = 1.5 * Te * ne * 1.380649e-23;
    for (int ir = 0; ir < m->nreactions; ++ir) {
        const vd_reaction *r = &m->rxn[ir];
        double k_f = orc_rate(m, r, T, Te, efm);
        double prod = sc[r->reac[0]];
        for (int t = 1; t < r->nreac; ++t) prod = prod * sc[r->reac[t]];
        double q = k_f * prod;
        for (int t = 0; t < r->nterms; ++t) gw[r->term_sp[t]] += fabs(r->term_coef[t] * q);
        if (r->rxntype != VD_RXN_NONE) {
            double e = 0.0;
            orc_comp_ener_exch(m, q, 0.0, sc, k_f, r->rxntype, r->eexci, r->elidx, &e, Ue, T, Te);
            *ge += fabs(e);
        }
    }
    if (m->elastic_loss) {
        double ndens = 0.0;
        for (int sp = 0; sp < ns; sp++) ndens += sc[sp] * N_A;
        double mu = orc_specmob(m, m->e_id, Te, ndens, EN * ndens * 1.0e-21, T);
        double nu = -ECHARGE / ME / mu;
        *ge += fabs(3.0 / 2.0 * K_B * sc[m->e_id] * N_A * (Te - T) * nu * (2.0 * ME / m->elastic_mass));
    }
}

/* dsdt scale of every species and the energy (NS+1 components over bx):
 * sum_d (S_lo + S_hi)/dx_d + gross(rxn_s) (+ the Joule terms for the energy), with
 * S the face scale of orc_face_scale. */
int orc_update_scale(const vd_mech *m, const vd_box *bx, const vd_array4 *sb, const vd_array4 *ef,
                     const vd_array4 *gne, const vd_array4 *scale, const vd_array4 *flux_ws,
                     const vd_params *p)
{
    int ns = m->nspecies, dim = bx->dim;
    for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
        for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
            for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                double sc[VD_MAX_SPECIES], gw[VD_MAX_SPECIES], ge = 0.0;
                for (int sp = 0; sp < ns; sp++) sc[sp] = A4(sb, i, j, k, sp) * 1.0e-6 / N_A * 1.0e6;
                if (p->do_reactions)
                    orc_production_gross(m, gw, sc, p->Tg, A4(sb, i, j, k, VD_ETEMP(ns)),
                                         A4(sb, i, j, k, VD_REF(ns)), &ge);
                else
                    for (int sp = 0; sp < ns; sp++) gw[sp] = 0.0;
                for (int sp = 0; sp < ns; sp++) A4(scale, i, j, k, sp) = gw[sp] * 1.0e-6 * N_A * 1.0e6;
                A4(scale, i, j, k, ns) = ge;
            }
    for (int s = 0; s <= ns; s++) {
        int is_energy = (s == ns);
        if (is_energy && !p->elecenergy_solve) continue;
        if (!is_energy && ((p->bg_mask >> s) & 1ull)) continue;
        if (!p->do_transport) continue;
        int cls = orc_class(m, s);
        for (int d = 0; d < dim; d++) {
            int fhi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
            fhi[d] += 1;
            for (int k = bx->lo[2]; k <= fhi[2]; ++k)
                for (int j = bx->lo[1]; j <= fhi[1]; ++j)
                    for (int i = bx->lo[0]; i <= fhi[0]; ++i)
                        A4(&flux_ws[d], i, j, k, 0) = orc_face_scale(m, i, j, k, d, s, sb, p->Tg, p->hyp_order,
                                                                     p->user_defined_vel, p->user_vel,
                                                                     p->vel_species);
            (void)cls;
            for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
                for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
                    for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                        int h[3] = {i, j, k};
                        h[d] += 1;
                        A4(scale, i, j, k, s) += (fabs(A4(&flux_ws[d], i, j, k, 0)) +
                                                  fabs(A4(&flux_ws[d], h[0], h[1], h[2], 0))) / p->dx[d];
                    }
        }
    }
    if (p->elecenergy_solve) {
        /* Joule: 0.5 * sum over faces |q mu ne E^2| + |q D grad(ne) E| */
        int eidx = m->e_id;
        double charge = fabs((double)m->charge[eidx] * ECHARGE);
        for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
            for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
                for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                    double g = 0.0;
                    for (int idim = 0; idim < dim; idim++)
                        for (int f = 0; f < 2; f++) {
                            int face[3] = {i, j, k};
                            face[idim] += f;
                            if (face[idim] == p->domlo[idim]) face[idim] += 1;
                            if (face[idim] == (p->domhi[idim] + 1)) face[idim] -= 1;
                            int l[3] = {face[0], face[1], face[2]};
                            l[idim] -= 1;
                            double etemp = 0.5 * (A4(sb, l[0], l[1], l[2], VD_ETEMP(ns)) +
                                                  A4(sb, face[0], face[1], face[2], VD_ETEMP(ns)));
                            double ne = 0.5 * (A4(sb, l[0], l[1], l[2], eidx) + A4(sb, face[0], face[1], face[2], eidx));
                            double ndens = 0.0;
                            for (int sp = 0; sp < ns; sp++)
                                ndens += 0.5 * (A4(sb, l[0], l[1], l[2], sp) + A4(sb, face[0], face[1], face[2], sp));
                            double efc = p->cs_technique
                                             ? 0.5 * (A4(sb, l[0], l[1], l[2], VD_EFX(ns) + idim) +
                                                      A4(sb, face[0], face[1], face[2], VD_EFX(ns) + idim))
                                             : A4(&ef[idim], face[0], face[1], face[2], 0);
                            double gn = A4(&gne[idim], face[0], face[1], face[2], 0);
                            double esum = 0.0;
                            for (int d = 0; d < dim; d++)
                                esum += sq(0.5 * (A4(sb, l[0], l[1], l[2], VD_EFX(ns) + d) +
                                                  A4(sb, face[0], face[1], face[2], VD_EFX(ns) + d)));
                            double emag = sqrt(esum);
                            double mu = p->const_ele_trans ? p->ele_mob / ndens
                                                           : orc_specmob(m, eidx, etemp, ndens, emag, p->Tg);
                            double dc = p->const_ele_trans ? p->ele_diff / ndens
                                                           : orc_specdiff(m, eidx, etemp, ndens, emag, p->Tg);
                            g += charge * (fabs(mu * ne * efc * efc) + fabs(dc * gn * efc));
                        }
                    A4(scale, i, j, k, ns) += 0.5 * g;
                }
    }
    return 0;
}
