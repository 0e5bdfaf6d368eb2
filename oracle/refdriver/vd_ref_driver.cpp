/*
 * vd_ref_driver.cpp -- runs the reference's own hot-path code on the CPU
 * (TEST INFRASTRUCTURE ONLY; built into oracle/_ref/, never shipped).
 *
 * Compiled per (case directory, AMREX_SPACEDIM) exactly as the reference compiles
 * one executable per case: the case's Chemistry.H / UserFunctions.H / ProbParm.H
 * and the reference's Source/compute_explicit_flux.H + Source/PlasmaChem.H are
 * included UNMODIFIED from the reference tree; only AMReX is replaced by the small
 * shim in oracle/refshim.  The reference's per-box loops are member functions of
 * Vidyut bound to MultiFab/MFIter, so the thin loops around the reference device
 * functions are restated here (cited line by line):
 *   ref_reaction_source        Source/ScalarSolve.cpp:143-165 (calls CKWC)
 *   ref_compute_explicit_flux  Source/ScalarSolve.cpp:226-250 (calls compute_flux)
 *   ref_compute_dsdt           Source/ScalarSolve.cpp:44-53
 *   ref_elecenergy_source      Source/ElecEnergySource.cpp:65-171 (calls specMob/specDiff)
 *   ref_explicit_update_all    Source/Evolve.cpp:203-288 call sequence (explicit parts)
 * The loops run under OpenMP, as the reference's MFIter loops can.
 */
#include "vd_amrex_shim.H"
#include <ProbParm.H>
#include <Chemistry.H>
#include <VarDefines.H>  /* before UserFunctions.H, as Vidyut.H orders them */
#include <UserFunctions.H>
#include <compute_explicit_flux.H>
#include "../../include/vidyut_b200.h"

/* Source/PlasmaChem.cpp:10,34-37 (the rest of that file needs the full AMReX app) */
namespace plasmachem {
AMREX_GPU_DEVICE_MANAGED int spec_chrg[NUM_SPECIES] = {0};
AMREX_GPU_HOST_DEVICE int get_charge(int specid) { return spec_chrg[specid]; }
} // namespace plasmachem

static amrex::Array4<amrex::Real> to_a4(const vd_array4& a)
{
    amrex::Array4<amrex::Real> r;
    r.p = a.p;
    r.jstride = a.jstride;
    r.kstride = a.kstride;
    r.nstride = a.nstride;
    r.begin = {a.begin[0], a.begin[1], a.begin[2]};
    r.end = {a.end[0], a.end[1], a.end[2]};
    r.ncomp = a.ncomp;
    return r;
}

template <class T>
static amrex::GpuArray<T, AMREX_SPACEDIM> to_ga(const T* v)
{
    amrex::GpuArray<T, AMREX_SPACEDIM> g;
    for (int d = 0; d < AMREX_SPACEDIM; d++) g[d] = v[d];
    return g;
}

static void set_probparm(ProbParm& pp, const double* uvel, int vel_species)
{
    (void)pp;
    (void)uvel;
    (void)vel_species;
#ifdef VD_PROBPARM_HAS_VEL
    pp.velx = uvel[0];
    pp.vely = uvel[1];
    pp.velz = uvel[2];
#endif
#ifdef VD_PROBPARM_HAS_VEL_SPECIES
    pp.vel_species = vel_species;
#endif
}

extern "C" {

int ref_init(void)
{
    CKCHRG(plasmachem::spec_chrg); /* plasmachem::init, Source/PlasmaChem.cpp:19-26 */
    return 0;
}
int ref_nspecies(void) { return NUM_SPECIES; }
int ref_dim(void) { return AMREX_SPACEDIM; }
int ref_e_id(void) { return E_ID; }

int ref_reaction_source(const vd_box* bx, vd_array4 sb4, vd_array4 rxn4, double Tg, double Pg,
                        double time)
{
    (void)Pg;
    (void)time;
    auto sborder_arr = to_a4(sb4);
    auto rxn_arr = to_a4(rxn4);
    amrex::Real captured_gastemp = Tg;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
        for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
            for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                amrex::Real spec_C[NUM_SPECIES];
                amrex::Real spec_wdot[NUM_SPECIES];
                amrex::Real Te = sborder_arr(i, j, k, ETEMP_ID);
                amrex::Real EN = sborder_arr(i, j, k, REF_ID);
                amrex::Real ener_exch = 0.0;
                for (int sp = 0; sp < NUM_SPECIES; sp++) spec_C[sp] = sborder_arr(i, j, k, sp) * 1.0e-6 / N_A;
                CKWC(captured_gastemp, spec_C, spec_wdot, Te, EN, &ener_exch);
                for (int sp = 0; sp < NUM_SPECIES; sp++) rxn_arr(i, j, k, sp) = spec_wdot[sp] * N_A * 1.0e6;
                rxn_arr(i, j, k, NUM_SPECIES) = ener_exch;
            }
    return 0;
}

int ref_compute_explicit_flux(const vd_box* bx, int dir, int specid, vd_array4 phi4,
                              const int32_t* bclo_, const int32_t* bchi_, const int32_t* domlo_,
                              const int32_t* domhi_, vd_array4 fx4, double Tg, double Pg, double time,
                              const double* dx_, double dt, int hyp_order, int udv, int weno_scheme,
                              const double* uvel, int vel_species)
{
    auto sborder_arr = to_a4(phi4);
    auto fx = to_a4(fx4);
    auto bclo = to_ga<int>(bclo_);
    auto bchi = to_ga<int>(bchi_);
    auto domlo = to_ga<int>(domlo_);
    auto domhi = to_ga<int>(domhi_);
    auto dx = to_ga<amrex::Real>(dx_);
    ProbParm pp;
    set_probparm(pp, uvel, vel_species);
    int hi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
    hi[dir] += 1; /* convert(bx, e_dir): nodal in the sweep direction */
    try {
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = bx->lo[2]; k <= hi[2]; ++k)
            for (int j = bx->lo[1]; j <= hi[1]; ++j)
                for (int i = bx->lo[0]; i <= hi[0]; ++i)
                    compute_flux(i, j, k, dir, specid, sborder_arr, bclo, bchi, domlo, domhi, fx, Tg,
                                 Pg, time, dx, dt, pp, hyp_order, udv, weno_scheme);
    } catch (...) {
        return -2;
    }
    return 0;
}

int ref_compute_dsdt(const vd_box* bx, int specid, const vd_array4* flux4, vd_array4 rxn4,
                     vd_array4 dsdt4, const double* dx)
{
    auto rxn_arr = to_a4(rxn4);
    auto dsdt_arr = to_a4(dsdt4);
    amrex::Array4<amrex::Real> flux_arr[3];
    for (int d = 0; d < AMREX_SPACEDIM; d++) flux_arr[d] = to_a4(flux4[d]);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
        for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
            for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                dsdt_arr(i, j, k) = (flux_arr[0](i, j, k) - flux_arr[0](i + 1, j, k)) / dx[0] +
                                    rxn_arr(i, j, k, specid);
#if AMREX_SPACEDIM > 1
                dsdt_arr(i, j, k) += (flux_arr[1](i, j, k) - flux_arr[1](i, j + 1, k)) / dx[1];
#if AMREX_SPACEDIM == 3
                dsdt_arr(i, j, k) += (flux_arr[2](i, j, k) - flux_arr[2](i, j, k + 1)) / dx[2];
#endif
#endif
            }
    return 0;
}

int ref_elecenergy_source(const vd_box* bx, vd_array4 sb4, vd_array4 rxn4, const vd_array4* ef4,
                          const vd_array4* gne4, vd_array4 dsdt4, vd_array4 phinew4,
                          const vd_params* prm)
{
    auto sborder_arr = to_a4(sb4);
    auto rxn_arr = to_a4(rxn4);
    auto dsdt_arr = to_a4(dsdt4);
    auto phi_arr = to_a4(phinew4);
    amrex::Array4<amrex::Real> ef_arr[3], gradne_arr[3];
    for (int d = 0; d < AMREX_SPACEDIM; d++) {
        ef_arr[d] = to_a4(ef4[d]);
        gradne_arr[d] = to_a4(gne4[d]);
    }
    auto domlo = to_ga<int>(prm->domlo);
    auto domhi = to_ga<int>(prm->domhi);
    int consteletrans = prm->const_ele_trans;
    int captured_cs_technique = prm->cs_technique;
    amrex::Real elemob = prm->ele_mob, elediff = prm->ele_diff;
    amrex::Real captured_gastemp = prm->Tg;
    int floor_jh = prm->floor_jh;
    int eidx = E_ID;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
        for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
            for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                amrex::Real mu, dcoeff, etemp, ne, efield_face, gradne_face, current_density;
                amrex::Real charge = plasmachem::get_charge(eidx) * ECHARGE;
                amrex::Real elec_jheat = 0.0;
                for (int idim = 0; idim < AMREX_SPACEDIM; idim++) {
                    for (int f = 0; f < 2; f++) {
                        amrex::IntVect face{AMREX_D_DECL(i, j, k)};
                        face[idim] += f;
                        if (face[idim] == domlo[idim]) face[idim] += 1;
                        if (face[idim] == (domhi[idim] + 1)) face[idim] -= 1;
                        amrex::IntVect lcell{AMREX_D_DECL(face[0], face[1], face[2])};
                        amrex::IntVect rcell{AMREX_D_DECL(face[0], face[1], face[2])};
                        lcell[idim] -= 1;
                        etemp = 0.5 * (sborder_arr(lcell, ETEMP_ID) + sborder_arr(rcell, ETEMP_ID));
                        amrex::Real Esum = 0.0;
                        amrex::Real efieldvec_face[AMREX_SPACEDIM];
                        for (int d = 0; d < AMREX_SPACEDIM; d++) {
                            efieldvec_face[d] = 0.5 * (sborder_arr(lcell, EFX_ID + d) + sborder_arr(rcell, EFX_ID + d));
                            Esum += std::pow(efieldvec_face[d], 2.0);
                        }
                        amrex::Real efield_mag = std::sqrt(Esum);
                        ne = 0.5 * (sborder_arr(lcell, eidx) + sborder_arr(rcell, eidx));
                        efield_face = (captured_cs_technique) ? efieldvec_face[idim] : ef_arr[idim](face);
                        gradne_face = gradne_arr[idim](face);
                        amrex::Real ndens = 0.0;
                        for (int sp = 0; sp < NUM_SPECIES; sp++)
                            ndens += 0.5 * (sborder_arr(lcell, sp) + sborder_arr(rcell, sp));
                        mu = (consteletrans) ? elemob / ndens
                                             : specMob(eidx, etemp, ndens, efield_mag, captured_gastemp);
                        dcoeff = (consteletrans) ? elediff / ndens
                                                 : specDiff(eidx, etemp, ndens, efield_mag, captured_gastemp);
                        current_density = charge * (mu * ne * efield_face - dcoeff * gradne_face);
                        elec_jheat += current_density * efield_face;
                    }
                }
                elec_jheat *= 0.5;
                if (floor_jh) {
                    if (elec_jheat < 0.0) elec_jheat = 0.0;
                }
                dsdt_arr(i, j, k) += (elec_jheat);
                phi_arr(i, j, k, EJH_ID) = elec_jheat;
                phi_arr(i, j, k, EIH_ID) = rxn_arr(i, j, k, EEN_ID);
            }
    return 0;
}

static vd_array4 comp_view(const vd_array4& a, int n)
{
    vd_array4 v = a;
    v.p = a.p + (int64_t)n * a.nstride;
    v.ncomp = 1;
    return v;
}

/* The explicit part of one corrector (Source/Evolve.cpp:203-288): rxnsrc; per
 * transported species (electrons, energy, ions, neutrals) flux + dsdt (+ Joule for
 * the energy); background species n += dt*rxn; followed by the explicit
 * accumulation n_new = n + dt*dsdt that replaces the implicit solve here, and the
 * Te update of Source/ScalarSolve.cpp:659-666 when requested.                      */
int ref_explicit_update_all(const vd_box* bx, vd_array4 sb, const vd_array4* ef, const vd_array4* gne,
                            vd_array4 phi_new, vd_array4 dsdt, vd_array4 rxn, const vd_array4* flux_ws,
                            const vd_params* p)
{
    const int ns = NUM_SPECIES;
    auto sb_arr = to_a4(sb);
    auto pn_arr = to_a4(phi_new);
    auto rx_arr = to_a4(rxn);
    if (p->do_reactions) ref_reaction_source(bx, sb, rxn, p->Tg, p->Pg, p->time);
    else
        for (int n = 0; n <= ns; n++)
            for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
                for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
                    for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) rx_arr(i, j, k, n) = 0.0;
    for (int s = 0; s <= ns; s++) {
        bool energy = (s == ns);
        if (energy && !p->elecenergy_solve) continue;
        bool bg = !energy && ((p->bg_mask >> s) & 1ull);
        vd_array4 dv4 = comp_view(dsdt, s);
        auto dv = to_a4(dv4);
        if (bg) {
            for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
                for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
                    for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                        double v = sb_arr(i, j, k, s);
                        if (p->do_bg_reactions) {
                            v += rx_arr(i, j, k, s) * p->dt;
                            if (v < p->min_species_density && p->bound_specden) v = p->min_species_density;
                        }
                        pn_arr(i, j, k, s) = v;
                        dv(i, j, k) = rx_arr(i, j, k, s);
                    }
            continue;
        }
        int cls = energy ? VD_CLASS_ENERGY
                         : (s == E_ID ? VD_CLASS_ELECTRON
                                      : (plasmachem::get_charge(s) != 0 ? VD_CLASS_ION : VD_CLASS_NEUTRAL));
        for (int d = 0; d < AMREX_SPACEDIM; d++) {
            if (p->do_transport) {
                int rc = ref_compute_explicit_flux(bx, d, s, sb, p->bc_lo[cls], p->bc_hi[cls], p->domlo,
                                                   p->domhi, flux_ws[d], p->Tg, p->Pg, p->time, p->dx, p->dt,
                                                   p->hyp_order, p->user_defined_vel, p->weno_scheme,
                                                   p->user_vel, p->vel_species);
                if (rc) return rc;
            } else {
                auto fa = to_a4(flux_ws[d]);
                int hi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
                hi[d] += 1;
                for (int k = bx->lo[2]; k <= hi[2]; ++k)
                    for (int j = bx->lo[1]; j <= hi[1]; ++j)
                        for (int i = bx->lo[0]; i <= hi[0]; ++i) fa(i, j, k) = 0.0;
            }
        }
        ref_compute_dsdt(bx, s, flux_ws, rxn, dv4, p->dx);
        if (energy) ref_elecenergy_source(bx, sb, rxn, ef, gne, dv4, phi_new, p);
        for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
            for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
                for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                    pn_arr(i, j, k, s) = sb_arr(i, j, k, s) + p->dt * dv(i, j, k);
                    /* the species solve's clipping (Source/ScalarSolve.cpp:597-622) */
                    if (p->bound_specden && !energy) {
                        double floor_ = (s == E_ID) ? p->min_electron_density : p->min_species_density;
                        if (pn_arr(i, j, k, s) < floor_) pn_arr(i, j, k, s) = floor_;
                    }
                }
    }
    if (p->update_te && p->elecenergy_solve) {
        for (int k = bx->lo[2]; k <= bx->hi[2]; ++k)
            for (int j = bx->lo[1]; j <= bx->hi[1]; ++j)
                for (int i = bx->lo[0]; i <= bx->hi[0]; ++i) {
                    pn_arr(i, j, k, ETEMP_ID) = twothird / K_B * pn_arr(i, j, k, EEN_ID) / sb_arr(i, j, k, E_ID);
                    if (pn_arr(i, j, k, ETEMP_ID) < p->min_electron_temp) {
                        pn_arr(i, j, k, ETEMP_ID) = p->min_electron_temp;
                        pn_arr(i, j, k, EEN_ID) = 1.5 * K_B * pn_arr(i, j, k, E_ID) * p->min_electron_temp;
                    }
                }
    }
    return 0;
}

} // extern "C"
