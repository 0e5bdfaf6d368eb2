/*
 * vidyut_b200.h -- C ABI of the B200 (sm_100a) explicit species / electron-energy
 * update of the Vidyut plasma fluid solver.
 *
 * The entry points take the same box / Array4 / scalar arguments as the per-box
 * loops of the reference solver, so an AMReX host can call them where those loops
 * sit today.  All device pointers are owned by the caller; every call is
 * asynchronous on the caller's stream and returns VD_OK (0) or a negative status
 * (the reference calls amrex::Abort in the same situations).
 *
 * Reference interfaces replaced (paths relative to the hsitaram/vidyut3d tree):
 *   vd_mech_init               plasmachem::init (Source/PlasmaChem.cpp:19-26) plus the
 *                              compile-time case header Chemistry.H (CKWC, productionRate,
 *                              comp_ener_exch, specMob, specDiff, CKCHRG, mw; e.g.
 *                              test/models/Ar_DC_1d/Chemistry.H:177-506)
 *   vd_compute_explicit_flux   the ParallelFor over one face box that calls compute_flux
 *                              (Source/ScalarSolve.cpp:226-250, Source/compute_explicit_flux.H:200-326)
 *   vd_compute_dsdt            Vidyut::compute_dsdt (Source/ScalarSolve.cpp:17-55)
 *   vd_reaction_source         the rxnsrc lambda of Vidyut::update_rxnsrc_at_all_levels
 *                              (Source/ScalarSolve.cpp:113-168)
 *   vd_elecenergy_source       Vidyut::compute_elecenergy_source (Source/ElecEnergySource.cpp:16-173)
 *   vd_explicit_update_all     one explicit step of the whole path: rxnsrc, every transported
 *                              species' flux + dsdt (Source/ScalarSolve.cpp:57-111), the Joule
 *                              term, the background-species update (Source/Evolve.cpp:267-287)
 *                              and the accumulation n += dt*dsdt, fused into two launches
 *                              (three in FP64, where the Joule term has a pass of its own).
 *   vd_implicit_species_solve  Vidyut::implicit_solve_scalar (Source/ScalarSolve.cpp:289-680):
 *                              the implicit diffusion solve of one species, on this library's
 *                              multigrid in place of AMReX's MLMG.
 *   vd_write_plotfile          Vidyut::WritePlotFile (Source/Plot.cpp:29-39): the plotfile layout
 *                              that amrex::WriteMultiLevelPlotfile writes, for one level.
 *   vd_write_checkpoint,       Vidyut::WriteCheckpointFile / ReadCheckpointFile
 *   vd_read_checkpoint         (Source/Plot.cpp:41-178), for one level.
 *   vd_batch_*                 no single reference counterpart: the per-box MFIter loops of the
 *                              functions above run over many independent boxes in one
 *                              persistent launch (the reference iterates boxes with MFIter).
 *   vd_server_*                no reference counterpart (continuous-batching request loop).
 */
#ifndef VIDYUT_B200_H
#define VIDYUT_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VD_ABI_VERSION 2

/* ---- limits of the runtime mechanism table ---------------------------------- */
#define VD_MAX_SPECIES   64
#define VD_MAX_REACTIONS 448
#define VD_MAX_FITS      48   /* reactions with Janev / F-fit rates              */
#define VD_MAX_REACTANTS 3
#define VD_MAX_TERMS     6

/* ---- status codes ---------------------------------------------------------- */
#define VD_OK             0
#define VD_ERR_ARG       -1   /* null pointer, empty/inverted box, bad component count      */
#define VD_ERR_SCHEME    -2   /* hyp_order not 1/2/5 or weno_scheme not 1/2/3               */
#define VD_ERR_GHOST     -3   /* input Array4 does not cover the stencil (too few ghosts)   */
#define VD_ERR_DIM       -4   /* dim not 1, 2 or 3                                          */
#define VD_ERR_MECH      -5   /* no mechanism loaded, or the mechanism table is invalid     */
#define VD_ERR_CUDA      -6   /* a CUDA runtime call failed (vd_last_error has the text)    */
#define VD_ERR_TIMEOUT   -7   /* a bounded wait ran out (vd_server_wait)                    */
#define VD_ERR_NOMEM     -8   /* device scratch could not be obtained                       */
#define VD_ERR_NONFINITE -9   /* NaN/Inf in an input or result (vd_params.check_finite)     */
#define VD_ERR_BUDGET   -10   /* serving: case does not fit the HBM budget                  */
#define VD_ERR_STATE    -11   /* call out of order (e.g. batch not built)                   */

/* ---- species / BC codes (Source/VarDefines.H:5-22) -------------------------- */
/* State component n of an Array4 with NVAR = nspecies + 10 components:
 *   [0, NS)      species number densities [1/m^3]
 *   NS+0 EEN     electron energy density [J/m^3]
 *   NS+1 ETEMP   electron temperature [K]
 *   NS+2 POT     potential [V]
 *   NS+3..5      cell-centred E field x, y, z [V/m]
 *   NS+6 EJH     Joule heating diagnostic, NS+7 EIH inelastic, NS+8 EEH elastic
 *   NS+9 REF     reduced field E/N [Td]                                         */
#define VD_EEN(ns)   ((ns) + 0)
#define VD_ETEMP(ns) ((ns) + 1)
#define VD_POT(ns)   ((ns) + 2)
#define VD_EFX(ns)   ((ns) + 3)
#define VD_EFY(ns)   ((ns) + 4)
#define VD_EFZ(ns)   ((ns) + 5)
#define VD_EJH(ns)   ((ns) + 6)
#define VD_EIH(ns)   ((ns) + 7)
#define VD_EEH(ns)   ((ns) + 8)
#define VD_REF(ns)   ((ns) + 9)
#define VD_NVAR(ns)  ((ns) + 10)

#define VD_BC_PER   0
#define VD_BC_DIRC  1
#define VD_BC_HNEU  2
#define VD_BC_IHNEU 3   /* compute_flux forces a zero face flux on such domain faces */
#define VD_BC_ROBIN 4

/* species classes used to pick the boundary codes (Source/Evolve.cpp:208-288) */
#define VD_CLASS_ELECTRON 0
#define VD_CLASS_ENERGY   1
#define VD_CLASS_ION      2
#define VD_CLASS_NEUTRAL  3

/* ---- data descriptors ------------------------------------------------------ */
/* Same fields and byte layout as amrex::Array4<amrex::Real>: element (i,j,k,n) is
 * p[(i-begin[0]) + (j-begin[1])*jstride + (k-begin[2])*kstride + n*nstride];
 * end[] is exclusive.  A 2-D caller has begin[2] = 0, end[2] = 1.              */
typedef struct vd_array4 {
    double*  p;
    int64_t  jstride, kstride, nstride;
    int32_t  begin[3], end[3];
    int32_t  ncomp;
} vd_array4;

/* amrex::Box: smallEnd lo[], bigEnd hi[] (inclusive), index type itype[] (0 cell,
 * 1 node) and the spatial dimension of the caller's build (AMREX_SPACEDIM).      */
typedef struct vd_box {
    int32_t lo[3], hi[3], itype[3];
    int32_t dim;
} vd_box;

/* ---- runtime mechanism (replaces the compile-time Chemistry.H) --------------- */
/* rate kinds: k_f as a function of Te [K] (productionRate in the case header)     */
#define VD_RATE_ARRHENIUS_TE 0   /* k = A * Te^b * exp(-C/Te)                      */
#define VD_RATE_CONST        1   /* k = A                                           */
#define VD_RATE_ARRHENIUS_TG 2   /* k = A * Tg^b * exp(-C/Tg)                       */
/* electron-impact fits in Te_eV = Te/11595 (test/Reactor/CO2_H2_Ar_mechanism_reduced/
 * Chemistry.H:940-1030), coefficients in vd_mech.fits[fit], k in m^3/mol/s:       */
#define VD_RATE_JANEV        3   /* k = jA exp(sum_{j=0..8} jc_j ln(Te_eV)^j) NA    */
#define VD_RATE_FFIT         4   /* k = fA exp(sum_{j=0..3} fc_j Te_eV^-(j+1)) NA    */
#define VD_RATE_JANEV_FFIT   5   /* Janev below Te_eV = switch_ev, F-fit from there  */
/* field-driven ionisation (test/verification/Streamer/Chemistry.H:266-280) with
 * E = EN * N * 1e-21 (EN the cell's reduced field REF [Td], N the density sum) and
 * c = fits[fit].jc: k = ((c0 + c1/E^3) exp(-c2/E) - c3) * c4 E^c5 * E  [1/s]     */
#define VD_RATE_TOWNSEND     6

/* electron-energy exchange types (comp_ener_exch, rxntype) */
#define VD_RXN_NONE       0
#define VD_RXN_EXCITATION 1
#define VD_RXN_IONIZATION 2
#define VD_RXN_RECOMB     3
#define VD_RXN_ATTACH     4   /* -mean electron energy * q, the CO2 reactor header's     */
#define VD_RXN_DETACH     7   /* +mean electron energy * q  comp_ener_exch (:872-881)    */
#define VD_RXN_ELASTIC    5

/* mobility models (specMob): mob_kind[s] for s in [0, NS]; s = NS is the energy  */
#define VD_MOB_ZERO      0   /* mu = 0                                                     */
#define VD_MOB_ELECTRON  1   /* nu = sqrt(8 kB Te/(pi me)) N sigma;  mu = -e/me/nu         */
#define VD_MOB_ION_TG    2   /* nu = sqrt(8 kB Tg/(pi M)) N sigma;   mu =  e/M/nu          */
#define VD_MOB_SCALED    3   /* mu = p0 * mu[ref]                                          */
#define VD_MOB_CONST_N   4   /* mu = p0 / N                                                */
#define VD_MOB_CONST     5   /* mu = p0                                                    */
#define VD_MOB_POW_EMAG  6   /* mu = p0 * |E|^p1 (test/verification/Streamer/Chemistry.H:169) */
/* the two models of test/verification/He_RF_1d/Chemistry.H:218-265, coefficients
 * c = fits[mob_ref].jc (mob_ref is the fit index for these two kinds):          */
#define VD_MOB_EN_POLY   7   /* mu = p0 * (1 + c0 x^2 + c1 x^4)^p1, x = |E|/N               */
#define VD_MOB_EXP_MEANE 8   /* mu = p0 * exp(c0 + c1 ln m + c2/m + c3/m^2 + c4/m^3) / N,
                                m = 1.5 Te/eV (the mean electron energy in eV)             */
/* diffusion models (specDiff) */
#define VD_DIFF_ZERO       0
#define VD_DIFF_TE_ABSMOB  1   /* D = (factor * Te/eV) * |mu[ref]|  */
#define VD_DIFF_TG_MOB     2   /* D = (factor * Tg/eV) *  mu[ref]   */
#define VD_DIFF_CONST      3   /* D = factor (e.g. test/models/ionelec_DC_1d/Chemistry.H:190-209) */
#define VD_DIFF_POW_EMAG   4   /* D = factor * |E|^diff_p1 (Streamer/Chemistry.H:189)            */
/* pressure-scaled coefficients, P_r = 101325 / (N kB Tg) (He_RF_1d/Chemistry.H:267-299) */
#define VD_DIFF_PRES       5   /* D = factor * P_r                                               */
#define VD_DIFF_TE_PRES    6   /* D = factor * (Te / diff_p1) * P_r                              */
#define VD_DIFF_SCALED     7   /* D = factor * D[ref]                                            */
/* |E| in mobilities and diffusion coefficients: the magnitude of the cell-centred
 * field of the state (EFX..EFZ) for the drift velocity and the diffusion solve;
 * of the two cells' average over the active directions for the Joule term
 * (Source/ElecEnergySource.cpp:103-119); EN * N * 1e-21 in the chemistry.       */

typedef struct vd_reaction {
    int32_t kind;                       /* VD_RATE_*                                   */
    int32_t nreac;                      /* q_f = k_f * sc[reac[0]] * ... (in order)    */
    int32_t reac[VD_MAX_REACTANTS];
    int32_t rxntype;                    /* VD_RXN_*                                    */
    int32_t elidx;                      /* collision partner for VD_RXN_ELASTIC        */
    int32_t nterms;                     /* wdot[term_sp[t]] += term_coef[t] * qdot     */
    int32_t term_sp[VD_MAX_TERMS];
    double  term_coef[VD_MAX_TERMS];
    double  A, b, C;                    /* C in kelvin, A in (m^3/mol)^(nreac-1)/s     */
    double  eexci;                      /* threshold energy [eV]                       */
    int32_t fit;                        /* index into vd_mech.fits (fit rate kinds)    */
    int32_t pad0;
} vd_reaction;

/* coefficients of a Janev / F-fit rate (NA = 6.02214085774e23 as in the headers) */
typedef struct vd_rate_fit {
    double jA, jc[9];                   /* Janev: A [cm^3/s] and the 9 coefficients    */
    double fA, fc[4];                   /* F-fit: A and the 4 coefficients             */
    double switch_ev;                   /* VD_RATE_JANEV_FFIT: the Te [eV] switch      */
} vd_rate_fit;

typedef struct vd_mech {
    int32_t nspecies, nreactions;
    int32_t e_id;                                   /* electron species index         */
    int32_t charge[VD_MAX_SPECIES];                 /* CKCHRG                         */
    double  mw[VD_MAX_SPECIES];                     /* g/mol (get_mw)                 */
    int32_t mob_kind[VD_MAX_SPECIES + 1];
    int32_t mob_ref[VD_MAX_SPECIES + 1];            /* SCALED: species; 7, 8: fit     */
    double  mob_p0[VD_MAX_SPECIES + 1];             /* cross section [m^2] / factor   */
    double  mob_p1[VD_MAX_SPECIES + 1];             /* particle mass [kg] / exponent  */
    int32_t diff_kind[VD_MAX_SPECIES + 1];
    int32_t diff_ref[VD_MAX_SPECIES + 1];
    double  diff_factor[VD_MAX_SPECIES + 1];
    double  diff_p1[VD_MAX_SPECIES + 1];            /* VD_DIFF_POW_EMAG exponent      */
    int32_t elastic_loss;                           /* trailing elastic-collision loss */
    int32_t pad0;
    double  elastic_mass;                           /* heavy-partner mass [kg]        */
    vd_reaction rxn[VD_MAX_REACTIONS];
    int32_t nfits, pad1;
    vd_rate_fit fits[VD_MAX_FITS];
} vd_mech;

/* ---- run parameters (Vidyut::ReadParameters keys, Source/Vidyut.cpp:258-392) -- */
#define VD_PREC_FP64  0
#define VD_PREC_MIXED 1   /* FP32 WENO / rates / flux arithmetic, FP64 accumulation */

typedef struct vd_params {
    int32_t dim;                 /* AMREX_SPACEDIM of the caller                  */
    int32_t hyp_order;           /* vidyut.hyp_order: 1, 2 or 5                    */
    int32_t weno_scheme;         /* vidyut.weno_scheme: 1 JS, 2 M, 3 Z              */
    int32_t user_defined_vel;    /* 1: constant velocity user_vel for vel_species  */
    int32_t vel_species;
    int32_t precision;           /* VD_PREC_*                                       */
    double  user_vel[3];
    double  Tg, Pg, time, dt;
    double  dx[3];
    int32_t domlo[3], domhi[3];
    int32_t bc_lo[4][3], bc_hi[4][3];   /* per VD_CLASS_*, per direction             */
    int32_t elecenergy_solve, do_reactions, do_transport, do_bg_reactions;
    int32_t floor_jh, const_ele_trans, cs_technique, bound_specden;
    double  ele_mob, ele_diff;
    double  min_species_density, min_electron_density, min_electron_temp;
    uint64_t bg_mask;            /* bit s: species s is a background species       */
    int32_t update_te;           /* 1: Te = (2/3) eps/(kB ne_old), floored         */
    int32_t gradne_from_state;   /* 1: gradne_fc = face difference of ne (state)   */
    int32_t check_finite;        /* 1: vd_explicit_update_all[_noalloc] waits for its
                                    kernels and returns VD_ERR_NONFINITE when a NaN or
                                    infinity was met: in the E field, Te or density sum
                                    of a cell the stencil reads, or in an updated value
                                    (so also in a density, the energy, a face field or a
                                    rate feeding one).  The outputs are then written but
                                    not meaningful.  0: no check, no synchronisation.  */
    int32_t pad1;
} vd_params;

/* ---- library ------------------------------------------------------------- */
int         vd_abi_version(void);
/* sizeof of the ABI structs, for binding checks: which = 0 vd_array4, 1 vd_box,
 * 2 vd_reaction, 3 vd_mech, 4 vd_params, 5 vd_poisson_params,
 * 6 vd_diffusion_params, 7 vd_batch_stats, 8 vd_server_stats (no reference
 * counterpart).                                                                  */
size_t      vd_sizeof(int which);
const char* vd_last_error(void);           /* text of the last failure on this thread */
const char* vd_status_string(int status);

/* Validates and loads the mechanism on the current device (the reference compiles
 * it into the binary).  Must be called before any compute entry point.           */
int vd_mech_init(const vd_mech* m);

/* Mechanism-specialised chemistry (no reference counterpart; the reference gets
 * the same effect by compiling Chemistry.H into each case executable).
 * vd_mech_init also generates CUDA source for the chemistry with the loaded
 * mechanism folded in and compiles it with NVRTC; vd_mech_specialized() returns 1
 * when those kernels run, 0 when the table-driven kernels do (NVRTC missing or
 * failed, or switched off with vd_set_specialize(0) before vd_mech_init);
 * vd_mech_specialize_status() says why.                                         */
int         vd_mech_specialized(void);
const char* vd_mech_specialize_status(void);
int         vd_set_specialize(int on);
/* Kernel-variant knobs (no reference counterpart), chosen by the tuner
 * (vidyut_b200/tune.py) and settable by hand:
 *   "transport_minblocks_<1|2|3>d_<fp64|mixed>"  1 or 2 resident transport blocks
 *                                                 per SM (2 caps registers at 64).
 * vd_tune_get returns the value or a negative status.                            */
int         vd_tune_set(const char* key, int value);
int         vd_tune_get(const char* key);
/* Generates and compiles (without loading; no GPU needed) the specialised kernels
 * of a mechanism; VD_OK, or VD_ERR_MECH with the compiler log in vd_last_error(). */
int         vd_mech_specialize_check(const vd_mech* m, size_t* cubin_bytes);

/* Face fluxes of one species in one sweep direction over the face box
 * convert(bx, dir) (Source/ScalarSolve.cpp:208-250).  phi holds NVAR components
 * with at least 1/2/3 ghost cells for hyp_order 1/2/5; fx is the face array.     */
int vd_compute_explicit_flux(const vd_box* bx, int dir, int specid, vd_array4 phi,
                             const int32_t bclo[3], const int32_t bchi[3],
                             const int32_t domlo[3], const int32_t domhi[3],
                             vd_array4 fx, double Tg, double Pg, double time,
                             const double dx[3], double dt, int hyp_order,
                             int user_defined_vel, int weno_scheme,
                             const double user_vel[3], int vel_species, void* stream);

/* dsdt(i,j,k) = sum_d (F_d(lo) - F_d(hi)) / dx_d + rxn(i,j,k,specid). */
int vd_compute_dsdt(const vd_box* bx, int specid, const vd_array4 flux[3],
                    vd_array4 rxn, vd_array4 dsdt, const double dx[3], void* stream);

/* rxn(i,j,k,0..NS-1) = species production rates [1/m^3/s], rxn(i,j,k,NS) = electron
 * energy exchange [W/m^3] from CKWC of the loaded mechanism.                      */
int vd_reaction_source(const vd_box* bx, vd_array4 sborder, vd_array4 rxn,
                       double Tg, double Pg, double time, void* stream);

/* Joule heating: dsdt += Q_J, phi_new(EJH) = Q_J, phi_new(EIH) = rxn(NS).        */
int vd_elecenergy_source(const vd_box* bx, vd_array4 sborder, vd_array4 rxn,
                         const vd_array4 efield_ec[3], const vd_array4 gradne_fc[3],
                         vd_array4 dsdt, vd_array4 phi_new, const vd_params* prm,
                         void* stream);

/* One explicit step over one box: phi_new = sborder + dt * dsdt for every
 * transported species and the electron energy (when elecenergy_solve), background
 * species += dt * rxn (when do_bg_reactions), EJH/EIH diagnostics.  dsdt (NT = NS+1
 * components, species index order) and rxn (NS+1 components) are optional outputs
 * (p == NULL to skip).  efield_ec/gradne_fc are the face arrays of the reference
 * (gradne_fc ignored when prm->gradne_from_state).                               */
int vd_explicit_update_all(const vd_box* bx, vd_array4 sborder,
                           const vd_array4 efield_ec[3], const vd_array4 gradne_fc[3],
                           vd_array4 phi_new, vd_array4 dsdt, vd_array4 rxn,
                           const vd_params* prm, void* stream);

/* Allocation-free form of vd_explicit_update_all (no counterpart in the reference).
 * For hosts that cannot let a library allocate device memory during a step: an
 * AMReX application normally hands most of the GPU to its own memory arena at
 * start-up, and some callers forbid any allocation inside their time-step loop.
 * Same arguments, work and results as vd_explicit_update_all, but the per-call
 * scratch (a status word, the per-cell density sums on the stencil-grown box, plus
 * the reaction source when rxn.p is NULL) comes from one fixed array compiled into
 * the library: VD_NOALLOC_SCRATCH_BYTES on every GPU the library is set up on,
 * held until the process exits.  The array is reserved on a device, and its
 * device address looked up, when vd_mech_init runs with that device current (or
 * at the first call of any entry point on another device); make that happen
 * before the host's arena takes the GPU, and before any stream capture.  After
 * it, this entry point allocates nothing.  A box whose scratch would not fit is
 * rejected with VD_ERR_NOMEM before anything is launched (pass rxn to need less
 * scratch).  All calls share the one array: calls that overlap on the GPU
 * (different streams, or another host thread) race on it, so order them on one
 * stream.  Each call clears the status word it uses and writes every other
 * scratch value before reading it.                                               */
#define VD_NOALLOC_SCRATCH_BYTES (64u << 20)
int vd_explicit_update_all_noalloc(const vd_box* bx, vd_array4 sborder,
                                   const vd_array4 efield_ec[3], const vd_array4 gradne_fc[3],
                                   vd_array4 phi_new, vd_array4 dsdt, vd_array4 rxn,
                                   const vd_params* prm, void* stream);

/* Per-box FP64 checksums of an update (conservation checks; no reference counterpart):
 * out[0] = sum over cells of sum_s charge_s * rxn_s   (charge production; 0 up to rounding)
 * out[1] = sum over cells of sum_s |charge_s * rxn_s| (scale for out[0])
 * out[2] = sum over cells of rxn(NS)                  (energy exchange)
 * out[3] = sum over cells and species of phi_new_s    (total particle count)
 * out is a device pointer to 4 doubles.                                           */
int vd_box_checksums(const vd_box* bx, vd_array4 rxn, vd_array4 phi_new,
                     double* out_dev, void* stream);

/* Explicit time scales of one box (Vidyut::find_time_scales, Source/TimeStep.cpp:34-116):
 * out[0] = min_d dx_d / max(|mu_e| |E|)  (electron drift),
 * out[1] = min_d dx_d^2 / (2 dim max D_e)  (electron diffusion),
 * out[2] = eps0 / (e max(|mu_e| n_e))  (dielectric relaxation);
 * DBL_MAX where the maximum is 0.  Synchronises the stream (the host gets the
 * numbers).  With several boxes the caller takes the minimum over boxes.          */
int vd_time_scales(const vd_box* bx, vd_array4 state, const vd_params* prm, double out[3], void* stream);

/* Ghost refill of one box (FillPatch with first-order extrapolation on
 * non-periodic faces, Source/Vidyut.cpp:90-101; periodic wrap elsewhere):
 * components comps[0..ncomp-1] of the `ghost` layers of face-adjacent ghost cells
 * are copied from the nearest valid cell (or the periodic image).  Corner and edge
 * ghosts are not written: no kernel of this library reads them.  periodic may be
 * NULL (no periodic direction).                                                   */
int vd_fill_ghosts(const vd_box* bx, vd_array4 state, int ghost, const int32_t* comps, int ncomp,
                   const int32_t periodic[3], void* stream);

/* Potential and electric field of one box that is the whole domain, before the
 * update (replaces the MLMG solve of Source/PotentialSolve.cpp:188-378 with the
 * same discrete problem, and Vidyut::update_cc_efields,
 * Source/PotentialSolve.cpp:391-430): del^2 phi = -(e/eps0) sum_k z_k n_k on the
 * cell-centred grid, faces with bc_* == VD_BC_DIRC hold phi = value_* at the face,
 * the others zero normal gradient.  Geometric multigrid from the state's POT
 * component as initial guess: FP64 defect correction of the potential with FP32
 * V(2,2) cycles of the correction equation, until the FP64 max|residual| <=
 * tol_rel * max|rhs| (tol_rel > 0; one host synchronisation per cycle) or
 * max_vcycles (tol_rel == 0: exactly max_vcycles, no synchronisation).  Writes POT,
 * EFX..EFZ (centred differences, one-sided at domain faces), REF (|E|/N in Td) in
 * the valid cells and refills their ghosts, and efield_ec[d] = -dphi/dx_d on the
 * face boxes (Dirichlet faces: to the face value over half a cell; unless
 * prm->cs_technique).  user_rhs (p == NULL: none) is added to the right-hand side
 * cell by cell (one component covering the box, in the units of del^2 phi): the
 * reference's user_sources::add_user_potential_sources
 * (Source/PotentialSolve.cpp:220-222).  Scratch (2 doubles per cell, and 3
 * floats per cell over the hierarchy) comes from the library's stream-ordered
 * pool. */
typedef struct {
    int32_t bc_lo[3], bc_hi[3];
    double  value_lo[3], value_hi[3];
    int32_t max_vcycles;
    int32_t pad0;
    double  tol_rel;
    vd_array4 user_rhs;
} vd_poisson_params;
int vd_poisson_solve(const vd_box* bx, vd_array4 state, const vd_array4 efield_ec[3],
                     const vd_params* prm, const vd_poisson_params* pp,
                     int32_t* vcycles_done, double* rel_residual, void* stream);

/* Implicit diffusion solve of one species on one box that is the whole domain
 * (replaces Vidyut::implicit_solve_scalar, Source/ScalarSolve.cpp:289-680, whose
 * MLABecLaplacian/MLMG solve is replaced by this library's multigrid on the same
 * discrete problem): (1/dt) n - div(D grad n) = n_old/dt + dsdt for species
 * dp->spec (NS: the electron energy).  D from specDiff of `state` (the current
 * state, covering the box grown by one) at cells, harmonic means on faces.  Domain
 * faces by prm->bc_lo/bc_hi of the species' class, valued by species_bc
 * (Source/PlasmaChem.H:75-184): VD_BC_DIRC holds that value at the face,
 * VD_BC_IHNEU takes it as the derivative along the direction, VD_BC_HNEU and
 * VD_BC_ROBIN (species_bc's default robin coefficients) zero gradient; a periodic
 * direction (VD_BC_PER on both sides, an even number of cells, the state's ghost
 * cells filled periodically) couples its first and last cells (odd counts and
 * one-sided VD_BC_PER are refused, VD_ERR_ARG).  n_old from state_old, the explicit source
 * from component dp->dsdt_comp of dsdt.  The initial guess is the current state;
 * FP64 V(2,2) cycles until max|residual| <= tol_rel * max|rhs| (tol_rel > 0, one
 * host synchronisation per cycle) or max_vcycles (tol_rel == 0: exactly that many,
 * no synchronisation).  Writes component spec of phi_new on the valid cells,
 * floored when prm->bound_specden (not the energy); for the electrons, when
 * gradne_fc is not NULL, the face gradients dn/dx_d on the face boxes
 * (getGradSolution); for the electron energy also ETEMP = (2/3) eps / (kB n_e)
 * with n_e from `state`, floored at min_electron_temp (then EEN = 1.5 kB n_e Te
 * with n_e from phi_new).  Scratch from the stream-ordered allocator. */
typedef struct {
    int32_t spec;          /* 0..NS-1 a species, NS the electron energy             */
    int32_t dsdt_comp;     /* component of dsdt holding this species' explicit source */
    int32_t max_vcycles;
    int32_t pad0;
    double  tol_rel;
    /* 1: the domain faces take the given Robin coefficients instead of species_bc:
     * a n + b dn/dnu = f on the face, nu the outward normal ([side][direction],
     * side 0 low, 1 high); the reference's case files set them through
     * user_transport::species_bc (e.g. test/verification/MMS/UserFunctions.H:60-104),
     * whose robin_a/b/f arrays MLMG reads.  a = 1, b = 0 holds the value f.       */
    int32_t user_robin;
    int32_t pad1;
    double  robin_a[2][3], robin_b[2][3], robin_f[2][3];
} vd_diffusion_params;
int vd_implicit_species_solve(const vd_box* bx, vd_array4 state, vd_array4 state_old, vd_array4 dsdt,
                              vd_array4 phi_new, const vd_array4 gradne_fc[3], const vd_params* prm,
                              const vd_diffusion_params* dp, int32_t* vcycles_done, double* rel_residual,
                              void* stream);

/* Plotfile of one box that is the whole domain (replaces Vidyut::WritePlotFile,
 * Source/Plot.cpp:29-39, which calls amrex::WriteMultiLevelPlotfile): writes the
 * single-level plotfile layout -- dir/Header, dir/Level_0/Cell_H and
 * dir/Level_0/Cell_D_00000 -- from HOST memory: data holds ncomp components of the
 * box's cells, component slowest, x fastest; names the ncomp variable names (the
 * reference uses the species names then Electron_energy, Electron_Temp, Potential,
 * Efieldx..z, Electron_Jheat, Electron_inelasticHeat, Electron_elasticHeat,
 * ReducedEF, Source/Vidyut.cpp:32-52); the domain starts at prob_lo with cells of
 * dx.  Synchronous file output; creates dir and dir/Level_0 when missing.        */
int vd_write_plotfile(const char* dir, const vd_box* bx, const double* data, int ncomp,
                      const char* const* names, const double prob_lo[3], const double dx[3], double time,
                      int step);

/* Checkpoint of one box (replaces Vidyut::WriteCheckpointFile and
 * ReadCheckpointFile, Source/Plot.cpp:41-178, on one level): dir/Header with the
 * title line "Checkpoint file for Vidyut", the finest level (0), the step, dt and
 * time lines and the box array; the state (host memory, ncomp components, component
 * slowest, x fastest) as the multi-fab dir/Level_0/phi in the plotfile's layout.
 * vd_read_checkpoint fills bx, ncomp, istep, dt and time; with data == NULL it only
 * reports them (a size query), otherwise it reads the values into data, which
 * must hold capacity >= cells * ncomp doubles.  Synchronous file I/O.            */
int vd_write_checkpoint(const char* dir, const vd_box* bx, const double* data, int ncomp, int istep, double dt,
                        double time);
int vd_read_checkpoint(const char* dir, vd_box* bx, double* data, int64_t capacity, int* ncomp, int* istep,
                       double* dt, double* time);

/* ---- batched cases (no single reference counterpart: the reference loops over
 * boxes with MFIter and calls the per-box functions above for each) -----------
 * A batch owns a device arena of hbm_budget_bytes and keeps every resident case's
 * state there (two copies: a step reads one and writes the other), with its
 * density-sum and reaction-source scratch and its Joule face arrays.  All cases
 * use the mechanism loaded when the batch was created and the batch's precision;
 * each has its own box, domain, dt, Tg, scheme and flags (vd_params).
 * vd_batch_step(n) advances every resident case by min(n, its remaining steps)
 * explicit steps: per step the density sums + chemistry of all cases, the fused
 * transport update of all cases (one launch per dimension present) and the ghost
 * refill of the written state (species, EEN and ETEMP; vd_fill_ghosts), each a
 * persistent kernel over a work list of (case, chunk-or-tile) items.  The n steps
 * are captured once as a CUDA graph and replayed while the set of cases stays the
 * same.  The fields the hot path only reads (E, its face values, the potential)
 * stay as given; gradne_fc is recomputed from the state when
 * prm->gradne_from_state, else kept as given.
 * State layout (add/read): dense, Array4 order (i fastest, component slowest) over
 * the box grown by the stencil halo H (1, 2 or 3 for hyp_order 1, 2, 5) in each of
 * its dim directions, VD_NVAR(NS) components; ghosts filled.  efield_ec / gradne_fc:
 * dense over the face box of direction d, one component; may be NULL when not used
 * (cs_technique, gradne_from_state, no electron energy).  Pointers may be host or
 * device memory.  Calls on one batch must come from one host thread at a time;
 * add/remove/tune wait for the batch's queued work first.                      */
typedef struct vd_batch vd_batch;
typedef struct {
    int32_t  ncases;
    int32_t  ncases_dim[4];      /* resident cases per dimension (index 1..3)     */
    int64_t  cells;              /* valid cells over resident cases               */
    uint64_t bytes_used;         /* arena bytes held by resident cases            */
    uint64_t bytes_budget;
    int64_t  steps_run;          /* case-steps completed since creation           */
    int64_t  graph_builds;       /* CUDA graph captures                           */
    int32_t  tile_variant[4];    /* transport tile variant per dimension (1..3)   */
    int32_t  launches_per_step;  /* kernels per step of the current case set      */
} vd_batch_stats;

int      vd_batch_create(vd_batch** out, int precision, uint64_t hbm_budget_bytes, int max_cases);
int      vd_batch_destroy(vd_batch* b);
uint64_t vd_batch_case_bytes(const vd_box* bx, const vd_params* prm);  /* 0 if invalid */
/* nsteps: steps this case takes in total (< 0: no limit).  VD_ERR_BUDGET when the
 * case does not fit the arena (or max_cases is reached): nothing is changed. */
int      vd_batch_add_case(vd_batch* b, const vd_box* bx, const double* state,
                           const double* const efield_ec[3], const double* const gradne_fc[3],
                           const vd_params* prm, const int32_t periodic[3], int64_t nsteps,
                           void* stream, int32_t* case_id);
int      vd_batch_remove_case(vd_batch* b, int32_t case_id);
int      vd_batch_step(vd_batch* b, int nsteps, void* stream);
int      vd_batch_case_info(vd_batch* b, int32_t case_id, int64_t* steps_done, int64_t* steps_left);
/* *nonfinite = 1 when a step of the case met a NaN or infinity (in the E field,
 * Te or density sum of a cell its stencil reads, or in an updated value); the
 * case then takes no further steps (vd_batch_load_case clears it).  Waits for the
 * batch's queued work.  The reference aborts the run in that situation. */
int      vd_batch_case_status(vd_batch* b, int32_t case_id, int32_t* nonfinite);
int      vd_batch_read_case(vd_batch* b, int32_t case_id, double* state, void* stream);
/* replaces a resident case's state (same layout as add; both copies are written)
 * and restarts its step count with nsteps; the arena region and the captured
 * graph are kept, so this is the cheap way to start a new solve of the same shape */
int      vd_batch_load_case(vd_batch* b, int32_t case_id, const double* state, int64_t nsteps,
                            void* stream);
/* autotuner: times the transport kernel of each tile variant on the resident cases
 * (trials launches each; the state is not advanced), keeps the fastest per
 * dimension and makes it the default of later batches.  ms_out (32 doubles or
 * NULL): ms_out[dim*8 + variant], -1 where not timed.                           */
int      vd_batch_tune(vd_batch* b, int trials, void* stream, double* ms_out);
int      vd_batch_set_tile_variant(vd_batch* b, int dim, int variant);
/* tile shape and target resident CTAs per SM of a transport variant (min_blocks may
 * be NULL); returns the number of variants of that dimension                    */
int      vd_batch_tile_shape(int dim, int variant, int32_t tile[3], int32_t* min_blocks);
int      vd_batch_set_graph(vd_batch* b, int on);  /* 0: launch kernels directly */
int      vd_batch_get_stats(vd_batch* b, vd_batch_stats* out);

/* ---- serving (no reference counterpart: the reference runs one case per process)
 * A continuous-batching request loop on one GPU over a vd_batch of
 * hbm_budget_bytes.  vd_server_submit copies the request's inputs (layouts as for
 * vd_batch_add_case) into host memory the server owns and queues it; a worker
 * thread admits queued requests oldest first as arena room frees up (smaller
 * ones may backfill past a request that does not fit until it has waited 200 ms),
 * steps all resident cases together quantum_steps explicit steps at a time,
 * and retires finished cases to host memory.  vd_server_wait blocks until the
 * request is done (timeout_s < 0: no limit; VD_ERR_TIMEOUT otherwise), copies its
 * final state (the ghost-grown layout) to state_out when not NULL, gives its
 * latency (submission to result in host memory) and forgets the request; a
 * request that failed returns its status, VD_ERR_NONFINITE when one of its steps
 * met a NaN or infinity (vd_batch_case_status).
 * A request larger than the whole budget is rejected at submission with
 * VD_ERR_BUDGET.  The server uses the device current at creation and the
 * mechanism loaded then.                                                         */
typedef struct vd_server vd_server;
typedef struct {
    int64_t  submitted, completed, failed, queued;
    double   p50_ms, p99_ms, max_ms;    /* latency of completed requests            */
    double   span_s;                    /* first submission to last completion      */
    double   solves_per_s;              /* completed / span_s                       */
    double   cell_updates_per_s;        /* sum of cells x steps completed / span_s  */
    uint64_t bytes_budget, peak_bytes_used;
    int64_t  quanta, graph_builds;
} vd_server_stats;

int vd_server_create(vd_server** out, int precision, uint64_t hbm_budget_bytes, int max_cases,
                     int quantum_steps);
int vd_server_destroy(vd_server* s);   /* stops the worker; unfinished requests fail */
int vd_server_submit(vd_server* s, const vd_box* bx, const double* state,
                     const double* const efield_ec[3], const double* const gradne_fc[3],
                     const vd_params* prm, const int32_t periodic[3], int64_t nsteps,
                     int64_t* request_id);
int vd_server_wait(vd_server* s, int64_t request_id, double* state_out, double timeout_s,
                   double* latency_ms);
int vd_server_get_stats(vd_server* s, vd_server_stats* out);

/* ---- measurement (no reference counterpart; the reference only prints the
 * whole-run wall time, Source/main.cpp:45-46) --------------------------------
 * vd_launch_count: kernels launched by this library since load (all entry points).
 * vd_profile_enable(1): from now on every launch is bracketed by CUDA events on
 * its own stream; vd_profile_read synchronises those events and returns, per
 * kernel name, the number of launches and their summed device time [ms] (at most
 * max entries, names NUL-separated in names, up to names_len bytes).
 * vd_profile_enable(0) stops recording and clears the records.                  */
int64_t vd_launch_count(void);
int     vd_profile_enable(int on);
int     vd_profile_read(char* names, int names_len, int64_t* counts, double* ms, int max);

#ifdef __cplusplus
}
#endif
#endif /* VIDYUT_B200_H */
