// vd_kernels.cuh -- host-visible launch interface of the device code in vd_kernels.cu.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "vd_types.cuh"

namespace vd {

// Box-loop geometry: cells lo..hi inclusive.
struct BoxIdx {
    int lo[3], hi[3];
    int n[3];
    int64_t ncell;
};

// Arguments of the fused transport kernel (per box).
struct TransportArgs {
    A4 sb, pn, dsdt, rxn, Nv;
    A4 ef[3], gne[3];
    int lo[3], hi[3];
    int ntile[3];
    double dx[3], idx[3], dt, Tg, dxmin;
    int domlo[3], domhi[3];
    int8_t zlo[4][3], zhi[4][3];  // 1: IHNEUBC zero flux on that domain face, per class
    int ntr, nbg;
    int8_t tr_sp[VD_MAX_SPECIES + 1], tr_cls[VD_MAX_SPECIES + 1], tr_flux[VD_MAX_SPECIES + 1];
    int8_t bg_sp[VD_MAX_SPECIES];
    int ns, e_id, hyp_order, weno, udv, vel_sp;
    double uvel[3];
    int elecenergy, do_bg, bound_specden, floor_jh, const_ele_trans, cs_technique, gradne_from_state;
    int update_te, write_diag;
    double min_spec, min_elec, ele_mob, ele_diff, min_te, charge_e;
    int ghost;  // stencil half width H (1, 2 or 3)
    // Derived from the lists above (finish_species_lists): the transported species
    // with a drift flux, in update order, and those without.  A fluxed species'
    // face velocity is fl_K * (velocity basis fl_slot of the cell): the mobility
    // models of specMob factor into a species constant and a per-cell basis
    // (bkind 0: E/(sqrt(Te) N), 1: E/N, 2: E, 3: E |E|^p, 4: E (1 + c0 x^2 + c1 x^4)^p
    // with x = |E|/N, 5: E exp(c0 + c1 ln m + c2/m + c3/m^2 + c4/m^3) / N with
    // m = 1.5 Te/eV); fl_slot < 0 means the user velocity.
    int nfl, nnf, nb;
    int8_t fl_sp[VD_MAX_SPECIES + 1], fl_cls[VD_MAX_SPECIES + 1], fl_slot[VD_MAX_SPECIES + 1];
    int8_t nf_sp[VD_MAX_SPECIES + 1];
    int8_t bkind[4];
    int8_t bfit[4];   // bkind 4, 5: the mechanism fit holding c
    int8_t stage_emag;  // the staged cells need |E| (a basis of kind 3 or 4, or the electrons' models)
    double bpow[4];   // bkind 3, 4: the exponent p
    double fl_K[VD_MAX_SPECIES + 1];
    float fl_Kf[VD_MAX_SPECIES + 1];  // fl_K rounded to FP32 (the mixed path's constant)
    // zero-flux faces of a fluxed species: bit d set when its class has IHNEUBC at
    // the low domain face of direction d (zlo), bit 3 + d at the high one (zhi)
    int8_t fl_zm[VD_MAX_SPECIES + 1];
    // Non-finite check (null: off).  The tile sets bit 0 of *status when a staged
    // cell's E, Te or density sum, or an updated value of an own cell, is NaN or
    // infinite; a NaN or infinity anywhere in a cell's inputs reaches one of them.
    unsigned int* status;
};

// The mixed path evaluates the Joule faces inside the transport tile when the tile
// has a drift-flux barrier to publish them by; otherwise (and always in FP64) a
// Joule pass (launch_joule_pre) runs before the transport update.
__host__ __device__ inline bool joule_in_tile(const TransportArgs& a, int prec)
{
    return prec == PREC_MIXED && a.elecenergy && a.nfl > 0;
}

// Fills the derived fluxed / unfluxed lists and velocity bases of a from its tr_*
// lists and the mechanism table m (host).
void finish_species_lists(TransportArgs& a, const VdMechDev& m);
// A velocity basis: the per-cell factor of a mobility model times E (the kinds of
// TransportArgs::bkind, with their exponent and coefficient fit).
struct VelBasis {
    int kind;
    double pw;
    int fit;
};
// species s's mobility as K times a velocity basis; false when it has no drift (host)
bool velocity_basis(const VdMechDev& m, int s, double Tg, VelBasis* b, double* K);
// the two bases evaluate to the same values (host)
bool same_basis(const VdMechDev& m, const VelBasis& x, const VelBasis& y);
constexpr int kMaxBases = 3;  // velocity bases a tile stages

// Arguments of the per-cell prep kernel: N = sum_s n_s over the grown box, and
// rxn (chemistry) over the valid box.
struct PrepArgs {
    A4 sb, rxn, Nv;
    int glo[3], ghi[3];     // grown box
    int lo[3], hi[3];       // valid box
    double Tg;
    int do_reactions, write_n;
};

// Ghost refill of one box after a step: the components in comps[] of every
// face-adjacent ghost cell (first-order extrapolation, or periodic wrap) --
// what FillPatch does before the next step (Source/GridWork.cpp:112-140).
struct GhostArgs {
    A4 st;
    int lo[3], hi[3];
    int ghost, dim;
    int periodic[3];
    int ncomp;
    int8_t comps[VD_MAX_SPECIES + 4];
    int64_t count;  // number of ghost cells to fill
};

int upload_mech(const VdMechDev* h, cudaStream_t st);
cudaError_t upload_mech_batch(const VdMechDev* h, cudaStream_t st);      // vd_batch_kernels.cu
cudaError_t upload_mech_diffusion(const VdMechDev* h, cudaStream_t st);  // vd_diffusion.cu

// Step control of a batched launch.  ctrl[c] = {steps case c takes in this call,
// index (0/1) of the buffer holding its current state}.  At step t a work item of
// case c is skipped when t >= ctrl[c].x; otherwise it uses the argument record
// boxes[((t + ctrl[c].y) & 1) * nbox + c] (records of both buffer parities are
// stored, so a captured graph replays unchanged while the per-case counts vary).
struct BatchCtl {
    const int2* ctrl;
    int nbox;
    int t;
};

// Batched launches over a work list of int2 items (box index, chunk or tile index).
constexpr int kPrepChunk = 512;   // cells of the grown box per prep work item
constexpr int kGhostChunk = 256;  // ghost cells per ghost work item
cudaError_t launch_prep_batch(const PrepArgs* boxes, const int2* items, int nitems, BatchCtl ctl, int prec, int ns,
                              cudaStream_t st);
cudaError_t launch_transport_batch(const TransportArgs* boxes, const int2* items, int nitems, BatchCtl ctl, int dim,
                                   int prec, int variant, cudaStream_t st);
cudaError_t launch_ghost_batch(const GhostArgs* boxes, const int2* items, int nitems, BatchCtl ctl,
                               cudaStream_t st);
// launch_joule_pre over the (box, Joule tile) items of boxes of dimension dim
// (vd_batch_kernels.cu; tiles as joule_tile_count in vd_transport.cuh)
cudaError_t launch_joule_pre_batch(const TransportArgs* boxes, const int2* items, int nitems, BatchCtl ctl, int dim,
                                   int prec, cudaStream_t st);
cudaError_t launch_ghost(const GhostArgs& a, cudaStream_t st);
// tile shapes of the batched transport kernel: variant v of dimension dim
int batch_tile_variants(int dim);
void batch_tile_shape(int dim, int variant, int t[3]);
int batch_variant_minblocks(int dim, int variant);  // resident CTAs per SM the variant targets

cudaError_t launch_reaction_source(const BoxIdx& b, const A4& sb, const A4& rxn, double Tg, int prec, int ns,
                                   cudaStream_t st);
cudaError_t launch_face_flux(const BoxIdx& fb, int dir, int specid, const A4& phi, const A4& fx,
                             const int8_t zlo[3], const int8_t zhi[3], const int domlo[3], const int domhi[3],
                             double Tg, double dxmin, double dt, int hyp_order, int udv, int weno,
                             const double uvel[3], int vel_sp, int ns, cudaStream_t st);
cudaError_t launch_dsdt(const BoxIdx& b, int dim, int specid, const A4 flux[3], const A4& rxn, const A4& dsdt,
                        const double dx[3], cudaStream_t st);
cudaError_t launch_joule(const BoxIdx& b, int dim, const A4& sb, const A4& rxn, const A4 ef[3], const A4 gne[3],
                         const A4& dsdt, const A4& pn, const TransportArgs& cfg, cudaStream_t st);
cudaError_t launch_prep(const PrepArgs& a, int prec, int ns, cudaStream_t st);
// The Joule term of every valid cell of the box into the EJH component of a.pn; a
// transport update with an electron energy equation that does not evaluate it in
// the tile (joule_in_tile) reads it there, so this runs between launch_prep and
// launch_transport.
cudaError_t launch_joule_pre(const TransportArgs& a, int dim, int prec, cudaStream_t st);
cudaError_t launch_transport(const TransportArgs& a, int dim, int prec, cudaStream_t st);
cudaError_t launch_checksums(const BoxIdx& b, const A4& rxn, const A4& pn, double* out, cudaStream_t st);
cudaError_t launch_time_scales(const BoxIdx& b, int dim, const A4& st, const TransportArgs& a,
                               unsigned long long* out, cudaStream_t s);

// Tile shape used by the transport kernel for a given dimension (for host-side tiling).
void transport_tile(int dim, int tile[3]);

// Launch accounting: every launch increments a counter; when profiling is on it is
// bracketed by CUDA events on its stream (see vd_profile_* in the header).
int64_t launch_count();
void add_launches(int64_t n);     // kernels run by a graph replay
void prof_suspend(bool on);       // this thread: no event pairs (stream capture)
void prof_enable(bool on);
int prof_read(char* names, int names_len, int64_t* counts, double* ms, int max);

// Tiles of the Joule pass: 256 cells, each face of the tile evaluated once.
template <int DIM> struct JouleTile;
template <> struct JouleTile<1> { static constexpr int X = 256, Y = 1, Z = 1; };
template <> struct JouleTile<2> { static constexpr int X = 32, Y = 8, Z = 1; };
template <> struct JouleTile<3> { static constexpr int X = 8, Y = 8, Z = 4; };
constexpr int kJouleThreads = 256;
// faces of one direction, on the tile's box grown by one along every direction
// of the problem
template <int DIM> constexpr int joule_face_box()
{
    return (JouleTile<DIM>::X + 1) * (JouleTile<DIM>::Y + (DIM > 1)) * (JouleTile<DIM>::Z + (DIM > 2));
}

// number of JouleTile tiles covering box lo..hi
template <int DIM>
__host__ __device__ inline int64_t joule_tile_count(const int* lo, const int* hi)
{
    using JT = JouleTile<DIM>;
    return (int64_t)((hi[0] - lo[0] + JT::X) / JT::X) * ((hi[1] - lo[1] + JT::Y) / JT::Y) *
           ((hi[2] - lo[2] + JT::Z) / JT::Z);
}

// Kernel-variant knobs set by the tuner (vd_tune_set / vd_tune_get).
int tune_set(const char* key, int value);
int tune_get(const char* key);

// Mechanism-specialised chemistry compiled at vd_mech_init (vd_spec.cpp).
int spec_build(const VdMechDev& m);
bool spec_active();
void spec_set_enabled(bool on);
const char* spec_error();
cudaError_t spec_launch_prep(const PrepArgs& a, int prec, cudaStream_t st);
cudaError_t spec_launch_prep_batch(const PrepArgs* boxes, const int2* items, int nitems, BatchCtl ctl, int prec,
                                   cudaStream_t st);
int spec_compile_only(const VdMechDev& m, size_t* cubin_bytes);

struct ProfScope {
    int slot;
    cudaStream_t st;
    ProfScope(const char* name, cudaStream_t s);
    ~ProfScope();
};

}  // namespace vd
