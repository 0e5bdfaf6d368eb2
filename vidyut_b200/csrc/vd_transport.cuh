// vd_transport.cuh -- the fused transport update of one tile (included by vd_kernels.cu).
//
// One CTA updates a TX x TY x TZ tile of one box.
// (0) Once per tile, for every cell of the stencil lines of each sweep direction d
//     (cells rel -3 .. T_d+2 along d of each tile row), the velocity bases of the
//     mobility models -- E_d/(sqrt(Te) N), E_d/N, E_d, E_d |E|^p, E_d f(|E|/N),
//     E_d g(Te)/N, as the mechanism needs -- are computed from Te, E and the
//     density sum and kept in shared memory.  A species' face velocity is then its
//     constant times one basis (specMob).
// (1) The transported species with a drift flux go in groups of up to GRP: the
//     densities of the whole group on all staged lines are loaded at once (many
//     independent loads in flight), then every face flux of every species of the
//     group is computed once (all directions; faces spread over the threads one by
//     one in the mixed path, in runs along the lines in the FP64 path), then
//     each thread takes the divergence of its own cell, adds rxn (and the Joule
//     term for the electron energy) and writes n + dt*dsdt in FP64.  Two barriers
//     per group.  The Joule term: the mixed path evaluates every face of the
//     tile once in FP32 before the first barrier (joule_face_mixed); the FP64
//     path reads it from the EJH diagnostic, where a kernel run just before left
//     it (joule_tile): FP64 face arithmetic inside the tile kernel would raise the
//     register pressure of every phase.
// (2) Transported species without a drift flux, background species and the Te
//     update need no neighbours and no barrier.
// The tile body is a device function so that the per-box kernel (one CTA per
// tile) and the batched persistent kernel (CTAs loop over a work list of
// (box, tile) items of many boxes) share it.
#pragma once
#include <type_traits>
#include "vd_device.cuh"
#include "vd_kernels.cuh"

namespace vd {

// ---------------------------------------------------------------------------
// Joule heating at one cell (Source/ElecEnergySource.cpp:76-153).  USE_N: use the
// per-cell density sums Nv (fused path) instead of re-summing the species.
template <bool USE_N>
__device__ __forceinline__ double joule_cell(const TransportArgs& a, int dim, int i, int j, int k)
{
    const int ns = a.ns, eidx = a.e_id;
    double jheat = 0.0;
    for (int idim = 0; idim < dim; idim++) {
        for (int f = 0; f < 2; f++) {
            int face[3] = {i, j, k};
            face[idim] += f;
            if (face[idim] == a.domlo[idim]) face[idim] += 1;
            if (face[idim] == a.domhi[idim] + 1) face[idim] -= 1;
            int l[3] = {face[0], face[1], face[2]};
            l[idim] -= 1;
            const int64_t ol = a.sb.off(l[0], l[1], l[2]);
            const int64_t orr = a.sb.off(face[0], face[1], face[2]);
            const double* p = a.sb.p;
            const int64_t cs = a.sb.ns;
            double etemp = 0.5 * (p[ol + VD_ETEMP(ns) * cs] + p[orr + VD_ETEMP(ns) * cs]);
            const double evf_d = 0.5 * (p[ol + (VD_EFX(ns) + idim) * cs] + p[orr + (VD_EFX(ns) + idim) * cs]);
            // |E| of the face-averaged field over the active directions
            // (Source/ElecEnergySource.cpp:103-119)
            double esum = 0.0;
            for (int d = 0; d < dim; d++) {
                const double e = 0.5 * (p[ol + (VD_EFX(ns) + d) * cs] + p[orr + (VD_EFX(ns) + d) * cs]);
                esum += e * e;
            }
            const double emag = sqrt(esum);
            double nel = p[ol + eidx * cs], ner = p[orr + eidx * cs];
            double ne = 0.5 * (nel + ner);
            double ef = a.cs_technique ? evf_d : a.ef[idim](face[0], face[1], face[2]);
            double gn = a.gradne_from_state ? (ner - nel) / a.dx[idim] : a.gne[idim](face[0], face[1], face[2]);
            double ndens;
            if (USE_N) {
                ndens = 0.5 * (a.Nv(l[0], l[1], l[2]) + a.Nv(face[0], face[1], face[2]));
            } else {
                ndens = 0.0;
                for (int s = 0; s < ns; s++) ndens += 0.5 * (p[ol + s * cs] + p[orr + s * cs]);
            }
            double mu = a.const_ele_trans ? a.ele_mob / ndens : mob_fp64(eidx, etemp, ndens, a.Tg, emag);
            double dc = a.const_ele_trans ? a.ele_diff / ndens : diff_fp64(eidx, etemp, ndens, a.Tg, emag);
            double cur = a.charge_e * (mu * ne * ef - dc * gn);
            jheat += cur * ef;
        }
    }
    jheat *= 0.5;
    if (a.floor_jh && jheat < 0.0) jheat = 0.0;
    return jheat;
}

template <int X_, int Y_, int Z_, int NTH_>
struct TileShape {
    static constexpr int X = X_, Y = Y_, Z = Z_, NTH = NTH_;
};
template <int DIM> struct DefaultTile;
template <> struct DefaultTile<1> { using T = TileShape<256, 1, 1, 256>; };
template <> struct DefaultTile<2> { using T = TileShape<32, 8, 1, 256>; };
template <> struct DefaultTile<3> { using T = TileShape<8, 8, 8, 512>; };
template <int DIM> constexpr int default_nth() { return DIM == 3 ? 512 : 256; }

template <int DIM, class TS>
struct TileGeom {
    static constexpr int T[3] = {TS::X, TS::Y, TS::Z};
    static constexpr int NCELL = T[0] * T[1] * T[2];
    // staged line set of direction d: extent T_d + 6 along d
    template <int D> static constexpr int SE(int e) { return T[e] + (e == D ? 6 : 0); }
    template <int D> static constexpr int NS() { return D < DIM ? SE<D>(0) * SE<D>(1) * SE<D>(2) : 0; }
    template <int D> static constexpr int FE(int e) { return T[e] + (e == D ? 1 : 0); }
    template <int D> static constexpr int NF() { return D < DIM ? FE<D>(0) * FE<D>(1) * FE<D>(2) : 0; }
    static constexpr int SOFF1 = NS<0>(), SOFF2 = NS<0>() + NS<1>(), STOT = NS<0>() + NS<1>() + NS<2>();
    static constexpr int FOFF1 = NF<0>(), FOFF2 = NF<0>() + NF<1>(), FTOT = NF<0>() + NF<1>() + NF<2>();
};

template <int DIM, class TS, int RUN>
struct RunGeom {
    using G = TileGeom<DIM, TS>;
    static constexpr int NR(int D) { return D < DIM ? (G::T[D] + RUN) / RUN : 0; }  // runs per line
    static constexpr int NL(int D)                                                   // lines
    {
        return D < DIM ? (G::T[0] * G::T[1] * G::T[2]) / G::T[D] : 0;
    }
    static constexpr int R0 = NL(0) * NR(0), R1 = NL(1) * NR(1), R2 = NL(2) * NR(2);
    static constexpr int ROFF1 = R0, ROFF2 = R0 + R1, NRUN = R0 + R1 + R2;
    static_assert(RUN >= 1 && RUN <= 60, "run length fits the info fields");
};

template <int PREC> struct VelT { using T = double; };
template <> struct VelT<PREC_MIXED> { using T = float; };

// The mixed path of 1-D and 2-D tiles also stages the Joule inputs of every staged
// position: ne (FP64: its face differences are the density gradient), Te and the
// density sum (FP32), in the space of the staged densities (they are read before
// the first group is staged).  3-D tiles read them from global memory.
template <int DIM, int PREC> constexpr bool joule_staged() { return PREC == PREC_MIXED && DIM < 3; }
struct JStage {
    double* ne;
    float* te;
    float* nd;
};

__host__ __device__ constexpr size_t smem_align(size_t x) { return (x + 15) & ~(size_t)15; }

// The face phase of the FP64 path takes the faces in runs along the lines
// (run_faces: the WENO smoothness indicators and weights of a cell centre are
// shared by the faces and reconstructions that use them); the mixed path computes
// each face on its own (face_tab: fewer live registers, an even split of the faces
// over the threads), which measured faster for its FP32 arithmetic on B200.
template <int DIM, int PREC> constexpr bool by_runs() { return PREC == PREC_FP64; }
// Faces per run: 5 in 3-D, where the T + 1 = 9 faces of a line then make two runs
// (384 per species for an 8^3 tile: one pass of its 512 threads), else 3.  Timed
// on B200 for the 3-D workload: runs of 2, 3, 4, 5 faces 3.20, 3.19, 4.05,
// 3.09 ms (4 leaves a third pass with one face); for 2-D tiles 3 beats 2 and 4.
template <int DIM, class TS> constexpr int run_len() { return DIM == 3 ? 5 : 3; }

// Dynamic shared memory of one tile with nb velocity bases and species groups of
// GRP, in this order: the Joule term of every face (FP64, mixed path); the run
// info words (run_info); the state offsets of the staged positions; the group's
// face fluxes; the bases; the group's staged densities (or the staged Joule
// inputs).  Fluxes, bases and densities are FP32 in the mixed path: a mixed flux
// is an FP32 value times a power of two, so it is stored exactly.
template <int DIM, int PREC, class TS>
struct TileSmem {
    using G = TileGeom<DIM, TS>;
    using VT = typename VelT<PREC>::T;
    static constexpr size_t joule() { return PREC == PREC_MIXED ? smem_align((size_t)G::FTOT * sizeof(double)) : 0; }
    static constexpr size_t finfo()
    {
        return by_runs<DIM, PREC>() ? smem_align((size_t)RunGeom<DIM, TS, run_len<DIM, TS>()>::NRUN * sizeof(int2))
                                    : smem_align((size_t)G::FTOT * sizeof(int));
    }
    static constexpr size_t soffs() { return smem_align((size_t)G::STOT * sizeof(int)); }
    static constexpr size_t flux(int grp) { return smem_align((size_t)grp * G::FTOT * sizeof(VT)); }
    static constexpr size_t basis(int nb) { return smem_align((size_t)nb * G::STOT * sizeof(VT)); }
    static constexpr size_t dens(int grp)
    {
        const size_t d = (size_t)grp * G::STOT * sizeof(VT);
        const size_t j = joule_staged<DIM, PREC>() ? (size_t)G::STOT * (sizeof(double) + 2 * sizeof(float)) : 0;
        return d > j ? d : j;
    }
};

template <int DIM, int PREC, class TS, int GRP>
__host__ __device__ constexpr size_t transport_smem(int nb)
{
    using S = TileSmem<DIM, PREC, TS>;
    return S::joule() + S::finfo() + S::soffs() + S::flux(GRP) + S::basis(nb) + S::dens(GRP);
}

// Species per group for a kernel that must keep MINB CTAs resident per SM: the
// largest of 8, 4, 2, 1 (at most GMAX) whose tile (with up to three velocity
// bases, the batched kernel's copy of its record and the driver's reserve) fits
// MINB times into the SM's 228 KB of shared memory.  Larger groups mean fewer
// barriers and more loads in flight; smaller ones leave room for more resident
// CTAs and for the L1 cache, which shares the same 256 KB per SM.
template <int DIM, int PREC, class TS, int MINB, int GMAX = 8>
constexpr int group_fit()
{
    constexpr size_t per_sm = 228 * 1024, extra = 3 * 1024;
    if (GMAX >= 8 && (transport_smem<DIM, PREC, TS, 8>(3) + extra) * MINB <= per_sm) return 8;
    if (GMAX >= 4 && (transport_smem<DIM, PREC, TS, 4>(3) + extra) * MINB <= per_sm) return 4;
    if ((transport_smem<DIM, PREC, TS, 2>(3) + extra) * MINB <= per_sm) return 2;
    return 1;
}

// |E| of the field averaged over a face's two cells (state offsets ol, orr), over
// the active directions (Source/ElecEnergySource.cpp:103-119)
__device__ __forceinline__ double face_emag(const TransportArgs& a, int64_t ol, int64_t orr, int dim)
{
    const double* p = a.sb.p;
    const int64_t cs = a.sb.ns;
    double esum = 0.0;
    for (int d = 0; d < dim; d++) {
        const double e = 0.5 * (p[ol + (VD_EFX(a.ns) + d) * cs] + p[orr + (VD_EFX(a.ns) + d) * cs]);
        esum += e * e;
    }
    return sqrt(esum);
}

// Joule heating carried by face g of direction D (the face between cells g - e_D
// and g): q (mu ne E_f - D grad ne) E_f with face averages of Te, ne and the density
// sum (Source/ElecEnergySource.cpp:86-160, one face of the per-cell loop).  Each
// cell adds half of its faces' values, after the domain-face substitution.
__device__ __forceinline__ double joule_face(const TransportArgs& a, int D, const int* g, int dim)
{
    const int ns = a.ns, eidx = a.e_id;
    int l[3] = {g[0], g[1], g[2]};
    l[D] -= 1;
    const int64_t ol = a.sb.off(l[0], l[1], l[2]);
    const int64_t orr = a.sb.off(g[0], g[1], g[2]);
    const double* p = a.sb.p;
    const int64_t cs = a.sb.ns;
    const double etemp = 0.5 * (p[ol + VD_ETEMP(ns) * cs] + p[orr + VD_ETEMP(ns) * cs]);
    const double evf_d = 0.5 * (p[ol + (VD_EFX(ns) + D) * cs] + p[orr + (VD_EFX(ns) + D) * cs]);
    const double nel = p[ol + eidx * cs], ner = p[orr + eidx * cs];
    const double ne = 0.5 * (nel + ner);
    const double ef = a.cs_technique ? evf_d : a.ef[D](g[0], g[1], g[2]);
    const double gn = a.gradne_from_state ? (ner - nel) / a.dx[D] : a.gne[D](g[0], g[1], g[2]);
    const double ndens = 0.5 * (a.Nv.p[a.Nv.off(l[0], l[1], l[2])] + a.Nv.p[a.Nv.off(g[0], g[1], g[2])]);
    double emag = 0.0;
    if (c_mech.emag_e) emag = face_emag(a, ol, orr, dim);
    double mu, dc;
    if (a.const_ele_trans) {
        mu = a.ele_mob / ndens;
        dc = a.ele_diff / ndens;
    } else {
        mu = mob_fp64(eidx, etemp, ndens, a.Tg, emag);
        // the usual electron diffusion model refers to the electron mobility itself
        if (c_mech.diff_kind[eidx] == VD_DIFF_TE_ABSMOB && c_mech.diff_ref[eidx] == eidx)
            dc = c_mech.diff_factor[eidx] * (etemp / EV) * fabs(mu);
        else
            dc = diff_fp64(eidx, etemp, ndens, a.Tg, emag);
    }
    const double cur = a.charge_e * (mu * ne * ef - dc * gn);
    return cur * ef;
}

// the arithmetic of joule_face_mixed from the face's Te and density-sum averages,
// the two cells' ne, the face field and the density gradient
__device__ __forceinline__ double joule_mixed_core(const TransportArgs& a, float etemp, float ndens, double nel,
                                                   double ner, double ef, double gn, float emag)
{
    const int eidx = a.e_id;
    const float Tg = (float)a.Tg;
    float mu, dc;
    if (a.const_ele_trans) {
        const float rn = rcp_approx(ndens);
        mu = (float)a.ele_mob * rn;
        dc = (float)a.ele_diff * rn;
    } else {
        mu = mob_f32(eidx, etemp, ndens, Tg, emag);
        dc = diff_f32(eidx, etemp, ndens, Tg, emag, mu);
    }
    const double drift = (double)(mu * (float)(0.5 * (nel + ner)) * (float)ef);
    const double diffusion = (double)(dc * (float)gn);
    return a.charge_e * (drift - diffusion) * ef;
}

// joule_face of the mixed path: the face averages, mobility, diffusion and the
// two current products (mu ne E_f and D grad ne) in FP32 on the special-function
// unit's reciprocal and square root, as for the drift fluxes; their difference,
// the charge and the product with E_f in FP64.
__device__ __forceinline__ double joule_face_mixed(const TransportArgs& a, int D, const int* g, int dim)
{
    const int ns = a.ns, eidx = a.e_id;
    int l[3] = {g[0], g[1], g[2]};
    l[D] -= 1;
    const int64_t ol = a.sb.off(l[0], l[1], l[2]);
    const int64_t orr = a.sb.off(g[0], g[1], g[2]);
    const double* p = a.sb.p;
    const int64_t cs = a.sb.ns;
    const float etemp = 0.5f * ((float)p[ol + VD_ETEMP(ns) * cs] + (float)p[orr + VD_ETEMP(ns) * cs]);
    const double nel = p[ol + eidx * cs], ner = p[orr + eidx * cs];
    const double ef = a.cs_technique ? 0.5 * (p[ol + (VD_EFX(ns) + D) * cs] + p[orr + (VD_EFX(ns) + D) * cs])
                                     : a.ef[D](g[0], g[1], g[2]);
    const double gn = a.gradne_from_state ? (ner - nel) * a.idx[D] : a.gne[D](g[0], g[1], g[2]);
    const float ndens = 0.5f * ((float)a.Nv.p[a.Nv.off(l[0], l[1], l[2])] + (float)a.Nv.p[a.Nv.off(g[0], g[1], g[2])]);
    const float emag = c_mech.emag_e ? (float)face_emag(a, ol, orr, dim) : 0.0f;
    return joule_mixed_core(a, etemp, ndens, nel, ner, ef, gn, emag);
}

// Joule term of every valid cell of tile `tile` (x fastest over the box's
// JouleTile tiles, joule_tile_count): half the sum of joule_face over the cell's
// 2 DIM faces, a domain face replaced by the next face inward
// (Source/ElecEnergySource.cpp:84-94), halved and floored at 0 when floor_jh
// (:153-162); stored in the EJH component of the output, the reference's
// diagnostic (:168), where the transport update of the cell reads it.  The mixed
// path evaluates the faces with joule_face_mixed, the FP64 path with joule_face.
// Each face of the tile is evaluated once, by the thread of the cell above it
// (the last cells of the tile also take the face above them); a domain face that
// the substitution never reads is skipped.  Every thread of the CTA must call it; sJ
// holds DIM * joule_face_box<DIM>() doubles, and its reads are finished when the
// function returns only after a barrier (callers that reuse it synchronise).
template <int DIM, int PREC>
__device__ __forceinline__ void joule_tile(const TransportArgs& a, int tile, double* sJ)
{
    using JT = JouleTile<DIM>;
    constexpr int T[3] = {JT::X, JT::Y, JT::Z};
    constexpr int FB0 = JT::X + 1, FB1 = JT::Y + (DIM > 1), FBOX = joule_face_box<DIM>();
    const int tid = threadIdx.x;
    const int nt0 = (a.hi[0] - a.lo[0] + JT::X) / JT::X, nt1 = (a.hi[1] - a.lo[1] + JT::Y) / JT::Y;
    const int tix = tile % nt0, tr = tile / nt0;
    const int tiy = tr % nt1, tiz = tr / nt1;
    const int c[3] = {tid % JT::X, (tid / JT::X) % JT::Y, tid / (JT::X * JT::Y)};
    const int org[3] = {a.lo[0] + tix * JT::X, a.lo[1] + tiy * JT::Y, a.lo[2] + tiz * JT::Z};
    const int g[3] = {org[0] + c[0], org[1] + c[1], org[2] + c[2]};
    const bool own = g[0] <= a.hi[0] && g[1] <= a.hi[1] && g[2] <= a.hi[2];
    if (own) {
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const bool last = c[d] == T[d] - 1 || g[d] == a.hi[d];
#pragma unroll
            for (int f = 0; f < 2; f++) {
                if (f == 1 && !last) break;
                const int fe = g[d] + f;
                // a domain face is read only when the domain is one cell wide
                const bool skip = (fe == a.domlo[d] || fe == a.domhi[d] + 1) && a.domhi[d] > a.domlo[d];
                int gf[3] = {g[0], g[1], g[2]};
                gf[d] = fe;
                int l[3] = {c[0], c[1], c[2]};
                l[d] += f;
                double jf = 0.0;
                if (!skip) jf = PREC == PREC_FP64 ? joule_face(a, d, gf, DIM) : joule_face_mixed(a, d, gf, DIM);
                sJ[d * FBOX + l[0] + FB0 * (l[1] + FB1 * l[2])] = jf;
            }
        }
    }
    __syncthreads();
    if (own) {
        double jheat = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
#pragma unroll
            for (int f = 0; f < 2; f++) {
                int fe = g[d] + f;
                if (fe == a.domlo[d]) fe += 1;
                if (fe == a.domhi[d] + 1) fe -= 1;
                int l[3] = {c[0], c[1], c[2]};
                l[d] += fe - g[d];
                jheat += sJ[d * FBOX + l[0] + FB0 * (l[1] + FB1 * l[2])];
            }
        }
        jheat *= 0.5;
        if (a.floor_jh && jheat < 0.0) jheat = 0.0;
        a.pn(g[0], g[1], g[2], VD_EJH(a.ns)) = jheat;
    }
}

template <int DIM, int PREC, class TS, int GRP>
constexpr size_t transport_smem_max() { return transport_smem<DIM, PREC, TS, GRP>(3); }

// global cell of staged position cc of direction D's line set; false when the
// position lies outside what the box's stencil may read (those stage as zero)
template <int DIM, int D, class TS>
__device__ __forceinline__ bool staged_cell(const TransportArgs& a, int cc, const int* org, int* g)
{
    using G = TileGeom<DIM, TS>;
    constexpr int E0 = G::template SE<D>(0), E1 = G::template SE<D>(1);
    int l[3];
    l[0] = cc % E0;
    l[1] = (cc / E0) % E1;
    l[2] = cc / (E0 * E1);
    g[0] = org[0] + l[0];
    g[1] = org[1] + l[1];
    g[2] = org[2] + l[2];
    g[D] -= 3;
    bool ok = (g[D] >= a.lo[D] - a.ghost) && (g[D] <= a.hi[D] + a.ghost);
#pragma unroll
    for (int e = 0; e < DIM; e++)
        if (e != D) ok = ok && (g[e] <= a.hi[e]);
    return ok;
}

// velocity bases of staged position cc of direction D: sB[k*STOT + cc] for slot k;
// so[cc]: the position's cell offset in the state (-1: stages as zero), read by
// every species group's staging
template <int DIM, int PREC, int D, class TS>
__device__ __forceinline__ bool stage_basis(const TransportArgs& a, int cc, const int* org,
                                            typename VelT<PREC>::T* sB, JStage js, bool jst, int* so)
{
    bool bad = false;  // a NaN or infinity in the position's E, Te or density sum
    using G = TileGeom<DIM, TS>;
    using VT = typename VelT<PREC>::T;
    int g[3];
    const bool ok = staged_cell<DIM, D, TS>(a, cc, org, g);
    VT b[3] = {VT(0), VT(0), VT(0)};
    double ne = 0.0, Te = 0.0, N = 0.0;
    so[cc] = ok ? (int)a.sb.off(g[0], g[1], g[2]) : -1;
    if (ok) {
        const int ns = a.ns;
        const int64_t cs = a.sb.ns;
        const double* p = a.sb.p + a.sb.off(g[0], g[1], g[2]);
        const double E = p[(VD_EFX(ns) + D) * cs];
        N = a.Nv(g[0], g[1], g[2]);
        Te = p[VD_ETEMP(ns) * cs];
        bad = !(isfinite(E) && isfinite(Te) && isfinite(N));
        if (joule_staged<DIM, PREC>() && jst) ne = p[a.e_id * cs];
        // |E| of the three state components, as compute_vel takes it
        // (Source/PlasmaChem.H:194-196), for the models in |E| and |E|/N
        double emag = 0.0;
        if (a.stage_emag) {
            const double ex = p[VD_EFX(ns) * cs], ey = p[VD_EFY(ns) * cs], ez = p[VD_EFZ(ns) * cs];
            emag = sqrt(ex * ex + ey * ey + ez * ez);
        }
        for (int k = 0; k < a.nb; k++) {
            const int kind = a.bkind[k];
            if constexpr (PREC == PREC_FP64) {
                if (kind == 0) b[k] = E / (sqrt(Te) * N);
                else if (kind == 1) b[k] = E / N;
                else if (kind == 2) b[k] = E;
                else b[k] = basis_field_fp64(kind, a.bfit[k], a.bpow[k], E, emag, N, Te);
            } else {
                const float Ef = (float)E, rN = rcp_approx((float)N);
                if (kind == 0) b[k] = Ef * rsqrtf((float)Te) * rN;
                else if (kind == 1) b[k] = Ef * rN;
                else if (kind == 2) b[k] = Ef;
                else b[k] = basis_field_f32(kind, a.bfit[k], (float)a.bpow[k], Ef, (float)emag, (float)N, (float)Te);
            }
        }
    }
    for (int k = 0; k < a.nb; k++) sB[k * G::STOT + cc] = b[k];
    if (joule_staged<DIM, PREC>() && jst) {
        js.ne[cc] = ne;
        js.te[cc] = (float)Te;
        js.nd[cc] = (float)N;
    }
    return bad;
}

// density of species s at staged position cc of direction D
template <int DIM, int PREC, int D, class TS>
__device__ __forceinline__ typename VelT<PREC>::T stage_density(const TransportArgs& a, int cc, int s,
                                                                  const int* org)
{
    using VT = typename VelT<PREC>::T;
    int g[3];
    if (!staged_cell<DIM, D, TS>(a, cc, org, g)) return VT(0);
    return (VT)a.sb.p[a.sb.off(g[0], g[1], g[2]) + (int64_t)s * a.sb.ns];
}

// ---------------------------------------------------------------------------
// Single faces (the mixed path).  Face info word of face f of the tile (faces of
// all directions in one index range, direction D from FOFF_D, x fastest), built
// once per tile: bits 0-15 the staged index of the face's first stencil cell (rel
// cell f_d - 3 + q has staged index f_d + q along d), bits 16-17 the direction,
// then whether the box updates the face and whether it is the low or high domain
// face of its direction.
constexpr int kFaceOk = 1 << 18, kFaceDomLo = 1 << 19, kFaceDomHi = 1 << 20;
template <int DIM, class TS>
__device__ __forceinline__ int face_info(const TransportArgs& a, int f, const int* org)
{
    using G = TileGeom<DIM, TS>;
    static_assert(G::STOT < (1 << 16), "staged index fits 16 bits");
    int D = 0, ff = f;
    if (DIM > 2 && f >= G::FOFF2) {
        D = 2;
        ff = f - G::FOFF2;
    } else if (DIM > 1 && f >= G::FOFF1) {
        D = 1;
        ff = f - G::FOFF1;
    }
    const int F0 = TS::X + (D == 0), F1 = TS::Y + (D == 1);
    const int l[3] = {ff % F0, (ff / F0) % F1, ff / (F0 * F1)};
    const int S0 = TS::X + (D == 0 ? 6 : 0), S1 = TS::Y + (D == 1 ? 6 : 0);
    const int soff = D == 0 ? 0 : (D == 1 ? G::SOFF1 : G::SOFF2);
    const int g[3] = {org[0] + l[0], org[1] + l[1], org[2] + l[2]};
    bool ok = g[D] <= a.hi[D] + 1;
#pragma unroll
    for (int e = 0; e < DIM; e++)
        if (e != D) ok = ok && (g[e] <= a.hi[e]);
    return (soff + l[0] + S0 * (l[1] + S1 * l[2])) | (D << 16) | (ok ? kFaceOk : 0) |
           (g[D] == a.domlo[D] ? kFaceDomLo : 0) | (g[D] == a.domhi[D] + 1 ? kFaceDomHi : 0);
}

// Flux of one species through the face with info word `info`: sU / sB the
// species' staged densities and velocity basis over all line sets (sB null: the
// user velocity of the face's direction), k its velocity constant, zm its
// zero-flux mask (TransportArgs::fl_zm); zero for a face the box does not update
// or where IHNEUBC holds (Source/compute_explicit_flux.H:200-326).  W5: the
// caller has checked hyp_order == 5 (the WENO loop then holds no low-order code).
template <int DIM, int PREC, class TS, bool W5>
__device__ __forceinline__ typename VelT<PREC>::T face_tab(const TransportArgs& a, int info, int zm,
                                                           const typename VelT<PREC>::T* sU,
                                                           const typename VelT<PREC>::T* sB,
                                                           typename VelT<PREC>::T k)
{
    using VT = typename VelT<PREC>::T;
    if (!(info & kFaceOk)) return VT(0);
    const int D = (info >> 16) & 3, base = info & 0xffff;
    const int STR = D == 0 ? 1 : (D == 1 ? TS::X : TS::X * TS::Y);
    if (!sB) k = (VT)a.uvel[D];
    VT u[6], v[6];
#pragma unroll
    for (int q = 0; q < 6; q++) {
        u[q] = sU[base + q * STR];
        v[q] = sB ? k * sB[base + q * STR] : k;
    }
    VT F;
    if constexpr (PREC == PREC_FP64) F = face_flux_fp64(u, v, W5 ? 5 : a.hyp_order, a.weno, a.dxmin, a.dt);
    else F = face_flux_mixed32(u, v, W5 ? 5 : a.hyp_order, a.weno, a.dxmin, a.dt);
    if (((info & kFaceDomLo) && ((zm >> D) & 1)) || ((info & kFaceDomHi) && ((zm >> (3 + D)) & 1))) F = VT(0);
    return F;
}

// ---------------------------------------------------------------------------
// Runs of faces.  The faces of the tile along a line of direction D (T_D + 1 of
// them) are taken in runs of up to RUN consecutive faces; one thread computes a
// run: it loads the run's RUN + 5 stencil cells once, evaluates the WENO
// smoothness indicators and nonlinear weights once per cell centre
// (weno_center_*) and the candidate polynomials once per face, so that adjacent
// faces and the two reconstructions of a centre share them.
// Run info of run r (RunGeom numbering: direction, then line, then the segment
// along the line), built once per tile.
//   x: bits 0-15 staged index of the first stencil cell of the run's first face
//      (the staged index of rel cell f_d - 3 + q is f_d + q along d), bits 16-17
//      the direction, bits 18-23 the number of faces nf, bits 24-29 one plus the
//      position in the run of the high domain face (0: none);
//   y: bits 0-15 tile face index of the first face (faces of direction D from
//      FOFF_D, x fastest), bits
//      16-21 the number of leading faces the box updates (the others lie beyond
//      the box), bits 22-27 one plus the position of the low domain face.
template <int DIM, class TS, int RUN>
__device__ __forceinline__ int2 run_info(const TransportArgs& a, int r, const int* org)
{
    using G = TileGeom<DIM, TS>;
    using RG = RunGeom<DIM, TS, RUN>;
    static_assert(G::FTOT < (1 << 16), "face index fits 16 bits");
    int D = 0;
    if (DIM > 2 && r >= RG::ROFF2) {
        D = 2;
        r -= RG::ROFF2;
    } else if (DIM > 1 && r >= RG::ROFF1) {
        D = 1;
        r -= RG::ROFF1;
    }
    const int nr = D == 0 ? RG::NR(0) : (D == 1 ? RG::NR(1) : RG::NR(2));
    const int line = r / nr, seg = r - line * nr;
    const int TD = D == 0 ? TS::X : (D == 1 ? TS::Y : TS::Z);
    const int f0 = seg * RUN;
    const int nf = min(RUN, TD + 1 - f0);
    int l[3];  // local coordinates of the run's first face
    if (D == 0) {
        l[0] = f0;
        l[1] = line % TS::Y;
        l[2] = line / TS::Y;
    } else if (D == 1) {
        l[0] = line % TS::X;
        l[1] = f0;
        l[2] = line / TS::X;
    } else {
        l[0] = line % TS::X;
        l[1] = line / TS::X;
        l[2] = f0;
    }
    const int S0 = TS::X + (D == 0 ? 6 : 0), S1 = TS::Y + (D == 1 ? 6 : 0);
    const int soff = D == 0 ? 0 : (D == 1 ? G::SOFF1 : G::SOFF2);
    const int F0 = TS::X + (D == 0), F1 = TS::Y + (D == 1);
    const int foff = D == 0 ? 0 : (D == 1 ? G::FOFF1 : G::FOFF2);
    bool line_ok = true;
#pragma unroll
    for (int e = 0; e < DIM; e++)
        if (e != D) line_ok = line_ok && (org[e] + l[e] <= a.hi[e]);
    const int g0 = org[D] + f0;  // global index of the first face
    const int nok = line_ok ? max(0, min(nf, a.hi[D] + 2 - g0)) : 0;
    const int ilo = a.domlo[D] - g0, ihi = a.domhi[D] + 1 - g0;
    int2 w;
    w.x = (soff + l[0] + S0 * (l[1] + S1 * l[2])) | (D << 16) | (nf << 18) |
          ((ihi >= 0 && ihi < nf) ? (ihi + 1) << 24 : 0);
    w.y = (foff + l[0] + F0 * (l[1] + F1 * l[2])) | (nok << 16) | ((ilo >= 0 && ilo < nf) ? (ilo + 1) << 22 : 0);
    return w;
}

// The faces of one run for one species: sU / sB the species' staged densities and
// velocity basis over all line sets (sB null: the user velocity of the run's
// direction), k its velocity constant, zm its zero-flux mask
// (TransportArgs::fl_zm); writes the nf face fluxes to sF (tile face numbering),
// zero where the box updates no face or IHNEUBC holds
// (Source/compute_explicit_flux.H:200-326).
template <int DIM, int PREC, class TS, int RUN, bool W5>
__device__ __forceinline__ void run_faces(const TransportArgs& a, int2 ri, int zm,
                                          const typename VelT<PREC>::T* __restrict__ sU,
                                          const typename VelT<PREC>::T* __restrict__ sB,
                                          typename VelT<PREC>::T k, typename VelT<PREC>::T* sF)
{
    using VT = typename VelT<PREC>::T;
    constexpr int NC = RUN + 5;
    const int base = ri.x & 0xffff, D = (ri.x >> 16) & 3, nf = (ri.x >> 18) & 63;
    const int ihi = ((ri.x >> 24) & 63) - 1;
    const int fbase = ri.y & 0xffff, nok = (ri.y >> 16) & 63, ilo = ((ri.y >> 22) & 63) - 1;
    const int STR = D == 0 ? 1 : (D == 1 ? TS::X : TS::X * TS::Y);  // staged and face stride along D
    const bool zlo = (zm >> D) & 1, zhi = (zm >> (3 + D)) & 1;
    if (!sB) k = (VT)a.uvel[D];
    auto store = [&](int i, VT F) {
        if (i >= nok || (i == ilo && zlo) || (i == ihi && zhi)) F = VT(0);
        sF[fbase + i * STR] = F;
    };
    if constexpr (!W5) {
        // upwind / WAF: FP64 arithmetic on the face's own stencil
        for (int i = 0; i < nf; i++) {
            double ud[6], vd[6];
#pragma unroll
            for (int q = 0; q < 6; q++) {
                ud[q] = (double)sU[base + (i + q) * STR];
                vd[q] = (double)(sB ? k * sB[base + (i + q) * STR] : k);
            }
            store(i, (VT)face_flux_low(ud, vd, a.hyp_order, a.weno, a.dxmin, a.dt));
        }
        return;
    }
    // one field at a time (the densities u, then the drift fluxes f = u v), so that
    // only one field's run of cells is live; face i lies between centres i+2 (left)
    // and i+3 (right)
    static_assert(PREC == PREC_FP64, "runs of faces serve the FP64 path");
    const int scheme = a.weno;
    double w[NC];
#pragma unroll
    for (int i = 0; i < NC; i++) w[i] = i < nf + 5 ? (double)sU[base + i * STR] : 0.0;
    // the reconstructions of the field in w at each face of the run, handed to
    // emit(i, left-biased value, right-biased value) as they are made
    auto recon = [&](auto&& emit) {
        WenoY64 yl = weno_center_fp64(w[0], w[1], w[2], w[3], w[4], scheme);
#pragma unroll
        for (int i = 0; i < RUN; i++) {
            if (i >= nf) break;
            const WenoY64 yr = weno_center_fp64(w[i + 1], w[i + 2], w[i + 3], w[i + 4], w[i + 5], scheme);
            const double p2 = wpoly_mid(w[i + 1], w[i + 2], w[i + 3]), p3 = wpoly_near(w[i + 2], w[i + 3], w[i + 4]);
            emit(i, weno_combine_fp64(yl.y1, yl.y2, yl.y3, wpoly_end(w[i], w[i + 1], w[i + 2]), p2, p3, scheme),
                 weno_combine_fp64(yr.y3, yr.y2, yr.y1, wpoly_end(w[i + 5], w[i + 4], w[i + 3]), p3, p2, scheme));
            yl = yr;
        }
    };
    auto vel = [&](int i) -> double { return (double)(sB ? k * sB[base + i * STR] : k); };
    double up[RUN], um[RUN];
    recon([&](int i, double pl, double mi) {
        up[i] = pl;
        um[i] = mi;
    });
#pragma unroll
    for (int i = 0; i < NC; i++) w[i] *= i < nf + 5 ? vel(i) : 0.0;
    // the drift fluxes' reconstructions go straight into the face flux (the face's
    // |v| from the two cells' velocities, reloaded from shared memory)
    recon([&](int i, double fp, double fm) {
        const double l = fabs(0.5 * (vel(i + 2) + vel(i + 3)));
        store(i, (VT)fma(0.5, fma(l, up[i], fp), 0.5 * fma(-l, um[i], fm)));
    });
}

// Update tile `tile` (index over a.ntile) of the box described by a.  Every thread
// of the CTA must call it; it returns with all shared memory reads finished
// except those of the last group's divergence (callers that reuse the shared
// memory for another tile synchronise first).
template <int DIM, int PREC, class TS, int GRP>
__device__ __forceinline__ void transport_tile_update(const TransportArgs& a, int tile, unsigned char* smem)
{
    using G = TileGeom<DIM, TS>;
    using VT = typename VelT<PREC>::T;
    constexpr int NTH = TS::NTH;
    const int tid = threadIdx.x;
    int tb = tile;
    const int tix = tb % a.ntile[0];
    tb /= a.ntile[0];
    const int tiy = tb % a.ntile[1];
    const int tiz = tb / a.ntile[1];
    const int org[3] = {a.lo[0] + tix * G::T[0], a.lo[1] + tiy * G::T[1], a.lo[2] + tiz * G::T[2]};
    using SM = TileSmem<DIM, PREC, TS>;
    constexpr int RUN = run_len<DIM, TS>();
    using RG = RunGeom<DIM, TS, RUN>;
    double* sJ = reinterpret_cast<double*>(smem);  // mixed path only
    int2* sRI = reinterpret_cast<int2*>(smem + SM::joule());  // by_runs
    int* sFI = reinterpret_cast<int*>(smem + SM::joule());    // single faces
    int* sSO = reinterpret_cast<int*>(smem + SM::joule() + SM::finfo());
    const size_t o_f = SM::joule() + SM::finfo() + SM::soffs();
    VT* sF = reinterpret_cast<VT*>(smem + o_f);
    VT* sB = reinterpret_cast<VT*>(smem + o_f + SM::flux(GRP));
    unsigned char* const dens = smem + o_f + SM::flux(GRP) + SM::basis(a.nb);
    // staged positions by table when every cell offset of the state fits 32 bits
    const bool stab = a.sb.ns <= 0x7fffffffLL;
    VT* sU = reinterpret_cast<VT*>(dens);
    // the staged Joule inputs share the densities' space: read in phase (0'),
    // before a barrier that precedes the first group's staging
    const JStage js{reinterpret_cast<double*>(dens), reinterpret_cast<float*>(dens + G::STOT * sizeof(double)),
                    reinterpret_cast<float*>(dens + G::STOT * (sizeof(double) + sizeof(float)))};

    // own cell
    const int cx = tid % G::T[0], cy = (tid / G::T[0]) % G::T[1], cz = tid / (G::T[0] * G::T[1]);
    const int gi = org[0] + cx, gj = org[1] + cy, gk = org[2] + cz;
    const bool own = (tid < G::NCELL) && gi <= a.hi[0] && gj <= a.hi[1] && gk <= a.hi[2];
    const int ns = a.ns;
    const int64_t cs = a.sb.ns;
    const int64_t own_o = own ? a.sb.off(gi, gj, gk) : 0;
    // The own cell's state and reaction source are read-only in this kernel (the
    // update goes to a.pn): read through the non-coherent path, so that these
    // loads may be issued ahead of the cell's stores.
    const int64_t own_r = own ? a.rxn.off(gi, gj, gk) : 0;
    auto state = [&](int s) -> double { return __ldg(a.sb.p + own_o + s * cs); };
    auto rate = [&](int s) -> double { return __ldg(a.rxn.p + own_r + s * a.rxn.ns); };
    double ne_new = 0.0, een_new = 0.0;
    bool bad = false;  // this thread met a NaN or infinity (reported once per warp at the end)
    const int nfl = a.nfl;
    // the mixed path's Joule faces, evaluated here (a barrier follows them)
    const bool jin = joule_in_tile(a, PREC);

    // Joule term of the own cell from the tile's faces: half the sum of its faces,
    // each domain face replaced as the reference does
    // (Source/ElecEnergySource.cpp:84-94,153-162)
    auto joule_own = [&]() -> double {
        const int gc[3] = {gi, gj, gk}, lc[3] = {cx, cy, cz};
        double jheat = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const int foff = d == 0 ? 0 : (d == 1 ? G::FOFF1 : G::FOFF2);
            const int F0 = G::T[0] + (d == 0), F1 = G::T[1] + (d == 1);
            const int str = d == 0 ? 1 : (d == 1 ? F0 : F0 * F1);
            const int base = foff + lc[0] + F0 * (lc[1] + F1 * lc[2]);
#pragma unroll
            for (int f = 0; f < 2; f++) {
                int fe = gc[d] + f;
                if (fe == a.domlo[d]) fe += 1;
                if (fe == a.domhi[d] + 1) fe -= 1;
                jheat += sJ[base + (fe - gc[d]) * str];
            }
        }
        jheat *= 0.5;
        if (a.floor_jh && jheat < 0.0) jheat = 0.0;
        return jheat;
    };

    // one species' own-cell result
    // (st: the species' old value, state(s), loaded by the caller so that several
    // species' loads can be in flight together)
    auto finish = [&](int s, double acc, double st) {
        if (s == ns) {
            if (jin) {
                const double jh = joule_own();
                acc += jh;
                a.pn(gi, gj, gk, VD_EJH(ns)) = jh;
            } else {
                // the Joule term the joule_tile pass left in EJH
                acc += a.pn(gi, gj, gk, VD_EJH(ns));
            }
            if (a.write_diag) a.pn(gi, gj, gk, VD_EIH(ns)) = rate(ns);
        }
        double nn = st + a.dt * acc;
        if (a.bound_specden && s != ns) {
            // solution clipping of the species solve (Source/ScalarSolve.cpp:597-622)
            const double lo = (s == a.e_id) ? a.min_elec : a.min_spec;
            if (nn < lo) nn = lo;
        }
        bad |= !isfinite(nn);
        a.pn(gi, gj, gk, s) = nn;
        if (a.dsdt.p) a.dsdt(gi, gj, gk, s) = acc;
        if (s == a.e_id) ne_new = nn;
        if (s == ns) een_new = nn;
    };

    if (nfl > 0) {
        // (0) run or face info words and the velocity bases of every staged position
        if constexpr (by_runs<DIM, PREC>()) {
            for (int r = tid; r < RG::NRUN; r += NTH) sRI[r] = run_info<DIM, TS, RUN>(a, r, org);
        } else {
            for (int f = tid; f < G::FTOT; f += NTH) sFI[f] = face_info<DIM, TS>(a, f, org);
        }
        if constexpr (PREC == PREC_MIXED) {
            // one loop per direction's line set, two positions per iteration, so
            // that the loads of both positions are in flight together (measured
            // faster for the mixed tile, slower for the FP64 one, whose positions
            // then split less evenly over the threads)
            auto bases = [&](auto dtag) {
                constexpr int D = decltype(dtag)::value;
                constexpr int off = D == 0 ? 0 : (D == 1 ? G::SOFF1 : G::SOFF2);
                const JStage jd{js.ne + off, js.te + off, js.nd + off};
#pragma unroll 2
                for (int cc = tid; cc < G::template NS<D>(); cc += NTH)
                    bad |= stage_basis<DIM, PREC, D, TS>(a, cc, org, sB + off, jd, jin, sSO + off);
            };
            bases(std::integral_constant<int, 0>{});
            if constexpr (DIM > 1) bases(std::integral_constant<int, 1>{});
            if constexpr (DIM > 2) bases(std::integral_constant<int, 2>{});
        } else {
            for (int c = tid; c < G::STOT; c += NTH) {
                if (c < G::SOFF1) {
                    bad |= stage_basis<DIM, PREC, 0, TS>(a, c, org, sB, js, jin, sSO);
                } else if (DIM > 1 && c < G::SOFF2) {
                    const JStage j1{js.ne + G::SOFF1, js.te + G::SOFF1, js.nd + G::SOFF1};
                    bad |= stage_basis<DIM, PREC, (DIM > 1 ? 1 : 0), TS>(a, c - G::SOFF1, org, sB + G::SOFF1, j1,
                                                                         jin, sSO + G::SOFF1);
                } else if (DIM > 2) {
                    const JStage j2{js.ne + G::SOFF2, js.te + G::SOFF2, js.nd + G::SOFF2};
                    bad |= stage_basis<DIM, PREC, (DIM > 2 ? 2 : 0), TS>(a, c - G::SOFF2, org, sB + G::SOFF2, j2,
                                                                         jin, sSO + G::SOFF2);
                }
            }
        }
        // the offset table and the staged Joule inputs are read by other threads
        if (stab || (joule_staged<DIM, PREC>() && jin)) __syncthreads();
    }
    if constexpr (PREC == PREC_MIXED) {
        if (jin) {
            // (0') the Joule term of every face of the tile, once (from the staged
            // inputs of the face's two cells when they are staged, which the basis
            // loop above wrote before its barrier)
            for (int f = tid; f < G::FTOT; f += NTH) {
                int d = 0, ff = f;
                if (DIM > 1 && f >= G::FOFF1) {
                    d = (DIM > 2 && f >= G::FOFF2) ? 2 : 1;
                    ff = f - (d == 1 ? G::FOFF1 : G::FOFF2);
                }
                const int F0 = G::T[0] + (d == 0), F1 = G::T[1] + (d == 1);
                int g[3] = {org[0] + ff % F0, org[1] + (ff / F0) % F1, org[2] + ff / (F0 * F1)};
                bool ok = g[d] <= a.hi[d] + 1;
                for (int e = 0; e < DIM; e++)
                    if (e != d) ok = ok && g[e] <= a.hi[e];
                double jf = 0.0;
                // a field-dependent electron mobility needs the face's |E|: global reads
                if (joule_staged<DIM, PREC>() && !c_mech.emag_e) {
                    if (ok) {
                        // staged index of the face's rel cell (f_d - 3 + q) is f_d + q
                        // along d: the cells below and above are q = 2 and 3
                        const int S0 = G::T[0] + (d == 0 ? 6 : 0), S1 = G::T[1] + (d == 1 ? 6 : 0);
                        const int STR = d == 0 ? 1 : (d == 1 ? S0 : S0 * S1);
                        const int soff = d == 0 ? 0 : (d == 1 ? G::SOFF1 : G::SOFF2);
                        const int l0 = ff % F0, l1 = (ff / F0) % F1, l2 = ff / (F0 * F1);
                        const int pl = soff + l0 + S0 * (l1 + S1 * l2) + 2 * STR, pr = pl + STR;
                        const double nel = js.ne[pl], ner = js.ne[pr];
                        double ef;
                        if (a.cs_technique) {
                            int gl[3] = {g[0], g[1], g[2]};
                            gl[d] -= 1;
                            const int64_t cs = a.sb.ns, ce = (VD_EFX(ns) + d) * cs;
                            ef = 0.5 * (a.sb.p[a.sb.off(gl[0], gl[1], gl[2]) + ce] + a.sb.p[a.sb.off(g[0], g[1], g[2]) + ce]);
                        } else {
                            ef = a.ef[d](g[0], g[1], g[2]);
                        }
                        const double gn = a.gradne_from_state ? (ner - nel) * a.idx[d] : a.gne[d](g[0], g[1], g[2]);
                        jf = joule_mixed_core(a, 0.5f * (js.te[pl] + js.te[pr]), 0.5f * (js.nd[pl] + js.nd[pr]), nel,
                                              ner, ef, gn, 0.0f);
                    }
                } else {
                    if (ok) jf = joule_face_mixed(a, d, g, DIM);
                }
                sJ[f] = jf;
            }
            // the first group's staging overwrites the staged Joule inputs
            if constexpr (joule_staged<DIM, PREC>()) __syncthreads();
        }
    }
    for (int g0 = 0; g0 < nfl; g0 += GRP) {
        const int gn = nfl - g0 < GRP ? nfl - g0 : GRP;
        // (1) densities of the group on the staged lines
        if (stab) {
            // four positions per thread at a time: their loads in flight together
            constexpr int CH = 4;
            const int tot = gn * G::STOT;
            for (int q0 = tid; q0 < tot; q0 += CH * NTH) {
                VT u[CH];
#pragma unroll
                for (int k = 0; k < CH; k++) {
                    const int q = q0 + k * NTH;
                    u[k] = VT(0);
                    if (q < tot) {
                        const int j = q / G::STOT, c = q - j * G::STOT;
                        const int o = sSO[c];
                        if (o >= 0) u[k] = (VT)__ldg(a.sb.p + o + (int64_t)a.fl_sp[g0 + j] * cs);
                    }
                }
#pragma unroll
                for (int k = 0; k < CH; k++)
                    if (q0 + k * NTH < tot) sU[q0 + k * NTH] = u[k];
            }
        } else for (int q = tid; q < gn * G::STOT; q += NTH) {
            const int j = q / G::STOT, c = q - j * G::STOT;
            const int s = a.fl_sp[g0 + j];
            VT u;
            if (c < G::SOFF1) {
                u = stage_density<DIM, PREC, 0, TS>(a, c, s, org);
            } else if (DIM > 1 && c < G::SOFF2) {
                u = stage_density<DIM, PREC, (DIM > 1 ? 1 : 0), TS>(a, c - G::SOFF1, s, org);
            } else {
                u = stage_density<DIM, PREC, (DIM > 2 ? 2 : 0), TS>(a, c - G::SOFF2, s, org);
            }
            sU[q] = u;
        }
        __syncthreads();
        // (2) every face flux of the group: by runs of faces along the lines, or
        // face by face
        // face by face; one loop per scheme family, so that the WENO loop carries
        // no low-order code
        auto runs = [&](auto w5) {
            for (int q = tid; q < gn * RG::NRUN; q += NTH) {
                const int j = q / RG::NRUN, r = q - j * RG::NRUN;
                const int sl = a.fl_slot[g0 + j];
                run_faces<DIM, PREC, TS, RUN, decltype(w5)::value>(a, sRI[r], a.fl_zm[g0 + j], sU + j * G::STOT,
                                                                   sl >= 0 ? sB + sl * G::STOT : nullptr,
                                                                   (VT)a.fl_K[g0 + j], sF + j * G::FTOT);
            }
        };
        auto faces = [&](auto w5) {
            for (int q = tid; q < gn * G::FTOT; q += NTH) {
                const int j = q / G::FTOT, f = q - j * G::FTOT;
                const int sl = a.fl_slot[g0 + j];
                sF[q] = face_tab<DIM, PREC, TS, decltype(w5)::value>(a, sFI[f], a.fl_zm[g0 + j], sU + j * G::STOT,
                                                                     sl >= 0 ? sB + sl * G::STOT : nullptr,
                                                                     (VT)a.fl_Kf[g0 + j]);
            }
        };
        if constexpr (by_runs<DIM, PREC>()) {
            if (a.hyp_order == 5) runs(std::true_type{});
            else runs(std::false_type{});
        } else {
            if (a.hyp_order == 5) faces(std::true_type{});
            else faces(std::false_type{});
        }
        __syncthreads();
        // (3) divergence + sources of the own cell: dsdt = (Fx_lo - Fx_hi)/dx + rxn,
        // then += y and z terms (Source/ScalarSolve.cpp:45-51)
        if (own) {
            // the own cell's dsdt of species j of the group, with its rate r, in the
            // reference's order: x faces + rate, then y, then z
            // (Source/ScalarSolve.cpp:45-51)
            auto divergence = [&](int j, double r) -> double {
                const VT* Fj = sF + j * G::FTOT;
                double acc;
                {
                    constexpr int F0 = G::template FE<0>(0), F1 = G::template FE<0>(1);
                    const int lo_f = cx + F0 * (cy + F1 * cz);
                    acc = ((double)Fj[lo_f] - (double)Fj[lo_f + 1]) * a.idx[0] + r;
                }
                if constexpr (DIM > 1) {
                    constexpr int F0 = G::template FE<1>(0), F1 = G::template FE<1>(1);
                    const int lo_f = G::FOFF1 + cx + F0 * (cy + F1 * cz);
                    acc += ((double)Fj[lo_f] - (double)Fj[lo_f + F0]) * a.idx[1];
                }
                if constexpr (DIM > 2) {
                    constexpr int F0 = G::template FE<2>(0), F1 = G::template FE<2>(1);
                    const int lo_f = G::FOFF2 + cx + F0 * (cy + F1 * cz);
                    acc += ((double)Fj[lo_f] - (double)Fj[lo_f + F0 * F1]) * a.idx[2];
                }
                return acc;
            };
            // two species at a time: their four loads in flight together
#pragma unroll 1
            for (int j = 0; j < gn; j += 2) {
                const bool two = j + 1 < gn;
                const int s0 = a.fl_sp[g0 + j], s1 = two ? a.fl_sp[g0 + j + 1] : s0;
                const double r0 = rate(s0), r1 = rate(s1), st0 = state(s0), st1 = state(s1);
                finish(s0, divergence(j, r0), st0);
                if (two) finish(s1, divergence(j + 1, r1), st1);
            }
        }
        // the next group's staging overwrites sU only after every thread has passed
        // the barrier above; sF is rewritten only after the next staging barrier,
        // by which time every divergence read of this group is done
    }
    if (own) {
        // four species at a time: their loads in flight together
        constexpr int CH = 4;
#pragma unroll 1
        for (int j0 = 0; j0 < a.nnf; j0 += CH) {
            double r[CH], st[CH];
#pragma unroll
            for (int k = 0; k < CH; k++) {
                const int s = a.nf_sp[j0 + k < a.nnf ? j0 + k : a.nnf - 1];
                r[k] = rate(s);
                st[k] = state(s);
            }
#pragma unroll
            for (int k = 0; k < CH; k++)
                if (j0 + k < a.nnf) finish(a.nf_sp[j0 + k], r[k], st[k]);
        }
#pragma unroll 1
        for (int j0 = 0; j0 < a.nbg; j0 += CH) {
            double r[CH], v[CH];
#pragma unroll
            for (int k = 0; k < CH; k++) {
                const int s = a.bg_sp[j0 + k < a.nbg ? j0 + k : a.nbg - 1];
                r[k] = rate(s);
                v[k] = state(s);
            }
#pragma unroll
            for (int k = 0; k < CH; k++) {
                if (j0 + k >= a.nbg) continue;
                const int s = a.bg_sp[j0 + k];
                if (a.do_bg) {
                    v[k] += r[k] * a.dt;
                    if (v[k] < a.min_spec && a.bound_specden) v[k] = a.min_spec;
                }
                bad |= !isfinite(v[k]);
                a.pn(gi, gj, gk, s) = v[k];
                if (a.dsdt.p) a.dsdt(gi, gj, gk, s) = r[k];
            }
        }
        if (a.update_te && a.elecenergy) {
            // Source/ScalarSolve.cpp:659-666
            double te = (2.0 / 3.0) / K_B * een_new / state(a.e_id);
            if (te < a.min_te) {
                te = a.min_te;
                a.pn(gi, gj, gk, VD_EEN(ns)) = 1.5 * K_B * ne_new * te;
            }
            a.pn(gi, gj, gk, VD_ETEMP(ns)) = te;
        }
    }
    if (a.status) {  // uniform over the CTA; every lane of every warp reaches it
        const unsigned any = __ballot_sync(0xffffffffu, bad);
        if (any && (threadIdx.x & 31) == 0) atomicOr(a.status, 1u);
    }
}

// per-box kernel: one CTA per tile
template <int DIM, int PREC, int MINB>
__global__ void __launch_bounds__(default_nth<DIM>(), MINB) k_transport(const __grid_constant__ TransportArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using TS = typename DefaultTile<DIM>::T;
    transport_tile_update<DIM, PREC, TS, group_fit<DIM, PREC, TS, MINB>()>(a, blockIdx.x, smem_raw);
}

// batched persistent kernel: each CTA walks the work list of (box, tile) items
// with a grid stride.  Boxes are described by TransportArgs records in global
// memory; an item's record is copied to shared memory, so that the tile body's
// many reads of it are shared-memory loads rather than global ones.  Two record
// buffers: while a tile is updated, the next item's record (when it is another
// box's) is fetched into the other buffer with asynchronous copies.
template <int DIM, int PREC, class TS, int MINB, int GMAX>
__global__ void __launch_bounds__(TS::NTH, MINB)
    k_transport_batch(const TransportArgs* __restrict__ boxes, const int2* __restrict__ items, int nitems,
                      const BatchCtl ctl)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NW = (int)(sizeof(TransportArgs) / 8);
    static_assert(sizeof(TransportArgs) % 8 == 0, "record copied in 8-byte words");
    __shared__ __align__(16) long long sA_raw[2][NW];
    // record index of item it, or -1 when its box takes no step now (the same for
    // every thread of the CTA)
    auto record_of = [&](int it, int2& w) -> int {
        w = items[it];
        const int2 cc = ctl.ctrl[w.x];
        return ctl.t >= cc.x ? -1 : ((ctl.t + cc.y) & 1) * ctl.nbox + w.x;
    };
    auto fetch = [&](int buf, int rec) {
        const long long* src = reinterpret_cast<const long long*>(boxes + rec);
        for (int q = threadIdx.x; q < NW; q += TS::NTH) {
            const unsigned dst = (unsigned)__cvta_generic_to_shared(&sA_raw[buf][q]);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src + q) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    int2 w;
    int it = blockIdx.x, rec = -1;
    while (it < nitems && (rec = record_of(it, w)) < 0) it += gridDim.x;
    if (it >= nitems) return;
    int held0 = rec, held1 = -1, b = 0;  // record in each buffer; buffer of the current item
    fetch(0, rec);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    for (;;) {
        // the next item of this CTA; its record goes to the other buffer now (that
        // buffer was last read by the previous tile, before its barrier)
        int itn = it + gridDim.x;
        {
            int2 wn;
            int recn = -1;
            while (itn < nitems && (recn = record_of(itn, wn)) < 0) itn += gridDim.x;
            const int hb = b ? held1 : held0, ho = b ? held0 : held1;
            if (itn < nitems && recn != hb && recn != ho) {
                fetch(b ^ 1, recn);
                if (b) held0 = recn;
                else held1 = recn;
            }
        }
        transport_tile_update<DIM, PREC, TS, group_fit<DIM, PREC, TS, MINB, GMAX>()>(
            *reinterpret_cast<const TransportArgs*>(sA_raw[b]), w.y, smem_raw);
        if (itn >= nitems) break;
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        __syncthreads();  // the record is complete; the next staging may overwrite this tile's shared memory
        it = itn;
        rec = record_of(it, w);
        if (rec != (b ? held1 : held0)) b ^= 1;
    }
}

}  // namespace vd
