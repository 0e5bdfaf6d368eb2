// vd_transport.cuh -- the fused transport update of one tile (included by vd_kernels.cu).
//
// One CTA updates a TX x TY x TZ tile of one box.  Per transported species:
// (1) stage the stencil lines of every sweep direction in shared memory -- for
//     direction d the cells rel -3 .. T_d+2 along d of each tile row, with the
//     density and the drift velocity mu(Te, N) E_d computed once per staged cell;
// (2) compute every face flux of the tile once (all directions in one pass,
//     faces spread evenly over the threads);
// (3) each thread takes the divergence of its own cell, adds rxn (and the Joule
//     term for the electron energy) and writes n + dt*dsdt in FP64.
// Two barriers per species.  The tile body is a device function so that the
// per-box kernel (one CTA per tile) and the batched persistent kernel (CTAs loop
// over a work list of (box, tile) items of many boxes) share it.
#pragma once

namespace vd {

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

template <int PREC> struct VelT { using T = double; };
template <> struct VelT<PREC_MIXED> { using T = float; };

// dynamic shared memory of one tile: face fluxes (FP64), staged densities and
// velocities (FP32 in the mixed path)
template <int DIM, int PREC, class TS>
constexpr size_t transport_smem()
{
    using G = TileGeom<DIM, TS>;
    return (size_t)G::FTOT * sizeof(double) + (size_t)G::STOT * 2 * sizeof(typename VelT<PREC>::T);
}

// stage staged-cell cc of direction D's line set: density and drift velocity
template <int DIM, int PREC, int D, class TS>
__device__ __forceinline__ void stage_cell(const TransportArgs& a, int cc, int s, const int* org,
                                           typename VelT<PREC>::T* sU, typename VelT<PREC>::T* sV)
{
    using G = TileGeom<DIM, TS>;
    using VT = typename VelT<PREC>::T;
    constexpr int E0 = G::template SE<D>(0), E1 = G::template SE<D>(1);
    int l[3];
    l[0] = cc % E0;
    l[1] = (cc / E0) % E1;
    l[2] = cc / (E0 * E1);
    int g[3] = {org[0] + l[0], org[1] + l[1], org[2] + l[2]};
    g[D] -= 3;
    bool ok = (g[D] >= a.lo[D] - a.ghost) && (g[D] <= a.hi[D] + a.ghost);
#pragma unroll
    for (int e = 0; e < DIM; e++)
        if (e != D) ok = ok && (g[e] <= a.hi[e]);
    VT u = VT(0);
    VT v = VT(0);
    if (ok) {
        const int ns = a.ns;
        const int64_t cs = a.sb.ns;
        const double* p = a.sb.p + a.sb.off(g[0], g[1], g[2]);
        u = (VT)p[s * cs];
        if (a.udv) {
            v = (s == a.vel_sp) ? VT(a.uvel[D]) : VT(0);
        } else {
            const double Te = p[VD_ETEMP(ns) * cs];
            const double E = p[(VD_EFX(ns) + D) * cs];
            const double N = a.Nv(g[0], g[1], g[2]);
            if constexpr (PREC == PREC_FP64) v = mob_fp64(s, Te, N, a.Tg) * E;
            else v = mob_f32(s, (float)Te, (float)N, (float)a.Tg) * (float)E;
        }
    }
    sU[cc] = u;
    sV[cc] = v;
}

// flux of face ff of direction D from the staged lines
template <int DIM, int PREC, int D, class TS>
__device__ __forceinline__ double face_of(const TransportArgs& a, int ff, int cls, const int* org,
                                          const typename VelT<PREC>::T* sU, const typename VelT<PREC>::T* sV)
{
    using G = TileGeom<DIM, TS>;
    using VT = typename VelT<PREC>::T;
    constexpr int F0 = G::template FE<D>(0), F1 = G::template FE<D>(1);
    constexpr int S0 = G::template SE<D>(0), S1 = G::template SE<D>(1);
    constexpr int STR = (D == 0) ? 1 : ((D == 1) ? S0 : S0 * S1);
    int l[3];
    l[0] = ff % F0;
    l[1] = (ff / F0) % F1;
    l[2] = ff / (F0 * F1);
    int g[3] = {org[0] + l[0], org[1] + l[1], org[2] + l[2]};
    bool ok = g[D] <= a.hi[D] + 1;
#pragma unroll
    for (int e = 0; e < DIM; e++)
        if (e != D) ok = ok && (g[e] <= a.hi[e]);
    if (!ok) return 0.0;
    // staged index of rel cell (f_d - 3 + q) is f_d + q along d
    const int base = l[0] + S0 * (l[1] + S1 * l[2]);
    VT u[6];
    VT v[6];
#pragma unroll
    for (int q = 0; q < 6; q++) {
        u[q] = sU[base + q * STR];
        v[q] = sV[base + q * STR];
    }
    double F;
    if constexpr (PREC == PREC_FP64) F = face_flux_fp64(u, v, a.hyp_order, a.weno, a.dxmin, a.dt);
    else F = face_flux_mixed32(u, v, a.hyp_order, a.weno, a.dxmin, a.dt);
    if (g[D] == a.domlo[D] && a.zlo[cls][D]) F = 0.0;
    if (g[D] == a.domhi[D] + 1 && a.zhi[cls][D]) F = 0.0;
    return F;
}

// Update tile `tile` (index over a.ntile) of the box described by a.  Every thread
// of the CTA must call it; it returns with all shared memory reads finished.
template <int DIM, int PREC, class TS>
__device__ __forceinline__ void transport_tile_update(const TransportArgs& a, int tile, double* sF,
                                               typename VelT<PREC>::T* sU, typename VelT<PREC>::T* sV)
{
    using G = TileGeom<DIM, TS>;
    constexpr int NTH = TS::NTH;
    const int tid = threadIdx.x;
    int tb = tile;
    const int tix = tb % a.ntile[0];
    tb /= a.ntile[0];
    const int tiy = tb % a.ntile[1];
    const int tiz = tb / a.ntile[1];
    const int org[3] = {a.lo[0] + tix * G::T[0], a.lo[1] + tiy * G::T[1], a.lo[2] + tiz * G::T[2]};

    // own cell
    const int cx = tid % G::T[0], cy = (tid / G::T[0]) % G::T[1], cz = tid / (G::T[0] * G::T[1]);
    const int gi = org[0] + cx, gj = org[1] + cy, gk = org[2] + cz;
    const bool own = (tid < G::NCELL) && gi <= a.hi[0] && gj <= a.hi[1] && gk <= a.hi[2];
    const int ns = a.ns;
    const int64_t cs = a.sb.ns;
    const int64_t own_o = own ? a.sb.off(gi, gj, gk) : 0;

    double ne_new = 0.0, een_new = 0.0;
    const int ntr = a.ntr;
    for (int it = 0; it < ntr; it++) {
        const int s = a.tr_sp[it];
        const int cls = a.tr_cls[it];
        double acc = own ? a.rxn(gi, gj, gk, s) : 0.0;
        if (a.tr_flux[it]) {
            for (int c = tid; c < G::STOT; c += NTH) {
                if (c < G::SOFF1) stage_cell<DIM, PREC, 0, TS>(a, c, s, org, sU, sV);
                else if (DIM > 1 && c < G::SOFF2)
                    stage_cell<DIM, PREC, (DIM > 1 ? 1 : 0), TS>(a, c - G::SOFF1, s, org, sU + G::SOFF1,
                                                                 sV + G::SOFF1);
                else if (DIM > 2)
                    stage_cell<DIM, PREC, (DIM > 2 ? 2 : 0), TS>(a, c - G::SOFF2, s, org, sU + G::SOFF2,
                                                                 sV + G::SOFF2);
            }
            __syncthreads();
            for (int f = tid; f < G::FTOT; f += NTH) {
                double F;
                if (f < G::FOFF1) F = face_of<DIM, PREC, 0, TS>(a, f, cls, org, sU, sV);
                else if (DIM > 1 && f < G::FOFF2)
                    F = face_of<DIM, PREC, (DIM > 1 ? 1 : 0), TS>(a, f - G::FOFF1, cls, org, sU + G::SOFF1,
                                                                  sV + G::SOFF1);
                else
                    F = face_of<DIM, PREC, (DIM > 2 ? 2 : 0), TS>(a, f - G::FOFF2, cls, org, sU + G::SOFF2,
                                                                  sV + G::SOFF2);
                sF[f] = F;
            }
            __syncthreads();
            if (own) {
                // dsdt = (Fx_lo - Fx_hi)/dx + rxn, then += y and z terms (ScalarSolve.cpp:45-51)
                {
                    constexpr int F0 = G::template FE<0>(0), F1 = G::template FE<0>(1);
                    const int lo_f = cx + F0 * (cy + F1 * cz);
                    acc = (sF[lo_f] - sF[lo_f + 1]) * a.idx[0] + acc;
                }
                if constexpr (DIM > 1) {
                    constexpr int F0 = G::template FE<1>(0), F1 = G::template FE<1>(1);
                    const int lo_f = G::FOFF1 + cx + F0 * (cy + F1 * cz);
                    acc += (sF[lo_f] - sF[lo_f + F0]) * a.idx[1];
                }
                if constexpr (DIM > 2) {
                    constexpr int F0 = G::template FE<2>(0), F1 = G::template FE<2>(1);
                    const int lo_f = G::FOFF2 + cx + F0 * (cy + F1 * cz);
                    acc += (sF[lo_f] - sF[lo_f + F0 * F1]) * a.idx[2];
                }
            }
            // the next species' staging overwrites sU/sV only after every thread has
            // passed the barrier above; sF is rewritten only after the next staging
            // barrier, by which time every divergence read of this species is done
        }
        if (own) {
            if (s == ns) {
                double jh = joule_cell<true>(a, DIM, gi, gj, gk);
                acc += jh;
                if (a.write_diag) {
                    a.pn(gi, gj, gk, VD_EJH(ns)) = jh;
                    a.pn(gi, gj, gk, VD_EIH(ns)) = a.rxn(gi, gj, gk, ns);
                }
            }
            double nn = a.sb.p[own_o + s * cs] + a.dt * acc;
            if (a.bound_specden && s != ns) {
                // solution clipping of the species solve (Source/ScalarSolve.cpp:599-625)
                const double lo = (s == a.e_id) ? a.min_elec : a.min_spec;
                if (nn < lo) nn = lo;
            }
            a.pn(gi, gj, gk, s) = nn;
            if (a.dsdt.p) a.dsdt(gi, gj, gk, s) = acc;
            if (s == a.e_id) ne_new = nn;
            if (s == ns) een_new = nn;
        }
    }
    if (own) {
        for (int ib = 0; ib < a.nbg; ib++) {
            const int s = a.bg_sp[ib];
            double v = a.sb.p[own_o + s * cs];
            double r = a.rxn(gi, gj, gk, s);
            if (a.do_bg) {
                v += r * a.dt;
                if (v < a.min_spec && a.bound_specden) v = a.min_spec;
            }
            a.pn(gi, gj, gk, s) = v;
            if (a.dsdt.p) a.dsdt(gi, gj, gk, s) = r;
        }
        if (a.update_te && a.elecenergy) {
            // Source/ScalarSolve.cpp:659-666
            double te = (2.0 / 3.0) / K_B * een_new / a.sb.p[own_o + a.e_id * cs];
            if (te < a.min_te) {
                te = a.min_te;
                a.pn(gi, gj, gk, VD_EEN(ns)) = 1.5 * K_B * ne_new * te;
            }
            a.pn(gi, gj, gk, VD_ETEMP(ns)) = te;
        }
    }
}

// per-box kernel: one CTA per tile
template <int DIM, int PREC, int MINB>
__global__ void __launch_bounds__(default_nth<DIM>(), MINB) k_transport(const __grid_constant__ TransportArgs a)
{
    using TS = typename DefaultTile<DIM>::T;
    using G = TileGeom<DIM, TS>;
    using VT = typename VelT<PREC>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sF = reinterpret_cast<double*>(smem_raw);
    VT* sU = reinterpret_cast<VT*>(sF + G::FTOT);
    VT* sV = sU + G::STOT;
    transport_tile_update<DIM, PREC, TS>(a, blockIdx.x, sF, sU, sV);
}

// batched persistent kernel: each CTA walks the work list of (box, tile) items
// with a grid stride; boxes are described by TransportArgs records in global memory
template <int DIM, int PREC, class TS, int MINB>
__global__ void __launch_bounds__(TS::NTH, MINB)
    k_transport_batch(const TransportArgs* __restrict__ boxes, const int2* __restrict__ items, int nitems,
                      const BatchCtl ctl)
{
    using G = TileGeom<DIM, TS>;
    using VT = typename VelT<PREC>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sF = reinterpret_cast<double*>(smem_raw);
    VT* sU = reinterpret_cast<VT*>(sF + G::FTOT);
    VT* sV = sU + G::STOT;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const int2 cc = ctl.ctrl[w.x];
        if (ctl.t >= cc.x) continue;  // uniform over the CTA
        transport_tile_update<DIM, PREC, TS>(boxes[((ctl.t + cc.y) & 1) * ctl.nbox + w.x], w.y, sF, sU, sV);
        __syncthreads();  // the next item's staging must not overwrite a slow thread's reads
    }
}

}  // namespace vd
