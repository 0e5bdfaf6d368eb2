// vd_kernels.cu -- sm_100a kernels of the explicit species / electron-energy update.
//
//   k_reaction_source  one thread per cell: CKWC of the loaded mechanism
//                      (Source/ScalarSolve.cpp:143-165)
//   k_face_flux        one thread per face: compute_flux for one species and one
//                      sweep direction (Source/compute_explicit_flux.H:200-326)
//   k_dsdt             Source/ScalarSolve.cpp:44-53
//   k_joule            Source/ElecEnergySource.cpp:65-171
//   k_prep             fused path, pass 1: sum_s n_s on the grown box + chemistry
//   k_transport        fused path, pass 2: for every transported species and sweep
//                      direction, stage the stencil lines of a tile in shared memory,
//                      compute each face flux once, take the divergence, add rxn and
//                      the Joule term, and write n + dt*dsdt (FP64 accumulate).
//   k_checksums        per-box FP64 conservation sums
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include "vd_device.cuh"
#include "vd_kernels.cuh"

namespace vd {

// ---------------------------------------------------------------------------
// launch accounting and optional per-launch event timing
namespace {
std::atomic<int64_t> g_launches{0};
std::atomic<bool> g_prof{false};
std::mutex g_prof_mu;
struct ProfRec {
    std::string name;
    cudaEvent_t a, b;
};
std::vector<ProfRec> g_recs;
}  // namespace

int64_t launch_count() { return g_launches.load(); }

void prof_enable(bool on)
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (auto& r : g_recs) {
        cudaEventSynchronize(r.b);
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    g_recs.clear();
    g_prof.store(on);
}

ProfScope::ProfScope(const char* name, cudaStream_t s) : slot(-1), st(s)
{
    g_launches.fetch_add(1);
    if (!g_prof.load()) return;
    ProfRec r;
    r.name = name;
    if (cudaEventCreate(&r.a) != cudaSuccess) return;
    if (cudaEventCreate(&r.b) != cudaSuccess) {
        cudaEventDestroy(r.a);
        return;
    }
    cudaEventRecord(r.a, s);
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_recs.push_back(r);
    slot = (int)g_recs.size() - 1;
}

ProfScope::~ProfScope()
{
    if (slot < 0) return;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (slot < (int)g_recs.size()) cudaEventRecord(g_recs[slot].b, st);
}

int prof_read(char* names, int names_len, int64_t* counts, double* ms, int max)
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    std::vector<std::string> keys;
    std::vector<int64_t> cnt;
    std::vector<double> tot;
    for (auto& r : g_recs) {
        if (cudaEventSynchronize(r.b) != cudaSuccess) return -1;
        float t = 0.f;
        if (cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess) return -1;
        size_t i = 0;
        while (i < keys.size() && keys[i] != r.name) i++;
        if (i == keys.size()) {
            keys.push_back(r.name);
            cnt.push_back(0);
            tot.push_back(0.0);
        }
        cnt[i]++;
        tot[i] += t;
    }
    int n = 0, pos = 0;
    for (size_t i = 0; i < keys.size() && n < max; i++) {
        int len = (int)keys[i].size() + 1;
        if (pos + len > names_len) break;
        memcpy(names + pos, keys[i].c_str(), len);
        pos += len;
        counts[n] = cnt[i];
        ms[n] = tot[i];
        n++;
    }
    return n;
}

int upload_mech(const VdMechDev* h, cudaStream_t st)
{
    cudaError_t e = cudaMemcpyToSymbolAsync(c_mech, h, sizeof(VdMechDev), 0, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return (int)e;
    e = cudaStreamSynchronize(st);
    return (int)e;
}

__device__ __forceinline__ void cell_of(const BoxIdx& b, int64_t idx, int& i, int& j, int& k)
{
    int64_t nxy = (int64_t)b.n[0] * b.n[1];
    k = (int)(idx / nxy);
    int64_t r = idx - (int64_t)k * nxy;
    j = (int)(r / b.n[0]);
    i = (int)(r - (int64_t)j * b.n[0]);
    i += b.lo[0];
    j += b.lo[1];
    k += b.lo[2];
}

static inline unsigned grid_for(int64_t n, int bs)
{
    int64_t g = (n + bs - 1) / bs;
    if (g > 148LL * 64) g = 148LL * 64;
    if (g < 1) g = 1;
    return (unsigned)g;
}

// ---------------------------------------------------------------------------
template <int PREC>
__global__ void __launch_bounds__(128) k_reaction_source(BoxIdx b, A4 sb, A4 rxn, double Tg)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ns = c_mech.ns;
    const int st = blockDim.x;
    double* sc = reinterpret_cast<double*>(smem_raw) + threadIdx.x;
    double* wd = sc + ns * st;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < b.ncell;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(b, idx, i, j, k);
        const int64_t o = sb.off(i, j, k);
        for (int s = 0; s < ns; s++) sc[s * st] = sb.p[o + s * sb.ns];
        double Te = sb.p[o + (int64_t)VD_ETEMP(ns) * sb.ns];
        double ee = chem_cell<PREC>(sc, wd, st, Te, Tg);
        const int64_t r = rxn.off(i, j, k);
        for (int s = 0; s < ns; s++) rxn.p[r + s * rxn.ns] = wd[s * st];
        rxn.p[r + (int64_t)ns * rxn.ns] = ee;
    }
}

// dynamic shared memory of the chemistry kernels: sc and wd, ns doubles per thread each
static cudaError_t chem_smem(const void* fn, int ns, int threads, size_t* bytes)
{
    *bytes = (size_t)2 * ns * threads * sizeof(double);
    if (*bytes > 48 * 1024)
        return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*bytes);
    return cudaSuccess;
}

cudaError_t launch_reaction_source(const BoxIdx& b, const A4& sb, const A4& rxn, double Tg, int prec, int ns,
                                   cudaStream_t st)
{
    unsigned g = grid_for(b.ncell, 128);
    size_t sm = 0;
    const void* fn = prec == PREC_MIXED ? (const void*)k_reaction_source<PREC_MIXED>
                                        : (const void*)k_reaction_source<PREC_FP64>;
    cudaError_t e = chem_smem(fn, ns, 128, &sm);
    if (e != cudaSuccess) return e;
    ProfScope ps("k_reaction_source", st);
    if (prec == PREC_MIXED) k_reaction_source<PREC_MIXED><<<g, 128, sm, st>>>(b, sb, rxn, Tg);
    else k_reaction_source<PREC_FP64><<<g, 128, sm, st>>>(b, sb, rxn, Tg);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// velocity of species s at cell (i,j,k) in direction d (plasmachem_transport::compute_vel,
// Source/PlasmaChem.H:187-206, or the constant user velocity of the Advect case)
__device__ __forceinline__ double vel_cell(const A4& phi, int i, int j, int k, int d, int s, int ns, double Tg,
                                           int udv, const double* uvel, int vel_sp)
{
    if (udv) return (s == vel_sp) ? uvel[d] : 0.0;
    const int64_t o = phi.off(i, j, k);
    double N = 0.0;
    for (int q = 0; q < ns; q++) N += phi.p[o + q * phi.ns];
    double Te = phi.p[o + (int64_t)VD_ETEMP(ns) * phi.ns];
    double mu = mob_fp64(s, Te, N, Tg);
    return mu * phi.p[o + (int64_t)(VD_EFX(ns) + d) * phi.ns];
}

struct FaceFluxArgs {
    BoxIdx fb;
    int dir, specid, ns;
    A4 phi, fx;
    int8_t zlo, zhi;
    int domlo, domhi;
    double Tg, dxmin, dt;
    int hyp_order, udv, weno, vel_sp;
    double uvel[3];
};

__global__ void __launch_bounds__(128) k_face_flux(const __grid_constant__ FaceFluxArgs a)
{
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < a.fb.ncell;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int c[3];
        cell_of(a.fb, idx, c[0], c[1], c[2]);
        double u[6], v[6];
        const int H = (a.hyp_order == 5) ? 3 : a.hyp_order;
#pragma unroll
        for (int q = 0; q < 6; q++) {
            int off = q - 3;  // cells i-3 .. i+2 along dir
            if (off < -H || off > H - 1) {
                u[q] = 0.0;
                v[q] = 0.0;
                continue;
            }
            int g[3] = {c[0], c[1], c[2]};
            g[a.dir] += off;
            u[q] = a.phi(g[0], g[1], g[2], a.specid);
            v[q] = vel_cell(a.phi, g[0], g[1], g[2], a.dir, a.specid, a.ns, a.Tg, a.udv, a.uvel, a.vel_sp);
        }
        double F = face_flux_fp64(u, v, a.hyp_order, a.weno, a.dxmin, a.dt);
        int fd = c[a.dir];
        if (fd == a.domlo && a.zlo) F = 0.0;
        if (fd == a.domhi + 1 && a.zhi) F = 0.0;
        a.fx(c[0], c[1], c[2], 0) = F;
    }
}

cudaError_t launch_face_flux(const BoxIdx& fb, int dir, int specid, const A4& phi, const A4& fx,
                             const int8_t zlo[3], const int8_t zhi[3], const int domlo[3], const int domhi[3],
                             double Tg, double dxmin, double dt, int hyp_order, int udv, int weno,
                             const double uvel[3], int vel_sp, int ns, cudaStream_t st)
{
    FaceFluxArgs a;
    a.fb = fb;
    a.dir = dir;
    a.specid = specid;
    a.ns = ns;
    a.phi = phi;
    a.fx = fx;
    a.zlo = zlo[dir];
    a.zhi = zhi[dir];
    a.domlo = domlo[dir];
    a.domhi = domhi[dir];
    a.Tg = Tg;
    a.dxmin = dxmin;
    a.dt = dt;
    a.hyp_order = hyp_order;
    a.udv = udv;
    a.weno = weno;
    a.vel_sp = vel_sp;
    for (int d = 0; d < 3; d++) a.uvel[d] = uvel[d];
    ProfScope ps("k_face_flux", st);
    k_face_flux<<<grid_for(fb.ncell, 128), 128, 0, st>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_dsdt(BoxIdx b, int dim, int specid, A4 f0, A4 f1, A4 f2, A4 rxn, A4 dsdt,
                                              double dx0, double dx1, double dx2)
{
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < b.ncell;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(b, idx, i, j, k);
        double v = (f0(i, j, k) - f0(i + 1, j, k)) / dx0 + rxn(i, j, k, specid);
        if (dim > 1) v += (f1(i, j, k) - f1(i, j + 1, k)) / dx1;
        if (dim == 3) v += (f2(i, j, k) - f2(i, j, k + 1)) / dx2;
        dsdt(i, j, k) = v;
    }
}

cudaError_t launch_dsdt(const BoxIdx& b, int dim, int specid, const A4 flux[3], const A4& rxn, const A4& dsdt,
                        const double dx[3], cudaStream_t st)
{
    ProfScope ps("k_dsdt", st);
    k_dsdt<<<grid_for(b.ncell, 256), 256, 0, st>>>(b, dim, specid, flux[0], flux[1], flux[2], rxn, dsdt, dx[0],
                                                    dx[1], dx[2]);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Joule heating at one cell (Source/ElecEnergySource.cpp:76-153).  sumN: use the
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
            double Esum = 0.0, evf_d = 0.0;
            for (int d = 0; d < dim; d++) {
                double e = 0.5 * (p[ol + (VD_EFX(ns) + d) * cs] + p[orr + (VD_EFX(ns) + d) * cs]);
                Esum += e * e;
                if (d == idim) evf_d = e;
            }
            (void)Esum;
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
            double mu = a.const_ele_trans ? a.ele_mob / ndens : mob_fp64(eidx, etemp, ndens, a.Tg);
            double dc = a.const_ele_trans ? a.ele_diff / ndens : diff_fp64(eidx, etemp, ndens, a.Tg);
            double cur = a.charge_e * (mu * ne * ef - dc * gn);
            jheat += cur * ef;
        }
    }
    jheat *= 0.5;
    if (a.floor_jh && jheat < 0.0) jheat = 0.0;
    return jheat;
}

__global__ void __launch_bounds__(128) k_joule(BoxIdx b, int dim, const __grid_constant__ TransportArgs a)
{
    const int ns = a.ns;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < b.ncell;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(b, idx, i, j, k);
        double jh = joule_cell<false>(a, dim, i, j, k);
        a.dsdt(i, j, k) += jh;
        a.pn(i, j, k, VD_EJH(ns)) = jh;
        a.pn(i, j, k, VD_EIH(ns)) = a.rxn(i, j, k, ns);
    }
}

cudaError_t launch_joule(const BoxIdx& b, int dim, const A4& sb, const A4& rxn, const A4 ef[3], const A4 gne[3],
                         const A4& dsdt, const A4& pn, const TransportArgs& cfg, cudaStream_t st)
{
    TransportArgs a = cfg;
    a.sb = sb;
    a.rxn = rxn;
    a.dsdt = dsdt;
    a.pn = pn;
    for (int d = 0; d < 3; d++) {
        a.ef[d] = ef[d];
        a.gne[d] = gne[d];
    }
    ProfScope ps("k_joule", st);
    k_joule<<<grid_for(b.ncell, 128), 128, 0, st>>>(b, dim, a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
template <int PREC>
__global__ void __launch_bounds__(128) k_prep(const __grid_constant__ PrepArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ns = c_mech.ns;
    const int st = blockDim.x;
    double* sc = reinterpret_cast<double*>(smem_raw) + threadIdx.x;
    double* wd = sc + ns * st;
    const int gx = a.ghi[0] - a.glo[0] + 1, gy = a.ghi[1] - a.glo[1] + 1, gz = a.ghi[2] - a.glo[2] + 1;
    const int64_t ntot = (int64_t)gx * gy * gz;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < ntot;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int k = (int)(idx / ((int64_t)gx * gy));
        int64_t r = idx - (int64_t)k * gx * gy;
        int j = (int)(r / gx);
        int i = (int)(r - (int64_t)j * gx);
        i += a.glo[0];
        j += a.glo[1];
        k += a.glo[2];
        const int64_t o = a.sb.off(i, j, k);
        double N = 0.0;
        for (int s = 0; s < ns; s++) {
            const double v = a.sb.p[o + s * a.sb.ns];
            sc[s * st] = v;
            N += v;
        }
        if (a.write_n) a.Nv(i, j, k) = N;
        bool inside = i >= a.lo[0] && i <= a.hi[0] && j >= a.lo[1] && j <= a.hi[1] && k >= a.lo[2] && k <= a.hi[2];
        if (!inside) continue;
        const int64_t ro = a.rxn.off(i, j, k);
        if (a.do_reactions) {
            double Te = a.sb.p[o + (int64_t)VD_ETEMP(ns) * a.sb.ns];
            double ee = chem_cell<PREC>(sc, wd, st, Te, a.Tg);
            for (int s = 0; s < ns; s++) a.rxn.p[ro + s * a.rxn.ns] = wd[s * st];
            a.rxn.p[ro + (int64_t)ns * a.rxn.ns] = ee;
        } else {
            for (int s = 0; s <= ns; s++) a.rxn.p[ro + s * a.rxn.ns] = 0.0;
        }
    }
}

cudaError_t launch_prep(const PrepArgs& a, int prec, int ns, cudaStream_t st)
{
    {
        cudaError_t es = spec_launch_prep(a, prec, st);
        if (es != cudaErrorNotReady) return es;
    }
    int64_t n = (int64_t)(a.ghi[0] - a.glo[0] + 1) * (a.ghi[1] - a.glo[1] + 1) * (a.ghi[2] - a.glo[2] + 1);
    unsigned g = grid_for(n, 128);
    size_t sm = 0;
    const void* fn = prec == PREC_MIXED ? (const void*)k_prep<PREC_MIXED> : (const void*)k_prep<PREC_FP64>;
    cudaError_t e = chem_smem(fn, ns, 128, &sm);
    if (e != cudaSuccess) return e;
    ProfScope ps("k_prep", st);
    if (prec == PREC_MIXED) k_prep<PREC_MIXED><<<g, 128, sm, st>>>(a);
    else k_prep<PREC_FP64><<<g, 128, sm, st>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Fused transport kernel.  One CTA per TX x TY x TZ tile, NTH threads.  Per
// transported species: (1) stage the stencil lines of every sweep direction in
// shared memory -- for direction d the cells rel -3 .. T_d+2 along d of each tile
// row, with the density and the drift velocity mu(Te, N) E_d computed once per
// staged cell; (2) compute every face flux of the tile once (all directions in one
// pass, faces spread evenly over the threads); (3) each thread takes the
// divergence of its own cell, adds rxn (and the Joule term for the electron
// energy) and writes n + dt*dsdt in FP64.  Two barriers per species.
template <int DIM> struct Tile;
template <> struct Tile<1> { static constexpr int X = 256, Y = 1, Z = 1, NTH = 256; };
template <> struct Tile<2> { static constexpr int X = 32, Y = 8, Z = 1, NTH = 256; };
template <> struct Tile<3> { static constexpr int X = 8, Y = 8, Z = 8, NTH = 512; };

void transport_tile(int dim, int t[3])
{
    if (dim == 1) { t[0] = Tile<1>::X; t[1] = 1; t[2] = 1; }
    else if (dim == 2) { t[0] = Tile<2>::X; t[1] = Tile<2>::Y; t[2] = 1; }
    else { t[0] = Tile<3>::X; t[1] = Tile<3>::Y; t[2] = Tile<3>::Z; }
}

template <int DIM>
struct TileGeom {
    static constexpr int T[3] = {Tile<DIM>::X, Tile<DIM>::Y, Tile<DIM>::Z};
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

// stage staged-cell cc of direction D's line set: density and drift velocity
template <int DIM, int PREC, int D>
__device__ __forceinline__ void stage_cell(const TransportArgs& a, int cc, int s, const int* org,
                                           typename VelT<PREC>::T* sU, typename VelT<PREC>::T* sV)
{
    using G = TileGeom<DIM>;
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
template <int DIM, int PREC, int D>
__device__ __forceinline__ double face_of(const TransportArgs& a, int ff, int cls, const int* org,
                                          const typename VelT<PREC>::T* sU, const typename VelT<PREC>::T* sV)
{
    using G = TileGeom<DIM>;
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

template <int DIM, int PREC, int MINB>
__global__ void __launch_bounds__(Tile<DIM>::NTH, MINB) k_transport(const __grid_constant__ TransportArgs a)
{
    using G = TileGeom<DIM>;
    using VT = typename VelT<PREC>::T;
    constexpr int NTH = Tile<DIM>::NTH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sF = reinterpret_cast<double*>(smem_raw);
    VT* sU = reinterpret_cast<VT*>(sF + G::FTOT);  // staged densities (FP32 in the mixed path)
    VT* sV = sU + G::STOT;                          // staged drift velocities

    const int tid = threadIdx.x;
    int tb = blockIdx.x;
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
    for (int it = 0; it < a.ntr; it++) {
        const int s = a.tr_sp[it];
        const int cls = a.tr_cls[it];
        double acc = own ? a.rxn(gi, gj, gk, s) : 0.0;
        if (a.tr_flux[it]) {
            for (int c = tid; c < G::STOT; c += NTH) {
                if (c < G::SOFF1) stage_cell<DIM, PREC, 0>(a, c, s, org, sU, sV);
                else if (DIM > 1 && c < G::SOFF2)
                    stage_cell<DIM, PREC, (DIM > 1 ? 1 : 0)>(a, c - G::SOFF1, s, org, sU + G::SOFF1, sV + G::SOFF1);
                else if (DIM > 2)
                    stage_cell<DIM, PREC, (DIM > 2 ? 2 : 0)>(a, c - G::SOFF2, s, org, sU + G::SOFF2, sV + G::SOFF2);
            }
            __syncthreads();
            for (int f = tid; f < G::FTOT; f += NTH) {
                double F;
                if (f < G::FOFF1) F = face_of<DIM, PREC, 0>(a, f, cls, org, sU, sV);
                else if (DIM > 1 && f < G::FOFF2)
                    F = face_of<DIM, PREC, (DIM > 1 ? 1 : 0)>(a, f - G::FOFF1, cls, org, sU + G::SOFF1, sV + G::SOFF1);
                else
                    F = face_of<DIM, PREC, (DIM > 2 ? 2 : 0)>(a, f - G::FOFF2, cls, org, sU + G::SOFF2, sV + G::SOFF2);
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
            a.pn(gi, gj, gk, s) = nn;
            if (a.dsdt.p) a.dsdt(gi, gj, gk, s) = acc;
            if (s == a.e_id) ne_new = nn;
            if (s == ns) een_new = nn;
        }
    }
    if (!own) return;
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

template <int DIM, int PREC, int MINB>
static cudaError_t launch_tr(const TransportArgs& a, cudaStream_t st)
{
    using G = TileGeom<DIM>;
    using VT = typename VelT<PREC>::T;
    constexpr size_t smem = (size_t)G::STOT * 2 * sizeof(VT) + (size_t)G::FTOT * sizeof(double);
    static unsigned attr_set = 0;  // one bit per device
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(attr_set & (1u << (dev & 31)))) {
        cudaError_t e = cudaFuncSetAttribute(k_transport<DIM, PREC, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_set |= 1u << (dev & 31);
    }
    unsigned nt = (unsigned)a.ntile[0] * a.ntile[1] * a.ntile[2];
    ProfScope ps("k_transport", st);
    k_transport<DIM, PREC, MINB><<<nt, Tile<DIM>::NTH, smem, st>>>(a);
    return cudaGetLastError();
}

// Occupancy variant of the transport kernel per (dimension, precision): resident
// blocks per SM the compiler must fit (registers capped at 64K / (threads * n)).
// Set by the tuner (vd_tune_set "transport_minblocks_<dim>d_<fp64|mixed>").
// Defaults measured on B200 (2 beats 1 for every dimension and precision: the
// kernels are issue/latency bound and gain more from 2x the resident warps than
// they lose to the few spills of a 64-register cap in 3-D).
static int g_tr_minb[4][2] = {{2, 2}, {2, 2}, {2, 2}, {2, 2}};

static int tr_minb_max(int dim) { return dim == 3 ? 2 : 4; }  // 512- vs 256-thread blocks

int tune_set(const char* key, int value)
{
    for (int d = 1; d <= 3; d++)
        for (int p = 0; p < 2; p++) {
            char k[64];
            snprintf(k, sizeof(k), "transport_minblocks_%dd_%s", d, p ? "mixed" : "fp64");
            if (strcmp(k, key) == 0) {
                if (value < 1 || value > tr_minb_max(d)) return -1;
                g_tr_minb[d][p] = value;
                return 0;
            }
        }
    return -2;
}

int tune_get(const char* key)
{
    for (int d = 1; d <= 3; d++)
        for (int p = 0; p < 2; p++) {
            char k[64];
            snprintf(k, sizeof(k), "transport_minblocks_%dd_%s", d, p ? "mixed" : "fp64");
            if (strcmp(k, key) == 0) return g_tr_minb[d][p];
        }
    return -2;
}

template <int DIM, int PREC>
static cudaError_t launch_tr_v(const TransportArgs& a, cudaStream_t st)
{
    const int mb = g_tr_minb[DIM][PREC];
    if constexpr (DIM < 3) {
        if (mb == 4) return launch_tr<DIM, PREC, 4>(a, st);
        if (mb == 3) return launch_tr<DIM, PREC, 3>(a, st);
    }
    if (mb == 2) return launch_tr<DIM, PREC, 2>(a, st);
    return launch_tr<DIM, PREC, 1>(a, st);
}

cudaError_t launch_transport(const TransportArgs& a, int dim, int prec, cudaStream_t st)
{
    if (prec == PREC_MIXED) {
        if (dim == 1) return launch_tr_v<1, PREC_MIXED>(a, st);
        if (dim == 2) return launch_tr_v<2, PREC_MIXED>(a, st);
        return launch_tr_v<3, PREC_MIXED>(a, st);
    }
    if (dim == 1) return launch_tr_v<1, PREC_FP64>(a, st);
    if (dim == 2) return launch_tr_v<2, PREC_FP64>(a, st);
    return launch_tr_v<3, PREC_FP64>(a, st);
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_checksums(BoxIdx b, A4 rxn, A4 pn, double* out)
{
    const int ns = c_mech.ns;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < b.ncell;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(b, idx, i, j, k);
        for (int s = 0; s < ns; s++) {
            double z = (double)c_mech.charge[s] * rxn(i, j, k, s);
            s0 += z;
            s1 += fabs(z);
            s3 += pn(i, j, k, s);
        }
        s2 += rxn(i, j, k, ns);
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        s3 += __shfl_xor_sync(0xffffffffu, s3, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&out[0], s0);
        atomicAdd(&out[1], s1);
        atomicAdd(&out[2], s2);
        atomicAdd(&out[3], s3);
    }
}

cudaError_t launch_checksums(const BoxIdx& b, const A4& rxn, const A4& pn, double* out, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(out, 0, 4 * sizeof(double), st);
    if (e != cudaSuccess) return e;
    unsigned g = grid_for(b.ncell, 256);
    if (g > 148 * 4) g = 148 * 4;
    ProfScope ps("k_checksums", st);
    k_checksums<<<g, 256, 0, st>>>(b, rxn, pn, out);
    return cudaGetLastError();
}

}  // namespace vd
