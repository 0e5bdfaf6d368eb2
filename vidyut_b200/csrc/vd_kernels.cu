// vd_kernels.cu -- sm_100a kernels of the explicit species / electron-energy update.
//
//   k_reaction_source  one thread per cell: CKWC of the loaded mechanism
//                      (Source/ScalarSolve.cpp:143-165)
//   k_face_flux        one thread per face: compute_flux for one species and one
//                      sweep direction (Source/compute_explicit_flux.H:200-326)
//   k_dsdt             Source/ScalarSolve.cpp:44-53
//   k_joule            Source/ElecEnergySource.cpp:65-171
//   k_prep             fused path, pass 1: sum_s n_s on the grown box + chemistry
//   k_joule_pre        fused path, pass 2: the Joule term of every valid cell
//   k_transport        fused path, pass 3: for every transported species and sweep
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
#include "vd_transport.cuh"

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
thread_local bool t_prof_suspended = false;
}  // namespace

int64_t launch_count() { return g_launches.load(); }
void add_launches(int64_t n) { g_launches.fetch_add(n); }
void prof_suspend(bool on) { t_prof_suspended = on; }

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
    if (!g_prof.load() || t_prof_suspended) return;
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
    e = upload_mech_batch(h, st);  // the batched transport kernels' copy
    if (e != cudaSuccess) return (int)e;
    e = upload_mech_diffusion(h, st);  // the implicit species solve's copy
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
        const double EN = c_mech.need_en ? sb.p[o + (int64_t)VD_REF(ns) * sb.ns] : 0.0;
        double ee = chem_cell<PREC>(sc, wd, st, Te, Tg, EN);
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
    // |E| of the three state components, as compute_vel takes it
    double esum = 0.0;
    for (int q = 0; q < 3; q++) {
        const double e = phi.p[o + (int64_t)(VD_EFX(ns) + q) * phi.ns];
        esum += e * e;
    }
    double mu = mob_fp64(s, Te, N, Tg, sqrt(esum));
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
// One cell (linear index idx over the grown box) of the prep pass: density sum and,
// inside the valid box, the reaction source.  sc/wd: this thread's shared rows.
template <int PREC>
__device__ __forceinline__ void prep_cell(const PrepArgs& a, int64_t idx, double* sc, double* wd, int st)
{
    const int ns = c_mech.ns;
    const int gx = a.ghi[0] - a.glo[0] + 1, gy = a.ghi[1] - a.glo[1] + 1;
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
    if (!inside) return;
    const int64_t ro = a.rxn.off(i, j, k);
    if (a.do_reactions) {
        double Te = a.sb.p[o + (int64_t)VD_ETEMP(ns) * a.sb.ns];
        const double EN = c_mech.need_en ? a.sb.p[o + (int64_t)VD_REF(ns) * a.sb.ns] : 0.0;
        double ee = chem_cell<PREC>(sc, wd, st, Te, a.Tg, EN);
        for (int s = 0; s < ns; s++) a.rxn.p[ro + s * a.rxn.ns] = wd[s * st];
        a.rxn.p[ro + (int64_t)ns * a.rxn.ns] = ee;
    } else {
        for (int s = 0; s <= ns; s++) a.rxn.p[ro + s * a.rxn.ns] = 0.0;
    }
}

__device__ __forceinline__ int64_t grown_cells(const PrepArgs& a)
{
    return (int64_t)(a.ghi[0] - a.glo[0] + 1) * (a.ghi[1] - a.glo[1] + 1) * (a.ghi[2] - a.glo[2] + 1);
}

template <int PREC>
__global__ void __launch_bounds__(128) k_prep(const __grid_constant__ PrepArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ns = c_mech.ns;
    const int st = blockDim.x;
    double* sc = reinterpret_cast<double*>(smem_raw) + threadIdx.x;
    double* wd = sc + ns * st;
    const int64_t ntot = grown_cells(a);
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < ntot;
         idx += (int64_t)gridDim.x * blockDim.x)
        prep_cell<PREC>(a, idx, sc, wd, st);
}

// batched prep: item (box, chunk) covers grown-box cells [chunk*kPrepChunk, +kPrepChunk)
template <int PREC>
__global__ void __launch_bounds__(128) k_prep_batch(const PrepArgs* __restrict__ boxes, const int2* __restrict__ items,
                                                    int nitems, const BatchCtl ctl)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ns = c_mech.ns;
    const int st = blockDim.x;
    double* sc = reinterpret_cast<double*>(smem_raw) + threadIdx.x;
    double* wd = sc + ns * st;
    __shared__ long long sA_raw[sizeof(PrepArgs) / 8];  // the item's record, read from shared memory
    static_assert(sizeof(PrepArgs) % 8 == 0, "record copied in 8-byte words");
    const PrepArgs& sA = *reinterpret_cast<const PrepArgs*>(sA_raw);
    int cur = -1;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const int2 cc = ctl.ctrl[w.x];
        if (ctl.t >= cc.x) continue;
        const int rec = ((ctl.t + cc.y) & 1) * ctl.nbox + w.x;
        if (rec != cur) {
            __syncthreads();  // every thread is done with the previous record
            const long long* src = reinterpret_cast<const long long*>(boxes + rec);
            long long* dst = sA_raw;
            for (int q = threadIdx.x; q < (int)(sizeof(PrepArgs) / 8); q += blockDim.x) dst[q] = src[q];
            cur = rec;
            __syncthreads();
        }
        const int64_t ntot = grown_cells(sA);
        const int64_t base = (int64_t)w.y * kPrepChunk;
        for (int q = threadIdx.x; q < kPrepChunk; q += blockDim.x) {
            const int64_t idx = base + q;
            if (idx < ntot) prep_cell<PREC>(sA, idx, sc, wd, st);
        }
    }
}

cudaError_t launch_prep_batch(const PrepArgs* boxes, const int2* items, int nitems, BatchCtl ctl, int prec, int ns,
                              cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    {
        cudaError_t es = spec_launch_prep_batch(boxes, items, nitems, ctl, prec, st);
        if (es != cudaErrorNotReady) return es;
    }
    size_t sm = 0;
    const void* fn =
        prec == PREC_MIXED ? (const void*)k_prep_batch<PREC_MIXED> : (const void*)k_prep_batch<PREC_FP64>;
    cudaError_t e = chem_smem(fn, ns, 128, &sm);
    if (e != cudaSuccess) return e;
    unsigned g = (unsigned)(nitems < 148 * 16 ? nitems : 148 * 16);
    ProfScope ps("k_prep_batch", st);
    if (prec == PREC_MIXED) k_prep_batch<PREC_MIXED><<<g, 128, sm, st>>>(boxes, items, nitems, ctl);
    else k_prep_batch<PREC_FP64><<<g, 128, sm, st>>>(boxes, items, nitems, ctl);
    return cudaGetLastError();
}

// ghost cell idx (0 <= idx < a.count) of a box, ordered by direction d, side, then
// layer and the other coordinates: copy the components in comps[] from the
// nearest valid cell (first-order extrapolation) or the periodic image
__device__ __forceinline__ void ghost_cell(const GhostArgs& a, int64_t idx)
{
    const int G = a.ghost;
    int n[3];
    for (int e = 0; e < 3; e++) n[e] = a.hi[e] - a.lo[e] + 1;
    int d = 0;
    int64_t P = 1;
    for (; d < a.dim; d++) {
        P = 1;
        for (int e = 0; e < a.dim; e++)
            if (e != d) P *= n[e];
        const int64_t cnt = 2 * (int64_t)G * P;
        if (idx < cnt) break;
        idx -= cnt;
    }
    if (d >= a.dim) return;
    // x faces take their G layers fastest (a row's ghost cells of one side share a
    // sector), the other directions their transverse position (coalesced along x)
    const int side = (int)(idx / ((int64_t)G * P));
    const int g = d == 0 ? (int)(idx % G) + 1 : (int)((idx / P) % G) + 1;
    int64_t rest = d == 0 ? (idx / G) % P : idx % P;
    int c[3] = {a.lo[0], a.lo[1], a.lo[2]};
    for (int e = 0; e < a.dim; e++) {
        if (e == d) continue;
        c[e] = a.lo[e] + (int)(rest % n[e]);
        rest /= n[e];
    }
    int dst[3] = {c[0], c[1], c[2]}, src[3] = {c[0], c[1], c[2]};
    if (side == 0) {
        dst[d] = a.lo[d] - g;
        src[d] = a.periodic[d] ? a.hi[d] - ((g - 1) % n[d]) : a.lo[d];
    } else {
        dst[d] = a.hi[d] + g;
        src[d] = a.periodic[d] ? a.lo[d] + ((g - 1) % n[d]) : a.hi[d];
    }
    const int64_t od = a.st.off(dst[0], dst[1], dst[2]), os = a.st.off(src[0], src[1], src[2]);
    for (int q = 0; q < a.ncomp; q++) {
        const int64_t co = (int64_t)a.comps[q] * a.st.ns;
        a.st.p[od + co] = a.st.p[os + co];
    }
}

// batched ghost refill: item (box, chunk) covers ghost cells [chunk*kGhostChunk, +kGhostChunk)
__global__ void __launch_bounds__(kGhostChunk) k_ghost_batch(const GhostArgs* __restrict__ boxes,
                                                             const int2* __restrict__ items, int nitems,
                                                             const BatchCtl ctl)
{
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const int2 cc = ctl.ctrl[w.x];
        if (ctl.t >= cc.x) continue;
        const GhostArgs& a = boxes[((ctl.t + cc.y) & 1) * ctl.nbox + w.x];
        const int64_t idx = (int64_t)w.y * kGhostChunk + threadIdx.x;
        if (idx < a.count) ghost_cell(a, idx);
    }
}

// single box
__global__ void __launch_bounds__(256) k_ghost(const __grid_constant__ GhostArgs a)
{
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < a.count;
         idx += (int64_t)gridDim.x * blockDim.x)
        ghost_cell(a, idx);
}

cudaError_t launch_ghost(const GhostArgs& a, cudaStream_t st)
{
    if (a.count <= 0) return cudaSuccess;
    unsigned g = grid_for(a.count, 256);
    ProfScope ps("k_ghost", st);
    k_ghost<<<g, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_ghost_batch(const GhostArgs* boxes, const int2* items, int nitems, BatchCtl ctl, cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    unsigned g = (unsigned)(nitems < 148 * 8 ? nitems : 148 * 8);
    ProfScope ps("k_ghost_batch", st);
    k_ghost_batch<<<g, kGhostChunk, 0, st>>>(boxes, items, nitems, ctl);
    return cudaGetLastError();
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
// Fused transport kernel (vd_transport.cuh): tile shapes and the tile update.

// The mobility models of specMob (test/models/Ar_DC_1d/Chemistry.H:177-202) as a
// species constant K times a per-cell basis: electron-type mu = c/(sqrt(Te) N s0)
// gives K = c/s0 on E/(sqrt(Te) N); ion-type mu = c/(sqrt(Tg) N s0) gives
// K = c/(sqrt(Tg) s0) on E/N; mu = p0/N gives K = p0 on E/N; a constant mu gives
// K = p0 on E; mu = p0 |E|^p1 gives K = p0 on E |E|^p1 (one basis per exponent);
// a scaled model multiplies its reference's K.
bool velocity_basis(const VdMechDev& m, int s, double Tg, VelBasis* b, double* K)
{
    b->pw = 0.0;
    b->fit = 0;
    double scale = 1.0;
    int k = m.mob_kind[s];
    if (k == VD_MOB_SCALED) {
        scale = m.mob_p0[s];
        s = m.mob_ref[s];
        k = m.mob_kind[s];
    }
    switch (k) {
    case VD_MOB_ELECTRON: b->kind = 0; *K = scale * (m.mob_c[s] / m.mob_p0[s]); return true;
    case VD_MOB_ION_TG: b->kind = 1; *K = scale * (m.mob_c[s] / (std::sqrt(Tg) * m.mob_p0[s])); return true;
    case VD_MOB_CONST_N: b->kind = 1; *K = scale * m.mob_p0[s]; return true;
    case VD_MOB_CONST: b->kind = 2; *K = scale * m.mob_p0[s]; return true;
    case VD_MOB_POW_EMAG: b->kind = 3; *K = scale * m.mob_p0[s]; b->pw = m.mob_p1[s]; return true;
    case VD_MOB_EN_POLY:
        b->kind = 4;
        *K = scale * m.mob_p0[s];
        b->pw = m.mob_p1[s];
        b->fit = m.mob_ref[s];
        return true;
    case VD_MOB_EXP_MEANE: b->kind = 5; *K = scale * m.mob_p0[s]; b->fit = m.mob_ref[s]; return true;
    default: return false;
    }
}

bool same_basis(const VdMechDev& m, const VelBasis& x, const VelBasis& y)
{
    if (x.kind != y.kind || x.pw != y.pw) return false;
    if (x.kind < 4) return true;
    const int nc = x.kind == 4 ? 2 : 5;  // coefficients the kind reads
    for (int j = 0; j < nc; j++)
        if (m.fits[x.fit].jc[j] != m.fits[y.fit].jc[j]) return false;
    return true;
}

void finish_species_lists(TransportArgs& a, const VdMechDev& m)
{
    a.nfl = a.nnf = a.nb = 0;
    a.stage_emag = m.emag_e;
    VelBasis bs[4];
    for (int it = 0; it < a.ntr; it++) {
        const int s = a.tr_sp[it];
        if (!a.tr_flux[it]) {
            a.nf_sp[a.nnf++] = (int8_t)s;
            continue;
        }
        double K = 0.0;
        int slot = -1;
        if (a.udv) {
            K = 1.0;  // v = the user velocity of the sweep direction
        } else {
            VelBasis b;
            if (!velocity_basis(m, s, a.Tg, &b, &K)) {
                a.nf_sp[a.nnf++] = (int8_t)s;
                continue;
            }
            for (int q = 0; q < a.nb; q++)
                if (same_basis(m, bs[q], b)) slot = q;
            if (slot < 0) {  // vd_mech_init admits at most kMaxBases distinct bases
                slot = a.nb;
                bs[a.nb] = b;
                a.bkind[a.nb] = (int8_t)b.kind;
                a.bfit[a.nb] = (int8_t)b.fit;
                if (b.kind == 3 || b.kind == 4) a.stage_emag = 1;
                a.bpow[a.nb++] = b.pw;
            }
        }
        a.fl_sp[a.nfl] = (int8_t)s;
        a.fl_cls[a.nfl] = a.tr_cls[it];
        a.fl_slot[a.nfl] = (int8_t)slot;
        a.fl_K[a.nfl] = K;
        a.fl_Kf[a.nfl] = (float)K;
        int zm = 0;
        for (int d = 0; d < 3; d++) zm |= (a.zlo[a.tr_cls[it]][d] ? 1 : 0) << d | (a.zhi[a.tr_cls[it]][d] ? 1 : 0) << (3 + d);
        a.fl_zm[a.nfl] = (int8_t)zm;
        a.nfl++;
    }
}

void transport_tile(int dim, int t[3])
{
    if (dim == 1) { t[0] = DefaultTile<1>::T::X; t[1] = 1; t[2] = 1; }
    else if (dim == 2) { t[0] = DefaultTile<2>::T::X; t[1] = DefaultTile<2>::T::Y; t[2] = 1; }
    else { t[0] = DefaultTile<3>::T::X; t[1] = DefaultTile<3>::T::Y; t[2] = DefaultTile<3>::T::Z; }
}

template <int DIM, int PREC, int MINB>
static cudaError_t launch_tr(const TransportArgs& a, cudaStream_t st)
{
    using TS = typename DefaultTile<DIM>::T;
    constexpr int GRP = group_fit<DIM, PREC, TS, MINB>();
    const size_t smem = transport_smem<DIM, PREC, TS, GRP>(a.nb);
    static unsigned attr_set = 0;  // one bit per device
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(attr_set & (1u << (dev & 31)))) {
        cudaError_t e = cudaFuncSetAttribute(k_transport<DIM, PREC, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)transport_smem_max<DIM, PREC, TS, GRP>());
        if (e != cudaSuccess) return e;
        attr_set |= 1u << (dev & 31);
    }
    unsigned nt = (unsigned)a.ntile[0] * a.ntile[1] * a.ntile[2];
    ProfScope ps("k_transport", st);
    k_transport<DIM, PREC, MINB><<<nt, DefaultTile<DIM>::T::NTH, smem, st>>>(a);
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

// Tile-shape variant of the batched transport kernel per (dimension, precision),
// the default for new batches ("batch_tile_<dim>d_<fp64|mixed>"; vd_batch_tune
// stores its choice here).
static int g_batch_tile[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
int batch_tile_variants(int dim);

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
            snprintf(k, sizeof(k), "batch_tile_%dd_%s", d, p ? "mixed" : "fp64");
            if (strcmp(k, key) == 0) {
                if (value < 0 || value >= batch_tile_variants(d)) return -1;
                g_batch_tile[d][p] = value;
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
            snprintf(k, sizeof(k), "batch_tile_%dd_%s", d, p ? "mixed" : "fp64");
            if (strcmp(k, key) == 0) return g_batch_tile[d][p];
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

// one CTA per JouleTile tile of the box
template <int DIM, int PREC>
__global__ void __launch_bounds__(kJouleThreads, 3) k_joule_pre(const __grid_constant__ TransportArgs a, int64_t ntiles)
{
    __shared__ double sJ[DIM * joule_face_box<DIM>()];
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        joule_tile<DIM, PREC>(a, (int)t, sJ);
        __syncthreads();  // the next tile rewrites sJ
    }
}

template <int DIM, int PREC>
static cudaError_t launch_jp(const TransportArgs& a, cudaStream_t st)
{
    const int64_t nt = joule_tile_count<DIM>(a.lo, a.hi);
    if (nt <= 0) return cudaSuccess;
    const unsigned g = (unsigned)(nt < (1 << 30) ? nt : (1 << 30));
    ProfScope ps("k_joule_pre", st);
    k_joule_pre<DIM, PREC><<<g, kJouleThreads, 0, st>>>(a, nt);
    return cudaGetLastError();
}

cudaError_t launch_joule_pre(const TransportArgs& a, int dim, int prec, cudaStream_t st)
{
    if (prec == PREC_MIXED) {
        if (dim == 1) return launch_jp<1, PREC_MIXED>(a, st);
        if (dim == 2) return launch_jp<2, PREC_MIXED>(a, st);
        return launch_jp<3, PREC_MIXED>(a, st);
    }
    if (dim == 1) return launch_jp<1, PREC_FP64>(a, st);
    if (dim == 2) return launch_jp<2, PREC_FP64>(a, st);
    return launch_jp<3, PREC_FP64>(a, st);
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

// ---------------------------------------------------------------------------
// Time-scale maxima (Vidyut::find_time_scales, Source/TimeStep.cpp:34-116): over
// the valid cells, max |mu_e| |E|, max D_e and max |mu_e| n_e, as the bit patterns
// of non-negative doubles (which order like the values) in out[0..2].
__global__ void __launch_bounds__(256) k_time_scales(BoxIdx b, int dim, A4 st, TransportArgs a,
                                                     unsigned long long* out)
{
    const int ns = a.ns, eidx = a.e_id;
    double m[3] = {0.0, 0.0, 0.0};
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < b.ncell;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_of(b, idx, i, j, k);
        const int64_t o = st.off(i, j, k);
        const double etemp = st.p[o + (int64_t)VD_ETEMP(ns) * st.ns];
        double esum = 0.0;
        for (int d = 0; d < dim; d++) {
            const double e = st.p[o + (int64_t)(VD_EFX(ns) + d) * st.ns];
            esum += e * e;
        }
        const double emag = sqrt(esum);
        double nd = 0.0;
        for (int s = 0; s < ns; s++) nd += st.p[o + (int64_t)s * st.ns];
        const double dc = a.const_ele_trans ? a.ele_diff / nd : diff_fp64(eidx, etemp, nd, a.Tg, emag);
        const double mu = a.const_ele_trans ? a.ele_mob / nd : mob_fp64(eidx, etemp, nd, a.Tg, emag);
        m[0] = fmax(m[0], fabs(mu) * emag);
        m[1] = fmax(m[1], dc);
        m[2] = fmax(m[2], fabs(mu) * st.p[o + (int64_t)eidx * st.ns]);
    }
    for (int q = 0; q < 3; q++) {
        double v = m[q];
        for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
        if ((threadIdx.x & 31) == 0) atomicMax(out + q, (unsigned long long)__double_as_longlong(v));
    }
}

cudaError_t launch_time_scales(const BoxIdx& b, int dim, const A4& st, const TransportArgs& a,
                               unsigned long long* out, cudaStream_t s)
{
    unsigned g = grid_for(b.ncell, 256);
    if (g > 148 * 8) g = 148 * 8;
    ProfScope ps("k_time_scales", s);
    k_time_scales<<<g, 256, 0, s>>>(b, dim, st, a, out);
    return cudaGetLastError();
}

}  // namespace vd
