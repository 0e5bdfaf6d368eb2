// vd_abi.cu -- extern "C" entry points (include/vidyut_b200.h).
//
// Every entry point validates its arguments on the host before launching: the box,
// the dimension, the scheme codes, and that each Array4 covers every cell the
// kernels will read or write (the stencil halo included).  A call that fails
// validation launches nothing and returns a negative status; vd_last_error() holds
// the reason.  Scratch (per-cell density sums, the reaction source when the caller
// does not want it) is taken from the stream-ordered allocator on the caller's
// stream and returned on the same stream, so concurrent calls on different streams
// never share it.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>
#include "../../include/vidyut_b200.h"
#include "vd_host.h"
#include "vd_kernels.cuh"

using namespace vd;

namespace {

thread_local std::string g_err;
std::mutex g_mech_mu;
vd_mech* g_mech = nullptr;       // host copy of the loaded mechanism
VdMechDev* g_mech_dev = nullptr; // host image of the device table
std::vector<int> g_loaded_dev;   // devices holding the current table
int g_mech_gen = 0;

int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char* fmt, ...)
{
    char buf[4096];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    return fail(VD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// Per-device resources set up once per device, at vd_mech_init or the first call
// on that device: the mechanism table, the library's own stream-ordered memory
// pool for per-call scratch, and the allocation-free update's fixed array.
//
// The scratch pool is the library's, not the device's default pool, so a host's
// own cudaMallocAsync frees keep the release behaviour the host chose; this pool
// keeps what it has taken between calls (no release at synchronisation) so that a
// time-step loop does not map and unmap memory at every step.
constexpr int kMaxDev = 64;
cudaMemPool_t g_pool[kMaxDev] = {};

// The allocation-free update's scratch (vd_explicit_update_all_noalloc).  In host
// code the name below is only a host-side stand-in; the array's device address is
// looked up once per device, with that device current, and passed to the kernels.
// The lookup makes the runtime load this file's module, which is when the array
// is reserved on the device.
constexpr size_t kNoallocDoubles = VD_NOALLOC_SCRATCH_BYTES / sizeof(double);
static __device__ __align__(256) double g_noalloc_scratch[kNoallocDoubles];
double* g_noalloc_ptr[kMaxDev] = {nullptr};

int setup_device(int dev)
{
    if (!g_pool[dev]) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool;
        cudaError_t e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return cuda_fail(e, "creating the scratch memory pool");
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return cuda_fail(e, "configuring the scratch memory pool");
        }
        g_pool[dev] = pool;
    }
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(allocation-free scratch)");
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    return VD_OK;
}

// Loads the mechanism table onto the current device if it is not there yet, and
// sets the device up (setup_device).
int ensure_mech_on_device(cudaStream_t st)
{
    std::lock_guard<std::mutex> lk(g_mech_mu);
    if (!g_mech) return fail(VD_ERR_MECH, "no mechanism loaded: call vd_mech_init first");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDev) return fail(VD_ERR_ARG, "device ordinal %d not supported", dev);
    for (int d : g_loaded_dev)
        if (d == dev) return VD_OK;
    int rc = setup_device(dev);
    if (rc) return rc;
    rc = upload_mech(g_mech_dev, st);
    if (rc != 0) return cuda_fail((cudaError_t)rc, "uploading mechanism table");
    g_loaded_dev.push_back(dev);
    return VD_OK;
}

// Scratch of one call from the library's pool on the current device (set up by
// ensure_mech_on_device), stream-ordered on st; released with cudaFreeAsync.
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDev || !g_pool[dev]) return cudaErrorNotReady;
    return cudaMallocFromPoolAsync(p, bytes, g_pool[dev], st);
}

int nspecies()
{
    std::lock_guard<std::mutex> lk(g_mech_mu);
    return g_mech ? g_mech->nspecies : -1;
}

bool valid_box(const vd_box* bx)
{
    if (!bx) return false;
    if (bx->dim < 1 || bx->dim > 3) return false;
    for (int d = 0; d < 3; d++) {
        if (bx->hi[d] < bx->lo[d]) return false;
        if (d >= bx->dim && (bx->lo[d] != 0 || bx->hi[d] != 0)) return false;
    }
    return true;
}

// Array4 covers cells lo..hi (inclusive) with at least ncomp components and a
// non-overlapping layout.
bool covers(const vd_array4& a, const int lo[3], const int hi[3], int ncomp, std::string* why)
{
    char buf[256];
    if (!a.p) { *why = "null data pointer"; return false; }
    if (((uintptr_t)a.p) % 8) { *why = "data pointer not 8-byte aligned"; return false; }
    if (a.ncomp < ncomp) {
        snprintf(buf, sizeof(buf), "ncomp %d < %d", a.ncomp, ncomp);
        *why = buf;
        return false;
    }
    for (int d = 0; d < 3; d++) {
        if (a.begin[d] > lo[d] || a.end[d] <= hi[d]) {
            snprintf(buf, sizeof(buf), "index range [%d,%d) in direction %d does not cover [%d,%d]", a.begin[d],
                     a.end[d], d, lo[d], hi[d]);
            *why = buf;
            return false;
        }
    }
    int64_t nx = a.end[0] - a.begin[0], ny = a.end[1] - a.begin[1], nz = a.end[2] - a.begin[2];
    if (a.jstride < nx || a.kstride < a.jstride * ny || (ncomp > 1 && a.nstride < a.kstride * nz)) {
        *why = "strides overlap";
        return false;
    }
    return true;
}

BoxIdx box_idx(const int lo[3], const int hi[3])
{
    BoxIdx b;
    for (int d = 0; d < 3; d++) {
        b.lo[d] = lo[d];
        b.hi[d] = hi[d];
        b.n[d] = hi[d] - lo[d] + 1;
    }
    b.ncell = (int64_t)b.n[0] * b.n[1] * b.n[2];
    return b;
}

int stencil_halo(int hyp_order) { return hyp_order == 5 ? 3 : hyp_order; }

int check_scheme(int hyp_order, int weno)
{
    if (hyp_order != 1 && hyp_order != 2 && hyp_order != 5)
        return fail(VD_ERR_SCHEME, "hyp_order %d not implemented (1, 2 or 5)", hyp_order);
    if (hyp_order == 5 && (weno < 1 || weno > 3))
        return fail(VD_ERR_SCHEME, "Unknown WENO scheme %d (1 JS, 2 M, 3 Z)", weno);
    return VD_OK;
}

void fill_class_flags(const vd_params* p, int8_t zlo[4][3], int8_t zhi[4][3])
{
    for (int c = 0; c < 4; c++)
        for (int d = 0; d < 3; d++) {
            zlo[c][d] = p->bc_lo[c][d] == VD_BC_IHNEU;
            zhi[c][d] = p->bc_hi[c][d] == VD_BC_IHNEU;
        }
}

// fluxed / unfluxed species lists and velocity bases of a transport record
void finish_lists(TransportArgs& a)
{
    std::lock_guard<std::mutex> lk(g_mech_mu);
    finish_species_lists(a, *g_mech_dev);
}

}  // namespace

// ===========================================================================
extern "C" {

int vd_abi_version(void) { return VD_ABI_VERSION; }

size_t vd_sizeof(int which)
{
    switch (which) {
    case 0: return sizeof(vd_array4);
    case 1: return sizeof(vd_box);
    case 2: return sizeof(vd_reaction);
    case 3: return sizeof(vd_mech);
    case 4: return sizeof(vd_params);
    case 5: return sizeof(vd_poisson_params);
    case 6: return sizeof(vd_diffusion_params);
    case 7: return sizeof(vd_batch_stats);
    case 8: return sizeof(vd_server_stats);
    default: return 0;
    }
}

const char* vd_last_error(void) { return g_err.c_str(); }

const char* vd_status_string(int s)
{
    switch (s) {
    case VD_OK: return "ok";
    case VD_ERR_ARG: return "invalid argument";
    case VD_ERR_SCHEME: return "unknown scheme";
    case VD_ERR_GHOST: return "too few ghost cells";
    case VD_ERR_DIM: return "unsupported dimension";
    case VD_ERR_MECH: return "mechanism not loaded or invalid";
    case VD_ERR_CUDA: return "CUDA error";
    case VD_ERR_TIMEOUT: return "timeout";
    case VD_ERR_NOMEM: return "out of device memory";
    case VD_ERR_NONFINITE: return "non-finite input";
    case VD_ERR_BUDGET: return "over HBM budget";
    case VD_ERR_STATE: return "call out of order";
    default: return "unknown status";
    }
}

// Validates a mechanism table and builds its device image (no device access).
static int build_mech_table(const vd_mech* m, VdMechDev** out)
{
    if (!m) return fail(VD_ERR_ARG, "null mechanism");
    const int ns = m->nspecies, nr = m->nreactions;
    if (ns < 1 || ns > VD_MAX_SPECIES) return fail(VD_ERR_MECH, "nspecies %d outside [1,%d]", ns, VD_MAX_SPECIES);
    if (nr < 0 || nr > VD_MAX_REACTIONS)
        return fail(VD_ERR_MECH, "nreactions %d outside [0,%d]", nr, VD_MAX_REACTIONS);
    if (m->e_id < 0 || m->e_id >= ns) return fail(VD_ERR_MECH, "electron index %d invalid", m->e_id);
    if (m->nfits < 0 || m->nfits > VD_MAX_FITS) return fail(VD_ERR_MECH, "nfits %d outside [0,%d]", m->nfits, VD_MAX_FITS);
    for (int s = 0; s <= ns; s++) {
        int k = m->mob_kind[s];
        if (k < 0 || k > 8) return fail(VD_ERR_MECH, "species %d: unknown mobility kind %d", s, k);
        if ((k == VD_MOB_POW_EMAG || k == VD_MOB_EN_POLY) && !std::isfinite(m->mob_p1[s]))
            return fail(VD_ERR_MECH, "species %d: mobility exponent must be finite", s);
        if ((k == VD_MOB_EN_POLY || k == VD_MOB_EXP_MEANE) && (m->mob_ref[s] < 0 || m->mob_ref[s] >= m->nfits))
            return fail(VD_ERR_MECH, "species %d: mobility fit index %d outside [0,%d)", s, m->mob_ref[s], m->nfits);
        if (k == VD_MOB_SCALED) {
            int r = m->mob_ref[s];
            if (r < 0 || r > ns || m->mob_kind[r] == VD_MOB_SCALED)
                return fail(VD_ERR_MECH, "species %d: scaled mobility must refer to an unscaled model", s);
        }
        if ((k == VD_MOB_ELECTRON || k == VD_MOB_ION_TG) && !(m->mob_p0[s] > 0.0))
            return fail(VD_ERR_MECH, "species %d: cross section must be > 0", s);
        if (k == VD_MOB_ION_TG && !(m->mob_p1[s] > 0.0))
            return fail(VD_ERR_MECH, "species %d: particle mass must be > 0", s);
        int dk = m->diff_kind[s];
        if (dk < 0 || dk > 7) return fail(VD_ERR_MECH, "species %d: unknown diffusion kind %d", s, dk);
        if (dk == VD_DIFF_POW_EMAG && !std::isfinite(m->diff_p1[s]))
            return fail(VD_ERR_MECH, "species %d: |E| exponent must be finite", s);
        if (dk == VD_DIFF_TE_PRES && !(std::isfinite(m->diff_p1[s]) && m->diff_p1[s] != 0.0))
            return fail(VD_ERR_MECH, "species %d: temperature scale must be finite and nonzero", s);
        if ((dk == VD_DIFF_TE_ABSMOB || dk == VD_DIFF_TG_MOB || dk == VD_DIFF_SCALED) &&
            (m->diff_ref[s] < 0 || m->diff_ref[s] > ns))
            return fail(VD_ERR_MECH, "species %d: diffusion reference invalid", s);
        if (dk == VD_DIFF_SCALED && m->diff_kind[m->diff_ref[s]] == VD_DIFF_SCALED)
            return fail(VD_ERR_MECH, "species %d: scaled diffusion must refer to an unscaled model", s);
    }
    if (m->elastic_loss && !(m->elastic_mass > 0.0)) return fail(VD_ERR_MECH, "elastic_mass must be > 0");
    for (int f = 0; f < m->nfits; f++) {
        const vd_rate_fit& F = m->fits[f];
        bool ok = std::isfinite(F.jA) && std::isfinite(F.fA) && F.jA >= 0.0 && F.fA >= 0.0 && std::isfinite(F.switch_ev);
        for (int j = 0; j < 9; j++) ok = ok && std::isfinite(F.jc[j]);
        for (int j = 0; j < 4; j++) ok = ok && std::isfinite(F.fc[j]);
        if (!ok) return fail(VD_ERR_MECH, "fit %d: coefficients must be finite, A >= 0", f);
    }
    for (int r = 0; r < nr; r++) {
        const vd_reaction& R = m->rxn[r];
        if (R.kind < 0 || R.kind > 6) return fail(VD_ERR_MECH, "reaction %d: unknown rate kind %d", r, R.kind);
        if (R.kind >= VD_RATE_JANEV && (R.fit < 0 || R.fit >= m->nfits))
            return fail(VD_ERR_MECH, "reaction %d: fit index %d outside [0,%d)", r, R.fit, m->nfits);
        if (R.nreac < 1 || R.nreac > VD_MAX_REACTANTS)
            return fail(VD_ERR_MECH, "reaction %d: %d reactants", r, R.nreac);
        for (int t = 0; t < R.nreac; t++)
            if (R.reac[t] < 0 || R.reac[t] >= ns) return fail(VD_ERR_MECH, "reaction %d: bad reactant", r);
        if (R.nterms < 0 || R.nterms > VD_MAX_TERMS) return fail(VD_ERR_MECH, "reaction %d: bad term count", r);
        for (int t = 0; t < R.nterms; t++)
            if (R.term_sp[t] < 0 || R.term_sp[t] >= ns) return fail(VD_ERR_MECH, "reaction %d: bad term", r);
        if (R.rxntype < 0 || R.rxntype > 7 || R.rxntype == 6)
            return fail(VD_ERR_MECH, "reaction %d: unknown rxntype %d", r, R.rxntype);
        if (R.rxntype == VD_RXN_ELASTIC && (R.elidx < 0 || R.elidx >= ns))
            return fail(VD_ERR_MECH, "reaction %d: bad elidx", r);
        if (!(R.A >= 0.0) || !std::isfinite(R.A) || !std::isfinite(R.b) || !std::isfinite(R.C))
            return fail(VD_ERR_MECH, "reaction %d: A must be finite and >= 0, b and C finite", r);
    }

    VdMechDev* d = new VdMechDev;
    memset(d, 0, sizeof(*d));
    d->ns = ns;
    d->nr = nr;
    d->e_id = m->e_id;
    d->elastic_loss = m->elastic_loss;
    d->elastic_coef = m->elastic_loss ? (2.0 * ME / m->elastic_mass) : 0.0;
    for (int s = 0; s < ns; s++) d->charge[s] = (int8_t)m->charge[s];
    for (int s = 0; s <= ns; s++) {
        d->mob_kind[s] = (int8_t)m->mob_kind[s];
        d->mob_ref[s] = (int8_t)m->mob_ref[s];
        d->mob_p0[s] = m->mob_p0[s];
        d->mob_p1[s] = m->mob_p1[s];
        d->diff_kind[s] = (int8_t)m->diff_kind[s];
        d->diff_ref[s] = (int8_t)m->diff_ref[s];
        d->diff_factor[s] = m->diff_factor[s];
        d->diff_p1[s] = m->diff_p1[s];
        if (m->mob_kind[s] == VD_MOB_ELECTRON) d->mob_c[s] = (-ECHARGE / ME) / std::sqrt(8.0 * K_B / PI / ME);
        else if (m->mob_kind[s] == VD_MOB_ION_TG)
            d->mob_c[s] = (ECHARGE / m->mob_p1[s]) / std::sqrt(8.0 * K_B / PI / m->mob_p1[s]);
    }
    d->nfits = m->nfits;
    for (int f = 0; f < m->nfits; f++) {
        const vd_rate_fit& F = m->fits[f];
        VdFitDev& G = d->fits[f];
        G.jA = F.jA;
        G.fA = F.fA;
        for (int j = 0; j < 9; j++) G.jc[j] = F.jc[j];
        for (int j = 0; j < 4; j++) G.fc[j] = F.fc[j];
        G.switch_ev = F.switch_ev;
        G.l2jA = F.jA > 0.0 ? std::log2(F.jA * NA_CE) : -INFINITY;
        G.l2fA = F.fA > 0.0 ? std::log2(F.fA * NA_CE) : -INFINITY;
    }
    // |E| reaches the electrons' transport when their mobility (or the one it
    // scales, or their diffusion coefficient's) is a power of |E|
    // (or a function of |E|/N)
    auto mob_emag = [&](int s) {
        int k = m->mob_kind[s];
        if (k == VD_MOB_SCALED) k = m->mob_kind[m->mob_ref[s]];
        return k == VD_MOB_POW_EMAG || k == VD_MOB_EN_POLY;
    };
    auto diff_emag = [&](int s) {
        int dk = m->diff_kind[s];
        if (dk == VD_DIFF_SCALED) {
            s = m->diff_ref[s];
            dk = m->diff_kind[s];
        }
        return dk == VD_DIFF_POW_EMAG || ((dk == VD_DIFF_TE_ABSMOB || dk == VD_DIFF_TG_MOB) && mob_emag(m->diff_ref[s]));
    };
    {
        const int e = m->e_id;
        d->emag_e = (int8_t)(mob_emag(e) || diff_emag(e));
        bool en = m->elastic_loss && mob_emag(e);
        for (int r = 0; r < nr; r++) en = en || m->rxn[r].kind == VD_RATE_TOWNSEND;
        d->need_en = (int8_t)en;
    }
    {
        // the transport tile stages at most kMaxBases velocity bases
        VelBasis bs[VD_MAX_SPECIES + 1];
        int nb = 0;
        for (int s = 0; s <= ns; s++) {
            VelBasis b;
            double K;
            if (!velocity_basis(*d, s, 300.0, &b, &K)) continue;
            bool seen = false;
            for (int q = 0; q < nb; q++) seen = seen || same_basis(*d, bs[q], b);
            if (!seen) bs[nb++] = b;
        }
        if (nb > kMaxBases) {
            delete d;
            return fail(VD_ERR_MECH, "the mobility models need %d velocity bases (at most %d)", nb, kMaxBases);
        }
    }
    for (int r = 0; r < nr; r++) {
        const vd_reaction& R = m->rxn[r];
        VdRxnDev& D = d->rxn[r];
        D.A = R.A;
        D.b = R.b;
        D.C = R.C;
        D.lnA = (R.A > 0.0) ? std::log(R.A) : -INFINITY;
        D.l2A = (R.A > 0.0) ? std::log2(R.A) : -INFINITY;
        D.Cl2 = R.C * 1.4426950408889634073599;  // log2(e)
        if (R.rxntype == VD_RXN_EXCITATION || R.rxntype == VD_RXN_IONIZATION) D.ex = (R.eexci * EV2J) * NA_CE;
        else if (R.rxntype == VD_RXN_ELASTIC) D.ex = 3.0 * KB_CE * (m->mw[m->e_id] / m->mw[R.elidx]);
        D.kind = (int8_t)R.kind;
        D.nreac = (int8_t)R.nreac;
        D.rxntype = (int8_t)R.rxntype;
        D.elidx = (int8_t)R.elidx;
        D.nterms = (int8_t)R.nterms;
        D.fit = (int8_t)(R.kind >= VD_RATE_JANEV ? R.fit : 0);
        for (int t = 0; t < R.nreac; t++) D.reac[t] = (int8_t)R.reac[t];
        for (int t = 0; t < R.nterms; t++) {
            D.sp[t] = (int8_t)R.term_sp[t];
            D.coef[t] = R.term_coef[t];
        }
    }
    *out = d;
    return VD_OK;
}

int vd_mech_specialize_check(const vd_mech* m, size_t* cubin_bytes)
{
    VdMechDev* d = nullptr;
    int rc = build_mech_table(m, &d);
    if (rc) return rc;
    size_t n = 0;
    rc = spec_compile_only(*d, &n);
    delete d;
    if (cubin_bytes) *cubin_bytes = n;
    if (rc) return fail(VD_ERR_MECH, "%s", spec_error());
    fail(VD_OK, "%s", spec_error());  // the ptxas resource report, for the caller's information
    return VD_OK;
}

int vd_mech_init(const vd_mech* m)
{
    VdMechDev* d = nullptr;
    int brc = build_mech_table(m, &d);
    if (brc) return brc;
    vd_mech* hm = new vd_mech;
    memcpy(hm, m, sizeof(vd_mech));
    {
        std::lock_guard<std::mutex> lk(g_mech_mu);
        delete g_mech;
        delete g_mech_dev;
        g_mech = hm;
        g_mech_dev = d;
        g_loaded_dev.clear();
        g_mech_gen++;
    }
    int rc = ensure_mech_on_device(0);
    if (rc) return rc;
    spec_build(*d);  // table-driven chemistry stays in use if this fails
    return VD_OK;
}

int vd_mech_specialized(void) { return spec_active() ? 1 : 0; }

const char* vd_mech_specialize_status(void) { return spec_active() ? "specialised" : spec_error(); }

int vd_set_specialize(int on)
{
    spec_set_enabled(on != 0);
    return VD_OK;
}

int vd_tune_set(const char* key, int value)
{
    if (!key) return fail(VD_ERR_ARG, "null key");
    int rc = tune_set(key, value);
    if (rc == -2) return fail(VD_ERR_ARG, "unknown tuning key %s", key);
    if (rc) return fail(VD_ERR_ARG, "value %d out of range for %s", value, key);
    return VD_OK;
}

int vd_tune_get(const char* key)
{
    if (!key) return fail(VD_ERR_ARG, "null key");
    int v = tune_get(key);
    if (v == -2) return fail(VD_ERR_ARG, "unknown tuning key %s", key);
    return v;
}

// ---------------------------------------------------------------------------
int vd_compute_explicit_flux(const vd_box* bx, int dir, int specid, vd_array4 phi, const int32_t bclo[3],
                             const int32_t bchi[3], const int32_t domlo[3], const int32_t domhi[3], vd_array4 fx,
                             double Tg, double Pg, double time, const double dx[3], double dt, int hyp_order,
                             int user_defined_vel, int weno_scheme, const double user_vel[3], int vel_species,
                             void* stream)
{
    (void)Pg;
    (void)time;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_mech_on_device(st);
    if (rc) return rc;
    const int ns = nspecies();
    if (!valid_box(bx)) return fail(bx && (bx->dim < 1 || bx->dim > 3) ? VD_ERR_DIM : VD_ERR_ARG, "invalid box");
    if (dir < 0 || dir >= bx->dim) return fail(VD_ERR_ARG, "sweep direction %d outside [0,%d)", dir, bx->dim);
    if (specid < 0 || specid > ns) return fail(VD_ERR_ARG, "specid %d outside [0,%d]", specid, ns);
    if (!bclo || !bchi || !domlo || !domhi || !dx) return fail(VD_ERR_ARG, "null argument");
    if ((rc = check_scheme(hyp_order, weno_scheme))) return rc;
    if (user_defined_vel && !user_vel) return fail(VD_ERR_ARG, "user_defined_vel needs user_vel");
    const int H = stencil_halo(hyp_order);
    int lo[3] = {bx->lo[0], bx->lo[1], bx->lo[2]}, hi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
    int flo[3] = {lo[0], lo[1], lo[2]}, fhi[3] = {hi[0], hi[1], hi[2]};
    fhi[dir] += 1;
    int rlo[3] = {lo[0], lo[1], lo[2]}, rhi[3] = {hi[0], hi[1], hi[2]};
    rlo[dir] -= H;
    rhi[dir] += H;
    std::string why;
    if (!covers(phi, rlo, rhi, VD_NVAR(ns), &why)) return fail(VD_ERR_GHOST, "phi: %s", why.c_str());
    if (!covers(fx, flo, fhi, 1, &why)) return fail(VD_ERR_ARG, "fx: %s", why.c_str());
    int8_t zlo[3], zhi[3];
    for (int d = 0; d < 3; d++) {
        zlo[d] = bclo[d] == VD_BC_IHNEU;
        zhi[d] = bchi[d] == VD_BC_IHNEU;
    }
    double dxmin = dx[0];
    for (int d = 1; d < bx->dim; d++) dxmin = dx[d] < dxmin ? dx[d] : dxmin;
    double uv[3] = {0, 0, 0};
    if (user_vel)
        for (int d = 0; d < 3; d++) uv[d] = user_vel[d];
    int dl[3] = {domlo[0], domlo[1], domlo[2]}, dh[3] = {domhi[0], domhi[1], domhi[2]};
    cudaError_t e = launch_face_flux(box_idx(flo, fhi), dir, specid, A4(phi), A4(fx), zlo, zhi, dl, dh, Tg, dxmin,
                                     dt, hyp_order, user_defined_vel, weno_scheme, uv, vel_species, ns, st);
    if (e != cudaSuccess) return cuda_fail(e, "k_face_flux launch");
    return VD_OK;
}

int vd_compute_dsdt(const vd_box* bx, int specid, const vd_array4 flux[3], vd_array4 rxn, vd_array4 dsdt,
                    const double dx[3], void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const int ns = nspecies();
    if (ns < 0) return fail(VD_ERR_MECH, "no mechanism loaded: call vd_mech_init first");
    if (!valid_box(bx)) return fail(VD_ERR_ARG, "invalid box");
    if (!flux || !dx) return fail(VD_ERR_ARG, "null argument");
    if (specid < 0 || specid > ns) return fail(VD_ERR_ARG, "specid %d outside [0,%d]", specid, ns);
    std::string why;
    for (int d = 0; d < bx->dim; d++) {
        int fhi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
        fhi[d] += 1;
        if (!covers(flux[d], bx->lo, fhi, 1, &why)) return fail(VD_ERR_ARG, "flux[%d]: %s", d, why.c_str());
    }
    if (!covers(rxn, bx->lo, bx->hi, specid + 1, &why)) return fail(VD_ERR_ARG, "rxn: %s", why.c_str());
    if (!covers(dsdt, bx->lo, bx->hi, 1, &why)) return fail(VD_ERR_ARG, "dsdt: %s", why.c_str());
    A4 f[3];
    for (int d = 0; d < 3; d++) f[d] = (d < bx->dim) ? A4(flux[d]) : A4(flux[0]);
    cudaError_t e = launch_dsdt(box_idx(bx->lo, bx->hi), bx->dim, specid, f, A4(rxn), A4(dsdt), dx, st);
    if (e != cudaSuccess) return cuda_fail(e, "k_dsdt launch");
    return VD_OK;
}

int vd_reaction_source(const vd_box* bx, vd_array4 sborder, vd_array4 rxn, double Tg, double Pg, double time,
                       void* stream)
{
    (void)Pg;
    (void)time;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_mech_on_device(st);
    if (rc) return rc;
    const int ns = nspecies();
    if (!valid_box(bx)) return fail(VD_ERR_ARG, "invalid box");
    std::string why;
    if (!covers(sborder, bx->lo, bx->hi, VD_NVAR(ns), &why)) return fail(VD_ERR_ARG, "sborder: %s", why.c_str());
    if (!covers(rxn, bx->lo, bx->hi, ns + 1, &why)) return fail(VD_ERR_ARG, "rxn: %s", why.c_str());
    cudaError_t e = launch_reaction_source(box_idx(bx->lo, bx->hi), A4(sborder), A4(rxn), Tg, PREC_FP64, ns, st);
    if (e != cudaSuccess) return cuda_fail(e, "k_reaction_source launch");
    return VD_OK;
}

static int check_params(const vd_box* bx, const vd_params* p)
{
    if (!valid_box(bx)) return fail(bx && (bx->dim < 1 || bx->dim > 3) ? VD_ERR_DIM : VD_ERR_ARG, "invalid box");
    if (!p) return fail(VD_ERR_ARG, "null params");
    if (p->dim != bx->dim) return fail(VD_ERR_DIM, "params.dim %d != box.dim %d", p->dim, bx->dim);
    for (int d = 0; d < bx->dim; d++)
        if (!(p->dx[d] > 0.0) || !std::isfinite(p->dx[d])) return fail(VD_ERR_ARG, "dx[%d] must be finite and > 0", d);
    if (p->precision != VD_PREC_FP64 && p->precision != VD_PREC_MIXED)
        return fail(VD_ERR_ARG, "unknown precision %d", p->precision);
    // the chemistry takes log(Tg) and 1/Tg, the ion mobility sqrt(Tg)
    if (!(p->Tg > 0.0) || !std::isfinite(p->Tg)) return fail(VD_ERR_ARG, "Tg must be finite and > 0 (got %g)", p->Tg);
    if (!(p->dt >= 0.0) || !std::isfinite(p->dt)) return fail(VD_ERR_ARG, "dt must be finite and >= 0 (got %g)", p->dt);
    return check_scheme(p->hyp_order, p->weno_scheme);
}

// The loaded mechanism as the update's host code needs it.
static vd_host::MechInfo mech_snapshot()
{
    vd_host::MechInfo mi;
    memset(&mi, 0, sizeof(mi));
    std::lock_guard<std::mutex> lk(g_mech_mu);
    mi.ns = g_mech->nspecies;
    mi.e_id = g_mech->e_id;
    mi.generation = g_mech_gen;
    for (int s = 0; s <= g_mech->nspecies; s++) mi.mob_kind[s] = g_mech->mob_kind[s];
    for (int s = 0; s < g_mech->nspecies; s++) mi.charge[s] = g_mech->charge[s];
    return mi;
}

// Scalars of a transport record from the box and the parameters.
static void fill_cfg(TransportArgs& a, const vd_box* bx, const vd_params* p, int ns, int e_id, int e_charge)
{
    memset(&a, 0, sizeof(a));
    for (int d = 0; d < 3; d++) {
        a.lo[d] = bx->lo[d];
        a.hi[d] = bx->hi[d];
        a.dx[d] = (d < bx->dim) ? p->dx[d] : 1.0;
        a.idx[d] = 1.0 / a.dx[d];
        a.domlo[d] = p->domlo[d];
        a.domhi[d] = p->domhi[d];
        a.uvel[d] = p->user_vel[d];
    }
    a.dxmin = a.dx[0];
    for (int d = 1; d < bx->dim; d++) a.dxmin = a.dx[d] < a.dxmin ? a.dx[d] : a.dxmin;
    a.dt = p->dt;
    a.Tg = p->Tg;
    fill_class_flags(p, a.zlo, a.zhi);
    a.ns = ns;
    a.e_id = e_id;
    a.hyp_order = p->hyp_order;
    a.weno = p->weno_scheme;
    a.udv = p->user_defined_vel;
    a.vel_sp = p->vel_species;
    a.elecenergy = p->elecenergy_solve;
    a.do_bg = p->do_bg_reactions;
    a.bound_specden = p->bound_specden;
    a.floor_jh = p->floor_jh;
    a.const_ele_trans = p->const_ele_trans;
    a.cs_technique = p->cs_technique;
    a.gradne_from_state = p->gradne_from_state;
    a.update_te = p->update_te;
    a.min_spec = p->min_species_density;
    a.min_elec = p->min_electron_density;
    a.ele_mob = p->ele_mob;
    a.ele_diff = p->ele_diff;
    a.min_te = p->min_electron_temp;
    a.charge_e = (double)e_charge * ECHARGE;
    a.ghost = stencil_halo(p->hyp_order);
    a.write_diag = 1;
}

// The species of a transport record: transported species (and the electron
// energy when it is solved) in species order with their BC class and whether they
// have a drift flux, background species apart (Source/Evolve.cpp:208-288); then
// the derived fluxed / unfluxed lists and velocity bases (finish_species_lists).
static void fill_species(TransportArgs& a, const vd_params* p, const vd_host::MechInfo& m)
{
    const int ns = m.ns;
    a.ntr = 0;
    a.nbg = 0;
    for (int s = 0; s <= ns; s++) {
        const bool energy = (s == ns);
        if (energy && !p->elecenergy_solve) continue;
        if (!energy && ((p->bg_mask >> s) & 1ull)) {
            a.bg_sp[a.nbg++] = (int8_t)s;
            continue;
        }
        a.tr_sp[a.ntr] = (int8_t)s;
        const int cls = energy ? VD_CLASS_ENERGY
                               : (s == m.e_id ? VD_CLASS_ELECTRON : (m.charge[s] != 0 ? VD_CLASS_ION : VD_CLASS_NEUTRAL));
        a.tr_cls[a.ntr] = (int8_t)cls;
        const bool has_vel = p->user_defined_vel ? (s == p->vel_species) : (m.mob_kind[s] != VD_MOB_ZERO);
        a.tr_flux[a.ntr] = (p->do_transport && has_vel) ? 1 : 0;
        a.ntr++;
    }
    finish_lists(a);
}

// Validation beyond check_params that every update of a box makes.
static int check_update_species(const vd_params* p, const vd_host::MechInfo& m)
{
    if (p->bg_mask >> m.ns) return fail(VD_ERR_ARG, "bg_mask names species >= %d", m.ns);
    if (p->bg_mask & (1ull << m.e_id)) return fail(VD_ERR_ARG, "electrons cannot be a background species");
    if (p->user_defined_vel && (p->vel_species < 0 || p->vel_species > m.ns))
        return fail(VD_ERR_ARG, "vel_species invalid");
    return VD_OK;
}

// Views of the face arrays the Joule term reads (efield_ec unless cs_technique,
// gradne_fc unless gradne_from_state), each checked to cover the face box of its
// direction.
static int face_views(const vd_box* bx, const vd_params* prm, const vd_array4 efield_ec[3],
                      const vd_array4 gradne_fc[3], A4 ef[3], A4 gne[3])
{
    std::string why;
    for (int d = 0; d < bx->dim; d++) {
        int fhi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
        fhi[d] += 1;
        if (!prm->cs_technique) {
            if (!efield_ec) return fail(VD_ERR_ARG, "efield_ec is null");
            if (!covers(efield_ec[d], bx->lo, fhi, 1, &why))
                return fail(VD_ERR_ARG, "efield_ec[%d]: %s", d, why.c_str());
            ef[d] = A4(efield_ec[d]);
        }
        if (!prm->gradne_from_state) {
            if (!gradne_fc) return fail(VD_ERR_ARG, "gradne_fc is null");
            if (!covers(gradne_fc[d], bx->lo, fhi, 1, &why))
                return fail(VD_ERR_ARG, "gradne_fc[%d]: %s", d, why.c_str());
            gne[d] = A4(gradne_fc[d]);
        }
    }
    return VD_OK;
}

int vd_elecenergy_source(const vd_box* bx, vd_array4 sborder, vd_array4 rxn, const vd_array4 efield_ec[3],
                         const vd_array4 gradne_fc[3], vd_array4 dsdt, vd_array4 phi_new, const vd_params* prm,
                         void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_mech_on_device(st);
    if (rc) return rc;
    if (!valid_box(bx) || !prm) return fail(VD_ERR_ARG, "invalid box or params");
    if (prm->dim != bx->dim) return fail(VD_ERR_DIM, "params.dim != box.dim");
    if (!(prm->Tg > 0.0) || !std::isfinite(prm->Tg)) return fail(VD_ERR_ARG, "Tg must be finite and > 0");
    const vd_host::MechInfo m = mech_snapshot();
    const int ns = m.ns;
    std::string why;
    int glo[3] = {bx->lo[0], bx->lo[1], bx->lo[2]}, ghi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
    for (int d = 0; d < bx->dim; d++) {
        glo[d] -= 1;
        ghi[d] += 1;
    }
    if (!covers(sborder, glo, ghi, VD_NVAR(ns), &why)) return fail(VD_ERR_GHOST, "sborder: %s", why.c_str());
    if (!covers(rxn, bx->lo, bx->hi, ns + 1, &why)) return fail(VD_ERR_ARG, "rxn: %s", why.c_str());
    if (!covers(dsdt, bx->lo, bx->hi, 1, &why)) return fail(VD_ERR_ARG, "dsdt: %s", why.c_str());
    if (!covers(phi_new, bx->lo, bx->hi, VD_NVAR(ns), &why)) return fail(VD_ERR_ARG, "phi_new: %s", why.c_str());
    A4 ef[3], gne[3];
    if ((rc = face_views(bx, prm, efield_ec, gradne_fc, ef, gne))) return rc;
    TransportArgs cfg;
    fill_cfg(cfg, bx, prm, ns, m.e_id, m.charge[m.e_id]);
    cudaError_t e = launch_joule(box_idx(bx->lo, bx->hi), bx->dim, A4(sborder), A4(rxn), ef, gne, A4(dsdt),
                                 A4(phi_new), cfg, st);
    if (e != cudaSuccess) return cuda_fail(e, "k_joule launch");
    return VD_OK;
}

// ---------------------------------------------------------------------------
// One fused explicit update of a box (vd_explicit_update_all and its
// allocation-free form share all of it but the origin of the scratch).
//
// Scratch layout: the status word of the non-finite check (kStatusBytes, so the
// rest stays 256-byte aligned), the density sums N over the stencil-grown box,
// then the reaction source (NS+1 components over the valid box) when the caller
// passes no rxn array.
constexpr size_t kStatusBytes = 256;

struct UpdatePlan {
    TransportArgs a;
    PrepArgs pa;
    int glo[3], ghi[3];
    int64_t gn, vn;   // cells of the grown box and of the valid box
    bool own_rxn;     // the reaction source lives in scratch
    bool check;       // prm->check_finite
    int dim, prec;
    size_t scratch_bytes() const
    {
        return kStatusBytes + (size_t)gn * sizeof(double) + (own_rxn ? (size_t)vn * (a.ns + 1) * sizeof(double) : 0);
    }
};

// Validates the arguments and fills everything of the plan but the scratch
// pointers.  Launches nothing.
static int plan_update(const vd_box* bx, vd_array4 sborder, const vd_array4 efield_ec[3],
                       const vd_array4 gradne_fc[3], vd_array4 phi_new, vd_array4 dsdt, vd_array4 rxn,
                       const vd_params* prm, UpdatePlan* P)
{
    int rc;
    if ((rc = check_params(bx, prm))) return rc;
    const vd_host::MechInfo m = mech_snapshot();
    if ((rc = check_update_species(prm, m))) return rc;
    const int ns = m.ns, dim = bx->dim;
    const int H = stencil_halo(prm->hyp_order);
    std::string why;
    for (int d = 0; d < 3; d++) {
        P->glo[d] = bx->lo[d];
        P->ghi[d] = bx->hi[d];
    }
    for (int d = 0; d < dim; d++) {
        P->glo[d] -= H;
        P->ghi[d] += H;
    }
    // the stencil only reaches along one axis at a time; corners are never read,
    // but the per-cell density sums cover the whole grown box, so require it.
    if (!covers(sborder, P->glo, P->ghi, VD_NVAR(ns), &why)) return fail(VD_ERR_GHOST, "sborder: %s", why.c_str());
    if (!covers(phi_new, bx->lo, bx->hi, VD_NVAR(ns), &why)) return fail(VD_ERR_ARG, "phi_new: %s", why.c_str());
    if (dsdt.p && !covers(dsdt, bx->lo, bx->hi, ns + 1, &why)) return fail(VD_ERR_ARG, "dsdt: %s", why.c_str());
    if (rxn.p && !covers(rxn, bx->lo, bx->hi, ns + 1, &why)) return fail(VD_ERR_ARG, "rxn: %s", why.c_str());
    A4 ef[3], gne[3];
    if (prm->elecenergy_solve && (rc = face_views(bx, prm, efield_ec, gradne_fc, ef, gne))) return rc;

    TransportArgs& a = P->a;
    fill_cfg(a, bx, prm, ns, m.e_id, m.charge[m.e_id]);
    fill_species(a, prm, m);
    int tile[3];
    transport_tile(dim, tile);
    for (int d = 0; d < 3; d++) {
        const int n = bx->hi[d] - bx->lo[d] + 1;
        a.ntile[d] = (n + tile[d] - 1) / tile[d];
    }
    a.sb = A4(sborder);
    a.pn = A4(phi_new);
    a.dsdt = dsdt.p ? A4(dsdt) : A4();
    a.rxn = rxn.p ? A4(rxn) : A4();
    for (int d = 0; d < 3; d++) {
        a.ef[d] = ef[d];
        a.gne[d] = gne[d];
    }
    PrepArgs& pa = P->pa;
    memset(&pa, 0, sizeof(pa));
    pa.sb = a.sb;
    for (int d = 0; d < 3; d++) {
        pa.glo[d] = P->glo[d];
        pa.ghi[d] = P->ghi[d];
        pa.lo[d] = bx->lo[d];
        pa.hi[d] = bx->hi[d];
    }
    pa.Tg = prm->Tg;
    pa.do_reactions = prm->do_reactions;
    pa.write_n = 1;
    P->gn = (int64_t)(P->ghi[0] - P->glo[0] + 1) * (P->ghi[1] - P->glo[1] + 1) * (P->ghi[2] - P->glo[2] + 1);
    P->vn = (int64_t)(bx->hi[0] - bx->lo[0] + 1) * (bx->hi[1] - bx->lo[1] + 1) * (bx->hi[2] - bx->lo[2] + 1);
    P->own_rxn = rxn.p == nullptr;
    P->check = prm->check_finite != 0;
    P->dim = dim;
    P->prec = prm->precision;
    return VD_OK;
}

// Points the plan at its scratch and launches the update on st (prep, the FP64
// path's Joule pass, transport).  With the non-finite check it clears the status
// word first and afterwards reads it back, synchronising st.
static int launch_update(UpdatePlan& P, char* scratch, cudaStream_t st)
{
    unsigned int* status = reinterpret_cast<unsigned int*>(scratch);
    double* Np = reinterpret_cast<double*>(scratch + kStatusBytes);
    A4 Nv;
    Nv.p = Np;
    Nv.bx = P.glo[0];
    Nv.by = P.glo[1];
    Nv.bz = P.glo[2];
    Nv.js = P.ghi[0] - P.glo[0] + 1;
    Nv.ks = Nv.js * (P.ghi[1] - P.glo[1] + 1);
    Nv.ns = Nv.ks * (P.ghi[2] - P.glo[2] + 1);
    Nv.ncomp = 1;
    TransportArgs& a = P.a;
    if (P.own_rxn) {
        A4 R;
        R.p = Np + P.gn;
        R.bx = a.lo[0];
        R.by = a.lo[1];
        R.bz = a.lo[2];
        R.js = a.hi[0] - a.lo[0] + 1;
        R.ks = R.js * (a.hi[1] - a.lo[1] + 1);
        R.ns = R.ks * (a.hi[2] - a.lo[2] + 1);
        R.ncomp = a.ns + 1;
        a.rxn = R;
    }
    a.Nv = Nv;
    a.status = P.check ? status : nullptr;
    P.pa.rxn = a.rxn;
    P.pa.Nv = Nv;
    cudaError_t e = P.check ? cudaMemsetAsync(status, 0, sizeof(unsigned int), st) : cudaSuccess;
    if (e == cudaSuccess) e = launch_prep(P.pa, P.prec, a.ns, st);
    if (e == cudaSuccess && a.elecenergy && !joule_in_tile(a, P.prec)) e = launch_joule_pre(a, P.dim, P.prec, st);
    if (e == cudaSuccess) e = launch_transport(a, P.dim, P.prec, st);
    if (e != cudaSuccess) return cuda_fail(e, "fused update launch");
    if (P.check) {
        unsigned int h = 0;
        e = cudaMemcpyAsync(&h, status, sizeof(h), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "reading the non-finite status");
        if (h) return fail(VD_ERR_NONFINITE, "NaN or infinity in the inputs or results of the update");
    }
    return VD_OK;
}

int vd_explicit_update_all(const vd_box* bx, vd_array4 sborder, const vd_array4 efield_ec[3],
                           const vd_array4 gradne_fc[3], vd_array4 phi_new, vd_array4 dsdt, vd_array4 rxn,
                           const vd_params* prm, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_mech_on_device(st);
    if (rc) return rc;
    UpdatePlan P;
    if ((rc = plan_update(bx, sborder, efield_ec, gradne_fc, phi_new, dsdt, rxn, prm, &P))) return rc;
    const size_t bytes = P.scratch_bytes();
    void* scratch = nullptr;
    cudaError_t e = scratch_alloc(&scratch, bytes, st);
    if (e != cudaSuccess) return fail(VD_ERR_NOMEM, "scratch of %zu bytes: %s", bytes, cudaGetErrorString(e));
    rc = launch_update(P, static_cast<char*>(scratch), st);
    cudaError_t e2 = cudaFreeAsync(scratch, st);
    if (rc) return rc;
    if (e2 != cudaSuccess) return cuda_fail(e2, "scratch release");
    return VD_OK;
}

int64_t vd_launch_count(void) { return launch_count(); }

int vd_profile_enable(int on)
{
    prof_enable(on != 0);
    return VD_OK;
}

int vd_profile_read(char* names, int names_len, int64_t* counts, double* ms, int max)
{
    if (!names || !counts || !ms || max <= 0) return fail(VD_ERR_ARG, "null output");
    int n = prof_read(names, names_len, counts, ms, max);
    if (n < 0) return fail(VD_ERR_CUDA, "reading profile events");
    return n;
}

int vd_time_scales(const vd_box* bx, vd_array4 state, const vd_params* prm, double out[3], void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_mech_on_device(st);
    if (rc) return rc;
    if (!out) return fail(VD_ERR_ARG, "null output");
    if ((rc = check_params(bx, prm))) return rc;
    const vd_host::MechInfo m = mech_snapshot();
    const int ns = m.ns;
    std::string why;
    if (!covers(state, bx->lo, bx->hi, VD_NVAR(ns), &why)) return fail(VD_ERR_ARG, "state: %s", why.c_str());
    TransportArgs a;
    fill_cfg(a, bx, prm, ns, m.e_id, m.charge[m.e_id]);
    unsigned long long* d = nullptr;
    cudaError_t e = scratch_alloc(reinterpret_cast<void**>(&d), 3 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return fail(VD_ERR_NOMEM, "3 words of scratch: %s", cudaGetErrorString(e));
    unsigned long long h[3] = {0, 0, 0};
    e = cudaMemsetAsync(d, 0, sizeof(h), st);
    if (e == cudaSuccess) e = launch_time_scales(box_idx(bx->lo, bx->hi), bx->dim, A4(state), a, d, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "time scales");
    double mx[3];
    memcpy(mx, h, sizeof(mx));
    // Source/TimeStep.cpp:94-110
    const double big = 1.79769313486231570e308;
    out[0] = out[1] = out[2] = big;
    for (int d2 = 0; d2 < bx->dim; d2++) {
        if (mx[0] > 0) out[0] = std::min(out[0], prm->dx[d2] / mx[0]);
        if (mx[1] > 0) out[1] = std::min(out[1], 0.5 * prm->dx[d2] * prm->dx[d2] / mx[1] / bx->dim);
    }
    if (mx[2] > 0) out[2] = 8.854187817e-12 / ECHARGE / mx[2];
    return VD_OK;
}

int vd_fill_ghosts(const vd_box* bx, vd_array4 state, int ghost, const int32_t* comps, int ncomp,
                   const int32_t periodic[3], void* stream)
{
    if (!valid_box(bx)) return fail(VD_ERR_ARG, "invalid box");
    if (ghost < 0 || ghost > 8) return fail(VD_ERR_GHOST, "ghost %d outside [0,8]", ghost);
    if (ncomp < 0 || ncomp > VD_MAX_SPECIES + 4 || (ncomp && !comps))
        return fail(VD_ERR_ARG, "ncomp %d outside [0,%d]", ncomp, VD_MAX_SPECIES + 4);
    int glo[3] = {bx->lo[0], bx->lo[1], bx->lo[2]}, ghi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
    for (int d = 0; d < bx->dim; d++) {
        glo[d] -= ghost;
        ghi[d] += ghost;
    }
    int maxc = 0;
    for (int q = 0; q < ncomp; q++) {
        if (comps[q] < 0 || comps[q] > 127) return fail(VD_ERR_ARG, "component %d out of range", comps[q]);
        maxc = comps[q] + 1 > maxc ? comps[q] + 1 : maxc;
    }
    std::string why;
    if (!covers(state, glo, ghi, maxc, &why)) return fail(VD_ERR_GHOST, "state: %s", why.c_str());
    GhostArgs a;
    memset(&a, 0, sizeof(a));
    a.st = A4(state);
    a.ghost = ghost;
    a.dim = bx->dim;
    a.count = 0;
    for (int d = 0; d < 3; d++) {
        a.lo[d] = bx->lo[d];
        a.hi[d] = bx->hi[d];
        a.periodic[d] = (periodic && d < bx->dim) ? (periodic[d] != 0) : 0;
        if (a.periodic[d] && bx->hi[d] - bx->lo[d] + 1 < 1) return fail(VD_ERR_ARG, "empty periodic direction");
    }
    for (int d = 0; d < bx->dim; d++) {
        int64_t P = 1;
        for (int e = 0; e < bx->dim; e++)
            if (e != d) P *= bx->hi[e] - bx->lo[e] + 1;
        a.count += 2 * (int64_t)ghost * P;
    }
    a.ncomp = ncomp;
    for (int q = 0; q < ncomp; q++) a.comps[q] = (int8_t)comps[q];
    cudaError_t e = launch_ghost(a, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "k_ghost launch");
    return VD_OK;
}

int vd_box_checksums(const vd_box* bx, vd_array4 rxn, vd_array4 phi_new, double* out_dev, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_mech_on_device(st);
    if (rc) return rc;
    const int ns = nspecies();
    if (!valid_box(bx) || !out_dev) return fail(VD_ERR_ARG, "invalid box or output");
    std::string why;
    if (!covers(rxn, bx->lo, bx->hi, ns + 1, &why)) return fail(VD_ERR_ARG, "rxn: %s", why.c_str());
    if (!covers(phi_new, bx->lo, bx->hi, ns, &why)) return fail(VD_ERR_ARG, "phi_new: %s", why.c_str());
    cudaError_t e = launch_checksums(box_idx(bx->lo, bx->hi), A4(rxn), A4(phi_new), out_dev, st);
    if (e != cudaSuccess) return cuda_fail(e, "k_checksums launch");
    return VD_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free explicit update.
//
// Some hosts cannot let this library allocate device memory while they step: an
// AMReX application usually gives most of the GPU to its own arena when it
// starts, and some callers allow no allocation inside the time-step loop at all.
// For them the scratch of the fused update lives in the fixed array
// g_noalloc_scratch (top of this file), reserved and located per device by
// setup_device, instead of coming from the scratch pool.
extern "C" int vd_explicit_update_all_noalloc(const vd_box* bx, vd_array4 sborder, const vd_array4 efield_ec[3],
                                              const vd_array4 gradne_fc[3], vd_array4 phi_new, vd_array4 dsdt,
                                              vd_array4 rxn, const vd_params* prm, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_mech_on_device(st);
    if (rc) return rc;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    char* scratch = reinterpret_cast<char*>(g_noalloc_ptr[dev]);  // set by ensure_mech_on_device
    if (!scratch) return fail(VD_ERR_STATE, "allocation-free scratch not set up on device %d", dev);
    UpdatePlan P;
    if ((rc = plan_update(bx, sborder, efield_ec, gradne_fc, phi_new, dsdt, rxn, prm, &P))) return rc;
    // scratch need, checked against the fixed array before anything is launched
    const size_t need = P.scratch_bytes();
    if (need > (size_t)VD_NOALLOC_SCRATCH_BYTES)
        return fail(VD_ERR_NOMEM,
                    "box needs %zu bytes of scratch; the allocation-free update has %zu bytes "
                    "(pass a rxn array to need %zu bytes, or use vd_explicit_update_all)",
                    need, (size_t)VD_NOALLOC_SCRATCH_BYTES, kStatusBytes + (size_t)P.gn * sizeof(double));
    return launch_update(P, scratch, st);
}

// ===========================================================================
// Host services for the batch layer (vd_host.h).

namespace vd_host {

int set_error(int code, const char* msg) { return fail(code, "%s", msg); }

int ensure_mech(cudaStream_t st) { return ensure_mech_on_device(st); }

double species_mw(int s)
{
    std::lock_guard<std::mutex> lk(g_mech_mu);
    if (!g_mech || s < 0 || s >= g_mech->nspecies) return 0.0;
    return g_mech->mw[s];
}

int mech_info(MechInfo* out)
{
    {
        std::lock_guard<std::mutex> lk(g_mech_mu);
        if (!g_mech) return fail(VD_ERR_MECH, "no mechanism loaded: call vd_mech_init first");
    }
    *out = mech_snapshot();
    return VD_OK;
}

int check_update_params(const vd_box* bx, const vd_params* p, const MechInfo& m)
{
    int rc = check_params(bx, p);
    if (rc) return rc;
    return check_update_species(p, m);
}

void fill_transport_args(TransportArgs& a, const vd_box* bx, const vd_params* p, const MechInfo& m)
{
    fill_cfg(a, bx, p, m.ns, m.e_id, m.charge[m.e_id]);
    fill_species(a, p, m);
}

cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st) { return ::scratch_alloc(p, bytes, st); }

int stencil_halo(int hyp_order) { return ::stencil_halo(hyp_order); }

}  // namespace vd_host
