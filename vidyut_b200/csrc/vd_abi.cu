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

// Loads the mechanism table onto the current device if it is not there yet.
int ensure_mech_on_device(cudaStream_t st)
{
    std::lock_guard<std::mutex> lk(g_mech_mu);
    if (!g_mech) return fail(VD_ERR_MECH, "no mechanism loaded: call vd_mech_init first");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    for (int d : g_loaded_dev)
        if (d == dev) return VD_OK;
    int rc = upload_mech(g_mech_dev, st);
    if (rc != 0) return cuda_fail((cudaError_t)rc, "uploading mechanism table");
    // keep freed scratch in this process's default pool between calls instead of
    // handing it back to the driver at every synchronisation
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    g_loaded_dev.push_back(dev);
    return VD_OK;
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

int species_class(const vd_mech* m, int s)
{
    if (s == m->nspecies) return VD_CLASS_ENERGY;
    if (s == m->e_id) return VD_CLASS_ELECTRON;
    return m->charge[s] != 0 ? VD_CLASS_ION : VD_CLASS_NEUTRAL;
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
    for (int s = 0; s <= ns; s++) {
        int k = m->mob_kind[s];
        if (k < 0 || k > 5) return fail(VD_ERR_MECH, "species %d: unknown mobility kind %d", s, k);
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
        if (dk < 0 || dk > 2) return fail(VD_ERR_MECH, "species %d: unknown diffusion kind %d", s, dk);
        if (dk != VD_DIFF_ZERO && (m->diff_ref[s] < 0 || m->diff_ref[s] > ns))
            return fail(VD_ERR_MECH, "species %d: diffusion reference invalid", s);
    }
    if (m->elastic_loss && !(m->elastic_mass > 0.0)) return fail(VD_ERR_MECH, "elastic_mass must be > 0");
    for (int r = 0; r < nr; r++) {
        const vd_reaction& R = m->rxn[r];
        if (R.kind < 0 || R.kind > 2) return fail(VD_ERR_MECH, "reaction %d: unknown rate kind %d", r, R.kind);
        if (R.nreac < 1 || R.nreac > VD_MAX_REACTANTS)
            return fail(VD_ERR_MECH, "reaction %d: %d reactants", r, R.nreac);
        for (int t = 0; t < R.nreac; t++)
            if (R.reac[t] < 0 || R.reac[t] >= ns) return fail(VD_ERR_MECH, "reaction %d: bad reactant", r);
        if (R.nterms < 0 || R.nterms > VD_MAX_TERMS) return fail(VD_ERR_MECH, "reaction %d: bad term count", r);
        for (int t = 0; t < R.nterms; t++)
            if (R.term_sp[t] < 0 || R.term_sp[t] >= ns) return fail(VD_ERR_MECH, "reaction %d: bad term", r);
        if (R.rxntype != 0 && R.rxntype != 1 && R.rxntype != 2 && R.rxntype != 3 && R.rxntype != 5)
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
        if (m->mob_kind[s] == VD_MOB_ELECTRON) d->mob_c[s] = (-ECHARGE / ME) / std::sqrt(8.0 * K_B / PI / ME);
        else if (m->mob_kind[s] == VD_MOB_ION_TG)
            d->mob_c[s] = (ECHARGE / m->mob_p1[s]) / std::sqrt(8.0 * K_B / PI / m->mob_p1[s]);
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
        if (!(p->dx[d] > 0.0)) return fail(VD_ERR_ARG, "dx[%d] must be > 0", d);
    if (p->precision != VD_PREC_FP64 && p->precision != VD_PREC_MIXED)
        return fail(VD_ERR_ARG, "unknown precision %d", p->precision);
    return check_scheme(p->hyp_order, p->weno_scheme);
}

static void fill_cfg(TransportArgs& a, const vd_box* bx, const vd_params* p, const vd_mech* m)
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
    a.ns = m->nspecies;
    a.e_id = m->e_id;
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
    a.charge_e = (double)m->charge[m->e_id] * ECHARGE;
    a.ghost = stencil_halo(p->hyp_order);
    a.write_diag = 1;
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
    vd_mech mcopy;
    {
        std::lock_guard<std::mutex> lk(g_mech_mu);
        mcopy.nspecies = g_mech->nspecies;
        mcopy.e_id = g_mech->e_id;
        memcpy(mcopy.charge, g_mech->charge, sizeof(mcopy.charge));
    }
    const int ns = mcopy.nspecies;
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
    for (int d = 0; d < 3; d++) {
        if (d < bx->dim) {
            int fhi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
            fhi[d] += 1;
            if (!prm->cs_technique) {
                if (!efield_ec || !covers(efield_ec[d], bx->lo, fhi, 1, &why))
                    return fail(VD_ERR_ARG, "efield_ec[%d]: %s", d, why.c_str());
                ef[d] = A4(efield_ec[d]);
            }
            if (!prm->gradne_from_state) {
                if (!gradne_fc || !covers(gradne_fc[d], bx->lo, fhi, 1, &why))
                    return fail(VD_ERR_ARG, "gradne_fc[%d]: %s", d, why.c_str());
                gne[d] = A4(gradne_fc[d]);
            }
        }
    }
    TransportArgs cfg;
    fill_cfg(cfg, bx, prm, &mcopy);
    cudaError_t e = launch_joule(box_idx(bx->lo, bx->hi), bx->dim, A4(sborder), A4(rxn), ef, gne, A4(dsdt),
                                 A4(phi_new), cfg, st);
    if (e != cudaSuccess) return cuda_fail(e, "k_joule launch");
    return VD_OK;
}

int vd_explicit_update_all(const vd_box* bx, vd_array4 sborder, const vd_array4 efield_ec[3],
                           const vd_array4 gradne_fc[3], vd_array4 phi_new, vd_array4 dsdt, vd_array4 rxn,
                           const vd_params* prm, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_mech_on_device(st);
    if (rc) return rc;
    if ((rc = check_params(bx, prm))) return rc;
    vd_mech* m;
    {
        std::lock_guard<std::mutex> lk(g_mech_mu);
        m = g_mech;
    }
    const int ns = m->nspecies, dim = bx->dim;
    const int H = stencil_halo(prm->hyp_order);
    std::string why;
    int glo[3] = {bx->lo[0], bx->lo[1], bx->lo[2]}, ghi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
    for (int d = 0; d < dim; d++) {
        glo[d] -= H;
        ghi[d] += H;
    }
    // the stencil only reaches along one axis at a time; corners are never read,
    // but the per-cell density sums cover the whole grown box, so require it.
    if (!covers(sborder, glo, ghi, VD_NVAR(ns), &why)) return fail(VD_ERR_GHOST, "sborder: %s", why.c_str());
    if (!covers(phi_new, bx->lo, bx->hi, VD_NVAR(ns), &why)) return fail(VD_ERR_ARG, "phi_new: %s", why.c_str());
    if (dsdt.p && !covers(dsdt, bx->lo, bx->hi, ns + 1, &why)) return fail(VD_ERR_ARG, "dsdt: %s", why.c_str());
    if (rxn.p && !covers(rxn, bx->lo, bx->hi, ns + 1, &why)) return fail(VD_ERR_ARG, "rxn: %s", why.c_str());
    if (prm->bg_mask >> ns) return fail(VD_ERR_ARG, "bg_mask names species >= %d", ns);
    if (prm->bg_mask & (1ull << m->e_id)) return fail(VD_ERR_ARG, "electrons cannot be a background species");
    if (prm->user_defined_vel && (prm->vel_species < 0 || prm->vel_species > ns))
        return fail(VD_ERR_ARG, "vel_species invalid");
    A4 ef[3], gne[3];
    if (prm->elecenergy_solve) {
        for (int d = 0; d < dim; d++) {
            int fhi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
            fhi[d] += 1;
            if (!prm->cs_technique) {
                if (!efield_ec || !covers(efield_ec[d], bx->lo, fhi, 1, &why))
                    return fail(VD_ERR_ARG, "efield_ec[%d]: %s", d, why.c_str());
                ef[d] = A4(efield_ec[d]);
            }
            if (!prm->gradne_from_state) {
                if (!gradne_fc || !covers(gradne_fc[d], bx->lo, fhi, 1, &why))
                    return fail(VD_ERR_ARG, "gradne_fc[%d]: %s", d, why.c_str());
                gne[d] = A4(gradne_fc[d]);
            }
        }
    }

    TransportArgs a;
    fill_cfg(a, bx, prm, m);
    int tile[3];
    transport_tile(dim, tile);
    for (int d = 0; d < 3; d++) {
        int n = bx->hi[d] - bx->lo[d] + 1;
        a.ntile[d] = (n + tile[d] - 1) / tile[d];
    }
    a.sb = A4(sborder);
    a.pn = A4(phi_new);
    a.dsdt = dsdt.p ? A4(dsdt) : A4();
    for (int d = 0; d < 3; d++) {
        a.ef[d] = ef[d];
        a.gne[d] = gne[d];
    }
    a.ntr = 0;
    a.nbg = 0;
    for (int s = 0; s <= ns; s++) {
        bool energy = (s == ns);
        if (energy && !prm->elecenergy_solve) continue;
        if (!energy && ((prm->bg_mask >> s) & 1ull)) {
            a.bg_sp[a.nbg++] = (int8_t)s;
            continue;
        }
        a.tr_sp[a.ntr] = (int8_t)s;
        a.tr_cls[a.ntr] = (int8_t)species_class(m, s);
        bool has_vel = prm->user_defined_vel ? (s == prm->vel_species) : (m->mob_kind[s] != VD_MOB_ZERO);
        a.tr_flux[a.ntr] = (prm->do_transport && has_vel) ? 1 : 0;
        a.ntr++;
    }
    finish_lists(a);

    // scratch: N on the grown box, rxn on the valid box when the caller does not keep it
    const int64_t gn = (int64_t)(ghi[0] - glo[0] + 1) * (ghi[1] - glo[1] + 1) * (ghi[2] - glo[2] + 1);
    const int64_t vn = (int64_t)(bx->hi[0] - bx->lo[0] + 1) * (bx->hi[1] - bx->lo[1] + 1) * (bx->hi[2] - bx->lo[2] + 1);
    size_t bytes = (size_t)gn * sizeof(double) + (rxn.p ? 0 : (size_t)vn * (ns + 1) * sizeof(double));
    void* scratch = nullptr;
    cudaError_t e = cudaMallocAsync(&scratch, bytes, st);
    if (e != cudaSuccess) return fail(VD_ERR_NOMEM, "scratch of %zu bytes: %s", bytes, cudaGetErrorString(e));
    double* Np = (double*)scratch;
    A4 Nv;
    Nv.p = Np;
    Nv.bx = glo[0];
    Nv.by = glo[1];
    Nv.bz = glo[2];
    Nv.js = ghi[0] - glo[0] + 1;
    Nv.ks = Nv.js * (ghi[1] - glo[1] + 1);
    Nv.ns = Nv.ks * (ghi[2] - glo[2] + 1);
    Nv.ncomp = 1;
    A4 R;
    if (rxn.p) {
        R = A4(rxn);
    } else {
        R.p = Np + gn;
        R.bx = bx->lo[0];
        R.by = bx->lo[1];
        R.bz = bx->lo[2];
        R.js = bx->hi[0] - bx->lo[0] + 1;
        R.ks = R.js * (bx->hi[1] - bx->lo[1] + 1);
        R.ns = R.ks * (bx->hi[2] - bx->lo[2] + 1);
        R.ncomp = ns + 1;
    }
    a.Nv = Nv;
    a.rxn = R;

    PrepArgs pa;
    pa.sb = a.sb;
    pa.rxn = R;
    pa.Nv = Nv;
    for (int d = 0; d < 3; d++) {
        pa.glo[d] = glo[d];
        pa.ghi[d] = ghi[d];
        pa.lo[d] = bx->lo[d];
        pa.hi[d] = bx->hi[d];
    }
    pa.Tg = prm->Tg;
    pa.do_reactions = prm->do_reactions;
    pa.write_n = 1;
    e = launch_prep(pa, prm->precision, ns, st);
    if (e == cudaSuccess && a.elecenergy && !joule_in_tile(a, prm->precision))
        e = launch_joule_pre(a, dim, prm->precision, st);
    if (e == cudaSuccess) e = launch_transport(a, dim, prm->precision, st);
    cudaError_t e2 = cudaFreeAsync(scratch, st);
    if (e != cudaSuccess) return cuda_fail(e, "fused update launch");
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
    vd_mech* m;
    {
        std::lock_guard<std::mutex> lk(g_mech_mu);
        m = g_mech;
    }
    const int ns = m->nspecies;
    std::string why;
    if (!covers(state, bx->lo, bx->hi, VD_NVAR(ns), &why)) return fail(VD_ERR_ARG, "state: %s", why.c_str());
    TransportArgs a;
    fill_cfg(a, bx, prm, m);
    unsigned long long* d = nullptr;
    cudaError_t e = cudaMallocAsync(&d, 3 * sizeof(unsigned long long), st);
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
// For them the scratch of the fused update lives in this fixed array instead of
// coming from the stream-ordered allocator.  Every GPU that loads the library
// holds the array until the process exits.  In host code the name below is only a
// host-side stand-in, so its device address is looked up once per device (with
// that device current) and passed to the kernels.
namespace {

constexpr size_t kNoallocDoubles = VD_NOALLOC_SCRATCH_BYTES / sizeof(double);
static __device__ __align__(256) double g_noalloc_scratch[kNoallocDoubles];

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[64] = {nullptr};  // device address of the array, per device

// Once per device: find the array's device address.
int noalloc_scratch_for_current_device(double** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64) return fail(VD_ERR_ARG, "device ordinal %d not supported", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return VD_OK;
}

}  // namespace

extern "C" int vd_explicit_update_all_noalloc(const vd_box* bx, vd_array4 sborder, const vd_array4 efield_ec[3],
                                              const vd_array4 gradne_fc[3], vd_array4 phi_new, vd_array4 dsdt,
                                              vd_array4 rxn, const vd_params* prm, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_mech_on_device(st);
    if (rc) return rc;
    double* scratch = nullptr;
    if ((rc = noalloc_scratch_for_current_device(&scratch))) return rc;
    if ((rc = check_params(bx, prm))) return rc;
    vd_mech* m;
    {
        std::lock_guard<std::mutex> lk(g_mech_mu);
        m = g_mech;
    }
    const int ns = m->nspecies, dim = bx->dim;
    const int H = stencil_halo(prm->hyp_order);
    std::string why;
    int glo[3] = {bx->lo[0], bx->lo[1], bx->lo[2]}, ghi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
    for (int d = 0; d < dim; d++) {
        glo[d] -= H;
        ghi[d] += H;
    }
    if (!covers(sborder, glo, ghi, VD_NVAR(ns), &why)) return fail(VD_ERR_GHOST, "sborder: %s", why.c_str());
    if (!covers(phi_new, bx->lo, bx->hi, VD_NVAR(ns), &why)) return fail(VD_ERR_ARG, "phi_new: %s", why.c_str());
    if (dsdt.p && !covers(dsdt, bx->lo, bx->hi, ns + 1, &why)) return fail(VD_ERR_ARG, "dsdt: %s", why.c_str());
    if (rxn.p && !covers(rxn, bx->lo, bx->hi, ns + 1, &why)) return fail(VD_ERR_ARG, "rxn: %s", why.c_str());
    if (prm->bg_mask >> ns) return fail(VD_ERR_ARG, "bg_mask names species >= %d", ns);
    if (prm->bg_mask & (1ull << m->e_id)) return fail(VD_ERR_ARG, "electrons cannot be a background species");
    if (prm->user_defined_vel && (prm->vel_species < 0 || prm->vel_species > ns))
        return fail(VD_ERR_ARG, "vel_species invalid");
    A4 ef[3], gne[3];
    if (prm->elecenergy_solve) {
        for (int d = 0; d < dim; d++) {
            int fhi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
            fhi[d] += 1;
            if (!prm->cs_technique) {
                if (!efield_ec || !covers(efield_ec[d], bx->lo, fhi, 1, &why))
                    return fail(VD_ERR_ARG, "efield_ec[%d]: %s", d, why.c_str());
                ef[d] = A4(efield_ec[d]);
            }
            if (!prm->gradne_from_state) {
                if (!gradne_fc || !covers(gradne_fc[d], bx->lo, fhi, 1, &why))
                    return fail(VD_ERR_ARG, "gradne_fc[%d]: %s", d, why.c_str());
                gne[d] = A4(gradne_fc[d]);
            }
        }
    }
    // scratch need, checked against the fixed array before anything is launched
    const int64_t gn = (int64_t)(ghi[0] - glo[0] + 1) * (ghi[1] - glo[1] + 1) * (ghi[2] - glo[2] + 1);
    const int64_t vn =
        (int64_t)(bx->hi[0] - bx->lo[0] + 1) * (bx->hi[1] - bx->lo[1] + 1) * (bx->hi[2] - bx->lo[2] + 1);
    const int64_t need = gn + (rxn.p ? 0 : vn * (ns + 1));
    if (need > (int64_t)kNoallocDoubles)
        return fail(VD_ERR_NOMEM,
                    "box needs %lld bytes of scratch; the allocation-free update has %zu bytes "
                    "(pass a rxn array to need %lld bytes, or use vd_explicit_update_all)",
                    (long long)(need * 8), (size_t)VD_NOALLOC_SCRATCH_BYTES, (long long)(gn * 8));

    TransportArgs a;
    fill_cfg(a, bx, prm, m);
    int tile[3];
    transport_tile(dim, tile);
    for (int d = 0; d < 3; d++) {
        int n = bx->hi[d] - bx->lo[d] + 1;
        a.ntile[d] = (n + tile[d] - 1) / tile[d];
    }
    a.sb = A4(sborder);
    a.pn = A4(phi_new);
    a.dsdt = dsdt.p ? A4(dsdt) : A4();
    for (int d = 0; d < 3; d++) {
        a.ef[d] = ef[d];
        a.gne[d] = gne[d];
    }
    a.ntr = 0;
    a.nbg = 0;
    for (int s = 0; s <= ns; s++) {
        bool energy = (s == ns);
        if (energy && !prm->elecenergy_solve) continue;
        if (!energy && ((prm->bg_mask >> s) & 1ull)) {
            a.bg_sp[a.nbg++] = (int8_t)s;
            continue;
        }
        a.tr_sp[a.ntr] = (int8_t)s;
        a.tr_cls[a.ntr] = (int8_t)species_class(m, s);
        bool has_vel = prm->user_defined_vel ? (s == prm->vel_species) : (m->mob_kind[s] != VD_MOB_ZERO);
        a.tr_flux[a.ntr] = (prm->do_transport && has_vel) ? 1 : 0;
        a.ntr++;
    }
    finish_lists(a);
    A4 Nv;
    Nv.p = scratch;
    Nv.bx = glo[0];
    Nv.by = glo[1];
    Nv.bz = glo[2];
    Nv.js = ghi[0] - glo[0] + 1;
    Nv.ks = Nv.js * (ghi[1] - glo[1] + 1);
    Nv.ns = Nv.ks * (ghi[2] - glo[2] + 1);
    Nv.ncomp = 1;
    A4 R;
    if (rxn.p) {
        R = A4(rxn);
    } else {
        R.p = scratch + gn;
        R.bx = bx->lo[0];
        R.by = bx->lo[1];
        R.bz = bx->lo[2];
        R.js = bx->hi[0] - bx->lo[0] + 1;
        R.ks = R.js * (bx->hi[1] - bx->lo[1] + 1);
        R.ns = R.ks * (bx->hi[2] - bx->lo[2] + 1);
        R.ncomp = ns + 1;
    }
    a.Nv = Nv;
    a.rxn = R;
    PrepArgs pa;
    pa.sb = a.sb;
    pa.rxn = R;
    pa.Nv = Nv;
    for (int d = 0; d < 3; d++) {
        pa.glo[d] = glo[d];
        pa.ghi[d] = ghi[d];
        pa.lo[d] = bx->lo[d];
        pa.hi[d] = bx->hi[d];
    }
    pa.Tg = prm->Tg;
    pa.do_reactions = prm->do_reactions;
    pa.write_n = 1;
    cudaError_t e = launch_prep(pa, prm->precision, ns, st);
    if (e == cudaSuccess && a.elecenergy && !joule_in_tile(a, prm->precision))
        e = launch_joule_pre(a, dim, prm->precision, st);
    if (e == cudaSuccess) e = launch_transport(a, dim, prm->precision, st);
    if (e != cudaSuccess) return cuda_fail(e, "allocation-free update launch");
    return VD_OK;
}

// ===========================================================================
// Host services for the batch layer (vd_host.h).
#include "vd_host.h"

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
    std::lock_guard<std::mutex> lk(g_mech_mu);
    if (!g_mech) return fail(VD_ERR_MECH, "no mechanism loaded: call vd_mech_init first");
    out->ns = g_mech->nspecies;
    out->e_id = g_mech->e_id;
    out->generation = g_mech_gen;
    for (int s = 0; s <= g_mech->nspecies; s++) out->mob_kind[s] = g_mech->mob_kind[s];
    for (int s = 0; s < g_mech->nspecies; s++) out->charge[s] = g_mech->charge[s];
    return VD_OK;
}

int check_update_params(const vd_box* bx, const vd_params* p, const MechInfo& m)
{
    int rc = check_params(bx, p);
    if (rc) return rc;
    if (p->bg_mask >> m.ns) return fail(VD_ERR_ARG, "bg_mask names species >= %d", m.ns);
    if (p->bg_mask & (1ull << m.e_id)) return fail(VD_ERR_ARG, "electrons cannot be a background species");
    if (p->user_defined_vel && (p->vel_species < 0 || p->vel_species > m.ns))
        return fail(VD_ERR_ARG, "vel_species invalid");
    if (!(p->dt >= 0.0) || !std::isfinite(p->dt)) return fail(VD_ERR_ARG, "dt must be finite and >= 0");
    return VD_OK;
}

void fill_transport_args(TransportArgs& a, const vd_box* bx, const vd_params* p, const MechInfo& m)
{
    vd_mech* mm = new vd_mech;  // fill_cfg reads nspecies, e_id and the electron charge
    memset(mm, 0, sizeof(vd_mech));
    mm->nspecies = m.ns;
    mm->e_id = m.e_id;
    for (int s = 0; s < m.ns; s++) mm->charge[s] = m.charge[s];
    fill_cfg(a, bx, p, mm);
    delete mm;
    const int ns = m.ns;
    a.ntr = 0;
    a.nbg = 0;
    for (int s = 0; s <= ns; s++) {
        bool energy = (s == ns);
        if (energy && !p->elecenergy_solve) continue;
        if (!energy && ((p->bg_mask >> s) & 1ull)) {
            a.bg_sp[a.nbg++] = (int8_t)s;
            continue;
        }
        a.tr_sp[a.ntr] = (int8_t)s;
        int cls = energy ? VD_CLASS_ENERGY
                         : (s == m.e_id ? VD_CLASS_ELECTRON : (m.charge[s] != 0 ? VD_CLASS_ION : VD_CLASS_NEUTRAL));
        a.tr_cls[a.ntr] = (int8_t)cls;
        bool has_vel = p->user_defined_vel ? (s == p->vel_species) : (m.mob_kind[s] != VD_MOB_ZERO);
        a.tr_flux[a.ntr] = (p->do_transport && has_vel) ? 1 : 0;
        a.ntr++;
    }
    finish_lists(a);
}

int stencil_halo(int hyp_order) { return ::stencil_halo(hyp_order); }

}  // namespace vd_host
