// vd_batch.cu -- many independent cases stepped together (vd_batch_* in vidyut_b200.h).
//
// A batch owns one device arena of a fixed byte budget.  Each resident case holds
// in it: two copies of its state (the step reads one and writes the other), the
// per-cell density sums on the stencil-grown box, the reaction source on the
// valid box and the face arrays of the Joule term.  One step of the batch is
//   k_prep_batch       density sums + chemistry of every case
//   k_transport_batch  the fused flux / divergence / accumulate update, one launch
//                      per dimension present (1-D and 2-D cases run concurrently)
//   k_ghost_batch      refill of the written state's ghost cells
// each a persistent kernel walking a work list of (case, chunk-or-tile) items.
// A call of n steps is captured once as a CUDA graph and replayed while the set
// of cases stays the same; which cases take how many steps in a call, and which
// state copy is current, is a small per-case control array copied before each
// replay (kernels skip the items of cases that are done).
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include "vd_host.h"

using namespace vd;

namespace {

constexpr size_t kAlign = 256;
inline size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

// First-fit allocator over [0, cap): offsets of free blocks -> sizes.
struct Arena {
    size_t cap = 0, used = 0;
    std::map<size_t, size_t> free_;
    void init(size_t c)
    {
        cap = c;
        used = 0;
        free_.clear();
        if (c) free_[0] = c;
    }
    bool alloc(size_t n, size_t* off)
    {
        n = align_up(n);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                *off = it->first;
                size_t rest = it->second - n;
                size_t at = it->first + n;
                free_.erase(it);
                if (rest) free_[at] = rest;
                used += n;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t n)
    {
        n = align_up(n);
        used -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Layout {  // byte offsets of one case's arrays inside its arena region
    int dim, H;
    int glo[3], ghi[3];
    int64_t gcells, vcells, fcells[3];
    size_t st[2], nv, rxn, ef[3], gne[3], bytes;
    bool has_ef, has_gne;
};

bool make_layout(const vd_box* bx, const vd_params* p, int ns, Layout* L)
{
    L->dim = bx->dim;
    L->H = vd_host::stencil_halo(p->hyp_order);
    int64_t vn = 1, gn = 1;
    for (int d = 0; d < 3; d++) {
        int g = d < bx->dim ? L->H : 0;
        L->glo[d] = bx->lo[d] - g;
        L->ghi[d] = bx->hi[d] + g;
        vn *= bx->hi[d] - bx->lo[d] + 1;
        gn *= L->ghi[d] - L->glo[d] + 1;
    }
    L->vcells = vn;
    L->gcells = gn;
    for (int d = 0; d < 3; d++) {
        L->fcells[d] = 0;
        if (d < bx->dim) L->fcells[d] = vn / (bx->hi[d] - bx->lo[d] + 1) * (bx->hi[d] - bx->lo[d] + 2);
    }
    L->has_ef = p->elecenergy_solve && !p->cs_technique;
    L->has_gne = p->elecenergy_solve && !p->gradne_from_state;
    size_t o = 0;
    for (int b = 0; b < 2; b++) {
        L->st[b] = o;
        o += align_up((size_t)gn * VD_NVAR(ns) * sizeof(double));
    }
    L->nv = o;
    o += align_up((size_t)gn * sizeof(double));
    L->rxn = o;
    o += align_up((size_t)vn * (ns + 1) * sizeof(double));
    for (int d = 0; d < 3; d++) {
        L->ef[d] = L->gne[d] = 0;
        if (d >= bx->dim) continue;
        if (L->has_ef) {
            L->ef[d] = o;
            o += align_up((size_t)L->fcells[d] * sizeof(double));
        }
        if (L->has_gne) {
            L->gne[d] = o;
            o += align_up((size_t)L->fcells[d] * sizeof(double));
        }
    }
    L->bytes = o;
    return true;
}

// dense Array4 view over lo..hi (inclusive), ncomp components
A4 dense_view(double* p, const int lo[3], const int hi[3], int ncomp)
{
    A4 a;
    memset(&a, 0, sizeof(a));
    a.p = p;
    a.bx = lo[0];
    a.by = lo[1];
    a.bz = lo[2];
    a.js = hi[0] - lo[0] + 1;
    a.ks = a.js * (hi[1] - lo[1] + 1);
    a.ns = a.ks * (hi[2] - lo[2] + 1);
    a.ncomp = ncomp;
    a.ex = hi[0] + 1;
    a.ey = hi[1] + 1;
    a.ez = hi[2] + 1;
    return a;
}

struct Case {
    int id;
    vd_box box;
    vd_params prm;
    int periodic[3];
    Layout L;
    size_t off;
    int cur;              // state copy (0/1) holding the current state
    int64_t steps_done;
    int64_t steps_left;   // < 0: no limit
    int sslot;            // its word in vd_batch::d_status
    bool failed;          // a NaN or infinity was met: takes no more steps
};

}  // namespace

struct vd_batch {
    int dev = 0;
    int prec = VD_PREC_MIXED;
    int max_cases = 0;
    int mech_gen = -1;
    vd_host::MechInfo mech;
    char* arena_base = nullptr;
    Arena arena;
    std::vector<Case> cases;  // slot order
    int next_id = 1;
    bool dirty = true;
    bool use_graph = true;
    int variant[4] = {0, 0, 0, 0};
    // device tables (capacity max_cases) and work lists
    TransportArgs* d_tr = nullptr;
    PrepArgs* d_pr = nullptr;
    GhostArgs* d_gh = nullptr;
    int2* d_ctrl = nullptr;
    // Non-finite status word per case (max_cases words; a case keeps its word
    // while resident): the transport tiles set bit 0 when they meet a NaN or
    // infinity (TransportArgs::status).
    unsigned int* d_status = nullptr;
    std::vector<int> free_sslot;
    int2* d_items = nullptr;
    size_t items_cap = 0;
    int n_prep = 0, n_ghost = 0, n_tr[4] = {0, 0, 0, 0}, n_jl[4] = {0, 0, 0, 0};
    size_t off_prep = 0, off_ghost = 0, off_tr[4] = {0, 0, 0, 0}, off_jl[4] = {0, 0, 0, 0};
    int2* h_ctrl[2] = {nullptr, nullptr};  // pinned staging of the control array
    cudaEvent_t ctrl_done[2] = {nullptr, nullptr};
    int ctrl_slot = 0;
    cudaEvent_t last_done = nullptr;  // end of the last work this batch queued
    bool pending = false;
    cudaStream_t side[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[3] = {nullptr, nullptr, nullptr};
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    int64_t steps_run = 0, graph_builds = 0;
    int launches_per_step = 0;
};

namespace {

int err(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int err(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return vd_host::set_error(code, buf);
}

int cuda_err(cudaError_t e, const char* what) { return err(VD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e)); }

// Waits for the work this batch queued last (tables, items and arena regions may
// then be changed).
int settle(vd_batch* b)
{
    if (!b->pending) return VD_OK;
    cudaError_t e = cudaEventSynchronize(b->last_done);
    if (e != cudaSuccess) return cuda_err(e, "waiting for the batch's last step");
    b->pending = false;
    return VD_OK;
}

void drop_graph(vd_batch* b)
{
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = 0;
}

int slot_of(const vd_batch* b, int id)
{
    for (size_t i = 0; i < b->cases.size(); i++)
        if (b->cases[i].id == id) return (int)i;
    return -1;
}

// Rebuilds the argument records of both parities and the work lists.
int rebuild(vd_batch* b)
{
    const int nb = (int)b->cases.size();
    const int ns = b->mech.ns;
    std::vector<TransportArgs> tr(2 * (size_t)b->max_cases);
    std::vector<PrepArgs> pr(2 * (size_t)b->max_cases);
    std::vector<GhostArgs> gh(2 * (size_t)b->max_cases);
    std::vector<int2> prep, ghost, trn[4], jl[4];
    for (int c = 0; c < nb; c++) {
        Case& k = b->cases[c];
        const Layout& L = k.L;
        double* base = (double*)(b->arena_base + k.off);
        double* st[2] = {(double*)((char*)base + L.st[0]), (double*)((char*)base + L.st[1])};
        A4 Nv = dense_view((double*)((char*)base + L.nv), L.glo, L.ghi, 1);
        A4 R = dense_view((double*)((char*)base + L.rxn), k.box.lo, k.box.hi, ns + 1);
        A4 ef[3], gne[3];
        memset(ef, 0, sizeof(ef));
        memset(gne, 0, sizeof(gne));
        for (int d = 0; d < L.dim; d++) {
            int fhi[3] = {k.box.hi[0], k.box.hi[1], k.box.hi[2]};
            fhi[d] += 1;
            if (L.has_ef) ef[d] = dense_view((double*)((char*)base + L.ef[d]), k.box.lo, fhi, 1);
            if (L.has_gne) gne[d] = dense_view((double*)((char*)base + L.gne[d]), k.box.lo, fhi, 1);
        }
        int tile[3];
        batch_tile_shape(L.dim, b->variant[L.dim], tile);
        TransportArgs a;
        vd_host::fill_transport_args(a, &k.box, &k.prm, b->mech);
        int64_t ntiles = 1;
        for (int d = 0; d < 3; d++) {
            int n = k.box.hi[d] - k.box.lo[d] + 1;
            a.ntile[d] = (n + tile[d] - 1) / tile[d];
            ntiles *= a.ntile[d];
        }
        a.Nv = Nv;
        a.rxn = R;
        a.dsdt = A4();
        for (int d = 0; d < 3; d++) {
            a.ef[d] = ef[d];
            a.gne[d] = gne[d];
        }
        PrepArgs p;
        memset(&p, 0, sizeof(p));
        p.rxn = R;
        p.Nv = Nv;
        for (int d = 0; d < 3; d++) {
            p.glo[d] = L.glo[d];
            p.ghi[d] = L.ghi[d];
            p.lo[d] = k.box.lo[d];
            p.hi[d] = k.box.hi[d];
        }
        p.Tg = k.prm.Tg;
        p.do_reactions = k.prm.do_reactions;
        p.write_n = 1;
        GhostArgs g;
        memset(&g, 0, sizeof(g));
        int64_t gcount = 0;
        for (int d = 0; d < 3; d++) {
            g.lo[d] = k.box.lo[d];
            g.hi[d] = k.box.hi[d];
            g.periodic[d] = d < L.dim ? k.periodic[d] : 0;
        }
        g.ghost = L.H;
        g.dim = L.dim;
        for (int d = 0; d < L.dim; d++) gcount += 2 * (int64_t)L.H * (L.vcells / (k.box.hi[d] - k.box.lo[d] + 1));
        g.count = gcount;
        g.ncomp = 0;
        for (int s = 0; s < ns; s++) g.comps[g.ncomp++] = (int8_t)s;
        g.comps[g.ncomp++] = (int8_t)VD_EEN(ns);
        g.comps[g.ncomp++] = (int8_t)VD_ETEMP(ns);
        for (int par = 0; par < 2; par++) {
            A4 sb = dense_view(st[par], L.glo, L.ghi, VD_NVAR(ns));
            A4 pn = dense_view(st[par ^ 1], L.glo, L.ghi, VD_NVAR(ns));
            TransportArgs& t = tr[(size_t)par * b->max_cases + c];
            t = a;
            t.sb = sb;
            t.pn = pn;
            t.status = b->d_status + k.sslot;
            PrepArgs& q = pr[(size_t)par * b->max_cases + c];
            q = p;
            q.sb = sb;
            GhostArgs& h = gh[(size_t)par * b->max_cases + c];
            h = g;
            h.st = pn;
        }
        const int64_t npc = (L.gcells + kPrepChunk - 1) / kPrepChunk;
        for (int64_t q = 0; q < npc; q++) prep.push_back(make_int2(c, (int)q));
        for (int64_t q = 0; q < ntiles; q++) trn[L.dim].push_back(make_int2(c, (int)q));
        if (a.elecenergy && !joule_in_tile(a, b->prec)) {
            const int64_t njt = L.dim == 1   ? joule_tile_count<1>(k.box.lo, k.box.hi)
                                : L.dim == 2 ? joule_tile_count<2>(k.box.lo, k.box.hi)
                                             : joule_tile_count<3>(k.box.lo, k.box.hi);
            for (int64_t q = 0; q < njt; q++) jl[L.dim].push_back(make_int2(c, (int)q));
        }
        const int64_t ngc = (gcount + kGhostChunk - 1) / kGhostChunk;
        for (int64_t q = 0; q < ngc; q++) ghost.push_back(make_int2(c, (int)q));
    }
    // one items array: prep | ghost | transport 1-D | 2-D | 3-D | Joule 1-D | 2-D | 3-D
    size_t total = prep.size() + ghost.size();
    for (int d = 1; d <= 3; d++) total += trn[d].size() + jl[d].size();
    if (total > (size_t)INT32_MAX) return err(VD_ERR_ARG, "too many work items");
    if (total > b->items_cap) {
        if (b->d_items) cudaFree(b->d_items);
        b->d_items = nullptr;
        size_t cap = std::max<size_t>(total, b->items_cap * 2);
        cudaError_t e = cudaMalloc(&b->d_items, cap * sizeof(int2));
        if (e != cudaSuccess) {
            b->items_cap = 0;
            return err(VD_ERR_NOMEM, "work list of %zu items: %s", cap, cudaGetErrorString(e));
        }
        b->items_cap = cap;
    }
    std::vector<int2> all;
    all.reserve(total);
    b->off_prep = all.size();
    all.insert(all.end(), prep.begin(), prep.end());
    b->off_ghost = all.size();
    all.insert(all.end(), ghost.begin(), ghost.end());
    for (int d = 1; d <= 3; d++) {
        b->off_tr[d] = all.size();
        all.insert(all.end(), trn[d].begin(), trn[d].end());
        b->n_tr[d] = (int)trn[d].size();
    }
    for (int d = 1; d <= 3; d++) {
        b->off_jl[d] = all.size();
        all.insert(all.end(), jl[d].begin(), jl[d].end());
        b->n_jl[d] = (int)jl[d].size();
    }
    b->n_prep = (int)prep.size();
    b->n_ghost = (int)ghost.size();
    cudaError_t e = cudaSuccess;
    if (total) e = cudaMemcpy(b->d_items, all.data(), total * sizeof(int2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nb) {
        for (int par = 0; par < 2; par++) {
            size_t o = (size_t)par * b->max_cases;
            e = cudaMemcpy(b->d_tr + o, tr.data() + o, nb * sizeof(TransportArgs), cudaMemcpyHostToDevice);
            if (e == cudaSuccess)
                e = cudaMemcpy(b->d_pr + o, pr.data() + o, nb * sizeof(PrepArgs), cudaMemcpyHostToDevice);
            if (e == cudaSuccess)
                e = cudaMemcpy(b->d_gh + o, gh.data() + o, nb * sizeof(GhostArgs), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) break;
        }
    }
    if (e != cudaSuccess) return cuda_err(e, "uploading batch tables");
    int ndims = 0;
    for (int d = 1; d <= 3; d++) ndims += (b->n_tr[d] > 0) + (b->n_jl[d] > 0);
    b->launches_per_step = (b->n_prep > 0) + ndims + (b->n_ghost > 0);
    drop_graph(b);
    b->dirty = false;
    return VD_OK;
}

// Queues `nsteps` steps of the current work lists on st (captured or direct).
cudaError_t queue_steps(vd_batch* b, int nsteps, cudaStream_t st)
{
    const int nb = (int)b->cases.size();
    const int ns = b->mech.ns;
    int dims[3], nd = 0;
    for (int d = 1; d <= 3; d++)
        if (b->n_tr[d] > 0) dims[nd++] = d;
    for (int t = 0; t < nsteps; t++) {
        BatchCtl ctl{b->d_ctrl, b->max_cases, t};
        cudaError_t e = launch_prep_batch(b->d_pr, b->d_items + b->off_prep, b->n_prep, ctl, b->prec, ns, st);
        if (e != cudaSuccess) return e;
        for (int d = 1; d <= 3 && e == cudaSuccess; d++)
            e = launch_joule_pre_batch(b->d_tr, b->d_items + b->off_jl[d], b->n_jl[d], ctl, d, b->prec, st);
        if (e != cudaSuccess) return e;
        if (nd > 1) {
            // independent dimensions run side by side
            if ((e = cudaEventRecord(b->fork, st)) != cudaSuccess) return e;
            for (int i = 1; i < nd; i++)
                if ((e = cudaStreamWaitEvent(b->side[i], b->fork, 0)) != cudaSuccess) return e;
        }
        for (int i = 0; i < nd; i++) {
            cudaStream_t s = i == 0 ? st : b->side[i];
            int d = dims[i];
            e = launch_transport_batch(b->d_tr, b->d_items + b->off_tr[d], b->n_tr[d], ctl, d, b->prec,
                                       b->variant[d], s);
            if (e != cudaSuccess) return e;
        }
        for (int i = 1; i < nd; i++) {
            if ((e = cudaEventRecord(b->join[i], b->side[i])) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(st, b->join[i], 0)) != cudaSuccess) return e;
        }
        e = launch_ghost_batch(b->d_gh, b->d_items + b->off_ghost, b->n_ghost, ctl, st);
        if (e != cudaSuccess) return e;
    }
    (void)nb;
    return cudaSuccess;
}

int build_graph(vd_batch* b, int nsteps)
{
    drop_graph(b);
    cudaStream_t cap;
    cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_err(e, "capture stream");
    cudaGraph_t g = nullptr;
    prof_suspend(true);
    const int64_t before = launch_count();
    e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    cudaError_t eq = cudaSuccess;
    if (e == cudaSuccess) {
        eq = queue_steps(b, nsteps, cap);
        e = cudaStreamEndCapture(cap, &g);
    }
    prof_suspend(false);
    // the captured launches ran nothing yet: count them at each replay instead
    add_launches(-(launch_count() - before));
    cudaStreamDestroy(cap);
    if (eq != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_err(eq, "capturing the batch step");
    }
    if (e != cudaSuccess) return cuda_err(e, "capturing the batch step");
    cudaGraphExec_t x = nullptr;
    e = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_err(e, "instantiating the batch graph");
    b->graph = x;
    b->graph_steps = nsteps;
    b->graph_builds++;
    return VD_OK;
}

int check_mech(vd_batch* b)
{
    vd_host::MechInfo m;
    int rc = vd_host::mech_info(&m);
    if (rc) return rc;
    if (m.generation != b->mech_gen)
        return err(VD_ERR_STATE, "the mechanism changed since the batch was created (vd_mech_init)");
    return VD_OK;
}

int check_device(vd_batch* b)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetDevice");
    if (dev != b->dev) return err(VD_ERR_STATE, "batch lives on device %d, current device is %d", b->dev, dev);
    return VD_OK;
}

// Writes ctrl = {steps this call, current copy} for every slot into staging and
// queues its copy to the device on st.
int queue_ctrl(vd_batch* b, const std::vector<int>& steps, cudaStream_t st)
{
    const int nb = (int)b->cases.size();
    int s = b->ctrl_slot;
    b->ctrl_slot ^= 1;
    cudaError_t e = cudaEventSynchronize(b->ctrl_done[s]);  // staging slot free again
    if (e != cudaSuccess) return cuda_err(e, "control staging");
    for (int c = 0; c < nb; c++) b->h_ctrl[s][c] = make_int2(steps[c], b->cases[c].cur);
    e = cudaMemcpyAsync(b->d_ctrl, b->h_ctrl[s], nb * sizeof(int2), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(b->ctrl_done[s], st);
    if (e != cudaSuccess) return cuda_err(e, "control upload");
    return VD_OK;
}

}  // namespace

// ===========================================================================
extern "C" {

uint64_t vd_batch_case_bytes(const vd_box* bx, const vd_params* prm)
{
    vd_host::MechInfo m;
    if (vd_host::mech_info(&m)) return 0;
    if (vd_host::check_update_params(bx, prm, m)) return 0;
    Layout L;
    make_layout(bx, prm, m.ns, &L);
    return L.bytes;
}

int vd_batch_create(vd_batch** out, int precision, uint64_t hbm_budget_bytes, int max_cases)
{
    if (!out) return err(VD_ERR_ARG, "null output");
    *out = nullptr;
    if (precision != VD_PREC_FP64 && precision != VD_PREC_MIXED)
        return err(VD_ERR_ARG, "unknown precision %d", precision);
    if (max_cases < 1 || max_cases > (1 << 20)) return err(VD_ERR_ARG, "max_cases %d outside [1, 2^20]", max_cases);
    if (hbm_budget_bytes < kAlign) return err(VD_ERR_ARG, "budget of %llu bytes too small",
                                              (unsigned long long)hbm_budget_bytes);
    int rc = vd_host::ensure_mech(0);
    if (rc) return rc;
    vd_batch* b = new vd_batch;
    rc = vd_host::mech_info(&b->mech);
    if (rc) {
        delete b;
        return rc;
    }
    b->mech_gen = b->mech.generation;
    b->prec = precision;
    b->max_cases = max_cases;
    cudaGetDevice(&b->dev);
    for (int d = 1; d <= 3; d++) {
        char key[64];
        snprintf(key, sizeof(key), "batch_tile_%dd_%s", d, precision == VD_PREC_MIXED ? "mixed" : "fp64");
        int v = tune_get(key);
        b->variant[d] = v >= 0 ? v : 0;
    }
    cudaError_t e = cudaMalloc(&b->arena_base, hbm_budget_bytes);
    if (e != cudaSuccess) {
        delete b;
        return err(VD_ERR_NOMEM, "arena of %llu bytes: %s", (unsigned long long)hbm_budget_bytes,
                   cudaGetErrorString(e));
    }
    b->arena.init(hbm_budget_bytes);
    size_t mc = (size_t)max_cases;
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tr, 2 * mc * sizeof(TransportArgs));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_pr, 2 * mc * sizeof(PrepArgs));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_gh, 2 * mc * sizeof(GhostArgs));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ctrl, mc * sizeof(int2));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_status, mc * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(b->d_status, 0, mc * sizeof(unsigned int));
    for (int q = max_cases - 1; q >= 0; q--) b->free_sslot.push_back(q);
    for (int s = 0; s < 2 && e == cudaSuccess; s++) {
        e = cudaMallocHost(&b->h_ctrl[s], mc * sizeof(int2));
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ctrl_done[s], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->last_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int i = 1; i < 3 && e == cudaSuccess; i++) {
        e = cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        int r = err(VD_ERR_NOMEM, "batch tables: %s", cudaGetErrorString(e));
        vd_batch_destroy(b);
        return r;
    }
    *out = b;
    return VD_OK;
}

int vd_batch_destroy(vd_batch* b)
{
    if (!b) return VD_OK;
    int dev0 = 0;
    cudaGetDevice(&dev0);
    cudaSetDevice(b->dev);
    settle(b);
    drop_graph(b);
    cudaFree(b->arena_base);
    cudaFree(b->d_tr);
    cudaFree(b->d_pr);
    cudaFree(b->d_gh);
    cudaFree(b->d_ctrl);
    cudaFree(b->d_status);
    cudaFree(b->d_items);
    for (int s = 0; s < 2; s++) {
        if (b->h_ctrl[s]) cudaFreeHost(b->h_ctrl[s]);
        if (b->ctrl_done[s]) cudaEventDestroy(b->ctrl_done[s]);
    }
    if (b->last_done) cudaEventDestroy(b->last_done);
    if (b->fork) cudaEventDestroy(b->fork);
    for (int i = 1; i < 3; i++) {
        if (b->side[i]) cudaStreamDestroy(b->side[i]);
        if (b->join[i]) cudaEventDestroy(b->join[i]);
    }
    delete b;
    cudaSetDevice(dev0);
    return VD_OK;
}

int vd_batch_add_case(vd_batch* b, const vd_box* bx, const double* state, const double* const efield_ec[3],
                      const double* const gradne_fc[3], const vd_params* prm, const int32_t periodic[3],
                      int64_t nsteps, void* stream, int32_t* case_id)
{
    if (!b || !state || !case_id) return err(VD_ERR_ARG, "null argument");
    int rc;
    if ((rc = check_device(b)) || (rc = check_mech(b))) return rc;
    if ((rc = vd_host::check_update_params(bx, prm, b->mech))) return rc;
    if (prm->precision != b->prec)
        return err(VD_ERR_ARG, "case precision %d differs from the batch's %d", prm->precision, b->prec);
    for (int d = 0; d < 3; d++)
        if (prm->domlo[d] > bx->lo[d] || prm->domhi[d] < bx->hi[d])
            return err(VD_ERR_ARG, "box extends outside the case's domain in direction %d", d);
    if ((int)b->cases.size() >= b->max_cases) return err(VD_ERR_BUDGET, "batch holds max_cases = %d", b->max_cases);
    Layout L;
    make_layout(bx, prm, b->mech.ns, &L);
    if (L.has_ef && !efield_ec) return err(VD_ERR_ARG, "efield_ec needed (elecenergy_solve without cs_technique)");
    if (L.has_gne && !gradne_fc) return err(VD_ERR_ARG, "gradne_fc needed (elecenergy_solve without gradne_from_state)");
    for (int d = 0; d < bx->dim; d++) {
        if (L.has_ef && !efield_ec[d]) return err(VD_ERR_ARG, "efield_ec[%d] is null", d);
        if (L.has_gne && !gradne_fc[d]) return err(VD_ERR_ARG, "gradne_fc[%d] is null", d);
        if (periodic && periodic[d] && (bx->hi[d] - bx->lo[d] + 1) < L.H)
            return err(VD_ERR_GHOST, "periodic direction %d shorter than the stencil halo", d);
    }
    if ((rc = settle(b))) return rc;
    size_t off = 0;
    if (!b->arena.alloc(L.bytes, &off))
        return err(VD_ERR_BUDGET, "case needs %zu bytes; %zu of %zu budget bytes in use", L.bytes, b->arena.used,
                   b->arena.cap);
    cudaStream_t st = (cudaStream_t)stream;
    char* base = b->arena_base + off;
    const size_t sbytes = (size_t)L.gcells * VD_NVAR(b->mech.ns) * sizeof(double);
    cudaError_t e = cudaMemcpyAsync(base + L.st[0], state, sbytes, cudaMemcpyDefault, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + L.st[1], base + L.st[0], sbytes, cudaMemcpyDeviceToDevice, st);
    for (int d = 0; d < bx->dim && e == cudaSuccess; d++) {
        const size_t fb = (size_t)L.fcells[d] * sizeof(double);
        if (L.has_ef) e = cudaMemcpyAsync(base + L.ef[d], efield_ec[d], fb, cudaMemcpyDefault, st);
        if (e == cudaSuccess && L.has_gne) e = cudaMemcpyAsync(base + L.gne[d], gradne_fc[d], fb, cudaMemcpyDefault, st);
    }
    const int sslot = b->free_sslot.back();
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_status + sslot, 0, sizeof(unsigned int), st);
    if (e == cudaSuccess) e = cudaEventRecord(b->last_done, st);
    if (e != cudaSuccess) {
        b->arena.release(off, L.bytes);
        return cuda_err(e, "uploading the case");
    }
    b->free_sslot.pop_back();
    b->pending = true;
    Case k;
    k.id = b->next_id++;
    k.box = *bx;
    k.prm = *prm;
    for (int d = 0; d < 3; d++) k.periodic[d] = periodic ? periodic[d] : 0;
    k.L = L;
    k.off = off;
    k.cur = 0;
    k.steps_done = 0;
    k.steps_left = nsteps;
    k.sslot = sslot;
    k.failed = false;
    b->cases.push_back(k);
    b->dirty = true;
    *case_id = k.id;
    return VD_OK;
}

int vd_batch_remove_case(vd_batch* b, int32_t case_id)
{
    if (!b) return err(VD_ERR_ARG, "null batch");
    int c = slot_of(b, case_id);
    if (c < 0) return err(VD_ERR_ARG, "no case %d in the batch", case_id);
    int rc = settle(b);
    if (rc) return rc;
    b->arena.release(b->cases[c].off, b->cases[c].L.bytes);
    b->free_sslot.push_back(b->cases[c].sslot);
    b->cases.erase(b->cases.begin() + c);
    b->dirty = true;
    return VD_OK;
}

int vd_batch_step(vd_batch* b, int nsteps, void* stream)
{
    if (!b) return err(VD_ERR_ARG, "null batch");
    if (nsteps < 0) return err(VD_ERR_ARG, "nsteps %d < 0", nsteps);
    int rc;
    if ((rc = check_device(b)) || (rc = check_mech(b))) return rc;
    if ((rc = vd_host::ensure_mech((cudaStream_t)stream))) return rc;
    const int nb = (int)b->cases.size();
    std::vector<int> steps(nb);
    int maxs = 0;
    for (int c = 0; c < nb; c++) {
        int64_t s = b->cases[c].steps_left < 0 ? nsteps : std::min<int64_t>(nsteps, b->cases[c].steps_left);
        if (b->cases[c].failed) s = 0;
        steps[c] = (int)s;
        maxs = std::max(maxs, steps[c]);
    }
    if (nb == 0 || maxs == 0) return VD_OK;
    if (b->dirty) {
        if ((rc = settle(b))) return rc;
        if ((rc = rebuild(b))) return rc;
    }
    cudaStream_t st = (cudaStream_t)stream;
    // a graph of nsteps steps serves every call of that length (cases that are
    // done skip their items); the direct path launches only maxs steps
    if ((rc = queue_ctrl(b, steps, st))) return rc;
    cudaError_t e;
    if (b->use_graph) {
        if (!b->graph || b->graph_steps != nsteps)
            if ((rc = build_graph(b, nsteps))) return rc;
        e = cudaGraphLaunch(b->graph, st);
        if (e == cudaSuccess) add_launches((int64_t)b->launches_per_step * nsteps);
    } else {
        e = queue_steps(b, maxs, st);
    }
    if (e == cudaSuccess) e = cudaEventRecord(b->last_done, st);
    if (e != cudaSuccess) return cuda_err(e, "batch step");
    b->pending = true;
    for (int c = 0; c < nb; c++) {
        Case& k = b->cases[c];
        k.cur ^= steps[c] & 1;
        k.steps_done += steps[c];
        if (k.steps_left > 0) k.steps_left -= steps[c];
        b->steps_run += steps[c];
    }
    return VD_OK;
}

int vd_batch_case_info(vd_batch* b, int32_t case_id, int64_t* steps_done, int64_t* steps_left)
{
    if (!b) return err(VD_ERR_ARG, "null batch");
    int c = slot_of(b, case_id);
    if (c < 0) return err(VD_ERR_ARG, "no case %d in the batch", case_id);
    if (steps_done) *steps_done = b->cases[c].steps_done;
    if (steps_left) *steps_left = b->cases[c].steps_left;
    return VD_OK;
}

int vd_batch_case_status(vd_batch* b, int32_t case_id, int32_t* nonfinite)
{
    if (!b || !nonfinite) return err(VD_ERR_ARG, "null argument");
    int rc = check_device(b);
    if (rc) return rc;
    int c = slot_of(b, case_id);
    if (c < 0) return err(VD_ERR_ARG, "no case %d in the batch", case_id);
    if ((rc = settle(b))) return rc;
    unsigned int h = 0;
    cudaError_t e = cudaMemcpy(&h, b->d_status + b->cases[c].sslot, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_err(e, "reading the case status");
    if (h) b->cases[c].failed = true;
    *nonfinite = (h || b->cases[c].failed) ? 1 : 0;
    return VD_OK;
}

int vd_batch_read_case(vd_batch* b, int32_t case_id, double* state, void* stream)
{
    if (!b || !state) return err(VD_ERR_ARG, "null argument");
    int rc = check_device(b);
    if (rc) return rc;
    int c = slot_of(b, case_id);
    if (c < 0) return err(VD_ERR_ARG, "no case %d in the batch", case_id);
    const Case& k = b->cases[c];
    cudaStream_t st = (cudaStream_t)stream;
    // ordered after the batch's last step, whichever stream that ran on
    cudaError_t e = b->pending ? cudaStreamWaitEvent(st, b->last_done, 0) : cudaSuccess;
    const size_t sbytes = (size_t)k.L.gcells * VD_NVAR(b->mech.ns) * sizeof(double);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(state, b->arena_base + k.off + k.L.st[k.cur], sbytes, cudaMemcpyDefault, st);
    if (e != cudaSuccess) return cuda_err(e, "reading the case");
    return VD_OK;
}

int vd_batch_load_case(vd_batch* b, int32_t case_id, const double* state, int64_t nsteps, void* stream)
{
    if (!b || !state) return err(VD_ERR_ARG, "null argument");
    int rc = check_device(b);
    if (rc) return rc;
    int c = slot_of(b, case_id);
    if (c < 0) return err(VD_ERR_ARG, "no case %d in the batch", case_id);
    Case& k = b->cases[c];
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = b->pending ? cudaStreamWaitEvent(st, b->last_done, 0) : cudaSuccess;
    const size_t sbytes = (size_t)k.L.gcells * VD_NVAR(b->mech.ns) * sizeof(double);
    // both copies: the fields a step only reads (E, potential, ...) are read from
    // whichever copy is current
    char* cur = b->arena_base + k.off + k.L.st[k.cur];
    char* oth = b->arena_base + k.off + k.L.st[k.cur ^ 1];
    if (e == cudaSuccess) e = cudaMemcpyAsync(cur, state, sbytes, cudaMemcpyDefault, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(oth, cur, sbytes, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_status + k.sslot, 0, sizeof(unsigned int), st);
    if (e == cudaSuccess) e = cudaEventRecord(b->last_done, st);
    if (e != cudaSuccess) return cuda_err(e, "loading the case");
    b->pending = true;
    k.steps_done = 0;
    k.steps_left = nsteps;
    k.failed = false;
    return VD_OK;
}

int vd_batch_set_tile_variant(vd_batch* b, int dim, int variant)
{
    if (!b) return err(VD_ERR_ARG, "null batch");
    if (dim < 1 || dim > 3) return err(VD_ERR_DIM, "dim %d", dim);
    if (variant < 0 || variant >= batch_tile_variants(dim))
        return err(VD_ERR_ARG, "variant %d outside [0,%d)", variant, batch_tile_variants(dim));
    if (b->variant[dim] != variant) {
        int rc = settle(b);
        if (rc) return rc;
        b->variant[dim] = variant;
        b->dirty = true;
    }
    return VD_OK;
}

int vd_batch_tile_shape(int dim, int variant, int32_t tile[3], int32_t* min_blocks)
{
    if (dim < 1 || dim > 3) return err(VD_ERR_DIM, "dim %d", dim);
    if (variant < 0 || variant >= batch_tile_variants(dim)) return err(VD_ERR_ARG, "variant %d", variant);
    int t[3];
    batch_tile_shape(dim, variant, t);
    for (int d = 0; d < 3; d++) tile[d] = t[d];
    if (min_blocks) *min_blocks = batch_variant_minblocks(dim, variant);
    return batch_tile_variants(dim);
}

int vd_batch_set_graph(vd_batch* b, int on)
{
    if (!b) return err(VD_ERR_ARG, "null batch");
    b->use_graph = on != 0;
    return VD_OK;
}

// Times the transport kernel of every tile variant on the resident cases and keeps
// the fastest per dimension.  The state is not advanced: each trial reads the
// current copy and writes the other one, which the next real step overwrites.
int vd_batch_tune(vd_batch* b, int trials, void* stream, double* ms_out)
{
    if (!b) return err(VD_ERR_ARG, "null batch");
    if (trials < 1) trials = 1;
    int rc;
    if ((rc = check_device(b)) || (rc = check_mech(b))) return rc;
    const int nb = (int)b->cases.size();
    if (ms_out)
        for (int i = 0; i < 32; i++) ms_out[i] = -1.0;
    if (nb == 0) return VD_OK;
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<int> one(nb, 1);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int d = 1; d <= 3; d++) {
        if ((rc = settle(b))) break;
        if (b->dirty && (rc = rebuild(b))) break;
        if (b->n_tr[d] == 0) continue;
        int best = b->variant[d];
        float best_ms = 1e30f;
        for (int v = 0; v < batch_tile_variants(d); v++) {
            if ((rc = settle(b))) break;
            b->variant[d] = v;
            if ((rc = rebuild(b))) break;
            if ((rc = queue_ctrl(b, one, st))) break;
            BatchCtl ctl{b->d_ctrl, b->max_cases, 0};
            cudaError_t e =
                launch_prep_batch(b->d_pr, b->d_items + b->off_prep, b->n_prep, ctl, b->prec, b->mech.ns, st);
            if (e == cudaSuccess)
                e = launch_joule_pre_batch(b->d_tr, b->d_items + b->off_jl[d], b->n_jl[d], ctl, d, b->prec, st);
            // one untimed launch, then the timed ones
            if (e == cudaSuccess)
                e = launch_transport_batch(b->d_tr, b->d_items + b->off_tr[d], b->n_tr[d], ctl, d, b->prec, v, st);
            if (e == cudaSuccess) e = cudaEventRecord(e0, st);
            for (int i = 0; i < trials && e == cudaSuccess; i++)
                e = launch_transport_batch(b->d_tr, b->d_items + b->off_tr[d], b->n_tr[d], ctl, d, b->prec, v, st);
            if (e == cudaSuccess) e = cudaEventRecord(e1, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) {
                rc = cuda_err(e, "tuning launch");
                break;
            }
            ms /= trials;
            if (ms_out && v < 8) ms_out[d * 8 + v] = ms;
            if (ms < best_ms) {
                best_ms = ms;
                best = v;
            }
        }
        if (rc) break;
        b->variant[d] = best;
        b->dirty = true;
        char key[64];
        snprintf(key, sizeof(key), "batch_tile_%dd_%s", d, b->prec == VD_PREC_MIXED ? "mixed" : "fp64");
        tune_set(key, best);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

int vd_batch_get_stats(vd_batch* b, vd_batch_stats* out)
{
    if (!b || !out) return err(VD_ERR_ARG, "null argument");
    memset(out, 0, sizeof(*out));
    out->ncases = (int32_t)b->cases.size();
    for (const Case& k : b->cases) {
        out->ncases_dim[k.box.dim]++;
        out->cells += k.L.vcells;
    }
    out->bytes_used = b->arena.used;
    out->bytes_budget = b->arena.cap;
    out->steps_run = b->steps_run;
    out->graph_builds = b->graph_builds;
    for (int d = 0; d < 4; d++) out->tile_variant[d] = b->variant[d];
    out->launches_per_step = b->launches_per_step;
    return VD_OK;
}

}  // extern "C"

// ===========================================================================
namespace vd_host {

int batch_failed_cases(vd_batch* b, std::vector<int>* ids)
{
    ids->clear();
    int rc = settle(b);
    if (rc) return rc;
    std::vector<unsigned int> h((size_t)b->max_cases);
    cudaError_t e = cudaMemcpy(h.data(), b->d_status, h.size() * sizeof(unsigned int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_err(e, "reading the case statuses");
    for (Case& k : b->cases) {
        if (h[k.sslot]) k.failed = true;
        if (k.failed) ids->push_back(k.id);
    }
    return VD_OK;
}

}  // namespace vd_host
