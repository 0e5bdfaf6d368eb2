// vd_diffusion.cu -- the implicit diffusion solve of one species
// (vd_implicit_species_solve in vidyut_b200.h).
//
// The reference solves, per transported species after the explicit part of a
// step, (1/dt) n - div(D grad n) = n_old/dt + dsdt_expl with AMReX's
// MLABecLaplacian and MLMG (Vidyut::implicit_solve_scalar,
// Source/ScalarSolve.cpp:289-680).  AMReX is not part of this library, so this file
// carries a geometric multigrid for the same discrete problem on one box that is
// the whole domain, in FP64:
//  - D at every cell of the box grown by one from specDiff of the current state
//    (:478-490), on faces the harmonic mean of the two cells (:497-505); coarse
//    levels average the fine faces that cover a coarse face;
//  - domain faces from species_bc (Source/PlasmaChem.H:75-184): one value per face,
//    the value at the face for VD_BC_DIRC, the derivative along the coordinate
//    direction for VD_BC_IHNEU; VD_BC_HNEU and VD_BC_ROBIN (species_bc's default
//    robin a = 0, b = 1, f = 0) give zero gradient; a periodic direction (both
//    sides VD_BC_PER, an even number of cells) couples its first and last cells
//    through the face between them, whose coefficient comes from the state's
//    ghost cells as any face's (the caller fills them periodically, as FillPatch
//    does);
//  - V(2,2) cycles of red-black Gauss-Seidel, averaging restriction, linear
//    prolongation, a one-CTA bottom solve on the coarsest grid;
//  - afterwards the density floor (:590-617), the electrons' face gradients
//    (getGradSolution, :618-621) and, for the electron energy, the Te update with
//    its floor (:630-666).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>
#include "vd_device.cuh"
#include "vd_host.h"

namespace vd {

// this translation unit's copy of the mechanism table (vd_device.cuh)
cudaError_t upload_mech_diffusion(const VdMechDev* h, cudaStream_t st)
{
    return cudaMemcpyToSymbolAsync(c_mech, h, sizeof(VdMechDev), 0, cudaMemcpyHostToDevice, st);
}

namespace {

constexpr double M_AMU = 1.66054e-27;  // Source/UnivConstants.H:18

struct DLevel {
    int n[3];          // cells per direction (1 beyond dim)
    double idx2[3];    // 1/dx^2 (0 beyond dim)
    double idx[3];     // 1/dx
    double a;          // 1/dt
    double* phi;
    double* rhs;
    double* res;
    double* b[3];      // face coefficients: face (i,j,k) of direction d, n[d]+1 along d
    __host__ __device__ int64_t cells() const { return (int64_t)n[0] * n[1] * n[2]; }
};

// Domain faces: type per side and direction; on the finest level the value of each
// boundary face (val[side][d], laid out over the face plane, x fastest), none on
// the correction levels (homogeneous).
struct DBc {
    int type_lo[3], type_hi[3];
    const double* val_lo[3];
    const double* val_hi[3];
    // faces of type kBcUserRobin: a n + b dn/dnu = f (nu the outward normal), per
    // [side][direction]; f is zero on the correction levels
    double ra[2][3], rb[2][3], rf[2][3];
    int per[3];  // 1: periodic direction
};
// the caller's Robin coefficients (vd_diffusion_params.user_robin) on a face
constexpr int kBcUserRobin = 100;

// A face with a n_f + b (n_g - n_c)/h = f, n_f = (n_c + n_g)/2, between the cell
// value n_c and its ghost n_g: n_g - n_c = (f - a n_c) / (a/2 + b/h).
__device__ __forceinline__ double robin_den(const DBc& bc, int side, int d, double idx)
{
    return 0.5 * bc.ra[side][d] + bc.rb[side][d] * idx;
}

__device__ __forceinline__ int64_t dlin(const DLevel& L, int i, int j, int k)
{
    return (int64_t)i + (int64_t)L.n[0] * (j + (int64_t)L.n[1] * k);
}
// face (i,j,k) of direction d in its face array (n[d] + 1 along d)
__device__ __forceinline__ int64_t flin(const DLevel& L, int d, int i, int j, int k)
{
    const int n0 = L.n[0] + (d == 0), n1 = L.n[1] + (d == 1);
    return (int64_t)i + (int64_t)n0 * (j + (int64_t)n1 * k);
}
// boundary face plane of direction d at transverse position (c[e] for e != d)
__device__ __forceinline__ int64_t plin(const DLevel& L, int d, const int* c)
{
    const int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
    return (int64_t)c[e0] + (int64_t)L.n[e0] * c[e1];
}

// The cell's face coefficients and neighbour values, loaded before any is used
// (the neighbour through a periodic direction wraps; beyond a domain face the
// cell itself stands in, unused): a thread's loads are then in flight together.
template <int DIM>
struct DNbr {
    double blo[DIM], bhi[DIM], vlo[DIM], vhi[DIM];
};
template <int DIM>
__device__ __forceinline__ DNbr<DIM> dstencil_load(const DLevel& L, const DBc& bc, int i, int j, int k,
                                                   const double* phi)
{
    const int c[3] = {i, j, k};
    const int64_t str[3] = {1, L.n[0], (int64_t)L.n[0] * L.n[1]};
    const int64_t cc = dlin(L, i, j, k);
    DNbr<DIM> v;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        int p[3] = {i, j, k};
        p[d] += 1;
        v.blo[d] = L.b[d][flin(L, d, i, j, k)];
        v.bhi[d] = L.b[d][flin(L, d, p[0], p[1], p[2])];
        const int64_t wrap = (int64_t)(L.n[d] - 1) * str[d];
        v.vlo[d] = phi[c[d] > 0 ? cc - str[d] : (bc.per[d] ? cc + wrap : cc)];
        v.vhi[d] = phi[c[d] < L.n[d] - 1 ? cc + str[d] : (bc.per[d] ? cc - wrap : cc)];
    }
    return v;
}
// The operator row of cell (i,j,k): diag * n_c + off = a n_c - div(b grad n) with
// the domain faces folded in.  An inside neighbour adds b/dx^2 to diag and
// -b n_nb/dx^2 to off; a Dirichlet face holds n = v at the face (half a cell
// away: 2b/dx^2 to diag, -2b v/dx^2 to off); a face with a given derivative g
// along its direction carries the flux b g (sgn b g/dx moved to off with the
// opposite sign); a zero-gradient face adds nothing.
template <int DIM>
__device__ __forceinline__ void dstencil_apply(const DLevel& L, const DBc& bc, int i, int j, int k,
                                               const DNbr<DIM>& v, double& off, double& diag)
{
    const int c[3] = {i, j, k};
    off = 0.0;
    diag = L.a;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const double w = L.idx2[d];
        const double blo = v.blo[d], bhi = v.bhi[d];
        if (c[d] > 0 || bc.per[d]) {
            off -= blo * w * v.vlo[d];
            diag += blo * w;
        } else if (bc.type_lo[d] == VD_BC_DIRC) {
            diag += 2.0 * blo * w;
            if (bc.val_lo[d]) off -= 2.0 * blo * w * bc.val_lo[d][plin(L, d, c)];
        } else if (bc.type_lo[d] == VD_BC_IHNEU && bc.val_lo[d]) {
            off += blo * bc.val_lo[d][plin(L, d, c)] * L.idx[d];
        } else if (bc.type_lo[d] == kBcUserRobin) {
            // -b (n_g - n_c)/dx^2 with n_g - n_c = (f - a n_c)/den
            const double den = robin_den(bc, 0, d, L.idx[d]);
            diag += blo * w * bc.ra[0][d] / den;
            off -= blo * w * bc.rf[0][d] / den;
        }
        if (c[d] < L.n[d] - 1 || bc.per[d]) {
            off -= bhi * w * v.vhi[d];
            diag += bhi * w;
        } else if (bc.type_hi[d] == VD_BC_DIRC) {
            diag += 2.0 * bhi * w;
            if (bc.val_hi[d]) off -= 2.0 * bhi * w * bc.val_hi[d][plin(L, d, c)];
        } else if (bc.type_hi[d] == VD_BC_IHNEU && bc.val_hi[d]) {
            off -= bhi * bc.val_hi[d][plin(L, d, c)] * L.idx[d];
        } else if (bc.type_hi[d] == kBcUserRobin) {
            const double den = robin_den(bc, 1, d, L.idx[d]);
            diag += bhi * w * bc.ra[1][d] / den;
            off -= bhi * w * bc.rf[1][d] / den;
        }
    }
}
template <int DIM>
__device__ __forceinline__ void dstencil(const DLevel& L, const DBc& bc, int i, int j, int k, const double* phi,
                                         double& off, double& diag)
{
    dstencil_apply<DIM>(L, bc, i, j, k, dstencil_load<DIM>(L, bc, i, j, k, phi), off, diag);
}

// one red-black Gauss-Seidel half sweep: cells with (i + j + k) % 2 == color.  A
// thread takes two cells, `half` apart along the slowest active direction (k in
// 3-D, j in 2-D; half = 0 in 1-D: one cell), with all their loads issued first.
template <int DIM>
__global__ void __launch_bounds__(128) k_dif_rbgs(DLevel L, DBc bc, int color, int half)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int ii[2], jj[2], kk[2];
    bool ok[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        jj[h] = blockIdx.y + (DIM == 2 ? h * half : 0);
        kk[h] = blockIdx.z + (DIM == 3 ? h * half : 0);
        ii[h] = 2 * t + ((jj[h] + kk[h] + color) & 1);
        ok[h] = ii[h] < L.n[0] && jj[h] < L.n[1] && kk[h] < L.n[2] && (h == 0 || half > 0);
    }
    DNbr<DIM> v[2];
    double r[2];
#pragma unroll
    for (int h = 0; h < 2; h++)
        if (ok[h]) {
            v[h] = dstencil_load<DIM>(L, bc, ii[h], jj[h], kk[h], L.phi);
            r[h] = L.rhs[dlin(L, ii[h], jj[h], kk[h])];
        }
#pragma unroll
    for (int h = 0; h < 2; h++)
        if (ok[h]) {
            double off, diag;
            dstencil_apply<DIM>(L, bc, ii[h], jj[h], kk[h], v[h], off, diag);
            L.phi[dlin(L, ii[h], jj[h], kk[h])] = (r[h] - off) / diag;
        }
}

// blkmax (null: not wanted): max |residual| of each block, one value per block in
// block order, reduced by k_dif_maxabs afterwards (one atomic per warp on a single
// address would serialise in L2 on large grids)
template <int DIM>
__global__ void __launch_bounds__(128) k_dif_residual(DLevel L, DBc bc, double* blkmax)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    if (i < L.n[0]) {
        double off, diag;
        dstencil<DIM>(L, bc, i, j, k, L.phi, off, diag);
        const int64_t c = dlin(L, i, j, k);
        const double r = L.rhs[c] - (off + diag * L.phi[c]);
        L.res[c] = r;
        m = r == r ? fabs(r) : INFINITY;  // a NaN residual counts as the largest
    }
    if (blkmax) {
        __shared__ double wmax[4];  // one per warp of the 128-thread block
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x == 0)
            blkmax[blockIdx.x + (int64_t)gridDim.x * (blockIdx.y + (int64_t)gridDim.y * blockIdx.z)] =
                fmax(fmax(wmax[0], wmax[1]), fmax(wmax[2], wmax[3]));
    }
}

// coarse rhs = average of the 2^dim fine residuals; coarse correction starts at 0
template <int DIM>
__global__ void __launch_bounds__(128) k_dif_restrict(DLevel F, DLevel C)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C.n[0]) return;
    double s = 0.0;
#pragma unroll
    for (int dz = 0; dz < (DIM > 2 ? 2 : 1); dz++)
#pragma unroll
        for (int dy = 0; dy < (DIM > 1 ? 2 : 1); dy++)
#pragma unroll
            for (int dx = 0; dx < 2; dx++)
                s += F.res[dlin(F, 2 * i + dx, DIM > 1 ? 2 * j + dy : j, DIM > 2 ? 2 * k + dz : k)];
    const int64_t c = dlin(C, i, j, k);
    C.rhs[c] = s * (1.0 / (double)(1 << DIM));
    C.phi[c] = 0.0;
}

// coarse face coefficient of direction D: the average of the 2^(dim-1) fine faces
// that make up the coarse face
template <int DIM, int D>
__global__ void __launch_bounds__(128) k_dif_coarsen_b(DLevel F, DLevel C)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C.n[0] + (D == 0)) return;
    const int cf[3] = {i, j, k};
    double s = 0.0;
    int cnt = 0;
#pragma unroll
    for (int t1 = 0; t1 < 2; t1++)
#pragma unroll
        for (int t2 = 0; t2 < 2; t2++) {
            int f[3];
            bool used = true;
#pragma unroll
            for (int e = 0; e < 3; e++) {
                if (e == D) {
                    f[e] = 2 * cf[e];
                } else if (e < DIM) {
                    // the two transverse directions take t1 and t2 in order
                    const int t = (e == (D == 0 ? 1 : 0)) ? t1 : t2;
                    f[e] = 2 * cf[e] + t;
                } else {
                    f[e] = cf[e];
                    const int t = (e == (D == 0 ? 1 : 0)) ? t1 : t2;
                    used = used && t == 0;
                }
            }
            if (used) {
                s += F.b[D][flin(F, D, f[0], f[1], f[2])];
                cnt++;
            }
        }
    C.b[D][flin(C, D, cf[0], cf[1], cf[2])] = s / (double)cnt;
}

// fine phi += linear interpolation of the coarse correction; outside a domain face
// the correction's mirror value: -c for a Dirichlet face, the homogeneous ghost
// relation for a Robin face, c otherwise; across a periodic direction the cell on
// the other side
template <int DIM>
__global__ void __launch_bounds__(128) k_dif_prolong(DLevel F, DLevel C, DBc bc)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.n[0]) return;
    const int f[3] = {i, j, k};
    int ci[3] = {i, j, k}, nb[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        ci[d] = f[d] >> 1;
        nb[d] = (f[d] & 1) ? 1 : -1;
    }
    double acc = 0.0;
#pragma unroll
    for (int mz = 0; mz < (DIM > 2 ? 2 : 1); mz++)
#pragma unroll
        for (int my = 0; my < (DIM > 1 ? 2 : 1); my++)
#pragma unroll
            for (int mx = 0; mx < 2; mx++) {
                const int m[3] = {mx, my, mz};
                double w = 1.0, sign = 1.0;
                int q[3] = {ci[0], ci[1], ci[2]};
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                    w *= m[d] ? 0.25 : 0.75;
                    if (m[d]) {
                        q[d] += nb[d];
                        if (q[d] < 0 && bc.per[d]) {
                            q[d] = C.n[d] - 1;
                        } else if (q[d] >= C.n[d] && bc.per[d]) {
                            q[d] = 0;
                        } else if (q[d] < 0) {
                            q[d] = 0;
                            if (bc.type_lo[d] == VD_BC_DIRC) sign = -sign;
                            if (bc.type_lo[d] == kBcUserRobin)
                                sign *= 1.0 - bc.ra[0][d] / robin_den(bc, 0, d, C.idx[d]);
                        } else if (q[d] >= C.n[d]) {
                            q[d] = C.n[d] - 1;
                            if (bc.type_hi[d] == VD_BC_DIRC) sign = -sign;
                            if (bc.type_hi[d] == kBcUserRobin)
                                sign *= 1.0 - bc.ra[1][d] / robin_den(bc, 1, d, C.idx[d]);
                        }
                    }
                }
                acc += w * sign * C.phi[dlin(C, q[0], q[1], q[2])];
            }
    F.phi[dlin(F, i, j, k)] += acc;
}

constexpr int kDifBottomCells = 4096;

template <int DIM>
__global__ void __launch_bounds__(256) k_dif_bottom(DLevel L, DBc bc, int sweeps)
{
    const int n0 = L.n[0], n1 = L.n[1];
    const int nc = (int)L.cells();
    for (int s = 0; s < sweeps; s++)
        for (int color = 0; color < 2; color++) {
            for (int c = threadIdx.x; c < nc; c += blockDim.x) {
                const int k = c / (n0 * n1), r = c - k * n0 * n1, j = r / n0, i = r - j * n0;
                if (((i + j + k) & 1) != color) continue;
                double off, diag;
                dstencil<DIM>(L, bc, i, j, k, L.phi, off, diag);
                L.phi[c] = (L.rhs[c] - off) / diag;
            }
            __syncthreads();
        }
}

__global__ void k_dif_maxabs(const double* x, int64_t n, unsigned long long* out)
{
    double m = 0.0;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(x[c]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// ---------------------------------------------------------------------------
// Set-up and finishing kernels on the box

struct DifArgs {
    A4 st, old, dsdt, pn;
    int lo[3], hi[3];
    int ns, dim, spec, e_id, dsdt_comp;
    int bound, is_energy;
    double Tg, dt, min_spec, min_elec, min_te;
    double cbar_neutral;   // sqrt(8 kB Tg / (pi m)) of the species when neutral
    int8_t charge[VD_MAX_SPECIES];
};

// D of every cell of the box grown by one (dense, x fastest)
template <int DIM>
__global__ void __launch_bounds__(128) k_dif_cell_d(DifArgs a, double* Dg, int g0, int g1)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g0) return;
    const int ci = a.lo[0] - 1 + i, cj = a.lo[1] - (DIM > 1) + j, ck = a.lo[2] - (DIM > 2) + k;
    const int ns = a.ns;
    const int64_t o = a.st.off(ci, cj, ck);
    double nd = 0.0;
    for (int s = 0; s < ns; s++) nd += a.st.p[o + (int64_t)s * a.st.ns];
    const double te = a.st.p[o + (int64_t)VD_ETEMP(ns) * a.st.ns];
    // |E| over the active directions (Source/ScalarSolve.cpp:486-488)
    double esum = 0.0;
    for (int d = 0; d < DIM; d++) {
        const double e = a.st.p[o + (int64_t)(VD_EFX(ns) + d) * a.st.ns];
        esum += e * e;
    }
    Dg[(int64_t)i + (int64_t)g0 * (j + (int64_t)g1 * k)] = diff_fp64(a.spec, te, nd, a.Tg, sqrt(esum));
}

// level-0 face coefficients of direction D: harmonic mean of the two cells
template <int DIM, int D>
__global__ void __launch_bounds__(128) k_dif_face_b(DLevel L, const double* Dg, int g0, int g1)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n[0] + (D == 0)) return;
    // face (i,j,k) lies between grown cells (f - e_D) and f, grown index = valid + 1
    int g[3] = {i + 1, j + (DIM > 1), k + (DIM > 2)};
    const int64_t cr = (int64_t)g[0] + (int64_t)g0 * (g[1] + (int64_t)g1 * g[2]);
    const int64_t s = D == 0 ? 1 : (D == 1 ? (int64_t)g0 : (int64_t)g0 * g1);
    const double dl = Dg[cr - s], dr = Dg[cr];
    L.b[D][flin(L, D, i, j, k)] = (dl + dr) != 0.0 ? 2.0 * dl * dr / (dl + dr) : 0.0;
}

// species_bc (Source/PlasmaChem.H:75-184) at the domain face of direction D on side
// sgn for every transverse position of the face plane
template <int DIM, int D>
__global__ void __launch_bounds__(128) k_dif_bcval(DifArgs a, DLevel L, double* out, int sgn)
{
    constexpr int E0 = D == 0 ? 1 : 0, E1 = D == 2 ? 1 : 2;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, t1 = blockIdx.y;
    if (t0 >= L.n[E0] || t1 >= L.n[E1]) return;
    int face[3];
    face[E0] = t0;
    face[E1] = t1;
    face[D] = sgn < 0 ? 0 : L.n[D];
    int cint[3] = {face[0], face[1], face[2]};
    if (sgn > 0) cint[D] -= 1;
    const int ns = a.ns;
    const A4& s = a.st;
    auto at = [&](int comp, const int* c) -> double {
        return s.p[s.off(a.lo[0] + c[0], a.lo[1] + c[1], a.lo[2] + c[2]) + (int64_t)comp * s.ns];
    };
    double nd = 0.0;
    for (int q = 0; q < ns; q++) nd += at(q, cint);
    const double te = at(VD_ETEMP(ns), cint);
    // |E| of the three state components (Source/PlasmaChem.H:114-116)
    const double ex = at(VD_EFX(ns), cint), ey = at(VD_EFY(ns), cint), ez = at(VD_EFZ(ns), cint);
    const double emag = sqrt(ex * ex + ey * ey + ez * ez);
    const double Dc = diff_fp64(a.spec, te, nd, a.Tg, emag);
    double g;
    if (a.spec == a.e_id) {
        const double cbar = sqrt(8.0 * K_B * te / PI / ME);
        const double flx = at(a.e_id, cint) * cbar / 4.0 * (double)sgn;
        g = -flx / Dc;
    } else if (a.is_energy) {
        const double cbar = sqrt(8.0 * K_B * te / PI / ME);
        const double flx = (2.0 * K_B * te) * at(a.e_id, cint) * cbar / 4.0 * (double)sgn;
        g = -flx / Dc;
    } else if (a.charge[a.spec] != 0) {
        const double mu = mob_fp64(a.spec, te, nd, a.Tg, emag);
        const double drift = mu * at(a.spec, cint) * at(VD_EFX(ns) + D, cint);
        g = (drift * (double)sgn >= 0.0) ? (-drift / Dc) : 0.0;
    } else {
        // the reference reads the density at the face index (the ghost cell on the
        // high side)
        const double flx = at(a.spec, face) * a.cbar_neutral / 4.0 * (double)sgn;
        g = -flx / Dc;
    }
    out[(int64_t)t0 + (int64_t)L.n[E0] * t1] = g;
}

// rhs = n_old/dt + dsdt; initial guess = the current state
__global__ void __launch_bounds__(128) k_dif_rhs(DifArgs a, DLevel L)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n[0]) return;
    const int ci = a.lo[0] + i, cj = a.lo[1] + j, ck = a.lo[2] + k;
    const int64_t c = dlin(L, i, j, k);
    L.rhs[c] = a.old(ci, cj, ck, a.spec) / a.dt + a.dsdt(ci, cj, ck, a.dsdt_comp);
    L.phi[c] = a.st(ci, cj, ck, a.spec);
}

// floor, copy to the output; the electron energy's Te update and floor
__global__ void __launch_bounds__(128) k_dif_finish(DifArgs a, DLevel L)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n[0]) return;
    const int ci = a.lo[0] + i, cj = a.lo[1] + j, ck = a.lo[2] + k;
    const int64_t c = dlin(L, i, j, k);
    double v = L.phi[c];
    if (a.bound && !a.is_energy) {
        const double lo = a.spec == a.e_id ? a.min_elec : a.min_spec;
        if (v < lo) v = lo;
        L.phi[c] = v;  // the electrons' face gradients use the floored solution
    }
    a.pn(ci, cj, ck, a.spec) = v;
    if (a.is_energy) {
        const int ns = a.ns;
        double te = (2.0 / 3.0) / K_B * v / a.st(ci, cj, ck, a.e_id);
        if (te < a.min_te) {
            te = a.min_te;
            a.pn(ci, cj, ck, VD_EEN(ns)) = 1.5 * K_B * a.pn(ci, cj, ck, a.e_id) * te;
        }
        a.pn(ci, cj, ck, VD_ETEMP(ns)) = te;
    }
}

// electron face gradients dn/dx_D (getGradSolution): inside faces by the cell
// difference, domain faces by the face relation the operator uses
template <int D>
__global__ void __launch_bounds__(128) k_dif_grad(DLevel L, DBc bc, A4 out, int lo0, int lo1, int lo2)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n[0] + (D == 0)) return;
    const int f[3] = {i, j, k};
    const int64_t s1 = D == 0 ? 1 : (D == 1 ? (int64_t)L.n[0] : (int64_t)L.n[0] * L.n[1]);
    const int64_t c = dlin(L, i, j, k);  // the cell above the face (one past the box at the high face)
    const double h = 1.0 / L.idx[D];
    double g = 0.0;
    if (f[D] > 0 && f[D] < L.n[D]) {
        g = (L.phi[c] - L.phi[c - s1]) / h;
    } else if (bc.per[D]) {
        // the face between the last cell and the first
        const int64_t first = f[D] == 0 ? c : c - (int64_t)L.n[D] * s1;
        g = (L.phi[first] - L.phi[first + (int64_t)(L.n[D] - 1) * s1]) / h;
    } else if (f[D] == 0) {
        if (bc.type_lo[D] == VD_BC_DIRC) g = (L.phi[c] - bc.val_lo[D][plin(L, D, f)]) / (0.5 * h);
        else if (bc.type_lo[D] == VD_BC_IHNEU) g = bc.val_lo[D][plin(L, D, f)];
        else if (bc.type_lo[D] == kBcUserRobin)  // outward derivative (n_g - n_c)/h, outward = -x
            g = -(bc.rf[0][D] - bc.ra[0][D] * L.phi[c]) / robin_den(bc, 0, D, L.idx[D]) / h;
    } else {
        if (bc.type_hi[D] == VD_BC_DIRC) g = (bc.val_hi[D][plin(L, D, f)] - L.phi[c - s1]) / (0.5 * h);
        else if (bc.type_hi[D] == VD_BC_IHNEU) g = bc.val_hi[D][plin(L, D, f)];
        else if (bc.type_hi[D] == kBcUserRobin)
            g = (bc.rf[1][D] - bc.ra[1][D] * L.phi[c - s1]) / robin_den(bc, 1, D, L.idx[D]) / h;
    }
    out.p[out.off(lo0 + i, lo1 + j, lo2 + k)] = g;
}

dim3 dgrid(const DLevel& L, int extra_x = 0, int per_thread = 1)
{
    const int nx = (L.n[0] + extra_x + per_thread - 1) / per_thread;
    return dim3((unsigned)((nx + 127) / 128), (unsigned)L.n[1], (unsigned)L.n[2]);
}

int derr(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int derr(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return vd_host::set_error(code, buf);
}

bool covers(const vd_array4& a, const int lo[3], const int hi[3], int ncomp)
{
    if (!a.p || a.ncomp < ncomp) return false;
    for (int d = 0; d < 3; d++)
        if (a.begin[d] > lo[d] || a.end[d] <= hi[d]) return false;
    return true;
}

template <int DIM>
struct DifOps {
    static void rbgs(const DLevel& L, const DBc& b, int color, cudaStream_t st)
    {
        ProfScope ps("k_dif_rbgs", st);
        // pairs along the slowest active direction
        const int ns = DIM == 3 ? L.n[2] : (DIM == 2 ? L.n[1] : 1);
        const int half = DIM == 1 ? 0 : (ns + 1) / 2;
        dim3 g = dgrid(L, 0, 2);
        if (DIM == 3) g.z = (unsigned)half;
        else if (DIM == 2) g.y = (unsigned)half;
        k_dif_rbgs<DIM><<<g, 128, 0, st>>>(L, b, color, half);
    }
    static void residual(const DLevel& L, const DBc& b, double* mx, cudaStream_t st)
    {
        ProfScope ps("k_dif_residual", st);
        k_dif_residual<DIM><<<dgrid(L), 128, 0, st>>>(L, b, mx);
    }
    static void restrict_(const DLevel& F, const DLevel& C, cudaStream_t st)
    {
        ProfScope ps("k_dif_restrict", st);
        k_dif_restrict<DIM><<<dgrid(C), 128, 0, st>>>(F, C);
    }
    static void prolong(const DLevel& F, const DLevel& C, const DBc& b, cudaStream_t st)
    {
        ProfScope ps("k_dif_prolong", st);
        k_dif_prolong<DIM><<<dgrid(F), 128, 0, st>>>(F, C, b);
    }
    static void bottom(const DLevel& L, const DBc& b, int sweeps, cudaStream_t st)
    {
        ProfScope ps("k_dif_bottom", st);
        k_dif_bottom<DIM><<<1, 256, 0, st>>>(L, b, sweeps);
    }
    static void coarsen_b(const DLevel& F, const DLevel& C, cudaStream_t st)
    {
        ProfScope ps("k_dif_coarsen_b", st);
        k_dif_coarsen_b<DIM, 0><<<dgrid(C, 1), 128, 0, st>>>(F, C);
        if (DIM > 1) k_dif_coarsen_b<DIM, (DIM > 1 ? 1 : 0)><<<dim3((C.n[0] + 127) / 128, C.n[1] + 1, C.n[2]), 128, 0, st>>>(F, C);
        if (DIM > 2) k_dif_coarsen_b<DIM, (DIM > 2 ? 2 : 0)><<<dim3((C.n[0] + 127) / 128, C.n[1], C.n[2] + 1), 128, 0, st>>>(F, C);
    }
    static void setup(const DifArgs& a, const DLevel& L0, double* Dg, double* const bv_lo[3], double* const bv_hi[3],
                      cudaStream_t st)
    {
        const int g0 = L0.n[0] + 2, g1 = L0.n[1] + (DIM > 1 ? 2 : 0), g2 = L0.n[2] + (DIM > 2 ? 2 : 0);
        ProfScope ps("k_dif_setup", st);
        k_dif_cell_d<DIM><<<dim3((g0 + 127) / 128, g1, g2), 128, 0, st>>>(a, Dg, g0, g1);
        k_dif_face_b<DIM, 0><<<dgrid(L0, 1), 128, 0, st>>>(L0, Dg, g0, g1);
        if (DIM > 1)
            k_dif_face_b<DIM, (DIM > 1 ? 1 : 0)><<<dim3((L0.n[0] + 127) / 128, L0.n[1] + 1, L0.n[2]), 128, 0, st>>>(
                L0, Dg, g0, g1);
        if (DIM > 2)
            k_dif_face_b<DIM, (DIM > 2 ? 2 : 0)><<<dim3((L0.n[0] + 127) / 128, L0.n[1], L0.n[2] + 1), 128, 0, st>>>(
                L0, Dg, g0, g1);
        for (int d = 0; d < DIM; d++) {
            const int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
            const dim3 g((unsigned)((L0.n[e0] + 127) / 128), (unsigned)L0.n[e1]);
            if (d == 0) {
                if (bv_lo[0]) k_dif_bcval<DIM, 0><<<g, 128, 0, st>>>(a, L0, bv_lo[0], -1);
                if (bv_hi[0]) k_dif_bcval<DIM, 0><<<g, 128, 0, st>>>(a, L0, bv_hi[0], 1);
            } else if (d == 1) {
                if (bv_lo[1]) k_dif_bcval<DIM, (DIM > 1 ? 1 : 0)><<<g, 128, 0, st>>>(a, L0, bv_lo[1], -1);
                if (bv_hi[1]) k_dif_bcval<DIM, (DIM > 1 ? 1 : 0)><<<g, 128, 0, st>>>(a, L0, bv_hi[1], 1);
            } else {
                if (bv_lo[2]) k_dif_bcval<DIM, (DIM > 2 ? 2 : 0)><<<g, 128, 0, st>>>(a, L0, bv_lo[2], -1);
                if (bv_hi[2]) k_dif_bcval<DIM, (DIM > 2 ? 2 : 0)><<<g, 128, 0, st>>>(a, L0, bv_hi[2], 1);
            }
        }
        k_dif_rhs<<<dgrid(L0), 128, 0, st>>>(a, L0);
    }
};

struct DifTable {
    void (*rbgs)(const DLevel&, const DBc&, int, cudaStream_t);
    void (*residual)(const DLevel&, const DBc&, double*, cudaStream_t);
    void (*restrict_)(const DLevel&, const DLevel&, cudaStream_t);
    void (*prolong)(const DLevel&, const DLevel&, const DBc&, cudaStream_t);
    void (*bottom)(const DLevel&, const DBc&, int, cudaStream_t);
    void (*coarsen_b)(const DLevel&, const DLevel&, cudaStream_t);
    void (*setup)(const DifArgs&, const DLevel&, double*, double* const*, double* const*, cudaStream_t);
};

template <int DIM>
DifTable dif_table()
{
    return {DifOps<DIM>::rbgs,    DifOps<DIM>::residual,  DifOps<DIM>::restrict_, DifOps<DIM>::prolong,
            DifOps<DIM>::bottom,  DifOps<DIM>::coarsen_b, DifOps<DIM>::setup};
}

}  // namespace
}  // namespace vd

using namespace vd;

extern "C" int vd_implicit_species_solve(const vd_box* bx, vd_array4 state, vd_array4 state_old, vd_array4 dsdt,
                                         vd_array4 phi_new, const vd_array4 gradne_fc[3], const vd_params* prm,
                                         const vd_diffusion_params* dp, int32_t* vcycles_done, double* rel_residual,
                                         void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (!bx || !prm || !dp) return derr(VD_ERR_ARG, "null argument");
    int rc = vd_host::ensure_mech(st);
    if (rc) return rc;
    vd_host::MechInfo m;
    if ((rc = vd_host::mech_info(&m))) return rc;
    const int dim = bx->dim, ns = m.ns;
    if (dim < 1 || dim > 3 || prm->dim != dim) return derr(VD_ERR_DIM, "dimension %d (params %d)", dim, prm->dim);
    if (dp->spec < 0 || dp->spec > ns) return derr(VD_ERR_ARG, "species %d outside 0..%d", dp->spec, ns);
    if (!(prm->dt > 0.0)) return derr(VD_ERR_ARG, "dt must be positive");
    if (dp->max_vcycles < 1) return derr(VD_ERR_ARG, "max_vcycles must be at least 1");
    int n[3] = {1, 1, 1};
    for (int d = 0; d < 3; d++) {
        n[d] = bx->hi[d] - bx->lo[d] + 1;
        if (n[d] < 1) return derr(VD_ERR_ARG, "empty box");
        if (d >= dim && n[d] != 1) return derr(VD_ERR_DIM, "box extends along direction %d > dim", d);
        if (d < dim && (bx->lo[d] != prm->domlo[d] || bx->hi[d] != prm->domhi[d]))
            return derr(VD_ERR_ARG, "the box must be the whole domain (direction %d)", d);
    }
    const int spec = dp->spec;
    const int cls = spec == ns ? VD_CLASS_ENERGY
                               : (spec == m.e_id ? VD_CLASS_ELECTRON : (m.charge[spec] != 0 ? VD_CLASS_ION
                                                                                           : VD_CLASS_NEUTRAL));
    DBc bc;
    memset(&bc, 0, sizeof(bc));
    for (int d = 0; d < dim; d++) {
        bc.type_lo[d] = prm->bc_lo[cls][d];
        bc.type_hi[d] = prm->bc_hi[cls][d];
        if ((bc.type_lo[d] == VD_BC_PER) != (bc.type_hi[d] == VD_BC_PER))
            return derr(VD_ERR_ARG, "direction %d periodic on one side only", d);
        if (bc.type_lo[d] < VD_BC_PER || bc.type_lo[d] > VD_BC_ROBIN || bc.type_hi[d] < VD_BC_PER ||
            bc.type_hi[d] > VD_BC_ROBIN)
            return derr(VD_ERR_ARG, "unknown boundary code in direction %d", d);
        if (bc.type_lo[d] == VD_BC_PER) {
            // red-black sweeps couple the first and last cells through the wrap:
            // they must differ in colour on every level
            if (n[d] % 2) return derr(VD_ERR_ARG, "periodic direction %d needs an even number of cells", d);
            bc.per[d] = 1;
            continue;
        }
        if (dp->user_robin) {
            // the caller's species_bc coefficients replace the default face values
            for (int side = 0; side < 2; side++) {
                const double ra = dp->robin_a[side][d], rb = dp->robin_b[side][d], rf = dp->robin_f[side][d];
                if (!std::isfinite(ra) || !std::isfinite(rb) || !std::isfinite(rf) ||
                    !(std::fabs(0.5 * ra + rb / prm->dx[d]) > 0.0))
                    return derr(VD_ERR_ARG, "Robin coefficients of direction %d side %d invalid", d, side);
                bc.ra[side][d] = ra;
                bc.rb[side][d] = rb;
                bc.rf[side][d] = rf;
            }
            bc.type_lo[d] = bc.type_hi[d] = kBcUserRobin;
        }
    }
    int glo[3], ghi[3];
    for (int d = 0; d < 3; d++) {
        glo[d] = bx->lo[d] - (d < dim ? 1 : 0);
        ghi[d] = bx->hi[d] + (d < dim ? 1 : 0);
    }
    if (!covers(state, glo, ghi, VD_NVAR(ns))) return derr(VD_ERR_GHOST, "state must cover the box grown by one with NVAR components");
    if (!covers(state_old, bx->lo, bx->hi, spec + 1)) return derr(VD_ERR_ARG, "state_old does not cover the box");
    if (!covers(dsdt, bx->lo, bx->hi, dp->dsdt_comp + 1) || dp->dsdt_comp < 0)
        return derr(VD_ERR_ARG, "dsdt does not cover the box with component %d", dp->dsdt_comp);
    if (!covers(phi_new, bx->lo, bx->hi, VD_NVAR(ns))) return derr(VD_ERR_ARG, "phi_new does not cover the box");
    const bool want_grad = spec == m.e_id && gradne_fc;
    if (want_grad)
        for (int d = 0; d < dim; d++) {
            int fhi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
            fhi[d] += 1;
            if (!covers(gradne_fc[d], bx->lo, fhi, 1)) return derr(VD_ERR_ARG, "gradne_fc[%d] does not cover the face box", d);
        }
    double mw = 0.0;
    if (cls == VD_CLASS_NEUTRAL) {
        mw = vd_host::species_mw(spec);
        if (!(mw > 0.0)) return derr(VD_ERR_MECH, "species %d has no molecular weight", spec);
    }

    // hierarchy: halve every active direction while all stay even and above 2
    std::vector<DLevel> lv;
    {
        DLevel L0;
        memset(&L0, 0, sizeof(L0));
        for (int d = 0; d < 3; d++) {
            L0.n[d] = n[d];
            L0.idx2[d] = d < dim ? 1.0 / (prm->dx[d] * prm->dx[d]) : 0.0;
            L0.idx[d] = d < dim ? 1.0 / prm->dx[d] : 0.0;
        }
        L0.a = 1.0 / prm->dt;
        lv.push_back(L0);
        for (;;) {
            const DLevel& f = lv.back();
            bool ok = true;
            for (int d = 0; d < dim; d++) ok = ok && (f.n[d] % 2 == 0) && f.n[d] > 2;
            if (!ok || lv.size() >= 24) break;
            DLevel c = f;
            for (int d = 0; d < 3; d++) {
                c.n[d] = d < dim ? f.n[d] / 2 : f.n[d];
                c.idx2[d] = f.idx2[d] * 0.25;
                c.idx[d] = f.idx[d] * 0.5;
            }
            lv.push_back(c);
        }
    }
    auto faces = [&](const DLevel& L, int d) -> int64_t {
        return d < dim ? (int64_t)(L.n[0] + (d == 0)) * (L.n[1] + (d == 1)) * (L.n[2] + (d == 2)) : 0;
    };
    size_t total = 0;
    for (auto& L : lv) {
        total += 3 * (size_t)L.cells();
        for (int d = 0; d < 3; d++) total += (size_t)faces(L, d);
    }
    const int64_t gcells = (int64_t)(n[0] + 2) * (n[1] + (dim > 1 ? 2 : 0)) * (n[2] + (dim > 2 ? 2 : 0));
    total += (size_t)gcells;
    int64_t plane[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) {
        const int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
        plane[d] = (int64_t)n[e0] * n[e1];
        total += 2 * (size_t)plane[d];
    }
    const dim3 g0 = dgrid(lv[0]);
    const int64_t nblk0 = (int64_t)g0.x * g0.y * g0.z;  // residual blocks of the finest level
    total += (size_t)nblk0;
    double* buf = nullptr;
    cudaError_t e = vd_host::scratch_alloc(reinterpret_cast<void**>(&buf), (total + 1) * sizeof(double) + 64, st);
    if (e != cudaSuccess) return derr(VD_ERR_NOMEM, "solver scratch of %zu bytes: %s", total * 8, cudaGetErrorString(e));
    double* p = buf;
    for (auto& L : lv) {
        L.phi = p;
        p += L.cells();
        L.rhs = p;
        p += L.cells();
        L.res = p;
        p += L.cells();
        for (int d = 0; d < 3; d++) {
            L.b[d] = d < dim ? p : nullptr;
            p += faces(L, d);
        }
    }
    double* Dg = p;
    p += gcells;
    double* bv_lo[3] = {nullptr, nullptr, nullptr};
    double* bv_hi[3] = {nullptr, nullptr, nullptr};
    for (int d = 0; d < dim; d++) {
        if (bc.per[d]) {  // no domain faces
            p += 2 * plane[d];
            continue;
        }
        bv_lo[d] = p;
        p += plane[d];
        bv_hi[d] = p;
        p += plane[d];
        bc.val_lo[d] = bv_lo[d];
        bc.val_hi[d] = bv_hi[d];
    }
    double* blkmax = p;
    p += nblk0;
    unsigned long long* d_max = reinterpret_cast<unsigned long long*>(p);
    DBc bc0 = bc;  // homogeneous faces for the correction levels
    for (int d = 0; d < 3; d++) {
        bc0.val_lo[d] = bc0.val_hi[d] = nullptr;
        bc0.rf[0][d] = bc0.rf[1][d] = 0.0;
    }

    DifArgs a;
    memset(&a, 0, sizeof(a));
    a.st = A4(state);
    a.old = A4(state_old);
    a.dsdt = A4(dsdt);
    a.pn = A4(phi_new);
    for (int d = 0; d < 3; d++) {
        a.lo[d] = bx->lo[d];
        a.hi[d] = bx->hi[d];
    }
    a.ns = ns;
    a.dim = dim;
    a.spec = spec;
    a.e_id = m.e_id;
    a.dsdt_comp = dp->dsdt_comp;
    a.bound = prm->bound_specden;
    a.is_energy = spec == ns;
    a.Tg = prm->Tg;
    a.dt = prm->dt;
    a.min_spec = prm->min_species_density;
    a.min_elec = prm->min_electron_density;
    a.min_te = prm->min_electron_temp;
    a.cbar_neutral = mw > 0.0 ? sqrt(8.0 * K_B * prm->Tg / PI / (mw * M_AMU)) : 0.0;
    for (int s = 0; s < ns; s++) a.charge[s] = (int8_t)m.charge[s];

    const DifTable ops = dim == 1 ? dif_table<1>() : (dim == 2 ? dif_table<2>() : dif_table<3>());
    auto fail_launch = [&](const char* what) -> int {
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) {
            cudaFreeAsync(buf, st);
            return derr(VD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(le));
        }
        return VD_OK;
    };
    {
        // species_bc face values are needed only when the caller gives no coefficients
        double* const none[3] = {nullptr, nullptr, nullptr};
        ops.setup(a, lv[0], Dg, dp->user_robin ? none : bv_lo, dp->user_robin ? none : bv_hi, st);
    }
    for (size_t l = 1; l < lv.size(); l++) ops.coarsen_b(lv[l - 1], lv[l], st);
    if ((rc = fail_launch("solver set-up"))) return rc;

    auto vcycle = [&]() {
        const int nl = (int)lv.size();
        for (int l = 0; l < nl; l++) {
            const DBc& b = l == 0 ? bc : bc0;
            if (l == nl - 1 && lv[l].cells() <= kDifBottomCells) {
                ops.bottom(lv[l], b, 64, st);
            } else {
                const int sweeps = (l == nl - 1) ? 64 : 2;
                for (int s = 0; s < sweeps; s++) {
                    ops.rbgs(lv[l], b, 0, st);
                    ops.rbgs(lv[l], b, 1, st);
                }
            }
            if (l < nl - 1) {
                ops.residual(lv[l], b, nullptr, st);
                ops.restrict_(lv[l], lv[l + 1], st);
            }
        }
        for (int l = nl - 2; l >= 0; l--) {
            const DBc& b = l == 0 ? bc : bc0;
            ops.prolong(lv[l], lv[l + 1], bc0, st);
            for (int s = 0; s < 2; s++) {
                ops.rbgs(lv[l], b, 0, st);
                ops.rbgs(lv[l], b, 1, st);
            }
        }
    };
    auto maxabs = [&](bool resid, double* out) -> int {
        cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), st);
        if (resid) {
            ops.residual(lv[0], bc, blkmax, st);
            ProfScope ps("k_dif_maxabs", st);
            const unsigned g = (unsigned)std::min<int64_t>((nblk0 + 255) / 256, 148 * 32);
            k_dif_maxabs<<<g < 1 ? 1 : g, 256, 0, st>>>(blkmax, nblk0, d_max);
        } else {
            ProfScope ps("k_dif_maxabs", st);
            const int64_t nc = lv[0].cells();
            unsigned g = (unsigned)std::min<int64_t>((nc + 255) / 256, 148 * 32);
            k_dif_maxabs<<<g < 1 ? 1 : g, 256, 0, st>>>(lv[0].rhs, nc, d_max);
        }
        unsigned long long h = 0;
        cudaError_t ce = cudaMemcpyAsync(&h, d_max, sizeof(h), cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) return derr(VD_ERR_CUDA, "residual norm: %s", cudaGetErrorString(ce));
        memcpy(out, &h, sizeof(*out));
        return VD_OK;
    };
    int done = 0;
    double rel = -1.0;
    if (dp->tol_rel > 0.0) {
        double scale = 0.0, r = 0.0;
        if ((rc = maxabs(false, &scale))) {
            cudaFreeAsync(buf, st);
            return rc;
        }
        if (scale == 0.0) scale = 1.0;
        for (done = 0; done < dp->max_vcycles;) {
            vcycle();
            done++;
            if ((rc = maxabs(true, &r))) {
                cudaFreeAsync(buf, st);
                return rc;
            }
            rel = r / scale;
            if (rel <= dp->tol_rel) break;
        }
        if (!(rel < INFINITY)) {
            cudaFreeAsync(buf, st);
            return derr(VD_ERR_CUDA, "the species solve produced a non-finite residual");
        }
    } else {
        for (done = 0; done < dp->max_vcycles; done++) vcycle();
    }
    {
        ProfScope ps("k_dif_finish", st);
        k_dif_finish<<<dgrid(lv[0]), 128, 0, st>>>(a, lv[0]);
        if (want_grad) {
            const DLevel& L0 = lv[0];
            k_dif_grad<0><<<dgrid(L0, 1), 128, 0, st>>>(L0, bc, A4(gradne_fc[0]), bx->lo[0], bx->lo[1], bx->lo[2]);
            if (dim > 1)
                k_dif_grad<1><<<dim3((L0.n[0] + 127) / 128, L0.n[1] + 1, L0.n[2]), 128, 0, st>>>(
                    L0, bc, A4(gradne_fc[1]), bx->lo[0], bx->lo[1], bx->lo[2]);
            if (dim > 2)
                k_dif_grad<2><<<dim3((L0.n[0] + 127) / 128, L0.n[1], L0.n[2] + 1), 128, 0, st>>>(
                    L0, bc, A4(gradne_fc[2]), bx->lo[0], bx->lo[1], bx->lo[2]);
        }
    }
    if ((rc = fail_launch("solver finish"))) return rc;
    e = cudaFreeAsync(buf, st);
    if (e != cudaSuccess) return derr(VD_ERR_CUDA, "scratch release: %s", cudaGetErrorString(e));
    if (vcycles_done) *vcycles_done = done;
    if (rel_residual) *rel_residual = rel;
    return VD_OK;
}
