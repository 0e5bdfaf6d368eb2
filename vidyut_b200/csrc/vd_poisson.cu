// vd_poisson.cu -- the potential / electric-field step before the explicit update
// (vd_poisson_solve in vidyut_b200.h).
//
// The reference solves del^2 phi = -(e/eps0) sum_k z_k n_k with AMReX's MLMG
// (Source/PotentialSolve.cpp:188-378), takes the face field -grad phi from the
// solver and the cell field by centred (one-sided at domain faces) differences of
// phi, and the reduced field |E|/N (Source/PotentialSolve.cpp:391-430,
// Source/HelperFuncs.H:14-70).  AMReX is not part of this library, so this file
// carries a self-contained geometric multigrid for the same discrete problem on
// one box that is the whole domain: cell-centred 2D+1-point Laplacian, Dirichlet
// faces (the applied potential at the face) or zero-gradient faces, V(2,2) cycles
// of red-black Gauss-Seidel, full-weighting restriction, linear prolongation, a
// 64-sweep bottom solve on the coarsest grid.  The potential, its defect and the
// fields are FP64; the cycles solve for the correction in FP32 (half the bytes
// per sweep), and the defect of the corrected FP64 potential decides convergence,
// so the solution meets the same FP64 tolerance.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>
#include "vd_host.h"

namespace vd {
namespace {

constexpr double EPS0 = 8.854187817e-12;  // Source/UnivConstants.H:12

// One grid of the hierarchy.  The potential itself is FP64 (Level: phi, rhs); the
// V-cycles solve for its correction in FP32 (CLevel: phi the correction, rhs the
// defect, res the residual), with 1/dx^2 scaled so the correction equation has
// O(1) coefficients (defect correction: the defect of every cycle is formed from
// the FP64 potential, so the FP32 cycles only set how fast it converges).
template <class T>
struct LevelT {
    int n[3];          // cells per direction (1 beyond dim)
    double idx2[3];    // 1/dx^2 (0 beyond dim), times the scale on correction levels
    T* phi;
    T* rhs;
    T* res;
    __host__ __device__ int64_t cells() const { return (int64_t)n[0] * n[1] * n[2]; }
};
using Level = LevelT<double>;
using CLevel = LevelT<float>;

struct BcInfo {
    int dir_lo[3], dir_hi[3];    // 1: Dirichlet face
    double val_lo[3], val_hi[3]; // its value (0 on the correction levels)
};

template <class T>
__device__ __forceinline__ int64_t lin(const LevelT<T>& L, int i, int j, int k)
{
    return (int64_t)i + (int64_t)L.n[0] * (j + (int64_t)L.n[1] * k);
}

// Off-diagonal sum and diagonal of the Laplacian at cell (i,j,k), with the domain
// faces folded in.  Each face of the cell contributes (phi_out - phi_c)/dx^2: an
// inside neighbour adds phi_nb and -phi_c; a Dirichlet face holds phi = V at the
// face, so phi_out = 2V - phi_c (constant 2V/dx^2, diagonal -2/dx^2); a
// zero-gradient face has phi_out = phi_c and adds nothing.
template <int DIM, class T>
struct Nbr {
    T lo[DIM], hi[DIM];
};
// every neighbour load first, unconditionally (the cell itself stands in beyond a
// domain face, where its value is not used): the loads of a thread are then all
// in flight together, which these latency-bound sweeps need
template <int DIM, class T>
__device__ __forceinline__ Nbr<DIM, T> stencil_load(const LevelT<T>& L, int i, int j, int k, const T* phi)
{
    // offsets from the cell in 32 bits (a plane of the grid holds < 2^31 cells):
    // one 64-bit address, then one wide multiply-add per load
    const int c[3] = {i, j, k};
    const int str[3] = {1, L.n[0], L.n[0] * L.n[1]};
    const T* pc = phi + lin(L, i, j, k);
    Nbr<DIM, T> v;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        v.lo[d] = pc[c[d] > 0 ? -str[d] : 0];
        v.hi[d] = pc[c[d] < L.n[d] - 1 ? str[d] : 0];
    }
    return v;
}
template <int DIM, class T>
__device__ __forceinline__ void stencil_apply(const LevelT<T>& L, const BcInfo& bc, int i, int j, int k,
                                              const Nbr<DIM, T>& v, T& off, T& diag)
{
    const int c[3] = {i, j, k};
    off = T(0);
    diag = T(0);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const T w = (T)L.idx2[d];
        if (c[d] > 0) {
            off += w * v.lo[d];
            diag -= w;
        } else if (bc.dir_lo[d]) {
            off += T(2) * w * (T)bc.val_lo[d];
            diag -= T(2) * w;
        }
        if (c[d] < L.n[d] - 1) {
            off += w * v.hi[d];
            diag -= w;
        } else if (bc.dir_hi[d]) {
            off += T(2) * w * (T)bc.val_hi[d];
            diag -= T(2) * w;
        }
    }
}
template <int DIM, class T>
__device__ __forceinline__ void stencil(const LevelT<T>& L, const BcInfo& bc, int i, int j, int k, const T* phi,
                                        T& off, T& diag)
{
    stencil_apply<DIM>(L, bc, i, j, k, stencil_load<DIM>(L, i, j, k, phi), off, diag);
}

// Multigrid kernels: one thread per cell (or per cell of one colour) with i over
// the x threads and j, k from the y and z block indices, so no index division.
// The V-cycle kernels run on the FP32 correction levels.

// one red-black Gauss-Seidel half sweep: cells with (i + j + k) % 2 == color.  A
// thread takes two cells, `half` apart along the slowest active direction (k in
// 3-D, j in 2-D; half = 0 in 1-D: one cell), with all their loads issued first.
// corr (null: none): the last half sweep of a cycle on the finest correction
// level also adds the finished correction to the FP64 potential corr, for its
// two cells and their x neighbours of the other colour (so every cell once).
template <int DIM>
__global__ void __launch_bounds__(128) k_mg_rbgs(CLevel L, BcInfo bc, int color, int half, double* corr)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int ii[2], jj[2], kk[2];
    bool row[2], ok[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        jj[h] = blockIdx.y + (DIM == 2 ? h * half : 0);
        kk[h] = blockIdx.z + (DIM == 3 ? h * half : 0);
        ii[h] = 2 * t + ((jj[h] + kk[h] + color) & 1);
        row[h] = jj[h] < L.n[1] && kk[h] < L.n[2] && (h == 0 || half > 0);
        ok[h] = row[h] && ii[h] < L.n[0];
    }
    Nbr<DIM, float> v[2];
    float r[2];
#pragma unroll
    for (int h = 0; h < 2; h++)
        if (ok[h]) {
            v[h] = stencil_load<DIM>(L, ii[h], jj[h], kk[h], L.phi);
            r[h] = L.rhs[lin(L, ii[h], jj[h], kk[h])];
        }
#pragma unroll
    for (int h = 0; h < 2; h++) {
        if (ok[h]) {
            float off, diag;
            stencil_apply<DIM>(L, bc, ii[h], jj[h], kk[h], v[h], off, diag);
            // L phi = off + diag phi = rhs  ->  phi = (rhs - off) / diag
            const int64_t c = lin(L, ii[h], jj[h], kk[h]);
            // fast division (2 ulp): a smoother needs no correctly rounded quotient,
            // and the sweep is issue bound
            const float e = __fdividef(r[h] - off, diag);
            L.phi[c] = e;
            if (corr) corr[c] += (double)e;
        }
        const int io = ii[h] ^ 1;  // the other cell of the pair (2t, 2t + 1)
        if (corr && row[h] && io < L.n[0]) {
            const int64_t c = lin(L, io, jj[h], kk[h]);
            corr[c] += (double)L.phi[c];
        }
    }
}

template <int DIM>
__global__ void __launch_bounds__(128) k_mg_residual(CLevel L, BcInfo bc)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n[0]) return;
    float off, diag;
    stencil<DIM>(L, bc, i, j, k, L.phi, off, diag);
    const int64_t c = lin(L, i, j, k);
    L.res[c] = L.rhs[c] - (off + diag * L.phi[c]);
}

// The defect of the FP64 potential P, r = rhs - L phi (FP64, inhomogeneous faces),
// becomes the right-hand side of the finest correction level (times the scale of
// its coefficients, rounded to FP32), whose correction starts at zero.
// blkmax (null: not wanted): max |r| of each block, one value per block in block
// order, reduced by k_maxabs afterwards (one atomic per warp on a single address
// would serialise in L2: 1.8 M of them on a 384^3 grid).
template <int DIM>
__global__ void __launch_bounds__(128) k_mg_defect(Level P, BcInfo bc, CLevel E, double scale, int half,
                                                   double* blkmax)
{
    // two cells per thread, `half` apart along the slowest active direction (as in
    // k_mg_rbgs), with all their loads issued first
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int jj[2], kk[2];
    bool ok[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        jj[h] = blockIdx.y + (DIM == 2 ? h * half : 0);
        kk[h] = blockIdx.z + (DIM == 3 ? h * half : 0);
        ok[h] = i < P.n[0] && jj[h] < P.n[1] && kk[h] < P.n[2] && (h == 0 || half > 0);
    }
    Nbr<DIM, double> v[2];
    double rh[2], pc[2];
#pragma unroll
    for (int h = 0; h < 2; h++)
        if (ok[h]) {
            v[h] = stencil_load<DIM>(P, i, jj[h], kk[h], P.phi);
            const int64_t c = lin(P, i, jj[h], kk[h]);
            rh[h] = P.rhs[c];
            pc[h] = P.phi[c];
        }
    double m = 0.0;
#pragma unroll
    for (int h = 0; h < 2; h++)
        if (ok[h]) {
            double off, diag;
            stencil_apply<DIM>(P, bc, i, jj[h], kk[h], v[h], off, diag);
            const int64_t c = lin(P, i, jj[h], kk[h]);
            const double r = rh[h] - (off + diag * pc[h]);
            E.rhs[c] = (float)(r * scale);
            E.phi[c] = 0.0f;
            m = fmax(m, fabs(r));
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

// P phi += the correction of the finest correction level
__global__ void __launch_bounds__(128) k_mg_correct(Level P, CLevel E)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n[0]) return;
    const int64_t c = lin(P, i, j, k);
    P.phi[c] += (double)E.phi[c];
}

// coarse rhs = average of the 2^dim fine residuals (full weighting for cell centres)
template <int DIM>
__global__ void __launch_bounds__(128) k_mg_restrict(CLevel F, CLevel C)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C.n[0]) return;
    float s = 0.0f;
#pragma unroll
    for (int dz = 0; dz < (DIM > 2 ? 2 : 1); dz++)
#pragma unroll
        for (int dy = 0; dy < (DIM > 1 ? 2 : 1); dy++)
#pragma unroll
            for (int dx = 0; dx < 2; dx++)
                s += F.res[lin(F, 2 * i + dx, DIM > 1 ? 2 * j + dy : j, DIM > 2 ? 2 * k + dz : k)];
    const int64_t c = lin(C, i, j, k);
    C.rhs[c] = s * (1.0f / (float)(1 << DIM));
    C.phi[c] = 0.0f;
}

// fine phi += linear interpolation of the coarse correction (weights 3/4, 1/4 per
// direction; at a domain face the outside coarse value is the correction's
// boundary value: -c for a Dirichlet face (zero at the face), c for zero gradient)
template <int DIM>
__global__ void __launch_bounds__(128) k_mg_prolong(CLevel F, CLevel C, BcInfo bc)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.n[0]) return;
    const int f[3] = {i, j, k};
    // per direction the two coarse cells (as offsets) and their weights; beyond a
    // domain face the second is the parent itself, weighted -1/4 or 1/4; beyond dim
    // the coarse index is the fine one
    const int64_t str[3] = {1, C.n[0], (int64_t)C.n[0] * C.n[1]};
    int64_t off[3][2];
    float w[3][2];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        if (d >= DIM) {
            off[d][0] = off[d][1] = (int64_t)f[d] * str[d];
            w[d][0] = 1.0f;
            w[d][1] = 0.0f;
            continue;
        }
        const int ci = f[d] >> 1, q = ci + ((f[d] & 1) ? 1 : -1);
        off[d][0] = (int64_t)ci * str[d];
        w[d][0] = 0.75f;
        if (q < 0) {
            off[d][1] = off[d][0];
            w[d][1] = bc.dir_lo[d] ? -0.25f : 0.25f;
        } else if (q >= C.n[d]) {
            off[d][1] = off[d][0];
            w[d][1] = bc.dir_hi[d] ? -0.25f : 0.25f;
        } else {
            off[d][1] = (int64_t)q * str[d];
            w[d][1] = 0.25f;
        }
    }
    float acc = 0.0f;
#pragma unroll
    for (int mz = 0; mz < (DIM > 2 ? 2 : 1); mz++)
#pragma unroll
        for (int my = 0; my < (DIM > 1 ? 2 : 1); my++) {
            const int64_t row = off[1][my] + off[2][mz];
            const float v = w[0][0] * C.phi[row + off[0][0]] + w[0][1] * C.phi[row + off[0][1]];
            acc += (w[1][my] * w[2][mz]) * v;
        }
    F.phi[lin(F, i, j, k)] += acc;
}

// bottom solve of a small coarsest grid: one CTA runs every red-black sweep, with
// a barrier between half sweeps (cells <= kBottomCells)
constexpr int kBottomCells = 4096;

template <int DIM>
__global__ void __launch_bounds__(256) k_mg_bottom(CLevel L, BcInfo bc, int sweeps)
{
    const int n0 = L.n[0], n1 = L.n[1];
    const int nc = (int)L.cells();
    for (int s = 0; s < sweeps; s++)
        for (int color = 0; color < 2; color++) {
            for (int c = threadIdx.x; c < nc; c += blockDim.x) {
                const int k = c / (n0 * n1), r = c - k * n0 * n1, j = r / n0, i = r - j * n0;
                if (((i + j + k) & 1) != color) continue;
                float off, diag;
                stencil<DIM>(L, bc, i, j, k, L.phi, off, diag);
                L.phi[c] = __fdividef(L.rhs[c] - off, diag);
            }
            __syncthreads();
        }
}

template <class T>
dim3 grid_cells(const LevelT<T>& L, int per_thread = 1)
{
    const int nx = (L.n[0] + per_thread - 1) / per_thread;
    return dim3((unsigned)((nx + 127) / 128), (unsigned)L.n[1], (unsigned)L.n[2]);
}

// grid of the two-cells-per-thread kernels: the slowest active direction halved
// (half, returned, is the distance between a thread's two cells; 0 in 1-D)
template <class T>
dim3 grid_pairs(const LevelT<T>& L, int dim, int per_thread, int* half)
{
    dim3 g = grid_cells(L, per_thread);
    const int ns = dim == 3 ? L.n[2] : (dim == 2 ? L.n[1] : 1);
    *half = dim == 1 ? 0 : (ns + 1) / 2;
    if (dim == 3) g.z = (unsigned)*half;
    else if (dim == 2) g.y = (unsigned)*half;
    return g;
}

template <int DIM>
struct Mg {
    static void rbgs(const CLevel& L, const BcInfo& b, int color, double* corr, cudaStream_t st)
    {
        ProfScope ps("k_mg_rbgs", st);
        int half = 0;
        const dim3 g = grid_pairs(L, DIM, 2, &half);
        k_mg_rbgs<DIM><<<g, 128, 0, st>>>(L, b, color, half, corr);
    }
    static void residual(const CLevel& L, const BcInfo& b, cudaStream_t st)
    {
        ProfScope ps("k_mg_residual", st);
        k_mg_residual<DIM><<<grid_cells(L), 128, 0, st>>>(L, b);
    }
    static void restrict_(const CLevel& F, const CLevel& C, cudaStream_t st)
    {
        ProfScope ps("k_mg_restrict", st);
        k_mg_restrict<DIM><<<grid_cells(C), 128, 0, st>>>(F, C);
    }
    static void bottom(const CLevel& L, const BcInfo& b, int sweeps, cudaStream_t st)
    {
        ProfScope ps("k_mg_bottom", st);
        k_mg_bottom<DIM><<<1, 256, 0, st>>>(L, b, sweeps);
    }
    static void prolong(const CLevel& F, const CLevel& C, const BcInfo& b, cudaStream_t st)
    {
        ProfScope ps("k_mg_prolong", st);
        k_mg_prolong<DIM><<<grid_cells(F), 128, 0, st>>>(F, C, b);
    }
    static void defect(const Level& P, const BcInfo& b, const CLevel& E, double scale, double* blkmax,
                       cudaStream_t st)
    {
        ProfScope ps("k_mg_defect", st);
        int half = 0;
        const dim3 g = grid_pairs(P, DIM, 1, &half);
        k_mg_defect<DIM><<<g, 128, 0, st>>>(P, b, E, scale, half, blkmax);
    }
};

struct MgOps {
    void (*rbgs)(const CLevel&, const BcInfo&, int, double*, cudaStream_t);
    void (*residual)(const CLevel&, const BcInfo&, cudaStream_t);
    void (*restrict_)(const CLevel&, const CLevel&, cudaStream_t);
    void (*prolong)(const CLevel&, const CLevel&, const BcInfo&, cudaStream_t);
    void (*bottom)(const CLevel&, const BcInfo&, int, cudaStream_t);
    void (*defect)(const Level&, const BcInfo&, const CLevel&, double, double*, cudaStream_t);
};

MgOps mg_ops(int dim)
{
    if (dim == 1) return {Mg<1>::rbgs, Mg<1>::residual, Mg<1>::restrict_, Mg<1>::prolong, Mg<1>::bottom, Mg<1>::defect};
    if (dim == 2) return {Mg<2>::rbgs, Mg<2>::residual, Mg<2>::restrict_, Mg<2>::prolong, Mg<2>::bottom, Mg<2>::defect};
    return {Mg<3>::rbgs, Mg<3>::residual, Mg<3>::restrict_, Mg<3>::prolong, Mg<3>::bottom, Mg<3>::defect};
}

__global__ void k_maxabs(const double* x, int64_t n, unsigned long long* out)
{
    double m = 0.0;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(x[c]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

struct PoisArgs {
    A4 st;
    A4 urhs;  // user source added to the right-hand side (p null: none)
    int lo[3], hi[3];
    int ns, dim;
    int8_t charge[VD_MAX_SPECIES];
};

// rhs = -(e/eps0) sum_k z_k n_k (Source/PotentialSolve.cpp:199-215); initial guess
// phi = the state's potential
__global__ void k_pois_rhs(PoisArgs a, Level L)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.n[0]) {
        const int64_t c = lin(L, i, j, k);
        const int64_t o = a.st.off(a.lo[0] + i, a.lo[1] + j, a.lo[2] + k);
        double r = 0.0;
        for (int s = 0; s < a.ns; s++)
            if (a.charge[s] != 0) r += (double)a.charge[s] * a.st.p[o + (int64_t)s * a.st.ns];
        L.rhs[c] = r * (-ECHARGE / EPS0);
        if (a.urhs.p) L.rhs[c] += a.urhs(a.lo[0] + i, a.lo[1] + j, a.lo[2] + k);
        L.phi[c] = a.st.p[o + (int64_t)VD_POT(a.ns) * a.st.ns];
    }
}

// potential, cell field (Source/HelperFuncs.H:14-70) and reduced field
// (Source/PotentialSolve.cpp:419-424) of the valid cells
struct D3 {
    double v[3];
};

__global__ void __launch_bounds__(128) k_pois_cell_fields(PoisArgs a, Level L, D3 dxs)
{
    const int ns = a.ns;
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n[0]) return;
    const int64_t c = lin(L, i, j, k);
    const int cc[3] = {i, j, k};
    const int64_t str[3] = {1, (int64_t)L.n[0], (int64_t)L.n[0] * L.n[1]};
    const double* ph = L.phi;
    double E[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        if (d >= a.dim) break;
        const int n = L.n[d];
        const int64_t s1 = str[d];
        const double dx = dxs.v[d];
        if (cc[d] > 0 && cc[d] < n - 1) {
            E[d] = -0.5 * (ph[c + s1] - ph[c - s1]) / dx;
        } else if (cc[d] == 0 && n > 1) {
            if (n - 1 > 2) E[d] = -0.5 * (-ph[c + 2 * s1] + 4.0 * ph[c + s1] - 3.0 * ph[c]) / dx;
            else E[d] = -(ph[c + s1] - ph[c]) / dx;
        } else if (cc[d] == n - 1 && n > 1) {
            if (n - 1 > 2) E[d] = -0.5 * (ph[c - 2 * s1] - 4.0 * ph[c - s1] + 3.0 * ph[c]) / dx;
            else E[d] = -(ph[c] - ph[c - s1]) / dx;
        }
    }
    const int64_t o = a.st.off(a.lo[0] + i, a.lo[1] + j, a.lo[2] + k);
    const int64_t cs = a.st.ns;
    double nd = 0.0, es = 0.0;
    for (int s = 0; s < ns; s++) nd += a.st.p[o + (int64_t)s * cs];
#pragma unroll
    for (int d = 0; d < 3; d++)
        if (d < a.dim) es += E[d] * E[d];
    a.st.p[o + (int64_t)VD_POT(ns) * cs] = ph[c];
    a.st.p[o + (int64_t)VD_EFX(ns) * cs] = E[0];
    a.st.p[o + (int64_t)VD_EFY(ns) * cs] = E[1];
    a.st.p[o + (int64_t)VD_EFZ(ns) * cs] = E[2];
    // pow(Esum, 0.5) in the reference: the correctly rounded square root
    a.st.p[o + (int64_t)VD_REF(ns) * cs] = (sqrt(es) / nd) / 1.0e-21;
}

// face field -dphi/dx_D on the face box of direction D; at a Dirichlet domain face
// the gradient to the face value over half a cell, at a zero-gradient face 0
// (what MLMG's getGradSolution returns, negated)
template <int D>
__global__ void __launch_bounds__(128) k_pois_face_field(Level L, BcInfo bc, A4 ef, double dx)
{
    const int j = blockIdx.y, k = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nf0 = L.n[0] + (D == 0);
    if (i >= nf0) return;
    const int f[3] = {i, j, k};
    const int64_t s1 = D == 0 ? 1 : (D == 1 ? (int64_t)L.n[0] : (int64_t)L.n[0] * L.n[1]);
    // linear index of the cell above the face; the cell below is c - s1 (for
    // f[D] == n[D] the index runs one past the box and only c - s1 is read)
    const int64_t c = lin(L, i, j, k);
    double e;
    if (f[D] == 0) e = bc.dir_lo[D] ? -(L.phi[c] - bc.val_lo[D]) / (0.5 * dx) : 0.0;
    else if (f[D] == L.n[D]) e = bc.dir_hi[D] ? -(bc.val_hi[D] - L.phi[c - s1]) / (0.5 * dx) : 0.0;
    else e = -(L.phi[c] - L.phi[c - s1]) / dx;
    ef.p[ef.off(ef.bx + i, ef.by + j, ef.bz + k)] = e;
}

unsigned grid_of(int64_t n)
{
    int64_t g = (n + 255) / 256;
    if (g > 148LL * 32) g = 148LL * 32;
    return (unsigned)(g < 1 ? 1 : g);
}

int err(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int err(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return vd_host::set_error(code, buf);
}

}  // namespace
}  // namespace vd

using namespace vd;

extern "C" int vd_poisson_solve(const vd_box* bx, vd_array4 state, const vd_array4 efield_ec[3], const vd_params* prm,
                                const vd_poisson_params* pp, int32_t* vcycles_done, double* rel_residual,
                                void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int rc = vd_host::ensure_mech(st);  // sets the device up (scratch pool)
    if (rc) return rc;
    vd_host::MechInfo m;
    if ((rc = vd_host::mech_info(&m))) return rc;
    if (!bx || !prm || !pp) return err(VD_ERR_ARG, "null argument");
    if ((rc = vd_host::check_update_params(bx, prm, m))) return rc;
    const int dim = bx->dim, ns = m.ns;
    for (int d = 0; d < dim; d++)
        if (prm->domlo[d] != bx->lo[d] || prm->domhi[d] != bx->hi[d])
            return err(VD_ERR_ARG, "the potential solve needs the box to be the whole domain (direction %d)", d);
    if (pp->max_vcycles < 1 || pp->max_vcycles > 1000) return err(VD_ERR_ARG, "max_vcycles %d", pp->max_vcycles);
    // ghost layers of the state (refilled for the potential and the fields)
    int n[3], glo[3], ghi[3];
    for (int d = 0; d < 3; d++) {
        n[d] = bx->hi[d] - bx->lo[d] + 1;
        glo[d] = bx->lo[d];
        ghi[d] = bx->hi[d];
    }
    int G = 0;  // ghost layers available in every active direction
    {
        G = 1 << 20;
        for (int d = 0; d < dim; d++) {
            G = std::min(G, bx->lo[d] - state.begin[d]);
            G = std::min(G, state.end[d] - 1 - bx->hi[d]);
        }
        if (G < 0) G = 0;
        if (G > 8) G = 8;
    }
    for (int d = 0; d < dim; d++) {
        glo[d] -= G;
        ghi[d] += G;
    }
    if (!state.p || state.ncomp < VD_NVAR(ns) || state.begin[0] > glo[0] || state.end[0] <= ghi[0])
        return err(VD_ERR_ARG, "state does not cover the box with NVAR components");
    if (!prm->cs_technique)
        for (int d = 0; d < dim; d++) {
            if (!efield_ec || !efield_ec[d].p) return err(VD_ERR_ARG, "efield_ec[%d] is null", d);
            int fhi[3] = {bx->hi[0], bx->hi[1], bx->hi[2]};
            fhi[d] += 1;
            for (int e = 0; e < 3; e++)
                if (efield_ec[d].begin[e] > bx->lo[e] || efield_ec[d].end[e] <= fhi[e])
                    return err(VD_ERR_ARG, "efield_ec[%d] does not cover the face box", d);
        }
    if (pp->user_rhs.p) {
        const vd_array4& u = pp->user_rhs;
        if (u.ncomp < 1 || ((uintptr_t)u.p) % 8) return err(VD_ERR_ARG, "user_rhs: bad component count or alignment");
        for (int d = 0; d < 3; d++)
            if (u.begin[d] > bx->lo[d] || u.end[d] <= bx->hi[d])
                return err(VD_ERR_ARG, "user_rhs does not cover the box in direction %d", d);
    }
    BcInfo bc;
    memset(&bc, 0, sizeof(bc));
    for (int d = 0; d < dim; d++) {
        bc.dir_lo[d] = pp->bc_lo[d] == VD_BC_DIRC;
        bc.dir_hi[d] = pp->bc_hi[d] == VD_BC_DIRC;
        bc.val_lo[d] = pp->value_lo[d];
        bc.val_hi[d] = pp->value_hi[d];
    }
    bool any_dir = false;
    for (int d = 0; d < dim; d++) any_dir = any_dir || bc.dir_lo[d] || bc.dir_hi[d];
    if (!any_dir) return err(VD_ERR_ARG, "the potential needs at least one Dirichlet face");

    // the potential (FP64) and the hierarchy of its correction (FP32), whose
    // coefficients are 1/dx^2 times scale = min dx^2, so they are at most 1: the
    // correction of a potential in volts then stays far inside FP32's range.
    // Hierarchy: halve every active direction while all stay even and above 2.
    Level P;
    double scale = 0.0;
    for (int d = 0; d < 3; d++) {
        P.n[d] = n[d];
        P.idx2[d] = d < dim ? 1.0 / (prm->dx[d] * prm->dx[d]) : 0.0;
        scale = std::max(scale, P.idx2[d]);
    }
    scale = 1.0 / scale;
    std::vector<CLevel> lv;
    {
        CLevel L0;
        for (int d = 0; d < 3; d++) {
            L0.n[d] = n[d];
            L0.idx2[d] = P.idx2[d] * scale;
        }
        lv.push_back(L0);
        for (;;) {
            const CLevel& f = lv.back();
            bool ok = true;
            for (int d = 0; d < dim; d++) ok = ok && (f.n[d] % 2 == 0) && f.n[d] > 2;
            if (!ok || lv.size() >= 24) break;
            CLevel c;
            for (int d = 0; d < 3; d++) {
                c.n[d] = d < dim ? f.n[d] / 2 : f.n[d];
                c.idx2[d] = f.idx2[d] * 0.25;
            }
            lv.push_back(c);
        }
    }
    // scratch: P's phi and rhs, the block maxima of the defect, the max (FP64);
    // phi, rhs and res of every correction level (FP32)
    int half0 = 0;
    const dim3 g0 = grid_pairs(P, dim, 1, &half0);
    const int64_t nblk0 = (int64_t)g0.x * g0.y * g0.z;  // defect blocks
    size_t nf = 0;
    for (auto& L : lv) nf += 3 * (size_t)L.cells();
    const size_t nd = 2 * (size_t)P.cells() + (size_t)nblk0 + 1;
    double* buf = nullptr;
    const size_t bytes = nd * sizeof(double) + nf * sizeof(float) + 64;
    cudaError_t e = vd_host::scratch_alloc(reinterpret_cast<void**>(&buf), bytes, st);
    if (e != cudaSuccess) return err(VD_ERR_NOMEM, "multigrid scratch of %zu bytes: %s", bytes, cudaGetErrorString(e));
    P.phi = buf;
    P.rhs = buf + P.cells();
    P.res = nullptr;
    double* blkmax = buf + 2 * P.cells();
    unsigned long long* d_max = reinterpret_cast<unsigned long long*>(blkmax + nblk0);
    {
        float* p = reinterpret_cast<float*>(buf + nd);
        for (auto& L : lv) {
            L.phi = p;
            p += L.cells();
            L.rhs = p;
            p += L.cells();
            L.res = p;
            p += L.cells();
        }
    }
    BcInfo bc0;  // homogeneous version for the correction levels
    bc0 = bc;
    for (int d = 0; d < 3; d++) bc0.val_lo[d] = bc0.val_hi[d] = 0.0;

    PoisArgs pa;
    memset(&pa, 0, sizeof(pa));
    pa.st = A4(state);
    if (pp->user_rhs.p) pa.urhs = A4(pp->user_rhs);
    for (int d = 0; d < 3; d++) {
        pa.lo[d] = bx->lo[d];
        pa.hi[d] = bx->hi[d];
    }
    pa.ns = ns;
    pa.dim = dim;
    for (int s = 0; s < ns; s++) pa.charge[s] = (int8_t)m.charge[s];

    auto launch_check = [&](const char* what) -> int {
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) {
            cudaFreeAsync(buf, st);
            return err(VD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(le));
        }
        return VD_OK;
    };

    {
        ProfScope ps("k_pois_rhs", st);
        k_pois_rhs<<<grid_cells(P), 128, 0, st>>>(pa, P);
    }
    if ((rc = launch_check("k_pois_rhs"))) return rc;
    double rhs_scale = 0.0;
    const bool check = pp->tol_rel > 0.0;
    const MgOps ops = mg_ops(dim);
    // one V(2,2) cycle of the correction equation, from a zero correction, then the
    // correction added to the potential (inside the last half sweep)
    auto vcycle = [&]() {
        const int nl = (int)lv.size();
        for (int l = 0; l < nl; l++) {
            if (l == nl - 1 && lv[l].cells() <= kBottomCells) {
                ops.bottom(lv[l], bc0, 64, st);  // one CTA, all sweeps in one launch
            } else {
                const int sweeps = (l == nl - 1) ? 64 : 2;
                for (int s = 0; s < sweeps; s++) {
                    ops.rbgs(lv[l], bc0, 0, nullptr, st);
                    ops.rbgs(lv[l], bc0, 1, nullptr, st);
                }
            }
            if (l < nl - 1) {
                ops.residual(lv[l], bc0, st);
                ops.restrict_(lv[l], lv[l + 1], st);
            }
        }
        for (int l = nl - 2; l >= 0; l--) {
            ops.prolong(lv[l], lv[l + 1], bc0, st);
            for (int s = 0; s < 2; s++) {
                ops.rbgs(lv[l], bc0, 0, nullptr, st);
                ops.rbgs(lv[l], bc0, 1, (l == 0 && s == 1) ? P.phi : nullptr, st);
            }
        }
        if (nl == 1) {  // no coarser level: the cycle was the bottom solve
            ProfScope ps("k_mg_correct", st);
            k_mg_correct<<<grid_cells(P), 128, 0, st>>>(P, lv[0]);
        }
    };
    // the max of the n doubles (non-negative doubles order like their bit patterns)
    auto read_max = [&](const double* x, int64_t nx, double* out) -> int {
        cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), st);
        {
            ProfScope ps("k_maxabs", st);
            k_maxabs<<<grid_of(nx), 256, 0, st>>>(x, nx, d_max);
        }
        unsigned long long h = 0;
        cudaError_t ce = cudaMemcpyAsync(&h, d_max, sizeof(h), cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) return err(VD_ERR_CUDA, "residual norm: %s", cudaGetErrorString(ce));
        memcpy(out, &h, sizeof(*out));
        return VD_OK;
    };
    int done = 0;
    double rel = -1.0;
    if (check) {
        // scale of the relative residual: max |rhs|
        if ((rc = read_max(P.rhs, P.cells(), &rhs_scale))) {
            cudaFreeAsync(buf, st);
            return rc;
        }
        if (rhs_scale == 0.0) rhs_scale = 1.0;
    }
    ops.defect(P, bc, lv[0], scale, nullptr, st);
    for (done = 0; done < pp->max_vcycles;) {
        vcycle();
        done++;
        if (check) {
            // the defect of the corrected potential: the convergence test and the
            // right-hand side of the next cycle
            ops.defect(P, bc, lv[0], scale, blkmax, st);
            double r = 0.0;
            if ((rc = read_max(blkmax, nblk0, &r))) {
                cudaFreeAsync(buf, st);
                return rc;
            }
            rel = r / rhs_scale;
            if (rel <= pp->tol_rel) break;
        } else if (done < pp->max_vcycles) {
            ops.defect(P, bc, lv[0], scale, nullptr, st);
        }
    }
    if ((rc = launch_check("multigrid"))) return rc;
    D3 dxs{{prm->dx[0], prm->dx[1], prm->dx[2]}};
    {
        ProfScope ps("k_pois_cell_fields", st);
        k_pois_cell_fields<<<grid_cells(P), 128, 0, st>>>(pa, P, dxs);
    }
    if (!prm->cs_technique)
        for (int d = 0; d < dim; d++) {
            const Level& L = P;
            int nf[3] = {L.n[0], L.n[1], L.n[2]};
            nf[d] += 1;
            ProfScope ps("k_pois_face_field", st);
            const dim3 g((unsigned)((nf[0] + 127) / 128), (unsigned)nf[1], (unsigned)nf[2]);
            const A4 efd(efield_ec[d]);
            if (d == 0) k_pois_face_field<0><<<g, 128, 0, st>>>(P, bc, efd, prm->dx[0]);
            else if (d == 1) k_pois_face_field<1><<<g, 128, 0, st>>>(P, bc, efd, prm->dx[1]);
            else k_pois_face_field<2><<<g, 128, 0, st>>>(P, bc, efd, prm->dx[2]);
        }
    if ((rc = launch_check("potential fields"))) return rc;
    // ghosts of the potential, the cell field and the reduced field
    if (G > 0) {
        const int32_t comps[5] = {VD_POT(ns), VD_EFX(ns), VD_EFY(ns), VD_EFZ(ns), VD_REF(ns)};
        const int32_t per[3] = {0, 0, 0};
        rc = vd_fill_ghosts(bx, state, G, comps, 5, per, stream);
        if (rc) {
            cudaFreeAsync(buf, st);
            return rc;
        }
    }
    e = cudaFreeAsync(buf, st);
    if (e != cudaSuccess) return err(VD_ERR_CUDA, "scratch release: %s", cudaGetErrorString(e));
    if (vcycles_done) *vcycles_done = done;
    if (rel_residual) *rel_residual = rel;
    return VD_OK;
}
