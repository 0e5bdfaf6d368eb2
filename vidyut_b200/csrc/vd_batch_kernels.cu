// vd_batch_kernels.cu -- launch variants of the batched persistent transport kernel,
// and the batched Joule pre-pass that runs before it.
//
// A variant is a tile shape and a residency target (CTAs per SM the compiler must
// fit, which caps registers at 64K / (threads x CTAs)); the species group size
// follows from the shared memory that residency leaves (group_fit).  The batch
// autotuner (vd_batch_tune) times every variant of a dimension on the resident
// cases and keeps the fastest.  This translation unit has its own copy of the
// mechanism table in constant memory, uploaded with the other one.
#include <tuple>
#include "vd_device.cuh"
#include "vd_kernels.cuh"
#include "vd_transport.cuh"

namespace vd {

cudaError_t upload_mech_batch(const VdMechDev* h, cudaStream_t st)
{
    return cudaMemcpyToSymbolAsync(c_mech, h, sizeof(VdMechDev), 0, cudaMemcpyHostToDevice, st);
}

template <class TS_, int MINB_, int GMAX_ = 8>
struct BatchVariant {
    using TS = TS_;
    static constexpr int MINB = MINB_;
    static constexpr int GMAX = GMAX_;  // species group cap (group_fit)
};

using T1a = TileShape<256, 1, 1, 256>;
using T1b = TileShape<128, 1, 1, 128>;
using T2a = TileShape<32, 8, 1, 256>;
using T2b = TileShape<16, 16, 1, 256>;
using T3a = TileShape<8, 8, 8, 512>;
using T3b = TileShape<16, 8, 4, 512>;

template <int DIM> struct BatchVariants;
template <> struct BatchVariants<1> {
    using L = std::tuple<BatchVariant<T1a, 2>, BatchVariant<T1b, 2>, BatchVariant<T1a, 3>, BatchVariant<T1a, 4>,
                         BatchVariant<T1b, 4>>;
};
template <> struct BatchVariants<2> {
    using L = std::tuple<BatchVariant<T2a, 2>, BatchVariant<T2b, 2>, BatchVariant<T2a, 3>, BatchVariant<T2b, 3>,
                         BatchVariant<T2a, 4>, BatchVariant<T2b, 4>, BatchVariant<T2a, 4, 4>, BatchVariant<T2b, 4, 4>>;
};
template <> struct BatchVariants<3> {
    using L = std::tuple<BatchVariant<T3a, 2>, BatchVariant<T3b, 2>>;
};
template <int DIM> constexpr int n_variants() { return (int)std::tuple_size<typename BatchVariants<DIM>::L>::value; }

int batch_tile_variants(int dim)
{
    return dim == 1 ? n_variants<1>() : dim == 2 ? n_variants<2>() : n_variants<3>();
}

template <int DIM, int V = 0>
static void shape_of(int v, int t[3], int* minb)
{
    if constexpr (V < n_variants<DIM>()) {
        using BV = typename std::tuple_element<V, typename BatchVariants<DIM>::L>::type;
        if (v == V) {
            t[0] = BV::TS::X;
            t[1] = BV::TS::Y;
            t[2] = BV::TS::Z;
            *minb = BV::MINB;
            return;
        }
        shape_of<DIM, V + 1>(v, t, minb);
    }
}

void batch_tile_shape(int dim, int v, int t[3])
{
    int minb = 0;
    if (dim == 1) shape_of<1>(v, t, &minb);
    else if (dim == 2) shape_of<2>(v, t, &minb);
    else shape_of<3>(v, t, &minb);
}

int batch_variant_minblocks(int dim, int v)
{
    int t[3], minb = 0;
    if (dim == 1) shape_of<1>(v, t, &minb);
    else if (dim == 2) shape_of<2>(v, t, &minb);
    else shape_of<3>(v, t, &minb);
    return minb;
}

template <int DIM, int PREC, class BV>
static cudaError_t launch_trb(const TransportArgs* boxes, const int2* items, int nitems, BatchCtl ctl, cudaStream_t st)
{
    using TS = typename BV::TS;
    constexpr int MINB = BV::MINB;
    constexpr int GRP = group_fit<DIM, PREC, TS, MINB, BV::GMAX>();
    constexpr size_t smem = transport_smem_max<DIM, PREC, TS, GRP>();  // boxes differ in basis count
    auto fn = k_transport_batch<DIM, PREC, TS, MINB, BV::GMAX>;
    static int grid_of[32] = {0};  // persistent grid (SMs x resident CTAs), per device
    int dev = 0;
    cudaGetDevice(&dev);
    int& grid = grid_of[dev & 31];
    if (!grid) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int nsm = 148, per_sm = 1;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, TS::NTH, smem);
        if (e != cudaSuccess) return e;
        grid = nsm * (per_sm < 1 ? 1 : per_sm);
    }
    int g = grid < nitems ? grid : nitems;
    ProfScope ps("k_transport_batch", st);
    fn<<<g, TS::NTH, smem, st>>>(boxes, items, nitems, ctl);
    return cudaGetLastError();
}

template <int DIM, int PREC, int V = 0>
static cudaError_t launch_trb_v(const TransportArgs* boxes, const int2* items, int nitems, BatchCtl ctl, int v,
                                cudaStream_t st)
{
    if constexpr (V < n_variants<DIM>()) {
        if (v == V) {
            using BV = typename std::tuple_element<V, typename BatchVariants<DIM>::L>::type;
            return launch_trb<DIM, PREC, BV>(boxes, items, nitems, ctl, st);
        }
        return launch_trb_v<DIM, PREC, V + 1>(boxes, items, nitems, ctl, v, st);
    } else {
        return cudaErrorInvalidValue;
    }
}

// Joule pre-pass over (box, tile) items: each CTA walks the work list with a grid
// stride, keeping the item's record in shared memory like the transport kernel.
template <int DIM, int PREC>
__global__ void __launch_bounds__(kJouleThreads, 3)
    k_joule_pre_batch(const TransportArgs* __restrict__ boxes, const int2* __restrict__ items, int nitems,
                      const BatchCtl ctl)
{
    __shared__ long long sA_raw[sizeof(TransportArgs) / 8];
    __shared__ double sJ[DIM * joule_face_box<DIM>()];
    const TransportArgs& sA = *reinterpret_cast<const TransportArgs*>(sA_raw);
    int cur = -1;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const int2 cc = ctl.ctrl[w.x];
        if (ctl.t >= cc.x) continue;  // uniform over the CTA
        const int rec = ((ctl.t + cc.y) & 1) * ctl.nbox + w.x;
        if (rec != cur) {
            const long long* src = reinterpret_cast<const long long*>(boxes + rec);
            for (int q = threadIdx.x; q < (int)(sizeof(TransportArgs) / 8); q += kJouleThreads) sA_raw[q] = src[q];
            cur = rec;
            __syncthreads();
        }
        joule_tile<DIM, PREC>(sA, w.y, sJ);
        __syncthreads();  // the next item's record and faces must not overwrite a slow thread's reads
    }
}

cudaError_t launch_joule_pre_batch(const TransportArgs* boxes, const int2* items, int nitems, BatchCtl ctl, int dim,
                                   int prec, cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    static int nsm = 0;
    if (!nsm) {
        int dev = 0, n = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        nsm = n;
    }
    const int grid = nitems < nsm * 8 ? nitems : nsm * 8;
    ProfScope ps("k_joule_pre_batch", st);
    const bool mx = prec == PREC_MIXED;
    if (dim == 1 && mx) k_joule_pre_batch<1, PREC_MIXED><<<grid, kJouleThreads, 0, st>>>(boxes, items, nitems, ctl);
    else if (dim == 1) k_joule_pre_batch<1, PREC_FP64><<<grid, kJouleThreads, 0, st>>>(boxes, items, nitems, ctl);
    else if (dim == 2 && mx) k_joule_pre_batch<2, PREC_MIXED><<<grid, kJouleThreads, 0, st>>>(boxes, items, nitems, ctl);
    else if (dim == 2) k_joule_pre_batch<2, PREC_FP64><<<grid, kJouleThreads, 0, st>>>(boxes, items, nitems, ctl);
    else if (mx) k_joule_pre_batch<3, PREC_MIXED><<<grid, kJouleThreads, 0, st>>>(boxes, items, nitems, ctl);
    else k_joule_pre_batch<3, PREC_FP64><<<grid, kJouleThreads, 0, st>>>(boxes, items, nitems, ctl);
    return cudaGetLastError();
}

cudaError_t launch_transport_batch(const TransportArgs* boxes, const int2* items, int nitems, BatchCtl ctl, int dim,
                                   int prec, int variant, cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    if (prec == PREC_MIXED) {
        if (dim == 1) return launch_trb_v<1, PREC_MIXED>(boxes, items, nitems, ctl, variant, st);
        if (dim == 2) return launch_trb_v<2, PREC_MIXED>(boxes, items, nitems, ctl, variant, st);
        return launch_trb_v<3, PREC_MIXED>(boxes, items, nitems, ctl, variant, st);
    }
    if (dim == 1) return launch_trb_v<1, PREC_FP64>(boxes, items, nitems, ctl, variant, st);
    if (dim == 2) return launch_trb_v<2, PREC_FP64>(boxes, items, nitems, ctl, variant, st);
    return launch_trb_v<3, PREC_FP64>(boxes, items, nitems, ctl, variant, st);
}

}  // namespace vd
