// vd_spec.cpp -- chemistry kernels specialised to the loaded mechanism.
//
// vd_mech_init writes CUDA source for the prep pass (per-cell density sums and
// CKWC) with the mechanism folded in -- one straight-line block per reaction with
// its constants as exact hexadecimal literals, species concentrations and
// production rates in registers -- compiles it with NVRTC for sm_100a and loads it
// with the runtime's library API.  This removes what the table-driven kernel
// spends its instructions on (reading the reaction table, branching on kinds,
// indexing per-thread species arrays).  The arithmetic per reaction is the same
// as in chem_cell (vd_device.cuh).  When NVRTC is unavailable or fails, the
// table-driven kernel is used (still on the GPU); vd_mech_specialized() reports
// which one runs.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include <nvrtc.h>
#include "vd_kernels.cuh"

namespace vd {

namespace {

std::string hexd(double x)
{
    char b[64];
    if (std::isinf(x)) return x > 0 ? "(1.0/0.0)" : "(-1.0/0.0)";
    snprintf(b, sizeof(b), "%a", x);
    return b;
}

// Layout-identical device-side definitions of A4 and PrepArgs (vd_types.cuh,
// vd_kernels.cuh); the host checks sizeof(PrepArgs) against the value the
// generated code reports through vd_spec_sizeof.
const char* kPrelude = R"(
typedef long long i64;
struct A4 {
    double* p;
    i64 js, ks, ns;
    int bx, by, bz, ncomp;
    int ex, ey, ez;
    __device__ __forceinline__ i64 off(int i, int j, int k) const
    {
        return (i64)(i - bx) + (i64)(j - by) * js + (i64)(k - bz) * ks;
    }
};
struct PrepArgs {
    A4 sb, rxn, Nv;
    int glo[3], ghi[3];
    int lo[3], hi[3];
    double Tg;
    int do_reactions, write_n;
};
struct BatchCtl {
    const int2* ctrl;
    int nbox;
    int t;
};
extern "C" __global__ void vd_spec_sizeof(unsigned long long* out)
{
    out[0] = sizeof(PrepArgs);
    out[1] = sizeof(BatchCtl);
}
// The FP64 rate exponential, called out of line: inlined, its instructions
// repeated for every reaction made the straight-line chemistry overflow the
// instruction cache (stall "no instruction"); out of line the FP64 prep kernel of
// 150 reactions ran 10 % faster on B200, with bit-identical results.  The mixed
// path's exp2 stays inline (out of line it was slower).
__device__ __noinline__ double vd_exp64(double x) { return exp(x); }
// 2^x as FP32 from an FP64 exponent (same as exp2_split in vd_device.cuh)
__device__ __forceinline__ float exp2_split(double x)
{
    const double xi = rint(x);
    const float f = exp2f((float)(x - xi));
    int i = (int)fmax(fmin(xi, 128.0), -127.0);
    if (i <= -127) return 0.0f;
    if (i >= 128) return __int_as_float(0x7f800000);
    return f * __int_as_float((i + 127) << 23);
}
)";

// electron mobility of the table (mob_fp64 in vd_device.cuh) as an expression of
// Te, nd (density sum) and Tg
std::string mob_expr(const VdMechDev& m, int s, const char* Te, const char* nd, const char* Tg, const char* emag)
{
    int kind = m.mob_kind[s];
    double scale = 1.0;
    if (kind == VD_MOB_SCALED) {
        scale = m.mob_p0[s];
        s = m.mob_ref[s];
        kind = m.mob_kind[s];
    }
    std::ostringstream o;
    o << "(" << hexd(scale) << " * ";
    switch (kind) {
    case VD_MOB_ELECTRON: o << "(" << hexd(m.mob_c[s]) << " / (sqrt(" << Te << ") * " << nd << " * " << hexd(m.mob_p0[s]) << "))"; break;
    case VD_MOB_ION_TG: o << "(" << hexd(m.mob_c[s]) << " / (sqrt(" << Tg << ") * " << nd << " * " << hexd(m.mob_p0[s]) << "))"; break;
    case VD_MOB_CONST_N: o << "(" << hexd(m.mob_p0[s]) << " / " << nd << ")"; break;
    case VD_MOB_CONST: o << hexd(m.mob_p0[s]); break;
    case VD_MOB_POW_EMAG: o << "(" << hexd(m.mob_p0[s]) << " * pow(" << emag << ", " << hexd(m.mob_p1[s]) << "))"; break;
    case VD_MOB_EN_POLY: {  // mob_en_poly in vd_device.cuh
        const double* c = m.fits[m.mob_ref[s]].jc;
        const std::string x = std::string("(") + emag + " / " + nd + ")";
        o << "(" << hexd(m.mob_p0[s]) << " * pow(1.0 + " << hexd(c[0]) << " * pow(" << x << ", 2.0) + " << hexd(c[1])
          << " * pow(" << x << ", 4.0), " << hexd(m.mob_p1[s]) << "))";
        break;
    }
    case VD_MOB_EXP_MEANE: {  // mob_exp_meane in vd_device.cuh
        const double* c = m.fits[m.mob_ref[s]].jc;
        const std::string me = std::string("(1.5 * ") + Te + " / " + hexd(EV) + ")";
        o << "(" << hexd(m.mob_p0[s]) << " * exp(" << hexd(c[0]) << " + " << hexd(c[1]) << " * log(" << me << ") + "
          << hexd(c[2]) << " / " << me << " + " << hexd(c[3]) << " / pow(" << me << ", 2.0) + " << hexd(c[4])
          << " / pow(" << me << ", 3.0)) / " << nd << ")";
        break;
    }
    default: o << "0.0"; break;
    }
    o << ")";
    if (scale == 1.0) {
        std::string t = o.str();
        return t;
    }
    return o.str();
}

std::string gen_prep_kernel(const VdMechDev& m, int prec)
{
    const int ns = m.ns;
    const int eid = m.e_id;
    std::ostringstream o;
    // minimum resident blocks per SM (caps registers at 65536 / (128 * min)); 0 leaves
    // the choice to the compiler.  VD_SPEC_MINBLOCKS overrides it for tuning.
    // Default: about 4 registers per species plus 48 (FP64) or plus 32 (mixed: the
    // rates are FP32), measured best on B200 for the 8- and 24-species mechanisms
    // (FP64: 6 and 3 blocks of 128 threads per SM; mixed: 8 and 4).
    int minb = 65536 / (128 * (4 * ns + (prec == PREC_MIXED ? 32 : 48)));
    minb = minb < 1 ? 1 : (minb > 8 ? 8 : minb);
    if (const char* e = getenv("VD_SPEC_MINBLOCKS")) minb = atoi(e);
    const std::string sfx = prec == PREC_MIXED ? "mixed" : "fp64";
    const std::string lb = "__launch_bounds__(128" + (minb > 0 ? ", " + std::to_string(minb) : std::string()) + ")";
    // per-box kernel (grid-stride over the grown box) and batched kernel (work list
    // of (box, chunk of kPrepChunk cells)), both around one per-cell function
    o << "__device__ __forceinline__ void vd_spec_cell_" << sfx << "(const PrepArgs& a, i64 idx);\n";
    o << "extern \"C\" __global__ void " << lb << " vd_spec_prep_" << sfx << "(const PrepArgs a)\n{\n"
      << "  const i64 ntot = (i64)(a.ghi[0] - a.glo[0] + 1) * (a.ghi[1] - a.glo[1] + 1) * (a.ghi[2] - a.glo[2] + 1);\n"
      << "  for (i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x; idx < ntot; idx += (i64)gridDim.x * blockDim.x)\n"
      << "    vd_spec_cell_" << sfx << "(a, idx);\n}\n";
    o << "extern \"C\" __global__ void " << lb << " vd_spec_prep_batch_" << sfx
      << "(const PrepArgs* __restrict__ boxes, const int2* __restrict__ items, int nitems, const BatchCtl ctl)\n{\n"
      << "  __shared__ PrepArgs a;  // the item's record\n"
      << "  int cur = -1;\n"
      << "  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {\n"
      << "    const int2 w = items[it];\n"
      << "    const int2 cc = ctl.ctrl[w.x];\n"
      << "    if (ctl.t >= cc.x) continue;\n"
      << "    const int rec = ((ctl.t + cc.y) & 1) * ctl.nbox + w.x;\n"
      << "    if (rec != cur) {\n"
      << "      __syncthreads();\n"
      << "      const long long* src = reinterpret_cast<const long long*>(boxes + rec);\n"
      << "      long long* dst = reinterpret_cast<long long*>(&a);\n"
      << "      for (int q = threadIdx.x; q < (int)(sizeof(PrepArgs) / 8); q += blockDim.x) dst[q] = src[q];\n"
      << "      cur = rec;\n"
      << "      __syncthreads();\n"
      << "    }\n"
      << "    const i64 ntot = (i64)(a.ghi[0] - a.glo[0] + 1) * (a.ghi[1] - a.glo[1] + 1) * (a.ghi[2] - a.glo[2] + 1);\n"
      << "    for (int q = threadIdx.x; q < " << kPrepChunk << "; q += blockDim.x) {\n"
      << "      const i64 idx = (i64)w.y * " << kPrepChunk << " + q;\n"
      << "      if (idx < ntot) vd_spec_cell_" << sfx << "(a, idx);\n"
      << "    }\n  }\n}\n";
    o << "__device__ __forceinline__ void vd_spec_cell_" << sfx << "(const PrepArgs& a, i64 idx)\n{\n";
    o << "  const double N_A = " << hexd(N_A) << ", NA_CE = " << hexd(NA_CE) << ", KB_CE = " << hexd(KB_CE)
      << ", K_B = " << hexd(K_B) << ";\n";
    o << "  const int gx = a.ghi[0] - a.glo[0] + 1, gy = a.ghi[1] - a.glo[1] + 1;\n"
         "  const i64 cs = a.sb.ns, rs = a.rxn.ns;\n"
         "  {\n"
         "    int i, j, k;\n"
         "    const i64 gxy = (i64)gx * gy;\n"
         "    if (idx < 0xffffffffLL && gxy < 0xffffffffLL) {  // 32-bit division, the usual case\n"
         "      const unsigned u = (unsigned)idx, pl = (unsigned)gxy;\n"
         "      const unsigned kk = u / pl, rr = u - kk * pl, jj = rr / (unsigned)gx;\n"
         "      k = (int)kk; j = (int)jj; i = (int)(rr - jj * (unsigned)gx);\n"
         "    } else {\n"
         "      k = (int)(idx / gxy);\n"
         "      const i64 r = idx - (i64)k * gxy;\n"
         "      j = (int)(r / gx);\n"
         "      i = (int)(r - (i64)j * gx);\n"
         "    }\n"
         "    i += a.glo[0]; j += a.glo[1]; k += a.glo[2];\n"
         "    const double* p = a.sb.p + a.sb.off(i, j, k);\n";
    for (int s = 0; s < ns; s++) o << "    const double n" << s << " = p[" << s << " * cs];\n";
    o << "    double N = 0.0;\n";
    for (int s = 0; s < ns; s++) o << "    N += n" << s << ";\n";
    o << "    if (a.write_n) a.Nv.p[a.Nv.off(i, j, k)] = N;\n"
         "    if (i < a.lo[0] || i > a.hi[0] || j < a.lo[1] || j > a.hi[1] || k < a.lo[2] || k > a.hi[2]) return;\n"
         "    double* rx = a.rxn.p + a.rxn.off(i, j, k);\n"
         "    if (!a.do_reactions) {\n";
    for (int s = 0; s <= ns; s++) o << "      rx[" << s << " * rs] = 0.0;\n";
    o << "      return;\n    }\n";
    o << "    const double Te = p[" << (ns + 1) << " * cs];\n    const double Tg = a.Tg;\n";
    if (m.need_en) o << "    const double EN = p[" << (ns + 9) << " * cs];\n";  // REF
    for (int s = 0; s < ns; s++) o << "    const double sc" << s << " = n" << s << " * 1.0e-6 / N_A * 1.0e6;\n";
    for (int s = 0; s < ns; s++) o << "    double w" << s << " = 0.0;\n";
    o << "    const double ne = sc" << eid << " * NA_CE;\n"
         "    const double Ue = 1.5 * Te * ne * KB_CE;\n"
         "    const double mee_na = Ue / ne * NA_CE;\n"
         "    const double sefact = (tanh((Te - Tg) / 0.5) + 1.0) / 2.0;\n"
         "    const double dT = Te - Tg;\n";
    if (prec == PREC_FP64) o << "    const double lTe = log(Te), lTg = log(Tg);\n";
    else o << "    const double lTe = log2(Te), lTg = log2(Tg);\n";
    o << "    const double invTe = 1.0 / Te, invTg = 1.0 / Tg;\n    double ee = 0.0;\n";
    if (m.need_en) {
        // E = EN N 1e-21 of the field-driven rates (townsend_rate in vd_device.cuh)
        o << "    double mix = 0.0;\n";
        for (int s = 0; s < ns; s++) o << "    mix += sc" << s << ";\n";
        o << "    const double efm = EN * (mix * N_A) * 1e-21;\n";
    }
    if (m.nfits > 0) {
        // the powers the Janev / F-fit rates share (fit_powers in vd_device.cuh)
        o << "    const double teev = Te / " << hexd(TE_FIT_EV) << ", lte = log(teev);\n"
          << "    const double ite = (Te == 0) ? 1.0 : 1.0 / teev;\n";
        if (prec == PREC_FP64) {
            for (int j = 0; j < 9; j++) o << "    const double tep" << j << " = pow(lte, " << j << ".0);\n";
            for (int j = 0; j < 4; j++) o << "    const double itp" << j << " = pow(ite, " << (j + 1) << ".0);\n";
        } else {
            o << "    const double tep0 = 1.0;\n";
            for (int j = 1; j < 9; j++) o << "    const double tep" << j << " = tep" << (j - 1) << " * lte;\n";
            o << "    const double itp0 = ite;\n";
            for (int j = 1; j < 4; j++) o << "    const double itp" << j << " = itp" << (j - 1) << " * ite;\n";
        }
    }
    // a fit rate's sum, accumulated in order as the header does (fit_rate)
    auto fit_sum = [&](const VdFitDev& F, bool janev) {
        o << "        double sum = 0.0;\n";
        if (janev)
            for (int j = 0; j < 9; j++)
                o << "        sum = __dadd_rn(sum, __dmul_rn(" << hexd(F.jc[j]) << ", tep" << j << "));\n";
        else
            for (int j = 0; j < 4; j++)
                o << "        sum = __dadd_rn(sum, __dmul_rn(" << hexd(F.fc[j]) << ", itp" << j << "));\n";
        if (prec == PREC_FP64)
            o << "        k = " << hexd(janev ? F.jA : F.fA) << " * vd_exp64(sum) * NA_CE;\n";
        else
            o << "        k = (double)exp2_split(fma(sum, " << hexd(1.4426950408889634074) << ", "
              << hexd(janev ? F.l2jA : F.l2fA) << "));\n";
    };
    for (int r = 0; r < m.nr; r++) {
        const VdRxnDev& R = m.rxn[r];
        o << "    { // reaction " << r << "\n      double k;\n";
        if (R.kind == VD_RATE_CONST) {
            o << "      k = " << hexd(R.A) << ";\n";
        } else if (R.kind == VD_RATE_TOWNSEND) {
            const double* c = m.fits[R.fit].jc;
            o << "      {\n        const double alpha = (" << hexd(c[0]) << " + " << hexd(c[1]) << " / pow(efm, 3.0)) * exp(-"
              << hexd(c[2]) << " / efm);\n"
              << "        const double mu_e = " << hexd(c[4]) << " * pow(efm, " << hexd(c[5]) << ");\n"
              << "        k = (alpha - " << hexd(c[3]) << ") * mu_e * efm;\n      }\n";
        } else if (R.kind >= VD_RATE_JANEV) {
            const VdFitDev& F = m.fits[R.fit];
            if (R.kind == VD_RATE_JANEV_FFIT) {
                o << "      if (teev < " << hexd(F.switch_ev) << ") {\n";
                fit_sum(F, true);
                o << "      } else {\n";
                fit_sum(F, false);
                o << "      }\n";
            } else {
                o << "      {\n";
                fit_sum(F, R.kind == VD_RATE_JANEV);
                o << "      }\n";
            }
        } else if (!(R.A > 0.0)) {
            o << "      k = 0.0;\n";
        } else {
            const bool te = (R.kind == VD_RATE_ARRHENIUS_TE);
            const char* lT = te ? "lTe" : "lTg";
            const char* iT = te ? "invTe" : "invTg";
            if (prec == PREC_FP64) {
                o << "      k = vd_exp64(fma(" << hexd(R.b) << ", " << lT << ", " << hexd(R.lnA) << ") - " << hexd(R.C)
                  << " * " << iT << ");\n";
            } else {
                o << "      k = (double)exp2_split(fma(" << hexd(R.b) << ", " << lT << ", " << hexd(R.l2A) << ") - "
                  << hexd(R.Cl2) << " * " << iT << ");\n";
            }
        }
        o << "      const double q = k * ";
        for (int t = 0; t < R.nreac; t++) o << (t ? " * " : "(") << "sc" << (int)R.reac[t];
        o << ");\n";
        for (int t = 0; t < R.nterms; t++)
            o << "      w" << (int)R.sp[t] << " = fma(" << hexd(R.coef[t]) << ", q, w" << (int)R.sp[t] << ");\n";
        if (R.rxntype == VD_RXN_EXCITATION || R.rxntype == VD_RXN_IONIZATION)
            o << "      ee -= " << hexd(R.ex) << " * q * sefact;\n";
        else if (R.rxntype == VD_RXN_RECOMB || R.rxntype == VD_RXN_ATTACH)
            o << "      ee -= mee_na * q;\n";
        else if (R.rxntype == VD_RXN_DETACH)
            o << "      ee += mee_na * q;\n";
        else if (R.rxntype == VD_RXN_ELASTIC)
            o << "      ee -= " << hexd(R.ex) << " * dT * (sc" << eid << " * sc" << (int)R.elidx << " * k) * NA_CE;\n";
        o << "    }\n";
    }
    if (m.elastic_loss) {
        o << "    {\n      double nd = 0.0;\n";
        for (int s = 0; s < ns; s++) o << "      nd += sc" << s << " * N_A;\n";
        o << "      const double mu = "
          << mob_expr(m, eid, "Te", "nd", "Tg", m.need_en ? "(EN * nd * 1.0e-21)" : "0.0") << ";\n"
          << "      const double nu = " << hexd(-ECHARGE / ME) << " / mu;\n"
          << "      ee -= 1.5 * K_B * sc" << eid << " * N_A * dT * nu * " << hexd(m.elastic_coef) << ";\n    }\n";
    }
    for (int s = 0; s < ns; s++) o << "    rx[" << s << " * rs] = w" << s << " * 1.0e-6 * N_A * 1.0e6;\n";
    o << "    rx[" << ns << " * rs] = ee;\n  }\n}\n";
    return o.str();
}

struct SpecModule {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t prep[2] = {nullptr, nullptr};
    cudaKernel_t batch[2] = {nullptr, nullptr};
};

std::mutex g_spec_mu;
std::map<std::string, SpecModule*> g_cache;   // by generated source
SpecModule* g_active = nullptr;
bool g_enabled = true;
std::string g_spec_err;

}  // namespace

void spec_set_enabled(bool on)
{
    std::lock_guard<std::mutex> lk(g_spec_mu);
    g_enabled = on;
}

bool spec_active()
{
    std::lock_guard<std::mutex> lk(g_spec_mu);
    return g_active != nullptr;
}

const char* spec_error() { return g_spec_err.c_str(); }

// Generate, compile and load the specialised kernels for m (cached by source).
// Returns 0 when the specialised kernels are active, nonzero when the
// table-driven kernels stay in use (spec_error() says why).
int spec_build(const VdMechDev& m)
{
    std::lock_guard<std::mutex> lk(g_spec_mu);
    g_active = nullptr;
    g_spec_err.clear();
    if (!g_enabled) {
        g_spec_err = "specialisation switched off";
        return 1;
    }
    std::string src = std::string(kPrelude) + gen_prep_kernel(m, PREC_FP64) + gen_prep_kernel(m, PREC_MIXED);
    auto it = g_cache.find(src);
    if (it != g_cache.end()) {
        g_active = it->second;
        return 0;
    }
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "vd_spec_chem.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        g_spec_err = "nvrtcCreateProgram failed";
        return 2;
    }
    // 177: concentrations of species that are no reactant are declared but unused
    const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device", "--fmad=true",
                          "--extra-device-vectorization", "--diag-suppress=177"};
    nvrtcResult rc = nvrtcCompileProgram(prog, 6, opts);
    if (rc != NVRTC_SUCCESS) {
        size_t n = 0;
        nvrtcGetProgramLogSize(prog, &n);
        std::string log(n, '\0');
        if (n) nvrtcGetProgramLog(prog, &log[0]);
        g_spec_err = std::string("NVRTC: ") + nvrtcGetErrorString(rc) + ": " + log.substr(0, 400);
        nvrtcDestroyProgram(&prog);
        return 3;
    }
    size_t nbin = 0;
    nvrtcGetCUBINSize(prog, &nbin);
    std::vector<char> bin(nbin);
    nvrtcGetCUBIN(prog, bin.data());
    nvrtcDestroyProgram(&prog);
    SpecModule* mod = new SpecModule;
    cudaError_t e = cudaLibraryLoadData(&mod->lib, bin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&mod->prep[PREC_FP64], mod->lib, "vd_spec_prep_fp64");
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&mod->prep[PREC_MIXED], mod->lib, "vd_spec_prep_mixed");
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&mod->batch[PREC_FP64], mod->lib, "vd_spec_prep_batch_fp64");
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&mod->batch[PREC_MIXED], mod->lib, "vd_spec_prep_batch_mixed");
    if (e == cudaSuccess) {
        // layout check of the kernel argument struct
        cudaKernel_t sz;
        unsigned long long* d = nullptr;
        unsigned long long h[2] = {0, 0};
        e = cudaLibraryGetKernel(&sz, mod->lib, "vd_spec_sizeof");
        if (e == cudaSuccess) e = cudaMalloc(&d, sizeof(h));
        if (e == cudaSuccess) {
            void* args[] = {&d};
            e = cudaLaunchKernel((const void*)sz, dim3(1), dim3(1), args, 0, 0);
            if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
            cudaFree(d);
            if (e == cudaSuccess && (h[0] != sizeof(PrepArgs) || h[1] != sizeof(BatchCtl))) {
                g_spec_err = "specialised kernel argument layout differs";
                return 4;
            }
        }
    }
    if (e != cudaSuccess) {
        g_spec_err = std::string("loading specialised kernels: ") + cudaGetErrorString(e);
        cudaGetLastError();
        return 5;
    }
    g_cache[src] = mod;
    g_active = mod;
    return 0;
}

// Generate and compile (without loading) the specialised kernels: a check that
// needs no GPU.  Returns 0 on success; spec_error() holds the NVRTC log otherwise.
int spec_compile_only(const VdMechDev& m, size_t* cubin_bytes)
{
    std::string src = std::string(kPrelude) + gen_prep_kernel(m, PREC_FP64) + gen_prep_kernel(m, PREC_MIXED);
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "vd_spec_chem.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        g_spec_err = "nvrtcCreateProgram failed";
        return 2;
    }
    const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device", "--fmad=true",
                          "--ptxas-options=-v", "--diag-suppress=177"};
    nvrtcResult rc = nvrtcCompileProgram(prog, 6, opts);
    size_t n = 0;
    nvrtcGetProgramLogSize(prog, &n);
    std::string log(n, '\0');
    if (n) nvrtcGetProgramLog(prog, &log[0]);
    if (rc != NVRTC_SUCCESS) {
        g_spec_err = std::string("NVRTC: ") + nvrtcGetErrorString(rc) + ": " + log.substr(0, 2000);
        nvrtcDestroyProgram(&prog);
        return 3;
    }
    g_spec_err = log.substr(0, 2000);  // resource usage reported by ptxas
    nvrtcGetCUBINSize(prog, cubin_bytes);
    nvrtcDestroyProgram(&prog);
    return 0;
}

// Launch the specialised prep kernel if active; returns cudaErrorNotReady when the
// table-driven kernel must be used instead.
cudaError_t spec_launch_prep(const PrepArgs& a, int prec, cudaStream_t st)
{
    cudaKernel_t k;
    {
        std::lock_guard<std::mutex> lk(g_spec_mu);
        if (!g_active) return cudaErrorNotReady;
        k = g_active->prep[prec == PREC_MIXED ? PREC_MIXED : PREC_FP64];
    }
    int64_t n = (int64_t)(a.ghi[0] - a.glo[0] + 1) * (a.ghi[1] - a.glo[1] + 1) * (a.ghi[2] - a.glo[2] + 1);
    int64_t g = (n + 127) / 128;
    if (g > 148LL * 64) g = 148LL * 64;
    if (g < 1) g = 1;
    PrepArgs copy = a;
    void* args[] = {&copy};
    ProfScope ps("k_prep_spec", st);
    return cudaLaunchKernel((const void*)k, dim3((unsigned)g), dim3(128), args, 0, st);
}

// Batched form: boxes and items are device arrays; one CTA per work item (grid-stride).
cudaError_t spec_launch_prep_batch(const PrepArgs* boxes, const int2* items, int nitems, BatchCtl ctl, int prec,
                                   cudaStream_t st)
{
    cudaKernel_t k;
    {
        std::lock_guard<std::mutex> lk(g_spec_mu);
        if (!g_active) return cudaErrorNotReady;
        k = g_active->batch[prec == PREC_MIXED ? PREC_MIXED : PREC_FP64];
    }
    unsigned g = (unsigned)(nitems < 148 * 16 ? nitems : 148 * 16);
    void* args[] = {(void*)&boxes, (void*)&items, &nitems, &ctl};
    ProfScope ps("k_prep_batch_spec", st);
    return cudaLaunchKernel((const void*)k, dim3(g), dim3(128), args, 0, st);
}

}  // namespace vd
