// vd_types.cuh -- data layouts shared by the host launch code and the kernels:
// physical constants, the device image of the mechanism table and the Array4 view.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/vidyut_b200.h"

namespace vd {

// Source/UnivConstants.H:4-18 and the generated-header constants
// (test/models/Ar_DC_1d/Chemistry.H:327-329,387-388).
constexpr double N_A = 6.02214076e23;
constexpr double K_B = 1.380649e-23;
constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double ECHARGE = 1.60217662e-19;
constexpr double ME = 9.10938188e-31;
constexpr double EV = ECHARGE / K_B;          // kelvin per eV
constexpr double P_NTP = 101325.0;             // pressure at normal conditions [Pa]
constexpr double NA_CE = 6.02214085774e23;    // Avogadro as written in comp_ener_exch
constexpr double KB_CE = 1.380649e-23;
constexpr double EV2J = 1.602176620800000e-19;
constexpr double TE_FIT_EV = 11595.0;         // kelvin per eV of the Janev / F-fit headers

enum { PREC_FP64 = 0, PREC_MIXED = 1 };

// ---------------------------------------------------------------------------
// Mechanism table as the kernels see it (built on the host from vd_mech).
struct VdRxnDev {
    double lnA, b, C, A;      // ln(A) for the exp(lnA + b ln T - C/T) form
    double ex;                // rxntype 1/2: (eexci*eV2J)*NA ; rxntype 5: 3 kB (mw_e/mw_el)
    double coef[VD_MAX_TERMS];
    double l2A, Cl2;          // log2(A), C*log2(e) for the mixed-precision rate
    int8_t kind, nreac, rxntype, elidx, nterms;
    int8_t reac[VD_MAX_REACTANTS];
    int8_t sp[VD_MAX_TERMS];
    int8_t fit;               // index into VdMechDev::fits for the fit rate kinds
    int8_t pad;
};

// Janev / F-fit coefficients; l2jA = log2(jA NA), l2fA = log2(fA NA) for the
// mixed-precision rate
struct VdFitDev {
    double jA, jc[9], fA, fc[4], switch_ev, l2jA, l2fA;
};

struct VdMechDev {
    int32_t ns, nr, e_id, elastic_loss;
    double elastic_coef;                       // 2 me / M
    double mob_p0[VD_MAX_SPECIES + 1];
    double mob_p1[VD_MAX_SPECIES + 1];
    double mob_c[VD_MAX_SPECIES + 1];          // folded constant of the mobility model
    double diff_factor[VD_MAX_SPECIES + 1];
    double diff_p1[VD_MAX_SPECIES + 1];
    int8_t charge[VD_MAX_SPECIES];
    int8_t mob_kind[VD_MAX_SPECIES + 1];
    int8_t mob_ref[VD_MAX_SPECIES + 1];
    int8_t diff_kind[VD_MAX_SPECIES + 1];
    int8_t diff_ref[VD_MAX_SPECIES + 1];
    int8_t emag_e;        // the electron mobility or diffusion depends on |E|
    int8_t need_en;       // the chemistry reads the reduced field (REF)
    int8_t pad;
    int32_t nfits;
    VdRxnDev rxn[VD_MAX_REACTIONS];
    VdFitDev fits[VD_MAX_FITS];
};
static_assert(sizeof(VdMechDev) <= 64000, "mechanism table must fit in constant memory");

// ---------------------------------------------------------------------------
// Array4 view: element (i,j,k,n) = p[(i-bx)+(j-by)*js+(k-bz)*ks+n*ns]
struct A4 {
    double* p;
    int64_t js, ks, ns;
    int bx, by, bz, ncomp;
    int ex, ey, ez;  // exclusive end
    __host__ __device__ A4() : p(nullptr), js(0), ks(0), ns(0), bx(0), by(0), bz(0), ncomp(0), ex(0), ey(0), ez(0) {}
    __host__ A4(const vd_array4& a)
        : p(a.p), js(a.jstride), ks(a.kstride), ns(a.nstride), bx(a.begin[0]), by(a.begin[1]),
          bz(a.begin[2]), ncomp(a.ncomp), ex(a.end[0]), ey(a.end[1]), ez(a.end[2]) {}
    __device__ __forceinline__ int64_t off(int i, int j, int k) const
    {
        return (int64_t)(i - bx) + (int64_t)(j - by) * js + (int64_t)(k - bz) * ks;
    }
    __device__ __forceinline__ double& operator()(int i, int j, int k, int n = 0) const
    {
        return p[off(i, j, k) + (int64_t)n * ns];
    }
};

}  // namespace vd
