// vd_device.cuh -- device-side data layout and physics of the explicit species /
// electron-energy update (sm_100a).
//
// The mechanism lives in __constant__ memory (every thread of a warp reads the
// same reaction at the same time, so the constant cache broadcasts it).  Two
// arithmetic flavours share the code:
//   PREC_FP64   all arithmetic in FP64; results agree with the reference CPU build
//               to ~1e-14 (FMA contraction and exp(log) rate evaluation are the
//               only differences);
//   PREC_MIXED  WENO weights, reconstructions, flux arithmetic and mobilities in
//               FP32 (values rescaled by an exact power of two per stencil), rate
//               constants through the FP32 special-function unit, and FP64 for the
//               production/loss sums, the energy-exchange sum and n += dt*dsdt.
#pragma once
#include "vd_types.cuh"

namespace vd {

// The loaded mechanism.  Every translation unit that includes this header has its
// own copy (internal linkage; the library is compiled without relocatable device
// code) and uploads it through its own upload function (upload_mech in
// vd_kernels.cu, which also calls upload_mech_batch in vd_batch_kernels.cu and
// upload_mech_diffusion in vd_diffusion.cu).
static __constant__ VdMechDev c_mech;

// Approximate reciprocal on the special-function unit (rcp.approx.ftz.f32,
// ~1 ulp); arguments are normal positive numbers wherever it is used.
__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// 2^x for an FP64 exponent x as an FP32 value: x = i + f with i = rint(x) (exact in
// FP64), 2^f for f in [-1/2, 1/2] on the FP32 special-function unit (exp2f, ~2 ulp)
// and 2^i through the exponent bits.  Relative error ~2.4e-7 whatever |x|;
// results below 2^-126 flush to zero, above 2^127 saturate to infinity.
__device__ __forceinline__ float exp2_split(double x)
{
    const double xi = rint(x);
    const float f = exp2f((float)(x - xi));
    int i = (int)fmax(fmin(xi, 128.0), -127.0);
    if (i <= -127) return 0.0f;
    if (i >= 128) return __int_as_float(0x7f800000);
    return f * __int_as_float((i + 127) << 23);
}

// ---------------------------------------------------------------------------
// Mobility (specMob, test/models/Ar_DC_1d/Chemistry.H:177-202) by model kind.
// FP64: mob_c = -e/me / sqrt(8 kB/(pi me)) (electron) or e/M / sqrt(8 kB/(pi M))
// (ion), so mu = mob_c / (sqrt(T) N sigma): one sqrt and one division.  emag is
// the field magnitude |E| the caller's reference loop passes to specMob (power
// laws in |E|, test/verification/Streamer/Chemistry.H:165-183).
// The He_RF_1d header's models (test/verification/He_RF_1d/Chemistry.H:229-243),
// in its order of operations: the ion form (1 + c0 x^2 + c1 x^4)^p of x = |E|/N,
// and the electron form exp(c0 + c1 ln m + c2/m + c3/m^2 + c4/m^3) of the mean
// energy m = 1.5 Te/eV (the constant factor and the 1/N are the caller's).
__device__ __forceinline__ double mob_en_poly(const double* c, double p, double emag, double N)
{
    const double x = emag / N;
    return pow(1.0 + c[0] * pow(x, 2.0) + c[1] * pow(x, 4.0), p);
}
__device__ __forceinline__ double mob_exp_meane(const double* c, double Te)
{
    const double m = 1.5 * Te / EV;
    return exp(c[0] + c[1] * log(m) + c[2] / m + c[3] / pow(m, 2.0) + c[4] / pow(m, 3.0));
}
// The field-dependent models in FP64, out of line: their pow / exp / log code,
// inlined into the transport tile, would cost every mechanism registers that only
// these models use.
static __device__ __noinline__ double mob_field_fp64(int s, double Te, double N, double emag)
{
    switch (c_mech.mob_kind[s]) {
    case VD_MOB_POW_EMAG: return c_mech.mob_p0[s] * pow(emag, c_mech.mob_p1[s]);
    case VD_MOB_EN_POLY: return c_mech.mob_p0[s] * mob_en_poly(c_mech.fits[c_mech.mob_ref[s]].jc, c_mech.mob_p1[s], emag, N);
    case VD_MOB_EXP_MEANE: return c_mech.mob_p0[s] * mob_exp_meane(c_mech.fits[c_mech.mob_ref[s]].jc, Te) / N;
    default: return 0.0;
    }
}
// velocity basis kinds 3, 4 and 5 of the FP64 transport tile (E times the per-cell
// factor of VD_MOB_POW_EMAG / VD_MOB_EN_POLY / VD_MOB_EXP_MEANE), out of line
static __device__ __noinline__ double basis_field_fp64(int kind, int fit, double pw, double E, double emag, double N,
                                                       double Te)
{
    if (kind == 3) return E * pow(emag, pw);
    if (kind == 4) return E * mob_en_poly(c_mech.fits[fit].jc, pw, emag, N);
    return E * mob_exp_meane(c_mech.fits[fit].jc, Te) / N;
}
__device__ __forceinline__ double mob_base_fp64(int s, double Te, double N, double Tg, double emag)
{
    switch (c_mech.mob_kind[s]) {
    case VD_MOB_ELECTRON: return c_mech.mob_c[s] / (sqrt(Te) * N * c_mech.mob_p0[s]);
    case VD_MOB_ION_TG: return c_mech.mob_c[s] / (sqrt(Tg) * N * c_mech.mob_p0[s]);
    case VD_MOB_CONST_N: return c_mech.mob_p0[s] / N;
    case VD_MOB_CONST: return c_mech.mob_p0[s];
    case VD_MOB_POW_EMAG:
    case VD_MOB_EN_POLY:
    case VD_MOB_EXP_MEANE: return mob_field_fp64(s, Te, N, emag);
    default: return 0.0;
    }
}
__device__ __forceinline__ double mob_fp64(int s, double Te, double N, double Tg, double emag)
{
    if (c_mech.mob_kind[s] == VD_MOB_SCALED)
        return c_mech.mob_p0[s] * mob_base_fp64(c_mech.mob_ref[s], Te, N, Tg, emag);
    return mob_base_fp64(s, Te, N, Tg, emag);
}
// The He_RF_1d models for the mixed path: the polynomial in FP32; the
// mean-energy exponent (about 55, whose FP32 rounding alone would be 4e-6 of the
// mobility) summed in FP64 from an FP32 logarithm and raised by exp2_split.
__device__ __forceinline__ float mob_en_poly_f32(const double* c, float p, float emag, float N)
{
    const float x = emag * rcp_approx(N);
    const float x2 = x * x;
    const float q = fmaf((float)c[1], x2 * x2, fmaf((float)c[0], x2, 1.0f));
    return exp2f(p * log2f(q));
}
__device__ __forceinline__ float mob_exp_meane_f32(const double* c, float Te)
{
    constexpr double LN2 = 0.69314718055994530942, LOG2E = 1.4426950408889634074;
    const double m = 1.5 * (double)Te / EV;
    const double im = 1.0 / m;
    const double sum = fma((double)log2f((float)m), c[1] * LN2, c[0]) + im * fma(im, fma(im, c[4], c[3]), c[2]);
    return exp2_split(sum * LOG2E);
}
// velocity basis kinds 3, 4 and 5 of the mixed transport tile, out of line (as
// basis_field_fp64)
static __device__ __noinline__ float basis_field_f32(int kind, int fit, float pw, float E, float emag, float N,
                                                     float Te)
{
    if (kind == 3) return E * exp2f(pw * log2f(emag));
    if (kind == 4) return E * mob_en_poly_f32(c_mech.fits[fit].jc, pw, emag, N);
    return E * mob_exp_meane_f32(c_mech.fits[fit].jc, Te) * rcp_approx(N);
}
__device__ __forceinline__ float mob_base_f32(int s, float Te, float N, float Tg, float emag)
{
    switch (c_mech.mob_kind[s]) {
    case VD_MOB_ELECTRON: return (float)c_mech.mob_c[s] * rsqrtf(Te) * rcp_approx(N * (float)c_mech.mob_p0[s]);
    case VD_MOB_ION_TG: return (float)c_mech.mob_c[s] * rsqrtf(Tg) * rcp_approx(N * (float)c_mech.mob_p0[s]);
    case VD_MOB_CONST_N: return (float)c_mech.mob_p0[s] * rcp_approx(N);
    case VD_MOB_CONST: return (float)c_mech.mob_p0[s];
    case VD_MOB_POW_EMAG: return (float)c_mech.mob_p0[s] * exp2f((float)c_mech.mob_p1[s] * log2f(emag));
    // the exponential's argument is too large for FP32 (e^55 in the He_RF_1d fit)
    case VD_MOB_EN_POLY:
        return (float)c_mech.mob_p0[s] *
               mob_en_poly_f32(c_mech.fits[c_mech.mob_ref[s]].jc, (float)c_mech.mob_p1[s], emag, N);
    case VD_MOB_EXP_MEANE:
        return (float)c_mech.mob_p0[s] * mob_exp_meane_f32(c_mech.fits[c_mech.mob_ref[s]].jc, Te) * rcp_approx(N);
    default: return 0.0f;
    }
}
__device__ __forceinline__ float mob_f32(int s, float Te, float N, float Tg, float emag)
{
    if (c_mech.mob_kind[s] == VD_MOB_SCALED)
        return (float)c_mech.mob_p0[s] * mob_base_f32(c_mech.mob_ref[s], Te, N, Tg, emag);
    return mob_base_f32(s, Te, N, Tg, emag);
}
// specDiff (test/models/Ar_DC_1d/Chemistry.H:204-239) by model kind; the
// field- and pressure-dependent ones out of line, as mob_field_fp64.
static __device__ __noinline__ double diff_field_fp64(int s, double Te, double N, double Tg, double emag)
{
    switch (c_mech.diff_kind[s]) {
    case VD_DIFF_POW_EMAG: return c_mech.diff_factor[s] * pow(emag, c_mech.diff_p1[s]);
    // P_NTP / (N kB Tg) (test/verification/He_RF_1d/Chemistry.H:270-296)
    case VD_DIFF_PRES: return c_mech.diff_factor[s] * (P_NTP / (N * K_B * Tg));
    case VD_DIFF_TE_PRES: return c_mech.diff_factor[s] * (Te / c_mech.diff_p1[s]) * (P_NTP / (N * K_B * Tg));
    default: return 0.0;
    }
}
__device__ __forceinline__ double diff_base_fp64(int s, double Te, double N, double Tg, double emag)
{
    switch (c_mech.diff_kind[s]) {
    case VD_DIFF_TE_ABSMOB:
        return c_mech.diff_factor[s] * (Te / EV) * fabs(mob_fp64(c_mech.diff_ref[s], Te, N, Tg, emag));
    case VD_DIFF_TG_MOB:
        return c_mech.diff_factor[s] * (Tg / EV) * mob_fp64(c_mech.diff_ref[s], Te, N, Tg, emag);
    case VD_DIFF_CONST: return c_mech.diff_factor[s];
    case VD_DIFF_POW_EMAG:
    case VD_DIFF_PRES:
    case VD_DIFF_TE_PRES: return diff_field_fp64(s, Te, N, Tg, emag);
    default: return 0.0;
    }
}
// specDiff with the scaled model (D = factor * D[ref], the energy's 5/3 of the
// electrons' coefficient in the Streamer and He_RF_1d headers)
__device__ __forceinline__ double diff_fp64(int s, double Te, double N, double Tg, double emag)
{
    if (c_mech.diff_kind[s] == VD_DIFF_SCALED)
        return c_mech.diff_factor[s] * diff_base_fp64(c_mech.diff_ref[s], Te, N, Tg, emag);
    return diff_base_fp64(s, Te, N, Tg, emag);
}
__device__ __forceinline__ float diff_base_f32(int s, float Te, float N, float Tg, float emag, float mu_e)
{
    // mu_e: the electron mobility when s's model refers to it (saves its re-evaluation)
    const int dk = c_mech.diff_kind[s], dr = c_mech.diff_ref[s];
    const float f = (float)c_mech.diff_factor[s];
    switch (dk) {
    case VD_DIFF_TE_ABSMOB:
    case VD_DIFF_TG_MOB: {
        const float mr = dr == c_mech.e_id ? mu_e : mob_f32(dr, Te, N, Tg, emag);
        if (dk == VD_DIFF_TE_ABSMOB) return f * (Te * (float)(1.0 / EV)) * fabsf(mr);
        return f * (Tg * (float)(1.0 / EV)) * mr;
    }
    case VD_DIFF_CONST: return f;
    case VD_DIFF_POW_EMAG: return f * exp2f((float)c_mech.diff_p1[s] * log2f(emag));
    case VD_DIFF_PRES: return f * ((float)P_NTP * rcp_approx(N * (float)K_B * Tg));
    case VD_DIFF_TE_PRES:
        return f * (Te * (float)(1.0 / c_mech.diff_p1[s])) * ((float)P_NTP * rcp_approx(N * (float)K_B * Tg));
    default: return 0.0f;
    }
}
__device__ __forceinline__ float diff_f32(int s, float Te, float N, float Tg, float emag, float mu_e)
{
    if (c_mech.diff_kind[s] == VD_DIFF_SCALED)
        return (float)c_mech.diff_factor[s] * diff_base_f32(c_mech.diff_ref[s], Te, N, Tg, emag, mu_e);
    return diff_base_f32(s, Te, N, Tg, emag, mu_e);
}

// ---------------------------------------------------------------------------
// WENO-5 reconstruction at i+1/2 from (im2, im1, i, ip1, ip2)
// (Source/compute_explicit_flux.H:25-112).  SCHEME 1 JS, 2 M, 3 Z.
template <class R>
__device__ __forceinline__ R gk_map(R wk, R g)
{
    return wk * (g + g * g - R(3) * g * wk + wk * wk) / (g * g + wk * (R(1) - R(2) * g));
}

__device__ __forceinline__ double weno_fp64(double a, double b, double c, double d, double e, int scheme)
{
    const double eps = 1e-20;
    double p1 = (1.0 / 3.0) * a - (7.0 / 6.0) * b + (11.0 / 6.0) * c;
    double p2 = -(1.0 / 6.0) * b + (5.0 / 6.0) * c + (1.0 / 3.0) * d;
    double p3 = (1.0 / 3.0) * c + (5.0 / 6.0) * d - (1.0 / 6.0) * e;
    double t1 = a - 2.0 * b + c, t2 = a - 4.0 * b + 3.0 * c;
    double b1 = (13.0 / 12.0) * (t1 * t1) + 0.25 * (t2 * t2);
    double t3 = b - 2.0 * c + d, t4 = b - d;
    double b2 = (13.0 / 12.0) * (t3 * t3) + 0.25 * (t4 * t4);
    double t5 = c - 2.0 * d + e, t6 = 3.0 * c - 4.0 * d + e;
    double b3 = (13.0 / 12.0) * (t5 * t5) + 0.25 * (t6 * t6);
    double a1, a2, a3;
    if (scheme == 3) {
        double tau = fabs(b1 - b3);
        double r1 = tau / (b1 + eps), r2 = tau / (b2 + eps), r3 = tau / (b3 + eps);
        a1 = 0.1 * (1.0 + r1 * r1);
        a2 = 0.6 * (1.0 + r2 * r2);
        a3 = 0.3 * (1.0 + r3 * r3);
    } else {
        double q1 = b1 + eps, q2 = b2 + eps, q3 = b3 + eps;
        a1 = 0.1 / (q1 * q1);
        a2 = 0.6 / (q2 * q2);
        a3 = 0.3 / (q3 * q3);
        if (scheme == 2) {
            double s = a1 + a2 + a3;
            double w1 = a1 / s, w2 = a2 / s, w3 = a3 / s;
            a1 = gk_map(w1, 0.1);
            a2 = gk_map(w2, 0.6);
            a3 = gk_map(w3, 0.3);
        }
    }
    double s = a1 + a2 + a3;
    return (a1 / s) * p1 + (a2 / s) * p2 + (a3 / s) * p3;
}


// One FP32 reconstruction of values already scaled to O(1), from its three 4 beta_k
// and candidate polynomials.  The nonlinear weights are
// rescaled so that no term can overflow and the smoothest stencil always keeps a
// weight of order gamma (the sum never underflows to zero, whatever the spread of
// the smoothness indicators): with q_k = beta_k + eps and m = min_k q_k,
//   WENO-JS  alpha_k ~ gamma_k (m/q_k)^2
//   WENO-Z   alpha_k ~ gamma_k (1 + (tau/q_k)^2)              if tau <= m
//            alpha_k ~ gamma_k ((m/tau)^2 + (m/q_k)^2)        otherwise
// (each a positive multiple of the reference's alpha_k); WENO-M keeps its map.
// The smoothness indicators are kept as 4 beta_k (13/3 and 1 for the reference's
// 13/12 and 1/4) and eps4 is 4 eps: every weight is a ratio of these, and scaling
// by a power of two changes no rounding, so the result is the same and each
// indicator costs one multiply less.
__device__ __forceinline__ float weno_weights_f32(float b1, float b2, float b3, float p1, float p2, float p3, int scheme,
                                                  float eps4)
{
    const float q1 = b1 + eps4, q2 = b2 + eps4, q3 = b3 + eps4;
    const float m = fminf(q1, fminf(q2, q3));
    const float r1 = rcp_approx(q1), r2 = rcp_approx(q2), r3 = rcp_approx(q3);
    float a1, a2, a3;
    if (scheme == 3) {
        const float tau = fabsf(b1 - b3);
        const bool big = tau > m;
        const float cr = big ? m * rcp_approx(tau) : 1.0f;
        const float t = big ? m : tau;
        const float B1 = t * r1, B2 = t * r2, B3 = t * r3;
        const float c2 = cr * cr;
        a1 = 0.1f * fmaf(B1, B1, c2);
        a2 = 0.6f * fmaf(B2, B2, c2);
        a3 = 0.3f * fmaf(B3, B3, c2);
    } else {
        const float B1 = m * r1, B2 = m * r2, B3 = m * r3;
        a1 = 0.1f * (B1 * B1);
        a2 = 0.6f * (B2 * B2);
        a3 = 0.3f * (B3 * B3);
        if (scheme == 2) {
            const float is = rcp_approx(a1 + a2 + a3);
            a1 = gk_map(a1 * is, 0.1f);
            a2 = gk_map(a2 * is, 0.6f);
            a3 = gk_map(a3 * is, 0.3f);
        }
    }
    return fmaf(a1, p1, fmaf(a2, p2, a3 * p3)) * rcp_approx(a1 + a2 + a3);
}

// Both reconstructions of one field at a face from its six stencil values x0..x5:
// plus, the left-biased WENO-5 value from x0..x4, and minus, the right-biased one
// from x5..x1 (weno(e,d,c,b,a) of the reference).
// They share two of their three second differences (x1-2x2+x3, x2-2x3+x4) with
// their squared terms, and two of their candidate polynomials (the parabola
// through x1..x3 at x2+1/2 and through x2..x4 at x3+1/2), which are computed once.
__device__ __forceinline__ void weno_pair_f32(const float* x, int scheme, float eps4, float& plus, float& minus)
{
    // second differences and the 13/3 d^2 terms of the windows centred at x1..x4
    const float d1 = fmaf(-2.0f, x[1], x[0]) + x[2], d2 = fmaf(-2.0f, x[2], x[1]) + x[3];
    const float d3 = fmaf(-2.0f, x[3], x[2]) + x[4], d4 = fmaf(-2.0f, x[4], x[3]) + x[5];
    const float c2 = (13.0f / 3.0f) * (d2 * d2), c3 = (13.0f / 3.0f) * (d3 * d3);
    // the polynomials the two share
    const float pm = fmaf(-1.0f / 6.0f, x[1], fmaf(5.0f / 6.0f, x[2], (1.0f / 3.0f) * x[3]));
    const float pn = fmaf(1.0f / 3.0f, x[2], fmaf(5.0f / 6.0f, x[3], (-1.0f / 6.0f) * x[4]));
    {
        const float p1 = fmaf(1.0f / 3.0f, x[0], fmaf(-7.0f / 6.0f, x[1], (11.0f / 6.0f) * x[2]));
        const float t2 = fmaf(3.0f, x[2], fmaf(-4.0f, x[1], x[0])), t4 = x[1] - x[3];
        const float t6 = fmaf(3.0f, x[2], fmaf(-4.0f, x[3], x[4]));
        const float b1 = fmaf(13.0f / 3.0f, d1 * d1, t2 * t2), b2 = fmaf(t4, t4, c2), b3 = fmaf(t6, t6, c3);
        plus = weno_weights_f32(b1, b2, b3, p1, pm, pn, scheme, eps4);
    }
    {
        const float p1 = fmaf(1.0f / 3.0f, x[5], fmaf(-7.0f / 6.0f, x[4], (11.0f / 6.0f) * x[3]));
        const float t2 = fmaf(3.0f, x[3], fmaf(-4.0f, x[4], x[5])), t4 = x[4] - x[2];
        const float t6 = fmaf(3.0f, x[3], fmaf(-4.0f, x[2], x[1]));
        const float b1 = fmaf(13.0f / 3.0f, d4 * d4, t2 * t2), b2 = fmaf(t4, t4, c3), b3 = fmaf(t6, t6, c2);
        minus = weno_weights_f32(b1, b2, b3, p1, pn, pm, scheme, eps4);
    }
}

// ---------------------------------------------------------------------------
// Face flux from the 6-cell stencil u[0..5] = cells (i-3 .. i+2), velocities v[0..5]
// (compute_flux, Source/compute_explicit_flux.H:245-316).  hyp_order 1 and 2 use
// u[1..4] / v[2..3] only.
__device__ __forceinline__ double face_flux_fp64(const double* u, const double* v, int hyp_order,
                                                 int scheme, double dxmin, double dt)
{
    const double vL = v[2], vR = v[3], pL = u[2], pR = u[3];
    if (hyp_order == 1) {
        double fL = pL * vL, fR = pR * vR;
        double sgn = copysign(1.0, 0.5 * (vL + vR));
        return fL * 0.5 * (1.0 + sgn) + fR * 0.5 * (1.0 - sgn);
    }
    if (hyp_order == 2) {
        double dl = pL - u[1], dm = pR - pL, dr = u[4] - pR;
        double vmid = 0.5 * (vL + vR);
        double sgn = copysign(1.0, vmid);
        double cfl = vmid * dt / dxmin;
        double fL = pL * vL, fR = pR * vR;
        double r = (cfl >= 0.0) ? dl / (dm + 1.0e-30) : dr / (dm + 1.0e-30);
        double lim = (r <= 0.0) ? 1.0 : ((r <= 1.0) ? 1.0 - (1.0 - fabs(cfl)) * r : fabs(cfl));
        return 0.5 * (fL + fR) - 0.5 * sgn * lim * (fR - fL);
    }
    double f[6];
#pragma unroll
    for (int q = 0; q < 6; q++) f[q] = u[q] * v[q];
    double lam = fabs(0.5 * (vL + vR));
    double fp = weno_fp64(f[0], f[1], f[2], f[3], f[4], scheme);
    double fm = weno_fp64(f[5], f[4], f[3], f[2], f[1], scheme);
    double up = weno_fp64(u[0], u[1], u[2], u[3], u[4], scheme);
    double um = weno_fp64(u[5], u[4], u[3], u[2], u[1], scheme);
    return 0.5 * (fp + lam * up) + 0.5 * (fm - lam * um);
}

// Mixed-precision face flux from densities already staged in FP32 (|n| < 3e38).
// The six values are scaled by an exact power of two s = 2^-e chosen from the
// exponent bits of max|u| (so max|u*s| is in [1/2, 1)); eps = 1e-20 is carried
// into the scaled units as 1e-20 s^2, clamped to [1e-30, 1e30] (for tiny fields
// eps dominates the smoothness indicators and the weights become the ideal ones,
// as in FP64).  The flux is unscaled by the exact power of two; the result is
// returned in FP32, which holds it exactly while it is a normal FP32 value (the
// FP64 route serves the one scale, 2^-127, that FP32 cannot hold).
// The first- and second-order schemes (FP64 arithmetic in both paths), out of
// line: inlined beside the WENO arithmetic they would cost the tile registers and
// instruction-cache space on every face.
static __device__ __noinline__ double face_flux_low(const double* u, const double* v, int hyp_order, int scheme,
                                                    double dxmin, double dt)
{
    return face_flux_fp64(u, v, hyp_order, scheme, dxmin, dt);
}
__device__ __forceinline__ float face_flux_mixed32(const float* u, const float* v, int hyp_order, int scheme,
                                                   double dxmin, double dt)
{
    if (hyp_order != 5) {
        double ud[6], vd[6];
#pragma unroll
        for (int q = 0; q < 6; q++) {
            ud[q] = (double)u[q];
            vd[q] = (double)v[q];
        }
        return (float)face_flux_low(ud, vd, hyp_order, scheme, dxmin, dt);
    }
    const float m = fmaxf(fmaxf(fmaxf(fabsf(u[0]), fabsf(u[1])), fmaxf(fabsf(u[2]), fabsf(u[3]))),
                          fmaxf(fabsf(u[4]), fabsf(u[5])));
    const int eb = (__float_as_int(m) >> 23) & 0xff;  // biased exponent of max|u|
    int e = 0;                                        // scale 2^-e; 0 for zero/denormal/non-finite
    if (eb > 0 && eb < 255) e = eb - 126;             // m in [2^(e-1), 2^e)
    int bs = 127 - e;
    bs = bs < 1 ? 1 : (bs > 254 ? 254 : bs);
    const float s = __int_as_float(bs << 23);
    int b2 = 127 - 2 * e;
    b2 = b2 < 0 ? 0 : (b2 > 255 ? 255 : b2);
    const float s2 = __int_as_float(b2 << 23);        // 2^-2e, 0 or inf at the ends
    const float eps = 4.0f * fminf(fmaxf(1e-20f * s2, 1e-30f), 1e30f);  // the weights take 4 eps
    float us[6], fs[6];
#pragma unroll
    for (int q = 0; q < 6; q++) {
        us[q] = u[q] * s;
        fs[q] = us[q] * v[q];
    }
    const float lam = fabsf(0.5f * (v[2] + v[3]));
    float fp, fm, up, um;
    weno_pair_f32(fs, scheme, eps, fp, fm);
    weno_pair_f32(us, scheme, eps, up, um);
    const float F = 0.5f * (fmaf(lam, up, fp) + fmaf(-lam, um, fm));
    if (bs < 254) return F * __int_as_float((254 - bs) << 23);  // 2^(127-bs)
    return (float)((double)F * __longlong_as_double((long long)(1150 - bs) << 52));
}

// ---------------------------------------------------------------------------
// WENO-5 around one cell centre.  For the values a..e of cells c-2..c+2 the
// reference reconstructs the right face of c as weno(a,b,c,d,e) (the
// left-biased value of that face) and the left face of c as weno(e,d,c,b,a) (the
// right-biased value of that face).  Both use the same three smoothness
// indicators -- the left-face ones are the right-face ones in reverse order
// (b1' = b3, b2' = b2, b3' = b1) -- and the same tau = |b1 - b3|, so everything up
// to the nonlinear weights is computed once per centre as Y_1..Y_3, with
//   WENO-Z   alpha_k = gamma_k Y_k,  Y_k = 1 + (tau/(beta_k + eps))^2
//   WENO-JS  alpha_k = gamma_k Y_k,  Y_k = 1/(beta_k + eps)^2  (M: then the map)
// at the right face and alpha'_k = gamma_k Y_(4-k) at the left face
// (Source/compute_explicit_flux.H:38-109).  The candidate polynomials are linear
// in the values; the caller evaluates them once per face and window and shares
// them between the reconstructions that use them (weno_combine_*).
struct WenoY64 {
    double y1, y2, y3;
};
__device__ __forceinline__ WenoY64 weno_center_fp64(double a, double b, double c, double d, double e, int scheme)
{
    // every product-sum written as an explicit fma or as separate roundings, so the
    // compiler contracts nothing: a centre gives the same bits wherever in a run of
    // faces it is evaluated (the tile decomposition then cannot change a result)
    constexpr double C1312 = 13.0 / 12.0;
    const double eps = 1e-20;
    const double t1 = fma(-2.0, b, a) + c, t2 = fma(3.0, c, fma(-4.0, b, a));
    const double b1 = fma(C1312 * t1, t1, 0.25 * (t2 * t2));
    const double t3 = fma(-2.0, c, b) + d, t4 = b - d;
    const double b2 = fma(C1312 * t3, t3, 0.25 * (t4 * t4));
    const double t5 = fma(-2.0, d, c) + e, t6 = fma(3.0, c, fma(-4.0, d, e));
    const double b3 = fma(C1312 * t5, t5, 0.25 * (t6 * t6));
    const double r1 = 1.0 / (b1 + eps), r2 = 1.0 / (b2 + eps), r3 = 1.0 / (b3 + eps);
    WenoY64 y;
    if (scheme == 3) {
        const double tau = fabs(b1 - b3);
        const double s1 = tau * r1, s2 = tau * r2, s3 = tau * r3;
        y.y1 = fma(s1, s1, 1.0);
        y.y2 = fma(s2, s2, 1.0);
        y.y3 = fma(s3, s3, 1.0);
    } else {
        y.y1 = r1 * r1;
        y.y2 = r2 * r2;
        y.y3 = r3 * r3;
    }
    return y;
}
// fused multiply-add in the precision of R (fmaf for float, fma for double)
template <class R> __device__ __forceinline__ R fmx(R a, R b, R c)
{
    if constexpr (sizeof(R) == sizeof(float)) return fmaf(a, b, c);
    else return fma(a, b, c);
}
// the mapping of WENO-M (Henrick et al.) with its products and sums pinned as in
// weno_center_fp64
template <class R> __device__ __forceinline__ R gk_map_pinned(R wk, R g)
{
    const R num = fmx(wk, wk, fmx(R(-3) * g, wk, g + g * g));
    const R den = fmx(wk, R(1) - R(2) * g, g * g);
    return wk * num / den;
}
// sum_k alpha_k p_k / sum_k alpha_k with alpha = gamma (0.1, 0.6, 0.3) times (y1, y2, y3)
__device__ __forceinline__ double weno_combine_fp64(double y1, double y2, double y3, double p1, double p2, double p3,
                                                    int scheme)
{
    double a1 = 0.1 * y1, a2 = 0.6 * y2, a3 = 0.3 * y3;
    if (scheme == 2) {
        const double is = 1.0 / (a1 + a2 + a3);
        a1 = gk_map_pinned(a1 * is, 0.1);
        a2 = gk_map_pinned(a2 * is, 0.6);
        a3 = gk_map_pinned(a3 * is, 0.3);
    }
    const double is = 1.0 / (a1 + a2 + a3);
    return fma(a1 * is, p1, fma(a2 * is, p2, (a3 * is) * p3));
}
// the candidate polynomials: the value at x2 + 1/2 of the parabola through a window
// (x0, x1, x2) (p1 of the reference), at x1 + 1/2 (p2) and at x0 + 1/2 (p3), each
// as two explicit fmas (no contraction left to the compiler)
template <class R> __device__ __forceinline__ R wpoly_end(R x0, R x1, R x2)
{
    return fmx(R(11) / R(6), x2, fmx(-(R(7) / R(6)), x1, (R(1) / R(3)) * x0));
}
template <class R> __device__ __forceinline__ R wpoly_mid(R x0, R x1, R x2)
{
    return fmx(R(1) / R(3), x2, fmx(R(5) / R(6), x1, -(R(1) / R(6)) * x0));
}
template <class R> __device__ __forceinline__ R wpoly_near(R x0, R x1, R x2)
{
    return fmx(-(R(1) / R(6)), x2, fmx(R(5) / R(6), x1, (R(1) / R(3)) * x0));
}



// ---------------------------------------------------------------------------
// Janev / F-fit electron-impact rates (test/Reactor/CO2_H2_Ar_mechanism_reduced/
// Chemistry.H:940-1030): with Te_eV = Te/11595, tep[j] = ln(Te_eV)^j (j = 0..8) and
// itp[j] = Te_eV^-(j+1) (j = 0..3; 1 for Te = 0),
//   Janev  k = jA exp(sum_j jc_j tep[j]) NA,   F-fit  k = fA exp(sum_j fc_j itp[j]) NA,
// the sums accumulated in order.  FP64 takes the powers with pow() as the header
// does; the mixed path by products and the exponential on the FP32 unit.
template <int PREC>
__device__ __forceinline__ void fit_powers(double Te, double* tep, double* itp, double& teev)
{
    teev = Te / TE_FIT_EV;
    const double lte = log(teev);
    const double ite = (Te == 0) ? 1.0 : 1.0 / teev;
    if (PREC == PREC_FP64) {
#pragma unroll
        for (int j = 0; j < 9; j++) tep[j] = pow(lte, (double)j);
#pragma unroll
        for (int j = 0; j < 4; j++) itp[j] = pow(ite, (double)(j + 1));
    } else {
        tep[0] = 1.0;
#pragma unroll
        for (int j = 1; j < 9; j++) tep[j] = tep[j - 1] * lte;
        itp[0] = ite;
#pragma unroll
        for (int j = 1; j < 4; j++) itp[j] = itp[j - 1] * ite;
    }
}
template <int PREC>
__device__ __forceinline__ double fit_rate(int kind, const VdFitDev& F, const double* tep, const double* itp,
                                           double teev)
{
    const bool janev = kind == VD_RATE_JANEV || (kind == VD_RATE_JANEV_FFIT && teev < F.switch_ev);
    // products and sums rounded separately as the header's loop (no contraction):
    // the sums cancel terms up to ~1e5 times larger than the result
    double sum = 0.0;
    if (janev) {
#pragma unroll
        for (int j = 0; j < 9; j++) sum = __dadd_rn(sum, __dmul_rn(F.jc[j], tep[j]));
    } else {
#pragma unroll
        for (int j = 0; j < 4; j++) sum = __dadd_rn(sum, __dmul_rn(F.fc[j], itp[j]));
    }
    if (PREC == PREC_FP64) return (janev ? F.jA : F.fA) * exp(sum) * NA_CE;
    constexpr double LOG2E = 1.4426950408889634074;
    return (double)exp2_split(fma(sum, LOG2E, janev ? F.l2jA : F.l2fA));
}

// Field-driven ionisation rate (test/verification/Streamer/Chemistry.H:266-280):
// alpha = (c0 + c1/E^3) exp(-c2/E), the attachment c3, mu_e = c4 E^c5,
// k = (alpha - c3) mu_e E, in the header's order of operations (FP64 in both paths).
__device__ __forceinline__ double townsend_rate(const double* c, double E)
{
    const double alpha = (c[0] + c[1] / pow(E, 3.0)) * exp(-c[2] / E);
    const double mu_e = c[4] * pow(E, c[5]);
    return (alpha - c[3]) * mu_e * E;
}

// ---------------------------------------------------------------------------
// CKWC for one cell (Source/ScalarSolve.cpp:143-157 + the generated productionRate,
// test/models/Ar_DC_1d/Chemistry.H:315-506).  The thread's species arrays live in
// shared memory with a stride of the block size ([species][thread]): every thread
// of a warp works on the same reaction at the same time, so sc[reac*st + tid] and
// wd[sp*st + tid] are conflict-free rows, and nothing spills to local memory.
// On entry sc[s*st] holds the number density of species s [1/m^3]; on exit
// wd[s*st] holds rxn_s [1/m^3/s]; returns the energy exchange [W/m^3].
template <int PREC>
__device__ __forceinline__ double chem_cell(double* sc, double* wd, const int st, double Te, double Tg, double EN)
{
    const int ns = c_mech.ns;
    const int eid = c_mech.e_id;
    for (int s = 0; s < ns; s++) {
        sc[s * st] = sc[s * st] * 1.0e-6 / N_A * 1.0e6;
        wd[s * st] = 0.0;
    }
    const double sce = sc[eid * st];
    const double ne = sce * NA_CE;
    const double Ue = 1.5 * Te * ne * KB_CE;
    const double mee_na = Ue / ne * NA_CE;
    const double sefact = (tanh((Te - Tg) / 0.5) + 1.0) / 2.0;
    const double dT = Te - Tg;
    double lnTe, lnTg;
    if (PREC == PREC_FP64) {
        lnTe = log(Te);
        lnTg = log(Tg);
    } else {
        lnTe = log2(Te);
        lnTg = log2(Tg);
    }
    const double invTe = 1.0 / Te, invTg = 1.0 / Tg;
    // the powers of ln(Te_eV) and 1/Te_eV the fit rates share
    // (test/Reactor/CO2_H2_Ar_mechanism_reduced/Chemistry.H:945-952)
    double tep[9], itp[4], teev = 0.0;
    if (c_mech.nfits > 0) fit_powers<PREC>(Te, tep, itp, teev);
    // the field magnitude of the field-driven rates: E = EN N 1e-21
    // (test/verification/Streamer/Chemistry.H:262-264)
    double efm = 0.0;
    if (c_mech.need_en) {
        double mix = 0.0;
        for (int s = 0; s < ns; s++) mix += sc[s * st];
        efm = EN * (mix * N_A) * 1e-21;
    }
    double ee = 0.0;
    const int nr = c_mech.nr;
    for (int r = 0; r < nr; r++) {
        const VdRxnDev& R = c_mech.rxn[r];
        double k;
        if (R.kind == VD_RATE_CONST) {
            k = R.A;
        } else if (R.kind == VD_RATE_TOWNSEND) {
            k = townsend_rate(c_mech.fits[R.fit].jc, efm);
        } else if (R.kind >= VD_RATE_JANEV) {
            k = fit_rate<PREC>(R.kind, c_mech.fits[R.fit], tep, itp, teev);
        } else {
            const bool te = (R.kind == VD_RATE_ARRHENIUS_TE);
            const double lT = te ? lnTe : lnTg;
            const double iT = te ? invTe : invTg;
            if (PREC == PREC_FP64) {
                k = exp(fma(R.b, lT, R.lnA) - R.C * iT);
            } else {
                k = (double)exp2_split(fma(R.b, lT, R.l2A) - R.Cl2 * iT);
            }
        }
        double prod = sc[R.reac[0] * st];
        for (int t = 1; t < R.nreac; t++) prod *= sc[R.reac[t] * st];
        const double q = k * prod;
        for (int t = 0; t < R.nterms; t++) {
            double* w = wd + R.sp[t] * st;
            *w = fma(R.coef[t], q, *w);
        }
        if (R.rxntype == VD_RXN_EXCITATION || R.rxntype == VD_RXN_IONIZATION) {
            ee -= R.ex * q * sefact;
        } else if (R.rxntype == VD_RXN_RECOMB || R.rxntype == VD_RXN_ATTACH) {
            ee -= mee_na * q;
        } else if (R.rxntype == VD_RXN_DETACH) {
            ee += mee_na * q;
        } else if (R.rxntype == VD_RXN_ELASTIC) {
            ee -= R.ex * dT * (sce * sc[R.elidx * st] * k) * NA_CE;
        }
    }
    if (c_mech.elastic_loss) {
        double nd = 0.0;
        for (int s = 0; s < ns; s++) nd += sc[s * st] * N_A;
        // |E| = EN N 1e-21 (the He_RF_1d header's CKWC, Chemistry.H:618); the argon
        // headers pass 0 there, with mobilities that do not read it
        double mu = mob_fp64(eid, Te, nd, Tg, EN * nd * 1.0e-21);
        double nu = -ECHARGE / ME / mu;
        ee -= 1.5 * K_B * sce * N_A * dT * nu * c_mech.elastic_coef;
    }
    for (int s = 0; s < ns; s++) wd[s * st] = wd[s * st] * 1.0e-6 * N_A * 1.0e6;
    return ee;
}

}  // namespace vd
