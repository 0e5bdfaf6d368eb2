/*
 * vd_amrex_shim.H -- minimal stand-in for the AMReX types and macros that the
 * reference's hot-path headers use (TEST INFRASTRUCTURE ONLY).
 *
 * Lets Source/compute_explicit_flux.H, Source/PlasmaChem.H, Source/UnivConstants.H,
 * Source/VarDefines.H and a case's Chemistry.H / UserFunctions.H / ProbParm.H
 * compile unmodified with g++ on the CPU.  AMReX itself is not available here.
 * Only what those headers touch is provided: Real, Long, IntVect, Dim3, Array4,
 * GpuArray, Vector, Math::abs, min, Abort and the GPU/inline/dimension macros.
 */
#ifndef VD_AMREX_SHIM_H
#define VD_AMREX_SHIM_H

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <stdexcept>

#ifndef AMREX_SPACEDIM
#error "compile with -DAMREX_SPACEDIM=1|2|3"
#endif

#if AMREX_SPACEDIM == 1
#define AMREX_D_DECL(a, b, c) a
#elif AMREX_SPACEDIM == 2
#define AMREX_D_DECL(a, b, c) a, b
#else
#define AMREX_D_DECL(a, b, c) a, b, c
#endif

#define AMREX_GPU_DEVICE
#define AMREX_GPU_HOST_DEVICE
#define AMREX_GPU_CONSTANT
#define AMREX_GPU_DEVICE_MANAGED
#define AMREX_FORCE_INLINE inline
#define AMREX_INLINE inline
#define AMREX_DEVICE_COMPILE 0
#define AMREX_RESTRICT __restrict__
#define AMREX_PRAGMA_SIMD

namespace amrex {
using Real = double;
using Long = long long;
namespace literals {}

struct Dim3 { int x, y, z; };

struct IntVect {
    int vect[AMREX_SPACEDIM];
    IntVect(AMREX_D_DECL(int i, int j, int k)) : vect{AMREX_D_DECL(i, j, k)} {}
    int& operator[](int d) { return vect[d]; }
    const int& operator[](int d) const { return vect[d]; }
};

template <class T, int N>
struct GpuArray {
    T arr[N];
    T& operator[](int i) { return arr[i]; }
    const T& operator[](int i) const { return arr[i]; }
};

template <class T>
struct Array4 {
    T* p;
    Long jstride, kstride, nstride;
    Dim3 begin, end;
    int ncomp;
    T& operator()(int i, int j, int k) const
    {
        return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride];
    }
    T& operator()(int i, int j, int k, int n) const
    {
        return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride + n * nstride];
    }
#if AMREX_SPACEDIM == 1
    T& operator()(IntVect const& v) const { return (*this)(v[0], 0, 0); }
    T& operator()(IntVect const& v, int n) const { return (*this)(v[0], 0, 0, n); }
#elif AMREX_SPACEDIM == 2
    T& operator()(IntVect const& v) const { return (*this)(v[0], v[1], 0); }
    T& operator()(IntVect const& v, int n) const { return (*this)(v[0], v[1], 0, n); }
#else
    T& operator()(IntVect const& v) const { return (*this)(v[0], v[1], v[2]); }
    T& operator()(IntVect const& v, int n) const { return (*this)(v[0], v[1], v[2], n); }
#endif
};

template <class T>
class Vector : public std::vector<T> {
  public:
    using std::vector<T>::vector;
};

namespace Math {
template <class T> inline T abs(T x) { return std::abs(x); }
}

template <class T> inline T min(T a) { return a; }
template <class T, class... R> inline T min(T a, R... r)
{
    T b = min(r...);
    return (a < b) ? a : b;
}

[[noreturn]] inline void Abort(const char* msg) { throw std::runtime_error(msg); }
[[noreturn]] inline void Abort(const std::string& msg) { throw std::runtime_error(msg); }
} // namespace amrex

#endif
