// Test infrastructure (oracle): a minimal AMReX-compatible surface, just large enough to compile
// the reference's own header-only hot-path physics (include/Physics_*, include/Operators_*) on the
// CPU without AMReX. Every AMReX_*.H in this directory includes only this file.
//
// Semantics follow the public AMReX API that those headers use:
//   amrex::Real = double, amrex::Array = std::array, Array4 = SoA with component stride last
//   (index i + j*jstride + k*kstride + n*nstride relative to its lower corner), amrex::min/max as
//   std::min/max, AMREX_D_DECL/AMREX_D_TERM by AMREX_SPACEDIM, amrex::Abort throws.
// Nothing here is used by the product: only the oracle build under oracle/_ref links it.
#ifndef COMPAS_ORACLE_AMREX_SHIM_CORE_H_
#define COMPAS_ORACLE_AMREX_SHIM_CORE_H_

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <limits>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#ifndef AMREX_SPACEDIM
#error "AMREX_SPACEDIM must be defined (2 or 3)"
#endif

#define AMREX_GPU_DEVICE
#define AMREX_GPU_HOST
#define AMREX_GPU_HOST_DEVICE
#define AMREX_GPU_GLOBAL
#define AMREX_FORCE_INLINE inline __attribute__((always_inline))
#define AMREX_INLINE inline
#define AMREX_RESTRICT __restrict__
#define AMREX_IF_ON_DEVICE(x)
#define AMREX_IF_ON_HOST(x) { x }
#define BL_PROFILE(x)
#define BL_PROFILE_VAR(a, b)
#define BL_PROFILE_VAR_STOP(a)
#define AMREX_ASSERT(x)
#define AMREX_ALWAYS_ASSERT(x) do { if (!(x)) amrex::Abort("assertion failed: " #x); } while (0)
#define AMREX_ALWAYS_ASSERT_WITH_MESSAGE(x, m) do { if (!(x)) amrex::Abort(m); } while (0)

#if (AMREX_SPACEDIM == 1)
#define AMREX_D_DECL(a, b, c) a
#define AMREX_D_TERM(a, b, c) a
#define AMREX_D_PICK(a, b, c) a
#elif (AMREX_SPACEDIM == 2)
#define AMREX_D_DECL(a, b, c) a, b
#define AMREX_D_TERM(a, b, c) a b
#define AMREX_D_PICK(a, b, c) b
#else
#define AMREX_D_DECL(a, b, c) a, b, c
#define AMREX_D_TERM(a, b, c) a b c
#define AMREX_D_PICK(a, b, c) c
#endif

namespace amrex {

using Real = double;
using Long = long long;

constexpr Real operator""_rt(long double x) { return static_cast<Real>(x); }
constexpr Real operator""_rt(unsigned long long x) { return static_cast<Real>(x); }

template <class T, std::size_t N>
using Array = std::array<T, N>;

template <class T>
using Vector = std::vector<T>;

template <class T, int N>
struct GpuArray {
    T arr[N];
    T& operator[](int i) { return arr[i]; }
    const T& operator[](int i) const { return arr[i]; }
    T* data() { return arr; }
    const T* data() const { return arr; }
};

struct Dim3 { int x, y, z; };

template <class T>
constexpr const T& min(const T& a, const T& b) { return std::min(a, b); }
template <class T>
constexpr const T& max(const T& a, const T& b) { return std::max(a, b); }
template <class T, class... Ts>
constexpr const T& min(const T& a, const T& b, const Ts&... c) { return min(min(a, b), c...); }
template <class T, class... Ts>
constexpr const T& max(const T& a, const T& b, const Ts&... c) { return max(max(a, b), c...); }
template <class T>
constexpr T Math_abs(T a) { return std::abs(a); }
namespace Math {
template <class T>
constexpr T abs(T a) { return std::abs(a); }
}  // namespace Math

[[noreturn]] inline void Abort(const std::string& msg = "") { throw std::runtime_error(msg); }
[[noreturn]] inline void Abort(const char* msg) { throw std::runtime_error(msg ? msg : ""); }
inline void Warning(const std::string&) {}

template <class... Ts>
AMREX_FORCE_INLINE void ignore_unused(const Ts&...) {}

// SoA array view with its lower corner at begin; component stride last.
template <class T>
struct Array4 {
    T* p = nullptr;
    Long jstride = 0, kstride = 0, nstride = 0;
    Dim3 begin{0, 0, 0};
    Dim3 end{1, 1, 1};
    int ncomp = 1;

    Array4() = default;
    Array4(T* ptr, Dim3 lo, Dim3 hi_plus_one, int nc)
        : p(ptr), begin(lo), end(hi_plus_one), ncomp(nc) {
        jstride = (Long)(end.x - begin.x);
        kstride = jstride * (Long)(end.y - begin.y);
        nstride = kstride * (Long)(end.z - begin.z);
    }
    template <class U, class = typename std::enable_if<std::is_same<const U, T>::value>::type>
    Array4(const Array4<U>& a)
        : p(a.p), jstride(a.jstride), kstride(a.kstride), nstride(a.nstride),
          begin(a.begin), end(a.end), ncomp(a.ncomp) {}

    T& operator()(int i, int j, int k, int n = 0) const {
        return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride + n * nstride];
    }
};

// Parameters are filled directly by the oracle driver; queries leave the defaults untouched.
class ParmParse {
public:
    explicit ParmParse(const std::string& = "") {}
    template <class T> bool query(const char*, T&) const { return false; }
    template <class T> bool query(const char*, T&, int) const { return false; }
    template <class T> bool queryarr(const char*, T&) const { return false; }
    template <class T> bool queryAdd(const char*, T&) const { return false; }
    template <class T> void get(const char* name, T&) const {
        Abort(std::string("ParmParse::get not available in the oracle shim: ") + name);
    }
    template <class T> void getarr(const char* name, T&) const {
        Abort(std::string("ParmParse::getarr not available in the oracle shim: ") + name);
    }
    bool contains(const char*) const { return false; }
    int countval(const char*) const { return 0; }
};

struct PrintSink {
    template <class T> PrintSink& operator<<(const T&) { return *this; }
    PrintSink& operator<<(std::ostream& (*)(std::ostream&)) { return *this; }
};
inline PrintSink Print(int = 0) { return PrintSink{}; }
inline PrintSink AllPrint() { return PrintSink{}; }

// Compile-only stand-ins for the host loops over whole MultiFabs that some physics headers define
// next to their cell functions (e.g. PressureRelaxationInstantaneous of the N-phase six-equation
// model). The oracle calls the cell functions itself; constructing an MFIter aborts.
struct Box {};
class MultiFab;
class MFIter {
public:
    MFIter(const MultiFab&, bool) { Abort("MultiFab loops are not available in the oracle shim"); }
    bool isValid() const { return false; }
    MFIter& operator++() { return *this; }
    Box tilebox() const { return Box{}; }
};
class MultiFab {
public:
    Array4<Real const> const_array(const MFIter&) const { return Array4<Real const>(); }
    Array4<Real> array(const MFIter&) { return Array4<Real>(); }
};
inline bool TilingIfNotGPU() { return false; }
template <class F>
void ParallelFor(const Box&, F&&) {}

}  // namespace amrex

using amrex::operator""_rt;

#endif
