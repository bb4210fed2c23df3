// mg_tangent.cuh — forward-mode (tangent-linear) derivatives of the V-cycle.
//
// A Dual carries a value and its derivative along one parameter direction.  Each
// operation computes the value exactly as the FP64 engine does (same operation, same
// order, no contraction: the engine is built with --fmad=false), so the value part of
// a tangent run has the bits of the plain run, and the derivative part follows by the
// chain rule.  Branches and comparisons look at values only.  The non-smooth points
// take the derivative a central difference sees there: |x| at x = 0 has derivative
// 0, max(a, b) at a tie the mean of both.
//
// Tan is the access type (see Prim in mg_cells.cuh) of one level of a tangent run:
// every array a parameter can change has a derivative array of the same layout
// (LevelTan::t, indexed by slot); face areas and obstacle sources do not depend on
// the parameters and are read as plain FP64.
#pragma once

#include "mg_cells.cuh"

namespace mg {

struct Dual {
    double v, d;
    Dual() = default;
    __host__ __device__ constexpr Dual(double x) : v(x), d(0.0) {}
    __host__ __device__ constexpr Dual(double x, double y) : v(x), d(y) {}
};

__device__ __forceinline__ Dual operator-(const Dual &a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator+(const Dual &a, const Dual &b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator+(const Dual &a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, const Dual &b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(const Dual &a, const Dual &b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(const Dual &a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, const Dual &b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(const Dual &a, const Dual &b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator*(const Dual &a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, const Dual &b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(const Dual &a, const Dual &b)
{
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator/(const Dual &a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Dual operator/(double a, const Dual &b)
{
    const double q = a / b.v;
    return {q, -(q * b.d) / b.v};
}

__device__ __forceinline__ double val(const Dual &x) { return x.v; }
__device__ __forceinline__ Dual gabs(const Dual &x) { return {fabs(x.v), x.v > 0.0 ? x.d : x.v < 0.0 ? -x.d : 0.0}; }
__device__ __forceinline__ Dual gmax(const Dual &a, const Dual &b)
{
    if (a.v > b.v) return a;
    if (b.v > a.v) return b;
    return {fmax(a.v, b.v), 0.5 * (a.d + b.d)};
}

// Derivative storage of one level: one array per slot (nullptr for the slots the
// parameters cannot change), the pressure-copy buffer's derivative, and the
// derivatives of the level's viscosity and scalar diffusivity.
struct LevelTan {
    double *t[NSLOTS];
    double *pbuf_t;
    double amu_t, amusc_t;
};
struct CaseTan {
    LevelTan lv[MAXLEV];
};

struct Tan {
    using T = Dual;
    const LevelDev &L;
    const LevelTan &D;
    __device__ __forceinline__ Dual ld(int s, int q) const { return {L.f[s][q], D.t[s][q]}; }
    __device__ __forceinline__ void st(int s, int q, const Dual &x) const
    {
        L.f[s][q] = x.v;
        D.t[s][q] = x.d;
    }
    __device__ __forceinline__ double g(int s, int q) const { return L.f[s][q]; }
    __device__ __forceinline__ Dual amu() const { return {L.amu, D.amu_t}; }
    __device__ __forceinline__ Dual amusc() const { return {L.amusc, D.amusc_t}; }
    __device__ __forceinline__ Dual pb(int k) const { return {L.pbuf[k], D.pbuf_t[k]}; }
    __device__ __forceinline__ void set_pb(int k, const Dual &x) const
    {
        L.pbuf[k] = x.v;
        D.pbuf_t[k] = x.d;
    }
};

// The levels of one case as seen by the one-CTA kernel.
struct TanCase {
    const CaseDev &C;
    const CaseTan &D;
    __device__ __forceinline__ Tan io(int ig) const { return Tan{C.lv[ig], D.lv[ig]}; }
};

// Slots with no derivative: geometry and obstacle sources (read through IO::g), the
// previous-cycle level-0 state of the stop rule (plain FP64 bookkeeping).
__host__ __device__ constexpr bool tangent_slot(int s)
{
    return s != S_AREAX && s != S_AREAY && s != S_SPU && s != S_SPV && s != S_SPSC && s != S_RS && s < NSLOTS_LEVEL;
}

}  // namespace mg
