// Device helpers shared by the FP64 (mg_dmd.cu) and FP32 (mg_dmd32.cu) DMD kernels.
#pragma once

#include "mg_internal.h"

namespace mg {
namespace {

constexpr double kPiInSq = 0.564189583547756286948079451561;  // 1/sqrt(pi)

__device__ __forceinline__ int owner(const Dev& d, int j) { return j < d.natms ? j : d.root[j]; }

// c0..c3 of one spline knot (rows of 8 doubles, 64-byte aligned) as two
// read-only 16-byte loads
__device__ __forceinline__ double4 knot4(const double* __restrict__ row)
{
    double2 lo = __ldg(reinterpret_cast<const double2*>(row));
    double2 hi = __ldg(reinterpret_cast<const double2*>(row) + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}

template <int NT>
struct Slots {
    static constexpr int NC = NT * (NT + 1) / 2;
    static constexpr int RHO = 0, DRR = NT * NT, DRA = 2 * NT * NT, PHI = 3 * NT * NT, DPR = 3 * NT * NT + NC,
                         DPA = 3 * NT * NT + 2 * NC, TOTAL = 3 * NT * NT + 3 * NC;
};

__device__ __forceinline__ double calc_ent(double x)
{
    if (x < 1.0e-8 || 0.99999999 < x) return 0.0;
    return x * log(x) + (1 - x) * log(1 - x);
}

// F(E), F'(E) (and F''(E)) from the quartic embedding spline (ff_dmd_I.cpp:322-341,
// interpolate_m ff_dmd_I.cpp:1794-1836); index clamp nr-2 as in the reference.
__device__ __forceinline__ void embed_F(const Dev& d, int a, double Ev, double& tmp0, double& tmp1, double* dd)
{
    double p = Ev * d.drho_inv;
    int m = min((int)p, d.nr - 2);
    p -= m;
    p = fmin(p, 1.0);
    double p2 = p * p, p3 = p2 * p, p4 = p3 * p;
    const double* cf = d.FT + ((size_t)a * (d.nrho + 1) + m) * d.Fw;
    tmp0 = cf[4] * p4 + cf[3] * p3 + cf[2] * p2 + cf[1] * p + cf[0];
    tmp1 = cf[8] * p3 + cf[7] * p2 + cf[6] * p + cf[5];
    if (Ev > d.rho_max) tmp0 += tmp1 * (Ev - d.rho_max);
    if (dd) *dd = (3.0 * cf[8] * p2 + cf[7] * p + cf[6]) * d.drho_inv;
}

// pair scratch of the running form: FP64 (plain) or FP32 (precision form)
template <typename P>
__device__ __forceinline__ const P* pr_ptr(const Dev& d);
template <>
__device__ __forceinline__ const double* pr_ptr<double>(const Dev& d) { return d.pr; }
template <>
__device__ __forceinline__ const float* pr_ptr<float>(const Dev& d) { return d.prf; }

}  // namespace
}  // namespace mg
