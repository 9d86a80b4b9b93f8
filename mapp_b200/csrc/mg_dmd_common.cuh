// Device helpers shared by the FP64 (mg_dmd.cu), FP32 (mg_dmd32.cu) and learned
// (mg_mlp.cu) DMD kernels.
#pragma once

#include "mg_internal.h"

namespace mg {
namespace {

constexpr double kPiInSq = 0.564189583547756286948079451561;  // 1/sqrt(pi)

__device__ __forceinline__ int owner(const Dev& d, int j) { return j < d.natms ? j : d.root[j]; }

// c0..c3 of one spline knot (rows of 8 doubles, 64-byte aligned) as one
// read-only 32-byte load (one sector, one request per lane)
__device__ __forceinline__ double4 knot4(const double* __restrict__ row)
{
    double4 r;
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(row));
    return r;
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
    // the upper clamp is the reference's (nr - 2, defect kept); the lower one
    // only matters for a negative density, which the learned form's untrained
    // network can produce: the first knot's polynomial is extrapolated instead
    // of reading before the table
    int m = max(0, min((int)p, d.nr - 2));
    p -= m;
    p = fmin(p, 1.0);
    double p2 = p * p, p3 = p2 * p, p4 = p3 * p;
    const double* cf = d.FT + ((size_t)a * (d.nrho + 1) + m) * d.Fw;
    tmp0 = cf[4] * p4 + cf[3] * p3 + cf[2] * p2 + cf[1] * p + cf[0];
    tmp1 = cf[8] * p3 + cf[7] * p2 + cf[6] * p + cf[5];
    if (Ev > d.rho_max) tmp0 += tmp1 * (Ev - d.rho_max);
    if (dd) *dd = (3.0 * cf[8] * p2 + cf[7] * p + cf[6]) * d.drho_inv;
}

// One species pair of one site pair: the Gauss-Hermite smearing of r*rho and
// r*phi (ff_dmd_I.cpp:178-259) or the plain EAM values above alpha_max
// (ff_dmd_I.cpp:261-310).  Returns false when the reference writes nothing.
//
// NQ > 0 fixes the node count at compile time so the node loop unrolls and
// the table loads of all nodes issue together; NQ = 0 reads it from d.nq.
// The branch-deciding quantities (alpha against alpha_min / alpha_max, rsq
// against the cut-offs) are computed exactly as the reference does; powers of
// alpha and 1/r come from rsqrt, which moves results by ulps only (the node and
// table-index decisions they feed are continuous in the result).
// kPack: read the node knots from the paired table d.pk64 (record kslot =
// a*nt+b of the ordered species pair, rho at +0, phi at +4) instead of the
// separate rho / phi tables; the coefficients are the same doubles.
template <bool kPhi, bool kDeriv, int NQ, bool kPack = false>
__device__ __forceinline__ bool smear(const Dev& d, int rslot, int pslot, double r, double r_inv, double rsq,
                                      double alpha, double& g0, double& g_dr, double& g_da, double& f0, double& f_dr,
                                      double& f_da, int kslot = 0)
{
    if (d.alpha_min < alpha && alpha < d.alpha_max) {
        const int nq = NQ > 0 ? NQ : d.nq;
        double inv_asq = rsqrt(alpha);
        double asq = alpha * inv_asq;
        double inv_alpha = inv_asq * inv_asq;
        double upper = (r + d.rc) * asq, lower = (r - d.rc) * asq;
        if (!(lower < d.xi[nq - 1])) return false;
        double fa = 0.0, fb = 0.0, fc = 0.0, ga = 0.0, gb = 0.0, gc = 0.0;
        const double* rt = kPack ? d.pk64 + (size_t)kslot * d.nr * 8 : d.rhoT + (size_t)rslot * d.nr * 8;
        const double* pt = kPack ? rt + 4 : d.phiT + (size_t)pslot * d.nr * 8;
#pragma unroll
        for (int q = 0; q < (NQ > 0 ? NQ : kMaxQuad); q++) {
            if (NQ == 0 && q >= nq) break;
            double xq = d.xi[q];
            if (xq > lower && xq < upper) {
                double tmp0 = r - xq * inv_asq;
                double p = fabs(tmp0) * d.dr_inv;
                int m = min((int)p, d.nr - 2);
                p -= m;
                p = fmin(p, 1.0);
                double p2 = p * p, p3 = p2 * p;
                double4 cr = knot4(rt + 8 * m);
                double tmp2 = (cr.w * p3 + cr.z * p2 + cr.y * p + cr.x) * tmp0;
                ga += d.w0[q] * tmp2;
                if (kDeriv) {
                    gb += d.w1[q] * tmp2;
                    gc += d.w2[q] * tmp2;
                }
                if (kPhi) {
                    double4 cp = knot4(pt + 8 * m);
                    double tmp1 = cp.w * p3 + cp.z * p2 + cp.y * p + cp.x;
                    if (tmp0 < 0.0) tmp1 = -tmp1;
                    fa += d.w0[q] * tmp1;
                    if (kDeriv) {
                        fb += d.w1[q] * tmp1;
                        fc += d.w2[q] * tmp1;
                    }
                }
            }
        }
        double sc = kPiInSq * r_inv;
        g0 = ga * sc;
        if (kDeriv) {
            gb *= sc;
            gc *= sc;
            g_dr = -g0 * r_inv - 2.0 * asq * gb;
            g_da = (0.5 * g0 - gc) * inv_alpha;
        }
        if (kPhi) {
            f0 = fa * sc;
            if (kDeriv) {
                fb *= sc;
                fc *= sc;
                f_dr = -f0 * r_inv - 2.0 * asq * fb;
                f_da = (0.5 * f0 - fc) * inv_alpha;
            }
        }
        return true;
    }
    if (d.alpha_max <= alpha) {
        if (!(rsq < d.cut_sq)) return false;
        double p = r * d.dr_inv;
        int m = min((int)p, d.nr - 2);
        p -= m;
        p = fmin(p, 1.0);
        double p2 = p * p, p3 = p2 * p;
        const double* cr = d.rhoT + ((size_t)rslot * d.nr + m) * 8;
        g0 = cr[3] * p3 + cr[2] * p2 + cr[1] * p + cr[0];
        if (kDeriv) {
            g_da = 0.0;
            g_dr = cr[6] * p2 + cr[5] * p + cr[4];
        }
        if (kPhi) {
            const double* cp = d.phiT + ((size_t)pslot * d.nr + m) * 8;
            double z2 = cp[3] * p3 + cp[2] * p2 + cp[1] * p + cp[0];
            f0 = z2 * r_inv;
            if (kDeriv) {
                double z2p = cp[6] * p2 + cp[5] * p + cp[4];
                f_da = 0.0;
                f_dr = (z2p - z2 * r_inv) * r_inv;
            }
        }
        return true;
    }
    return false;
}

constexpr float kPiInSqF = 0.564189583547756286948079451561f;

struct F32Consts {
    float rc, dr_inv, alpha_min, alpha_max;
    int nr;
    float top, top_m;  // nr - 1 and nr - 2 as floats
};

__device__ __forceinline__ F32Consts f32_consts(const Dev& d)
{
    F32Consts c;
    c.rc = (float)d.rc;
    c.dr_inv = (float)d.dr_inv;
    c.alpha_min = (float)d.alpha_min;
    c.alpha_max = (float)d.alpha_max;
    c.nr = d.nr;
    c.top = (float)(d.nr - 1);
    c.top_m = (float)(d.nr - 2);
    return c;
}

// FP32 counterpart of smear(): one species pair of one site pair, tables
// packed one 32-byte sector per knot {rho c0..c3, phi c0..c3} (pk).
// one knot row of the packed table: read-only cache load from global memory,
// or a plain load when the table is a shared-memory copy (ld.global.nc must
// not be given a shared-memory address)
template <bool kShared>
__device__ __forceinline__ float4 knot_f(const float4* p)
{
    if (kShared) return *p;
    return __ldg(p);
}

// floor of 0 <= p < 2^22 as an int and as a float by the round-to-nearest of
// p - 1/2 against 1.5 * 2^23, on the FP32 / integer pipes instead of the
// conversion unit; at an exact integer p it may give p - 1 (then p - m = 1,
// the end of the previous interval, where the spline takes the same value)
__device__ __forceinline__ int floor_idx(float p, float& fm)
{
    const float t = __fadd_rn(__fadd_rn(p, -0.5f), 12582912.0f);
    fm = __fadd_rn(t, -12582912.0f);
    return __float_as_int(t) - 0x4B400000;
}

template <bool kPhi, int NQ, bool kShared = false>
__device__ __forceinline__ bool smear_f(const Dev& d, const F32Consts& k, const float4* __restrict__ pk, float r,
                                        float r_inv, bool below_rc, float alpha, float& g0, float& g_dr, float& g_da,
                                        float& f0, float& f_dr, float& f_da)
{
    if (k.alpha_min < alpha && alpha < k.alpha_max) {
        const int nq = NQ > 0 ? NQ : d.nq;
        float inv_asq = rsqrtf(alpha);
        float asq = alpha * inv_asq;
        float inv_alpha = inv_asq * inv_asq;
        float upper = (r + k.rc) * asq, lower = (r - k.rc) * asq;
        if (!(lower < d.xi_f[nq - 1])) return false;
        float fa = 0.f, fb = 0.f, fc = 0.f, ga = 0.f, gb = 0.f, gc = 0.f;
#pragma unroll
        for (int q = 0; q < (NQ > 0 ? NQ : kMaxQuad); q++) {
            if (NQ == 0 && q >= nq) break;
            float xq = d.xi_f[q];
            if (xq > lower && xq < upper) {
                float tmp0 = r - xq * inv_asq;
                float p = fminf(fabsf(tmp0) * k.dr_inv, k.top);
                float fm;
                int m = floor_idx(p, fm);
                if (m > k.nr - 2) {
                    m = k.nr - 2;
                    fm = k.top_m;
                }
                p -= fm;
                p = fminf(p, 1.0f);
                float p2 = p * p, p3 = p2 * p;
                float4 cr = knot_f<kShared>(pk + 2 * m);
                float tmp2 = (cr.w * p3 + cr.z * p2 + cr.y * p + cr.x) * tmp0;
                float w0 = d.w0_f[q], w1 = d.w1_f[q], w2 = d.w2_f[q];
                ga += w0 * tmp2;
                gb += w1 * tmp2;
                gc += w2 * tmp2;
                if (kPhi) {
                    float4 cp = knot_f<kShared>(pk + 2 * m + 1);
                    float tmp1 = cp.w * p3 + cp.z * p2 + cp.y * p + cp.x;
                    if (tmp0 < 0.0f) tmp1 = -tmp1;
                    fa += w0 * tmp1;
                    fb += w1 * tmp1;
                    fc += w2 * tmp1;
                }
            }
        }
        float sc = kPiInSqF * r_inv;
        g0 = ga * sc;
        gb *= sc;
        gc *= sc;
        g_dr = -g0 * r_inv - 2.0f * asq * gb;
        g_da = (0.5f * g0 - gc) * inv_alpha;
        if (kPhi) {
            f0 = fa * sc;
            fb *= sc;
            fc *= sc;
            f_dr = -f0 * r_inv - 2.0f * asq * fb;
            f_da = (0.5f * f0 - fc) * inv_alpha;
        }
        return true;
    }
    if (k.alpha_max <= alpha) {
        if (!below_rc) return false;
        float p = fminf(r * k.dr_inv, k.top);
        float fm;
        int m = floor_idx(p, fm);
        if (m > k.nr - 2) {
            m = k.nr - 2;
            fm = k.top_m;
        }
        p -= fm;
        p = fminf(p, 1.0f);
        float p2 = p * p, p3 = p2 * p;
        float4 cr = knot_f<kShared>(pk + 2 * m);
        g0 = cr.w * p3 + cr.z * p2 + cr.y * p + cr.x;
        g_da = 0.0f;
        g_dr = (cr.y + 2.0f * cr.z * p + 3.0f * cr.w * p2) * k.dr_inv;
        if (kPhi) {
            float4 cp = knot_f<kShared>(pk + 2 * m + 1);
            float z2 = cp.w * p3 + cp.z * p2 + cp.y * p + cp.x;
            float z2p = (cp.y + 2.0f * cp.z * p + 3.0f * cp.w * p2) * k.dr_inv;
            f0 = z2 * r_inv;
            f_da = 0.0f;
            f_dr = (z2p - z2 * r_inv) * r_inv;
        }
        return true;
    }
    return false;
}

// pair scratch of the running form: FP64 (plain) or FP32 (precision form)
template <typename P>
__device__ __forceinline__ const P* pr_ptr(const Dev& d);
template <>
__device__ __forceinline__ const double* pr_ptr<double>(const Dev& d) { return d.pr; }
template <>
__device__ __forceinline__ const float* pr_ptr<float>(const Dev& d) { return d.prf; }

// the per-pair densities (q = b*nt+a of species pair (a, b)) and pair energies
// (q = COMP(a, b)) that c_d_calc and calc_g read, at a list entry's slot: the
// pair scratch of the force call at the compact pair index, or, while the
// active sublist is on, its contiguous copy at the entry's CSR index
template <int NT, typename P>
struct PairVals {
    const P* pr;
    const double* av;
    long long pstride, astride;
    bool act;
    __device__ __forceinline__ explicit PairVals(const Dev& d)
        : pr(pr_ptr<P>(d)), av(d.act_pv), pstride(d.maxp), astride(d.act_cap), act(d.act_on != 0)
    {
    }
    __device__ __forceinline__ double rho(int q, long long slot) const
    {
        return act ? av[(size_t)q * astride + slot] : (double)pr[(size_t)(Slots<NT>::RHO + q) * pstride + slot];
    }
    __device__ __forceinline__ double phi(int q, long long slot) const
    {
        return act ? av[(size_t)(NT * NT + q) * astride + slot]
                   : (double)pr[(size_t)(Slots<NT>::PHI + q) * pstride + slot];
    }
};

}  // namespace
}  // namespace mg
