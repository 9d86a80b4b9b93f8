// FP32 smearing on the split table (Dev::pkS): the precision form's
// arithmetic of ForceField_DMD_I::force_calc's quadrature (ff_dmd_I.cpp:
// 178-310), shared by its force kernels (mg_dmd32.cu) and the learned form's
// quadrature fallback (mg_mlp_tc.cu).  The table pointers may be a
// shared-memory copy or the table in global memory.
#pragma once

#include "mg_internal.h"
#include "mg_dmd_common.cuh"

namespace mg {
namespace {

// ---- split-table smearing ---------------------------------------------------

struct SplitK {
    float rc, dr_inv, top, alpha_min, alpha_max;
};

// copies the first nslots slots of the split table into shared memory
__device__ __forceinline__ void load_split_table(const Dev& d, float4* sh, int nslots)
{
    const int n = nslots * d.nrS;
    for (int k = threadIdx.x; k < n; k += blockDim.x) sh[k] = __ldg(d.pkS + k);
    __syncthreads();
}

__device__ __forceinline__ SplitK split_consts(const Dev& d)
{
    SplitK k;
    k.rc = (float)d.rc;
    k.dr_inv = d.drS_inv;
    k.top = (float)(d.nrS - 1);
    k.alpha_min = (float)d.alpha_min;
    k.alpha_max = (float)d.alpha_max;
    return k;
}

// knot row and fraction of |x| on the split table: p = min(|x| / h, K - 1),
// row = floor(p) by a round-down add against 1.5 * 2^23 (exact for
// 0 <= p < 2^22; FP32 pipe, no conversion instruction), t = p - row in [0, 1)
struct Knot {
    int row;
    float t;
};

__device__ __forceinline__ Knot knot_at(float x, const SplitK& k)
{
    const float p = fminf(fabsf(x) * k.dr_inv, k.top);
    const float f = __fadd_rd(p, 12582912.0f);
    Knot r;
    r.row = __float_as_int(f) - 0x4B400000;
    r.t = p - (f - 12582912.0f);
    return r;
}

__device__ __forceinline__ float horner(const float4 c, float t) { return fmaf(fmaf(fmaf(c.w, t, c.z), t, c.y), t, c.x); }

__device__ __forceinline__ float horner_d(const float4 c, float t)
{
    return fmaf(fmaf(3.0f * c.w, t, 2.0f * c.z), t, c.y);
}

// v with the sign of t (the odd extension of r*phi, ff_dmd_I.cpp:214-215):
// one bit operation
__device__ __forceinline__ float with_sign_of(float v, float t)
{
    return __int_as_float(__float_as_int(v) ^ (__float_as_int(t) & 0x80000000));
}

// Node positions t_q = r - xi_q / sqrt(alpha) of the quadrature.  The
// reference's node test (ff_dmd_I.cpp:198) is |t_q| < rc; the table's zero
// row for |x| >= rc makes a rejected node add an exact zero, so no node is
// tested.  NQ = 3: three nodes whose middle one is 0, so it sits at r (knot
// k0); NQ = 0: d.nq nodes.
//
// kInRange: the caller has established alpha_min < alpha < alpha_max.

// Value of the smeared density of one ordered species pair (rho slot tr).
template <int NQ, bool kInRange>
__device__ __forceinline__ float dens_value(const Dev& d, const float4* tr, const SplitK& k, float r, float r_inv,
                                            bool below_rc, float alpha, const Knot& k0)
{
    if (kInRange || (k.alpha_min < alpha && alpha < k.alpha_max)) {
        const float ias = rsqrtf(alpha);
        float ga;
        if (NQ == 3) {
            const float tm = fmaf(-d.xi_f[0], ias, r), tp = fmaf(-d.xi_f[2], ias, r);
            const Knot km = knot_at(tm, k), kp = knot_at(tp, k);
            ga = d.w0_f[0] * (horner(tr[km.row], km.t) * tm);
            ga = fmaf(d.w0_f[1], horner(tr[k0.row], k0.t) * r, ga);
            ga = fmaf(d.w0_f[2], horner(tr[kp.row], kp.t) * tp, ga);
        } else {
            ga = 0.0f;
            for (int q = 0; q < d.nq; q++) {
                const float t0 = fmaf(-d.xi_f[q], ias, r);
                const Knot kq = knot_at(t0, k);
                ga = fmaf(d.w0_f[q], horner(tr[kq.row], kq.t) * t0, ga);
            }
        }
        return ga * kPiInSqF * r_inv;
    }
    if (k.alpha_max <= alpha && below_rc) return horner(tr[k0.row], k0.t);
    return 0.0f;
}

// Value of the smeared r*phi of one species pair (phi slot tp) over r: the
// pair energy term of ff_dmd_I.cpp:226-231 (values only).
template <int NQ>
__device__ __forceinline__ float phi_value(const Dev& d, const float4* tp, const SplitK& k, float r, float r_inv,
                                           bool below_rc, float alpha, const Knot& k0)
{
    if (k.alpha_min < alpha && alpha < k.alpha_max) {
        const float ias = rsqrtf(alpha);
        float fa = 0.0f;
        const int nq = NQ == 3 ? 3 : d.nq;
        for (int q = 0; q < (NQ == 3 ? 3 : kMaxQuad); q++) {
            if (q >= nq) break;
            const float t0 = (NQ == 3 && q == 1) ? r : fmaf(-d.xi_f[q], ias, r);
            const Knot kq = (NQ == 3 && q == 1) ? k0 : knot_at(t0, k);
            fa = fmaf(d.w0_f[q], with_sign_of(horner(tp[kq.row], kq.t), t0), fa);
        }
        return fa * kPiInSqF * r_inv;
    }
    if (k.alpha_max <= alpha && below_rc) return horner(tp[k0.row], k0.t) * r_inv;
    return 0.0f;
}

// value and r / alpha derivatives of one smeared function
struct VDer {
    float v, dr, da;
};

// Full smearing of one ordered species pair (ff_dmd_I.cpp:178-310): the rho
// slot tr always, the phi slot tp when kPhi; values and both derivatives with
// the reference's closing algebra (ff_dmd_I.cpp:231-259, 261-310).
template <int NQ, bool kPhi, bool kInRange>
__device__ __forceinline__ void smear_full(const Dev& d, const float4* tr, const float4* tp, const SplitK& k, float r,
                                           float r_inv, bool below_rc, float alpha, const Knot& k0, VDer& g, VDer& f)
{
    g.v = g.dr = g.da = 0.0f;
    f.v = f.dr = f.da = 0.0f;
    if (kInRange || (k.alpha_min < alpha && alpha < k.alpha_max)) {
        const float ias = rsqrtf(alpha), as = alpha * ias, inv_alpha = ias * ias;
        float ga = 0.f, gb = 0.f, gc = 0.f, fa = 0.f, fb = 0.f, fc = 0.f;
        const int nq = NQ == 3 ? 3 : d.nq;
#pragma unroll
        for (int q = 0; q < (NQ == 3 ? 3 : kMaxQuad); q++) {
            if (NQ != 3 && q >= nq) break;
            const float t0 = (NQ == 3 && q == 1) ? r : fmaf(-d.xi_f[q], ias, r);
            const Knot kq = (NQ == 3 && q == 1) ? k0 : knot_at(t0, k);
            const float vr = horner(tr[kq.row], kq.t) * t0;
            ga = fmaf(d.w0_f[q], vr, ga);
            gb = fmaf(d.w1_f[q], vr, gb);
            gc = fmaf(d.w2_f[q], vr, gc);
            if (kPhi) {
                const float vp = with_sign_of(horner(tp[kq.row], kq.t), t0);
                fa = fmaf(d.w0_f[q], vp, fa);
                fb = fmaf(d.w1_f[q], vp, fb);
                fc = fmaf(d.w2_f[q], vp, fc);
            }
        }
        const float sc = kPiInSqF * r_inv;
        g.v = ga * sc;
        g.dr = fmaf(-g.v, r_inv, -2.0f * as * (gb * sc));
        g.da = fmaf(0.5f, g.v, -gc * sc) * inv_alpha;
        if (kPhi) {
            f.v = fa * sc;
            f.dr = fmaf(-f.v, r_inv, -2.0f * as * (fb * sc));
            f.da = fmaf(0.5f, f.v, -fc * sc) * inv_alpha;
        }
        return;
    }
    if (k.alpha_max <= alpha && below_rc) {
        const float4 cr = tr[k0.row];
        g.v = horner(cr, k0.t);
        g.dr = horner_d(cr, k0.t) * k.dr_inv;
        if (kPhi) {
            const float4 cp = tp[k0.row];
            const float z2 = horner(cp, k0.t), z2p = horner_d(cp, k0.t) * k.dr_inv;
            f.v = z2 * r_inv;
            f.dr = (z2p - z2 * r_inv) * r_inv;
        }
    }
}

}  // namespace
}  // namespace mg
