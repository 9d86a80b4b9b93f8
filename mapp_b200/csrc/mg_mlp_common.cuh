// Pieces of the learned form (MG_FORM_MLP) shared by its training kernels
// (mg_mlp.cu) and its tensor-core deployment (mg_mlp_tc.cu).
//
// Network: 4 -> 64 -> 64 -> 64 -> 6, activation silu_p (below), BF16 weights
// and activations, FP32 accumulation.  Inputs (r, w_i, w_j, species-pair
// code) normalised over the training box; outputs standardised.
//
// What the network learns is the smearing correction, not the smeared value:
// for each output q the label is  quadrature_q(r, alpha) - base_q(r), with
// base the reference's unsmeared branch for alpha >= alpha_max
// (ff_dmd_I.cpp:261-310: phi(r), rho(r) and their r derivatives from the
// splines at r; 0 for the alpha derivatives).  At deployment the force pass
// adds base_q(r) back.  The correction is a few per cent of the value it
// corrects, so the network's relative error costs that much less in absolute
// terms.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

#include "mg_internal.h"

namespace mg {
namespace mlp {

constexpr int H = 64;  // hidden width
// parameter offsets of the FP32 master vector (W stored [in][out])
constexpr int OW1 = 0, OB1 = OW1 + 16 * H, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + H * H,
              OW4 = OB3 + H, OB4 = OW4 + H * 8, NPARAM = OB4 + 8, OLOSS = NPARAM, NPART = NPARAM + 1;

// Activation silu_p(z) = z * sigma_p(z), with sigma_p a polynomial stand-in for
// the logistic function that runs on the FP32 FMA pipe (no transcendental
// unit): x = z / 8, u = min(x^2, 1),
//     sigma_p(z) = clamp(1/2 + x Q(u), 0, 1),   Q(u) = sum_k q_k u^k  (degree 7),
// Q fitted here by iteratively reweighted least squares (a near-minimax fit)
// to sigma(8x) - 1/2 on [-1, 1] under the constraint Q(1) = 1/2, so that
// sigma_p(z) is 0 for z <= -8 and 1 for z >= 8 (to the rounding of the
// coefficients, 1e-7) and silu_p(z) vanishes for large negative z.  (For |x| > 1, u = 1 and 1/2 + x/2 lies outside [0, 1]:
// the clamp alone gives the two tails.)  Bounds (checked against the
// exp-based logistic on a dense grid, FP32 evaluation):
//     |sigma_p(z) - sigma(z)| <= 9.2e-4,  |silu_p(z) - silu(z)| <= 7.3e-3
// for every z (the second is at most 9.2e-4 |z|), below the 2^-9 relative
// rounding the BF16 activations carry.  Training and deployment use the same
// function, so the network is fitted with the activation it runs.
//
// The scale 8 is a power of two so that deployment can run the network on
// x = z / 8 instead of z with every value scaled exactly (no extra rounding):
// silu_p(z) / 8 = x sigma(x) with sigma a function of x alone, so the
// tensor-core pass feeds the inputs and biases of layer 1 divided by 8, the
// biases of layers 2 and 3 divided by 8, and multiplies layer 4 by 8.
constexpr float kSigQ0 = 1.981310478e+00f, kSigQ1 = -9.368737072e+00f, kSigQ2 = 3.989676019e+01f,
                kSigQ3 = -1.137893481e+02f, kSigQ4 = 2.023527075e+02f, kSigQ5 = -2.133724498e+02f,
                kSigQ6 = 1.215064055e+02f, kSigQ7 = -2.870664878e+01f;
constexpr float kSigZ = 8.0f, kSigInvZ = 0.125f;

__host__ __device__ __forceinline__ float sig_q(float u)
{
    float q = kSigQ7;
    q = fmaf(q, u, kSigQ6);
    q = fmaf(q, u, kSigQ5);
    q = fmaf(q, u, kSigQ4);
    q = fmaf(q, u, kSigQ3);
    q = fmaf(q, u, kSigQ2);
    q = fmaf(q, u, kSigQ1);
    q = fmaf(q, u, kSigQ0);
    return q;
}

// sigma_p as a function of x = z / 8
__host__ __device__ __forceinline__ float sigma_x(float x)
{
    const float u = fminf(x * x, 1.0f);
    return fminf(fmaxf(fmaf(x, sig_q(u), 0.5f), 0.0f), 1.0f);
}

__host__ __device__ __forceinline__ float sigma_p(float z) { return sigma_x(z * kSigInvZ); }

__host__ __device__ __forceinline__ float silu_p(float z) { return z * sigma_p(z); }

// d silu_p / dz = sigma_p + z sigma_p'; sigma_p' = (Q(u) + 2u Q'(u)) / 8
// where |z| < 8 and the clamp of sigma_p is not active, 0 elsewhere (the
// fitted polynomial reaches 0 and 1 slightly inside |z| = 8)
__host__ __device__ __forceinline__ float dsilu_p(float z)
{
    const float x = z * kSigInvZ;
    const float u = fminf(x * x, 1.0f);
    const float q = sig_q(u);
    float dq = 7.0f * kSigQ7;
    dq = fmaf(dq, u, 6.0f * kSigQ6);
    dq = fmaf(dq, u, 5.0f * kSigQ5);
    dq = fmaf(dq, u, 4.0f * kSigQ4);
    dq = fmaf(dq, u, 3.0f * kSigQ3);
    dq = fmaf(dq, u, 2.0f * kSigQ2);
    dq = fmaf(dq, u, kSigQ1);
    const float su = fmaf(x, q, 0.5f);
    const float s = fminf(fmaxf(su, 0.0f), 1.0f);
    const float ds = (fabsf(x) < 1.0f && su > 0.0f && su < 1.0f) ? (q + 2.0f * u * dq) * kSigInvZ : 0.0f;
    return s + z * ds;
}

// The other activation: SiLU with the logistic function from the
// transcendental unit, sigma(z) = (1 + tanh(z / 2)) / 2 with tanh.approx.f32
// (absolute error about 2^-11).
__device__ __forceinline__ float tanh_hw(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float silu_t(float z) { return z * fmaf(0.5f, tanh_hw(0.5f * z), 0.5f); }
__device__ __forceinline__ float dsilu_t(float z)
{
    const float s = fmaf(0.5f, tanh_hw(0.5f * z), 0.5f);
    return s * (1.0f + z * (1.0f - s));
}

// Activation kinds (MlpState::act, MG_MLP_ACT_*): 0 silu_p on every hidden
// unit; 1 silu_t on every hidden unit; 2 split: silu_t on the first
// kSplitTanh units of each hidden layer, silu_p on the rest.  The split keeps
// both pipes that can evaluate an activation busy at once: per element silu_t
// costs one transcendental-unit operation (that unit runs at an eighth of the
// FMA pipe's rate) and 4 FMA-pipe operations, silu_p 11 FMA-pipe operations:
// with a fraction f of silu_t units the FMA pipe carries 11 - 7f and the
// transcendental unit 8f FMA-equivalents per element, equal at f = 11/15,
// so 48 of 64.
constexpr int kSplitTanh = 48;

__device__ __forceinline__ bool tanh_unit(int act, int col) { return act == 1 || (act == 2 && col < kSplitTanh); }
__device__ __forceinline__ float act_rt(int act, int col, float z) { return tanh_unit(act, col) ? silu_t(z) : silu_p(z); }
__device__ __forceinline__ float dact_rt(int act, int col, float z)
{
    return tanh_unit(act, col) ? dsilu_t(z) : dsilu_p(z);
}

// ---- deployment forms on x = z / 8 (see above) --------------------------------
// g(x) = silu(8x) / 8.  Polynomial units: u = x^2 saturated to [0, 1], the
// Horner steps, the final fma saturated to [0, 1] (the same values as
// sigma_x: the .sat modifier is the clamp); tanh units: x (1 + tanh(4x)) / 2.
__device__ __forceinline__ float mul_sat(float a, float b)
{
    float d;
    asm("mul.rn.sat.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float fma_sat(float a, float b, float c)
{
    float d;
    asm("fma.rn.sat.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float gx_poly(float x) { return x * fma_sat(x, sig_q(mul_sat(x, x)), 0.5f); }
__device__ __forceinline__ float gx_tanh(float x) { return x * fmaf(0.5f, tanh_hw(4.0f * x), 0.5f); }
template <int ACT>
__device__ __forceinline__ float gx(int col, float x)
{
    return (ACT == 1 || (ACT == 2 && col < kSplitTanh)) ? gx_tanh(x) : gx_poly(x);
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// two FP32 values rounded to BF16 and packed (lo in the low half) with one
// paired conversion (cvt.rn.bf16x2.f32) instead of two single ones: the
// conversions of the network's activations are the busiest part of its
// epilogue
__device__ __forceinline__ uint32_t pack2f(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    // splitmix64 finaliser (Steele, Lea & Flood 2014)
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double u01(unsigned long long h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

// normalised network inputs of (r, w_i, w_j, code)
__device__ __forceinline__ void net_inputs(const MlpBox& b, float r, float wi, float wj, int code, float (&in)[4])
{
    in[0] = (r - 0.5f * (b.r_lo + b.r_hi)) / (0.5f * (b.r_hi - b.r_lo));
    in[1] = (wi - 0.5f * (b.w_lo + b.w_hi)) / (0.5f * (b.w_hi - b.w_lo));
    in[2] = (wj - 0.5f * (b.w_lo + b.w_hi)) / (0.5f * (b.w_hi - b.w_lo));
    in[3] = (float)code - 1.0f;
}

// The base of the learned outputs (phi, rho, dphi/dr, drho/dr, dphi/dalpha,
// drho/dalpha) at r: the reference's unsmeared branch (ff_dmd_I.cpp:261-310)
// on the FP64 splines (rho slot rs, phi slot ps, rows of 8 doubles, index
// clamp nr-2, p <= 1); the alpha derivatives are 0.
__device__ __forceinline__ void base_f64(const Dev& d, int rs, int ps, double r, double (&o)[6])
{
    double p = r * d.dr_inv;
    const int m = min((int)p, d.nr - 2);
    p -= m;
    p = fmin(p, 1.0);
    const double p2 = p * p, p3 = p2 * p, r_inv = 1.0 / r;
    const double* cr = d.rhoT + ((size_t)rs * d.nr + m) * 8;
    const double* cp = d.phiT + ((size_t)ps * d.nr + m) * 8;
    const double z2 = cp[3] * p3 + cp[2] * p2 + cp[1] * p + cp[0];
    const double z2p = cp[6] * p2 + cp[5] * p + cp[4];
    o[0] = z2 * r_inv;
    o[1] = cr[3] * p3 + cr[2] * p2 + cr[1] * p + cr[0];
    o[2] = (z2p - z2 * r_inv) * r_inv;
    o[3] = cr[6] * p2 + cr[5] * p + cr[4];
    o[4] = 0.0;
    o[5] = 0.0;
}

}  // namespace mlp
}  // namespace mg
