// Precision form (MG_FORM_FP32) of ForceField_DMD_I/II/DMD::force_calc
// (ff_dmd_I.cpp:88-450): the per-pair work -- pair geometry after the cut
// test, the Gauss-Hermite smearing, the spline lookups and the force
// projections -- runs in FP32; per-site density and force sums are
// compensated; the cut test on rsq, the per-site embedding F(E) and the energy
// and virial totals stay FP64.
//
// Tables: one 32-byte sector per ordered species pair (a,b) and knot,
// {rho c0..c3 of density slot b*nt+a, phi c0..c3 of slot COMP(a,b)}, so a
// quadrature node costs one sector where the FP64 form needs two.
//
// Per-site sums: a site's i-side pairs are summed inside the warp with TwoSum
// (error-free addition) steps, and every contribution is accumulated into the
// site's FP64 density / force with a fire-and-forget atomic add.  A Kahan
// (sum, compensation) float pair would need a compare-and-swap round trip per
// update, which measured 1.5x slower for the whole force call; the FP64
// accumulator is at least as accurate.
#include "mg_reduce.cuh"
#include "mg_dmd_common.cuh"

namespace mg {
namespace {

#ifndef MG_DMD32_MINB
#define MG_DMD32_MINB 4
#endif

// Accumulate a compensated (hi, lo) FP32 value into an FP64 per-site sum.
__device__ __forceinline__ void acc_add(double* dst, float hi, float lo)
{
    double v = (double)hi + (double)lo;
    if (v != 0.0) atomicAdd(dst, v);
}

// TwoSum-compensated sum over the caller's segment of lanes; the first lane of
// the segment receives (hi, lo) with value hi + lo.
__device__ __forceinline__ float2 seg_sum2(float v, const Seg& s)
{
    int lane = threadIdx.x & 31;
    float hi = v, lo = 0.0f;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        float h2 = __shfl_down_sync(0xffffffffu, hi, o);
        float l2 = __shfl_down_sync(0xffffffffu, lo, o);
        if (lane + o <= s.last) {
            float t = hi + h2;
            float bp = t - hi;
            float err = (hi - (t - bp)) + (h2 - bp);
            hi = t;
            lo = lo + l2 + err;
        }
    }
    return make_float2(hi, lo);
}

// ---- pass 1: FP32 smearing, compensated densities -------------------------
// kSmem = 1: the coarse table (d.pkC) is copied into shared memory first and
// every knot of the quadrature is read from there, one 1024-thread block per
// SM; kSmem = 0: the fine packed table through L1 / L2.
template <int NT, int NQ, int kSmem>
__global__ void __launch_bounds__(kSmem ? 1024 : kFFBlock, kSmem ? 1 : MG_DMD32_MINB) k_dmd32_pass1(Dev d, int row0)
{
    using S = Slots<NT>;
    extern __shared__ float4 tab_sh[];
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const size_t mp = (size_t)d.maxp;
    F32Consts kc = f32_consts(d);
    const float4* tab = d.pkT;
    if (kSmem) {
        const int n4 = NT * NT * d.nrC * 2;
        for (int k = threadIdx.x; k < n4; k += blockDim.x) tab_sh[k] = __ldg(d.pkC + k);
        __syncthreads();
        tab = tab_sh;
        kc.nr = d.nrC;
        kc.dr_inv = d.drC_inv;
        kc.top = (float)(d.nrC - 1);
        kc.top_m = (float)(d.nrC - 2);
    }
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (long long base = (long long)blockIdx.x * blockDim.x + threadIdx.x - lane; base < d.npairs; base += stride) {
        long long p = base + lane;
        bool valid = p < d.npairs;
        int i = valid ? d.pair_i[p] : -1;
        float Ei[NT];
#pragma unroll
        for (int a = 0; a < NT; a++) Ei[a] = 0.0f;
        const bool act = valid && site_active(d, i);
        double epair = 0.0;
        if (act) {
            int j = d.pair_j[p];
            double4 xi = d.pos[i], xj = d.pos[j];
            float ai[NT], ci[NT], aj[NT], cj[NT], Ej[NT];
#pragma unroll
            for (int a = 0; a < NT; a++) {
                ai[a] = (float)d.alpha[(size_t)i * NT + a];
                ci[a] = (float)d.c[(size_t)i * NT + a];
                aj[a] = (float)d.alpha[(size_t)j * NT + a];
                cj[a] = (float)d.c[(size_t)j * NT + a];
                Ej[a] = 0.0f;
            }
            double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
            double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
            bool own_j = j < d.natms;
            bool in_cut = rsq < d.cut_sq_mod;
            bool below_rc = rsq < d.cut_sq;
            float rsqf = (float)rsq;
            float r_inv = rsqrtf(rsqf);
            float r = rsqf * r_inv;
            double w = own_j ? 0.5 : 0.25;
            float* out = d.prf + p;
#pragma unroll
            for (int a = 0; a < NT; a++)
#pragma unroll
                for (int b = 0; b < NT; b++) {
                    const int rs = b * NT + a, ps = comp_idx(a, b);
                    const float4* pk = tab + (size_t)(a * NT + b) * kc.nr * 2;
                    float g0 = 0, gdr = 0, gda = 0, f0 = 0, fdr = 0, fda = 0;
                    bool hit = false;
                    if (in_cut) {
                        float alpha = __fdividef(ai[a] * aj[b], ai[a] + aj[b]);
                        hit = (a >= b) ? smear_f<true, NQ, kSmem != 0>(d, kc, pk, r, r_inv, below_rc, alpha, g0, gdr,
                                                                      gda, f0, fdr, fda)
                                       : smear_f<false, NQ, kSmem != 0>(d, kc, pk, r, r_inv, below_rc, alpha, g0, gdr,
                                                                       gda, f0, fdr, fda);
                    }
                    if (!hit) g0 = gdr = gda = f0 = fdr = fda = 0.0f;
                    __stcs(out + (S::RHO + rs) * mp, g0);
                    __stcs(out + (S::DRR + rs) * mp, gdr);
                    __stcs(out + (S::DRA + rs) * mp, gda);
                    if (a >= b) {
                        __stcs(out + (S::PHI + ps) * mp, f0);
                        __stcs(out + (S::DPR + ps) * mp, fdr);
                        __stcs(out + (S::DPA + ps) * mp, fda);
                        epair += w * (double)((cj[b] * ci[a] + cj[a] * ci[b]) * f0);
                    }
                    Ei[a] += g0 * cj[b];
                    Ej[b] += g0 * ci[a];
                }
            if (own_j && in_cut) {
#pragma unroll
                for (int b = 0; b < NT; b++) acc_add(&d.E[(size_t)j * NT + b], Ej[b], 0.0f);
            }
        }
        Seg sg = seg_of(i);
#pragma unroll
        for (int a = 0; a < NT; a++) {
            float2 t = seg_sum2(Ei[a], sg);
            if (valid && lane == sg.first) acc_add(&d.E[(size_t)i * NT + a], t.x, t.y);
        }
        if (d.site_cell) cell_energy_add(d, valid ? i : -1, epair);
        else acc[0] += epair;
    }
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// ---- per-site embedding (FP64, as in the plain form) ----------------------
template <int NT>
__global__ void __launch_bounds__(kFFBlock) k_dmd32_embed(Dev d, int row0)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    double e = 0.0;
    if (i < d.natms && site_active(d, i)) {
#pragma unroll
        for (int a = 0; a < NT; a++) {
            size_t q = (size_t)i * NT + a;
            double Ev = d.E[q];
            double tmp0, tmp1;
            embed_F(d, a, Ev, tmp0, tmp1, nullptr);
            double ca = d.c[q], al = d.alpha[q];
            d.E[q] = tmp0;
            d.dE[q] = tmp1;
            e += ca * tmp0;
            e += d.kbT * calc_ent(ca);
            e += 1.5 * d.kbT * ca * log(al) + ca * d.c0[a];
            d.f[(size_t)i * d.x_dim + 3 + a] -= 1.5 * d.kbT * ca / al;
        }
    }
    if (d.site_cell) cell_energy_add(d, i < d.natms ? i : -1, e);
    else acc[0] += e;
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// ---- pass 2: FP32 force projections, compensated force sums ----------------
template <int NT>
__global__ void __launch_bounds__(kFFBlock, MG_DMD32_MINB) k_dmd32_pass2(Dev d, int st_clc, int row0)
{
    using S = Slots<NT>;
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const size_t mp = (size_t)d.maxp;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (long long base = (long long)blockIdx.x * blockDim.x + threadIdx.x - lane; base < d.npairs; base += stride) {
        long long p = base + lane;
        bool valid = p < d.npairs;
        int i = valid ? d.pair_i[p] : -1;
        float fi[3 + NT];
#pragma unroll
        for (int q = 0; q < 3 + NT; q++) fi[q] = 0.0f;
        const bool act = valid && site_active(d, i);
        // pairs beyond the smeared cut contribute nothing and pass 1 stored no
        // derivatives for them: the same exact rsq test as pass 1 skips them
        bool in_cut = false;
        int j = 0;
        double4 xi = make_double4(0, 0, 0, 0), xj = xi;
        if (act) {
            j = d.pair_j[p];
            xi = d.pos[i];
            xj = d.pos[j];
            const double ex0 = xi.x - xj.x, ex1 = xi.y - xj.y, ex2 = xi.z - xj.z;
            in_cut = __dadd_rn(__dadd_rn(__dmul_rn(ex0, ex0), __dmul_rn(ex1, ex1)), __dmul_rn(ex2, ex2)) < d.cut_sq_mod;
        }
        if (in_cut) {
            const float* in = d.prf + p;
            float drr[NT * NT], dra[NT * NT], dpr[S::NC], dpa[S::NC];
#pragma unroll
            for (int q = 0; q < NT * NT; q++) {
                drr[q] = __ldcs(in + (S::DRR + q) * mp);
                dra[q] = __ldcs(in + (S::DRA + q) * mp);
            }
#pragma unroll
            for (int q = 0; q < S::NC; q++) {
                dpr[q] = __ldcs(in + (S::DPR + q) * mp);
                dpa[q] = __ldcs(in + (S::DPA + q) * mp);
            }
            int oj = owner(d, j);
            float ai[NT], ci[NT], dEi[NT], aj[NT], cj[NT], dEj[NT], fj[NT];
#pragma unroll
            for (int a = 0; a < NT; a++) {
                ai[a] = (float)d.alpha[(size_t)i * NT + a];
                ci[a] = (float)d.c[(size_t)i * NT + a];
                dEi[a] = (float)d.dE[(size_t)i * NT + a];
                aj[a] = (float)d.alpha[(size_t)j * NT + a];
                cj[a] = (float)d.c[(size_t)j * NT + a];
                dEj[a] = (float)d.dE[(size_t)oj * NT + a];
                fj[a] = 0.0f;
            }
            float dx0 = (float)(xi.x - xj.x), dx1 = (float)(xi.y - xj.y), dx2 = (float)(xi.z - xj.z);
            float r_inv = rsqrtf(dx0 * dx0 + dx1 * dx1 + dx2 * dx2);
            bool own_j = j < d.natms;
            float fsum = 0.0f;
#pragma unroll
            for (int a = 0; a < NT; a++)
#pragma unroll
                for (int b = 0; b < NT; b++) {
                    const int ab = a * NT + b, ba = b * NT + a, ps = comp_idx(a, b);
                    float cc = ci[a] * cj[b];
                    float fpair = -(drr[ab] * dEi[a] + drr[ba] * dEj[b] + dpr[ps]) * cc * r_inv;
                    float sa = ai[a] + aj[b];
                    float apair = -(dra[ab] * dEi[a] + dra[ba] * dEj[b] + dpa[ps]) * cc * __frcp_rn(sa * sa);
                    fsum += fpair;
                    fi[3 + a] += apair * aj[b] * aj[b];
                    fj[b] += apair * ai[a] * ai[a];
                }
            fi[0] = dx0 * fsum;
            fi[1] = dx1 * fsum;
            fi[2] = dx2 * fsum;
            if (st_clc) {
                double wf = (own_j ? 1.0 : 0.5) * (double)fsum;
                acc[1] -= wf * dx0 * dx0;
                acc[2] -= wf * dx1 * dx1;
                acc[3] -= wf * dx2 * dx2;
                acc[4] -= wf * dx1 * dx2;
                acc[5] -= wf * dx2 * dx0;
                acc[6] -= wf * dx0 * dx1;
            }
            if (own_j) {
                double* fj_out = d.f + (size_t)j * d.x_dim;
                if (fsum != 0.0f) {
                    acc_add(fj_out + 0, -dx0 * fsum, 0.0f);
                    acc_add(fj_out + 1, -dx1 * fsum, 0.0f);
                    acc_add(fj_out + 2, -dx2 * fsum, 0.0f);
                }
#pragma unroll
                for (int b = 0; b < NT; b++) acc_add(fj_out + 3 + b, fj[b], 0.0f);
            }
        }
        Seg sg = seg_of(i);
#pragma unroll
        for (int q = 0; q < 3 + NT; q++) {
            float2 t = seg_sum2(fi[q], sg);
            if (valid && lane == sg.first) acc_add(d.f + (size_t)i * d.x_dim + q, t.x, t.y);
        }
    }
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

template <int NT>
cudaError_t dmd32_force_nt(const Dev& d, int st_clc, int* nb, cudaStream_t st, cudaEvent_t* evs)
{
    int g1 = persistent_grid(d.npairs, d.tune_bps > 0 ? d.tune_bps : MG_DMD32_MINB), g2 = div_up(d.natms, kFFBlock);
    int g3 = persistent_grid(d.npairs, d.tune_bps2 > 0 ? d.tune_bps2 : MG_DMD32_MINB);
    const size_t tab_bytes = (size_t)NT * NT * d.nrC * 2 * sizeof(float4);
    const bool smem = d.pkC != nullptr && tab_bytes <= 200 * 1024;
    if (smem) {
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_dmd32_pass1<NT, 3, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            cudaFuncSetAttribute(k_dmd32_pass1<NT, 0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            attr = true;
        }
        long long need = div_up(d.npairs, 1024LL);
        g1 = (int)(need < num_sms() ? (need > 0 ? need : 1) : num_sms());
    }
    if (evs) cudaEventRecord(evs[0], st);
    if (smem) {
        if (d.nq == 3) k_dmd32_pass1<NT, 3, 1><<<g1, 1024, tab_bytes, st>>>(d, 0);
        else k_dmd32_pass1<NT, 0, 1><<<g1, 1024, tab_bytes, st>>>(d, 0);
    } else {
        if (d.nq == 3) k_dmd32_pass1<NT, 3, 0><<<g1, kFFBlock, 0, st>>>(d, 0);
        else k_dmd32_pass1<NT, 0, 0><<<g1, kFFBlock, 0, st>>>(d, 0);
    }
    if (evs) cudaEventRecord(evs[1], st);
    k_dmd32_embed<NT><<<g2, kFFBlock, 0, st>>>(d, g1);
    if (evs) cudaEventRecord(evs[2], st);
    k_dmd32_pass2<NT><<<g3, kFFBlock, 0, st>>>(d, st_clc, g1 + g2);
    if (evs) cudaEventRecord(evs[3], st);
    *nb = g1 + g2 + g3;
    return cudaGetLastError();
}

template <int NT>
cudaError_t dmd32_tail_nt(const Dev& d, int st_clc, int row0, int* nb, cudaStream_t st, cudaEvent_t* evs)
{
    int g1 = persistent_grid(d.npairs, d.tune_bps2 > 0 ? d.tune_bps2 : MG_DMD32_MINB), g2 = div_up(d.natms, kFFBlock);
    k_dmd32_embed<NT><<<g2, kFFBlock, 0, st>>>(d, row0);
    if (evs) cudaEventRecord(evs[2], st);
    k_dmd32_pass2<NT><<<g1, kFFBlock, 0, st>>>(d, st_clc, row0 + g2);
    if (evs) cudaEventRecord(evs[3], st);
    *nb = g1 + g2;
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_dmd_force_f32_after_pass1(const Dev& d, int st_clc, int row0, int* nb, cudaStream_t st,
                                             cudaEvent_t* evs)
{
    switch (d.nt) {
    case 1: return dmd32_tail_nt<1>(d, st_clc, row0, nb, st, evs);
    case 2: return dmd32_tail_nt<2>(d, st_clc, row0, nb, st, evs);
    case 3: return dmd32_tail_nt<3>(d, st_clc, row0, nb, st, evs);
    case 4: return dmd32_tail_nt<4>(d, st_clc, row0, nb, st, evs);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dmd_force_f32(const Dev& d, int st_clc, int* nb, cudaStream_t st, cudaEvent_t* evs)
{
    switch (d.nt) {
    case 1: return dmd32_force_nt<1>(d, st_clc, nb, st, evs);
    case 2: return dmd32_force_nt<2>(d, st_clc, nb, st, evs);
    case 3: return dmd32_force_nt<3>(d, st_clc, nb, st, evs);
    case 4: return dmd32_force_nt<4>(d, st_clc, nb, st, evs);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace mg
