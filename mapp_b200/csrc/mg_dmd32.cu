// Precision form (MG_FORM_FP32) of ForceField_DMD_I/II/DMD::force_calc
// (ff_dmd_I.cpp:88-450): the per-pair work -- pair geometry after the cut
// test, the Gauss-Hermite smearing, the spline lookups and the force
// projections -- runs in FP32; per-site density and force sums are carried in
// FP64; the cut test on rsq, the per-site embedding F(E) and the energy and
// virial totals stay FP64.
//
// Structure of one force call (no per-pair array reaches HBM):
//   k_dmd32_dens   densities only: per listed pair the cut test, then for the
//                  in-cut pairs the value of the smeared density of every
//                  ordered species pair (ff_dmd_I.cpp:178-230, weights w0
//                  only).  A warp queues its in-cut pairs in shared memory and
//                  evaluates them 32 at a time, so no lane idles on a pair
//                  beyond the cut; each full batch of 32 is also appended to
//                  the in-cut pair list `icut` (padded with i = -1), with the
//                  pair's geometry, so the force pass gathers no positions.
//   k_dmd32_embed  F(E), F'(E), entropy and alpha terms per site (FP64).
//   k_dmd32_force  per batch of `icut`: the smearing again, now with all three
//                  weight sets and the pair function, giving the per-pair
//                  derivatives the reference stores (ff_dmd_I.cpp:231-259),
//                  projected at once onto the forces (ff_dmd_I.cpp:357-436);
//                  pair energy and virial.
// Recomputing the smearing costs one table pass over the in-cut pairs; it
// replaces the reference's per-pair buffers (21 values per pair for two
// species), which in FP32 would move about 84 B per listed pair through HBM
// twice per call.  c_d_calc and calc_g read the per-pair densities and pair
// energies of the last force_calc; after a precision-form force call they are
// written on demand by k_dmd32_fill (launch_dmd32_pair_values).
//
// Tables: the splines resampled onto kSplitKnots knots over [0, rc] (cubic
// Hermite pieces through the fine spline's value and slope, FP32) and held in
// shared memory, one float4 {c0..c3} per knot and slot: the rho slots of the
// ordered species pairs first (slot a*nt+b holds density slot b*nt+a), then
// the phi slots in COMP order; row K-1 of a slot is zero, so a quadrature
// node the reference rejects (|r - xi_q / sqrt(alpha)| >= rc) adds an exact
// zero without a test.  Rho and phi are separate slots so the 16-byte knot
// loads of a warp spread over all eight bank groups.
//
// Per-site sums: densities are FP64 throughout -- a warp's i-side
// contributions summed by segmented FP64 shuffles (pairs are in i order
// inside a batch) and added with one FP64 atomic per site and batch, j-side
// contributions FP64 atomics; an FP64 accumulator of FP32 terms keeps more
// bits than a Kahan-compensated FP32 sum and needs no compare-and-swap loop.
// Forces: i-side runs summed in FP32 over at most 32 terms, then one FP64
// atomic per site and batch; j-side FP32 vector reductions into a per-site
// FP32 buffer that k_dmd32_fmerge adds to the FP64 forces.
#include <mutex>
#include <unordered_map>

#include "mg_reduce.cuh"
#include "mg_dmd_common.cuh"
#include "mg_split.cuh"

namespace mg {
namespace {

#ifndef MG_DMD32_MINB
#define MG_DMD32_MINB 4
#endif
// resident 256-thread blocks per SM the two precision-form pair passes are
// compiled for (bounds their registers): the force pass at 4 (64 registers,
// no spills) measured 3-5 % faster than unbounded (80 registers, 3 blocks)
#ifndef MG_FORCE_MINB
#define MG_FORCE_MINB 4
#endif
#if defined(MG_DENS_MINB) && MG_DENS_MINB > 0
#define MG_DENS_BOUNDS __launch_bounds__(kFFBlock, MG_DENS_MINB)
#else
#define MG_DENS_BOUNDS __launch_bounds__(kFFBlock)
#endif
#if defined(MG_FORCE_MINB) && MG_FORCE_MINB > 0
#define MG_FORCE_BOUNDS __launch_bounds__(kFFBlock, MG_FORCE_MINB)
#else
#define MG_FORCE_BOUNDS __launch_bounds__(kFFBlock)
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

// Segments of a warp whose keys are sorted (equal keys in contiguous lanes,
// padding lanes with key -1 at the end): boundaries from one shuffle and one
// ballot instead of a match instruction.
__device__ __forceinline__ Seg seg_sorted(int key)
{
    const int lane = threadIdx.x & 31;
    const int prev = __shfl_up_sync(0xffffffffu, key, 1);
    const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || prev != key);
    const unsigned upto = heads & (0xffffffffu >> (31 - lane));  // heads at or before this lane
    const unsigned after = heads & ~(0xffffffffu >> (31 - lane));
    Seg sg;
    sg.first = 31 - __clz(upto);
    sg.last = after ? __ffs(after) - 2 : 31;
    return sg;
}

// FP32 sum over the caller's segment (first lane of the segment receives it)
__device__ __forceinline__ float seg_sumf(float v, const Seg& s)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const float t = __shfl_down_sync(0xffffffffu, v, o);
        if (lane + o <= s.last) v += t;
    }
    return v;
}

// a site position as one 32-byte read-only load
__device__ __forceinline__ double4 pos_ld(const Dev& d, int i)
{
    double4 r;
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(d.pos + i));
    return r;
}

// alpha and c of site j from its FP32 record (srec: {alpha_0.., c_0..})
template <int NT>
__device__ __forceinline__ void load_rec(const Dev& d, int j, float (&al)[NT], float (&cc)[NT])
{
    float v[8];
    const float4 r0 = __ldg(d.srec + (size_t)j * kSiteRec);
    v[0] = r0.x;
    v[1] = r0.y;
    v[2] = r0.z;
    v[3] = r0.w;
    if (2 * NT > 4) {
        const float4 r1 = __ldg(d.srec + (size_t)j * kSiteRec + 1);
        v[4] = r1.x;
        v[5] = r1.y;
        v[6] = r1.z;
        v[7] = r1.w;
    }
#pragma unroll
    for (int a = 0; a < NT; a++) {
        al[a] = v[a];
        cc[a] = v[NT + a];
    }
}

// ---- set-up of a precision-form force call ----------------------------------
// the FP32 site records of every site (owned + ghost); for the owned sites
// being evaluated, f, E and the j-side force sums zeroed; the in-cut list
// emptied
template <int NT>
__global__ void __launch_bounds__(kFFBlock) k_dmd32_prep(Dev d)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) d.status[4] = 0;
    if (i < d.nall) {
        float v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int a = 0; a < NT; a++) {
            v[a] = (float)d.alpha[(size_t)i * NT + a];
            v[NT + a] = (float)d.c[(size_t)i * NT + a];
        }
        d.srec[(size_t)i * kSiteRec] = make_float4(v[0], v[1], v[2], v[3]);
        if (2 * NT > 4) d.srec[(size_t)i * kSiteRec + 1] = make_float4(v[4], v[5], v[6], v[7]);
    }
    if (i < d.natms && site_active(d, i)) {
        for (int q = 0; q < d.x_dim; q++) d.f[(size_t)i * d.x_dim + q] = 0.0;
#pragma unroll
        for (int a = 0; a < NT; a++) d.E[(size_t)i * NT + a] = 0.0;
        reinterpret_cast<float4*>(d.facc)[(size_t)i * 2] = make_float4(0.f, 0.f, 0.f, 0.f);
        reinterpret_cast<float4*>(d.facc)[(size_t)i * 2 + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// the j-side FP32 force sums added to the FP64 forces
template <int NT>
__global__ void __launch_bounds__(kFFBlock) k_dmd32_fmerge(Dev d)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.natms || !site_active(d, i)) return;
    const float4 a = reinterpret_cast<const float4*>(d.facc)[(size_t)i * 2];
    const float4 b = reinterpret_cast<const float4*>(d.facc)[(size_t)i * 2 + 1];
    const float v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    double* f = d.f + (size_t)i * d.x_dim;
#pragma unroll
    for (int q = 0; q < 3 + NT; q++) f[q] += (double)v[q];
}

// ---- pass A: densities, in-cut pair list ------------------------------------
constexpr int kQueue = 64;  // per-warp queue of in-cut pairs (two batches)

template <int NT, int NQ>
__global__ void MG_DENS_BOUNDS k_dmd32_dens(Dev d, int K)
{
    extern __shared__ float4 tab[];
    __shared__ int2 q_ij[kFFWarps][kQueue];
    __shared__ float4 q_x[kFFWarps][kQueue];  // dx, dy, dz (FP32), rsq
    load_split_table(d, tab, NT * NT);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const SplitK k = split_consts(d);
    const float cut_sq_f = (float)d.cut_sq;
    const long long stride = (long long)gridDim.x * kFFBlock;
    long long base = (long long)blockIdx.x * kFFBlock + w * 32;  // this warp's chunk of 32 listed pairs
    int cnt = 0;                                                 // queued in-cut pairs (warp-uniform)
    // this warp's region of the in-cut list: K batches of 32 (it tests at most
    // K chunks of 32 listed pairs), filled from the start; the batch count goes
    // to icut_n[warp]
    const int wg = blockIdx.x * kFFWarps + w;
    int4* region = d.icut + (size_t)wg * K * 32 * 2;
    int nbt = 0;
    // Software pipeline over this warp's chunks: while a batch is evaluated,
    // the positions of the next chunk and the pair indices of the one after
    // are already in flight (a chunk's cut test needs pair -> site -> position,
    // two dependent gathers).  A lane's j is -1 when it has no pair to test.
    auto load_idx = [&](long long b, int& i, int& j) {
        const long long p = b + lane;
        i = -1;
        j = -1;
        if (p < d.npairs) {
            i = d.pair_i[p];
            if (site_active(d, i)) j = d.pair_j[p];
        }
    };
    int i1, j1, i2, j2;
    load_idx(base, i1, j1);
    double4 xi1 = make_double4(0, 0, 0, 0), xj1 = xi1;
    if (j1 >= 0) {
        xi1 = pos_ld(d, i1);
        xj1 = pos_ld(d, j1);
    }
    load_idx(base + stride, i2, j2);
    while (true) {
        const bool have = base < d.npairs;
        if (have) {
            bool in = false;
            float4 gx = make_float4(0.f, 0.f, 0.f, 0.f);
            if (j1 >= 0) {
                const double dx0 = xi1.x - xj1.x, dx1 = xi1.y - xj1.y, dx2 = xi1.z - xj1.z;
                const double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
                in = rsq < d.cut_sq_mod;
                gx = make_float4((float)dx0, (float)dx1, (float)dx2, (float)rsq);
            }
            const unsigned m = __ballot_sync(0xffffffffu, in);
            if (in) {
                const int slot = cnt + __popc(m & lt);
                q_ij[w][slot] = make_int2(i1, j1);
                q_x[w][slot] = gx;
            }
            cnt += __popc(m);
            __syncwarp();
        }
        // advance the pipeline by one chunk
        i1 = i2;
        j1 = j2;
        if (j1 >= 0) {
            xi1 = pos_ld(d, i1);
            xj1 = pos_ld(d, j1);
        }
        load_idx(base + 2 * stride, i2, j2);
        const bool done = !have || base + stride >= d.npairs;
        // evaluate full batches, and the last partial one once this warp has no chunk left
        while (cnt >= 32 || (done && cnt > 0)) {
            const int nb = min(cnt, 32);
            const bool on = lane < nb;
            const int2 e = on ? q_ij[w][lane] : make_int2(-1, -1);
            const float4 gx = on ? q_x[w][lane] : make_float4(0.f, 0.f, 0.f, 1.f);
            const float rsqf = gx.w;
            __syncwarp();
            if (lane < cnt - nb) {
                q_ij[w][lane] = q_ij[w][nb + lane];
                q_x[w][lane] = q_x[w][nb + lane];
            }
            __syncwarp();
            cnt -= nb;
            // append the batch, padded to 32 with i = -1, to this warp's
            // region: per pair {i, j, owner of j} and {dx, dy, dz, rsq}
            if (nbt < K) {
                const int oj = on ? owner(d, e.y) : -1;
                // (a batch's 32 first halves, then its 32 second halves: each
                // store instruction writes 512 contiguous bytes)
                int4* o = region + (size_t)nbt * 64 + lane;
                o[0] = make_int4(e.x, e.y, oj, 0);
                o[32] = make_int4(__float_as_int(gx.x), __float_as_int(gx.y), __float_as_int(gx.z), __float_as_int(gx.w));
            } else if (lane == 0)
                d.status[4] = 1;
            nbt++;
            float Ei[NT], Ej[NT], ci[NT], cj[NT], al[NT * NT];
            float r = 1.0f, r_inv = 1.0f;
            bool below_rc = false, inr = true;
#pragma unroll
            for (int a = 0; a < NT; a++) Ei[a] = Ej[a] = ci[a] = cj[a] = 0.0f;
#pragma unroll
            for (int q = 0; q < NT * NT; q++) al[q] = 0.0f;
            if (on) {
                float ai[NT], aj[NT];
                load_rec<NT>(d, e.x, ai, ci);
                load_rec<NT>(d, e.y, aj, cj);
                r_inv = rsqrtf(rsqf);
                r = rsqf * r_inv;
                below_rc = rsqf < cut_sq_f;
#pragma unroll
                for (int a = 0; a < NT; a++)
#pragma unroll
                    for (int b = 0; b < NT; b++) {
                        const float alpha = __fdividef(ai[a] * aj[b], ai[a] + aj[b]);
                        al[a * NT + b] = alpha;
                        inr = inr && k.alpha_min < alpha && alpha < k.alpha_max;
                    }
            }
            // every lane's species pairs inside the smeared range: no branches
            const bool fast = __all_sync(0xffffffffu, inr);
            if (on) {
                const Knot k0 = knot_at(r, k);
#pragma unroll
                for (int a = 0; a < NT; a++)
#pragma unroll
                    for (int b = 0; b < NT; b++) {
                        const float4* tr = tab + (size_t)(a * NT + b) * d.nrS;
                        const float g0 = fast ? dens_value<NQ, true>(d, tr, k, r, r_inv, below_rc, al[a * NT + b], k0)
                                              : dens_value<NQ, false>(d, tr, k, r, r_inv, below_rc, al[a * NT + b], k0);
                        Ei[a] = fmaf(g0, cj[b], Ei[a]);
                        Ej[b] = fmaf(g0, ci[a], Ej[b]);
                    }
                if (e.y < d.natms) {
#pragma unroll
                    for (int b = 0; b < NT; b++)
                        if (Ej[b] != 0.0f) atomicAdd(&d.E[(size_t)e.y * NT + b], (double)Ej[b]);
                }
            }
            const Seg sg = seg_sorted(e.x);
#pragma unroll
            for (int a = 0; a < NT; a++) {
                const double t = seg_sum((double)Ei[a], sg);
                if (on && lane == sg.first && t != 0.0) atomicAdd(&d.E[(size_t)e.x * NT + a], t);
            }
        }
        if (done) break;
        base += stride;
    }
    if (lane == 0) d.icut_n[wg] = (unsigned)min(nbt, K);
}

// ---- pass B: smearing with derivatives, forces, pair energy, virial ---------
template <int NT, int NQ>
__global__ void MG_FORCE_BOUNDS k_dmd32_force(Dev d, int st_clc, int row0, int W, int K)
{
    using S = Slots<NT>;
    extern __shared__ float4 tab[];
    load_split_table(d, tab, NT * NT + S::NC);
    const int lane = threadIdx.x & 31;
    const SplitK k = split_consts(d);
    const float cut_sq_f = (float)d.cut_sq;
    // slots (region rg, batch b) of the density pass's W regions of K
    // batches, region by region (region-major spreads the warps running
    // together over the system, so their j-side reductions seldom meet on the
    // same sites; batch-major measured slower)
    const long long nslot = (long long)W * K;
    const long long wstride = (long long)gridDim.x * kFFWarps;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    // this thread's virial terms (a few dozen pairs) in FP32; the block and
    // grid totals are FP64
    float vir[6] = {0, 0, 0, 0, 0, 0};
    for (long long t = (long long)blockIdx.x * kFFWarps + (threadIdx.x >> 5); t < nslot; t += wstride) {
        const long long rg = t / K;
        if (t - rg * K >= (long long)__ldg(d.icut_n + rg)) continue;  // past the region's last batch
        const int4 e = d.icut[(size_t)t * 64 + lane];
        const int4 ex = d.icut[(size_t)t * 64 + 32 + lane];
        const bool on = e.x >= 0;
        float fi[3 + NT];
#pragma unroll
        for (int q = 0; q < 3 + NT; q++) fi[q] = 0.0f;
        double epair = 0.0;
        float ai[NT], ci[NT], aj[NT], cj[NT], al[NT * NT];
        bool inr = true;
#pragma unroll
        for (int a = 0; a < NT; a++) ai[a] = ci[a] = aj[a] = cj[a] = 0.0f;
#pragma unroll
        for (int q = 0; q < NT * NT; q++) al[q] = 0.0f;
        if (on) {
            load_rec<NT>(d, e.x, ai, ci);
            load_rec<NT>(d, e.y, aj, cj);
#pragma unroll
            for (int a = 0; a < NT; a++)
#pragma unroll
                for (int b = 0; b < NT; b++) {
                    const float alpha = __fdividef(ai[a] * aj[b], ai[a] + aj[b]);
                    al[a * NT + b] = alpha;
                    inr = inr && k.alpha_min < alpha && alpha < k.alpha_max;
                }
        }
        // every lane's species pairs inside the smeared range: no branches
        const bool fast = __all_sync(0xffffffffu, inr);
        if (on) {
            const int i = e.x, j = e.y, oj = e.z;
            const float dx0 = __int_as_float(ex.x), dx1 = __int_as_float(ex.y), dx2 = __int_as_float(ex.z);
            const float rsqf = __int_as_float(ex.w);
            const float r_inv = rsqrtf(rsqf), r = rsqf * r_inv;
            const bool below_rc = rsqf < cut_sq_f;
            const bool own_j = j < d.natms;
            float dEi[NT], dEj[NT];
            if (NT == 2) {
                const float2 ei = __ldg(reinterpret_cast<const float2*>(d.dE32) + i);
                const float2 ej = __ldg(reinterpret_cast<const float2*>(d.dE32) + oj);
                dEi[0] = ei.x;
                dEi[NT - 1] = ei.y;
                dEj[0] = ej.x;
                dEj[NT - 1] = ej.y;
            } else {
#pragma unroll
                for (int a = 0; a < NT; a++) {
                    dEi[a] = __ldg(d.dE32 + (size_t)i * NT + a);
                    dEj[a] = __ldg(d.dE32 + (size_t)oj * NT + a);
                }
            }
            const Knot k0 = knot_at(r, k);
            // the per-pair derivatives the reference stores, in its slot order
            float drr[NT * NT], dra[NT * NT], dpr[S::NC], dpa[S::NC];
            float ep = 0.0f;
#pragma unroll
            for (int a = 0; a < NT; a++)
#pragma unroll
                for (int b = 0; b < NT; b++) {
                    const int rs = b * NT + a, ps = comp_idx(a, b);
                    const float alpha = al[a * NT + b];
                    const float4* tr = tab + (size_t)(a * NT + b) * d.nrS;
                    const float4* tp = tab + (size_t)(NT * NT + ps) * d.nrS;
                    VDer g, f;
                    if (fast) {
                        if (a >= b) smear_full<NQ, true, true>(d, tr, tp, k, r, r_inv, below_rc, alpha, k0, g, f);
                        else smear_full<NQ, false, true>(d, tr, tp, k, r, r_inv, below_rc, alpha, k0, g, f);
                    } else {
                        if (a >= b) smear_full<NQ, true, false>(d, tr, tp, k, r, r_inv, below_rc, alpha, k0, g, f);
                        else smear_full<NQ, false, false>(d, tr, tp, k, r, r_inv, below_rc, alpha, k0, g, f);
                    }
                    drr[rs] = g.dr;
                    dra[rs] = g.da;
                    if (a >= b) {
                        dpr[ps] = f.dr;
                        dpa[ps] = f.da;
                        ep = fmaf(cj[b] * ci[a] + cj[a] * ci[b], f.v, ep);
                    }
                }
            epair = (own_j ? 0.5 : 0.25) * (double)ep;
            // projections (ff_dmd_I.cpp:370-392)
            float fj[NT];
            float fsum = 0.0f;
#pragma unroll
            for (int b = 0; b < NT; b++) fj[b] = 0.0f;
#pragma unroll
            for (int a = 0; a < NT; a++)
#pragma unroll
                for (int b = 0; b < NT; b++) {
                    const int ab = a * NT + b, ba = b * NT + a, ps = comp_idx(a, b);
                    const float cc = ci[a] * cj[b];
                    const float fpair = -(drr[ab] * dEi[a] + drr[ba] * dEj[b] + dpr[ps]) * cc * r_inv;
                    const float sa = ai[a] + aj[b];
                    const float apair = -(dra[ab] * dEi[a] + dra[ba] * dEj[b] + dpa[ps]) * __fdividef(cc, sa * sa);
                    fsum += fpair;
                    fi[3 + a] = fmaf(apair, aj[b] * aj[b], fi[3 + a]);
                    fj[b] = fmaf(apair, ai[a] * ai[a], fj[b]);
                }
            fi[0] = dx0 * fsum;
            fi[1] = dx1 * fsum;
            fi[2] = dx2 * fsum;
            if (st_clc) {
                const float wf = (own_j ? 1.0f : 0.5f) * fsum;
                vir[0] = fmaf(-wf, dx0 * dx0, vir[0]);
                vir[1] = fmaf(-wf, dx1 * dx1, vir[1]);
                vir[2] = fmaf(-wf, dx2 * dx2, vir[2]);
                vir[3] = fmaf(-wf, dx1 * dx2, vir[3]);
                vir[4] = fmaf(-wf, dx2 * dx0, vir[4]);
                vir[5] = fmaf(-wf, dx0 * dx1, vir[5]);
            }
            if (own_j) {
                // j-side sums in FP32, vector reductions (merged into f by k_dmd32_fmerge)
                float4* fo = reinterpret_cast<float4*>(d.facc) + (size_t)j * 2;
                atomicAdd(fo, make_float4(-dx0 * fsum, -dx1 * fsum, -dx2 * fsum, fj[0]));
                if (NT == 2) atomicAdd(reinterpret_cast<float*>(fo + 1), fj[NT - 1]);
                else if (NT > 2) {
                    float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
                    t.x = fj[1 % NT];
                    if (NT > 2) t.y = fj[2 % NT];
                    if (NT > 3) t.z = fj[3 % NT];
                    atomicAdd(fo + 1, t);
                }
            }
        }
        // i-side forces: FP32 sums over the batch's run of each site (at most 32
        // terms, tree order), one FP64 atomic per site and component
        const Seg sg = seg_sorted(e.x);
#pragma unroll
        for (int q = 0; q < 3 + NT; q++) {
            const float t = seg_sumf(fi[q], sg);
            if (on && lane == sg.first && t != 0.0f) atomicAdd(d.f + (size_t)e.x * d.x_dim + q, (double)t);
        }
        if (d.site_cell) cell_energy_add(d, on ? e.x : -1, epair);
        else acc[0] += epair;
    }
#pragma unroll
    for (int q = 0; q < 6; q++) acc[1 + q] = (double)vir[q];
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// ---- per-pair densities and pair energies for c_d_calc / calc_g -------------
// One thread per listed pair: the values k_dmd32_dens and k_dmd32_force
// compute, stored in the reference's slot order into the FP32 pair scratch
// (rho and phi blocks only; the derivative blocks are not read there).
template <int NT, int NQ>
__global__ void __launch_bounds__(kFFBlock) k_dmd32_fill(Dev d)
{
    using S = Slots<NT>;
    extern __shared__ float4 tab[];
    load_split_table(d, tab, NT * NT + S::NC);
    const SplitK k = split_consts(d);
    const float cut_sq_f = (float)d.cut_sq;
    const size_t mp = (size_t)d.maxp;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < d.npairs;
         p += (long long)gridDim.x * blockDim.x) {
        const int i = d.pair_i[p], j = d.pair_j[p];
        const double4 xi = d.pos[i], xj = d.pos[j];
        const double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
        const double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
        const bool in = rsq < d.cut_sq_mod;
        const float rsqf = (float)rsq;
        const float r_inv = rsqrtf(rsqf), r = rsqf * r_inv;
        const bool below_rc = rsqf < cut_sq_f;
        float ai[NT], ci[NT], aj[NT], cj[NT];
#pragma unroll
        for (int a = 0; a < NT; a++) {
            ai[a] = (float)d.alpha[(size_t)i * NT + a];
            ci[a] = (float)d.c[(size_t)i * NT + a];
            aj[a] = (float)d.alpha[(size_t)j * NT + a];
            cj[a] = (float)d.c[(size_t)j * NT + a];
        }
        const Knot k0 = knot_at(r, k);
        float* out = d.prf + p;
#pragma unroll
        for (int a = 0; a < NT; a++)
#pragma unroll
            for (int b = 0; b < NT; b++) {
                const int rs = b * NT + a, ps = comp_idx(a, b);
                const float alpha = __fdividef(ai[a] * aj[b], ai[a] + aj[b]);
                float g0 = 0.0f, f0 = 0.0f;
                if (in) {
                    g0 = dens_value<NQ, false>(d, tab + (size_t)(a * NT + b) * d.nrS, k, r, r_inv, below_rc, alpha, k0);
                    if (a >= b)
                        f0 = phi_value<NQ>(d, tab + (size_t)(NT * NT + ps) * d.nrS, k, r, r_inv, below_rc, alpha, k0);
                }
                out[(S::RHO + rs) * mp] = g0;
                if (a >= b) out[(S::PHI + ps) * mp] = f0;
            }
    }
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
            if (d.dE32) d.dE32[q] = (float)tmp1;
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

// resident blocks per SM of a force kernel at its dynamic shared memory,
// cached per device, kernel and size
int resident_blocks(const void* fn, size_t smem)
{
    static std::mutex mu;
    static std::unordered_map<std::string, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    char key[96];
    snprintf(key, sizeof(key), "%d:%p:%zu", dev, fn, smem);
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    if (smem > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kFFBlock, smem) != cudaSuccess) {
        cudaGetLastError();
        nb = 0;
    }
    nb = std::max(0, std::min(nb, kMaxPassBlocksPerSM));
    cache[key] = nb;
    return nb;
}

// grid of a persistent pair kernel: resident blocks per SM (capped by the
// tuning hint when given) on every SM, never more blocks than 256-pair chunks
int pair_grid(long long npairs, int resident, int hint)
{
    int bps = resident;
    if (hint > 0) bps = std::min(bps, hint);
    bps = std::max(bps, 1);
    return persistent_grid(npairs, bps);
}

template <int NT>
cudaError_t dmd32_force_nt(const Dev& d, int st_clc, int* nb, cudaStream_t st, cudaEvent_t* evs)
{
    constexpr int NC = NT * (NT + 1) / 2;
    if (!d.pkS || !d.icut || !d.icut_n) return cudaErrorInvalidValue;
    const size_t smA = (size_t)NT * NT * d.nrS * sizeof(float4), smB = (size_t)(NT * NT + NC) * d.nrS * sizeof(float4);
    const bool mid0 = d.nq == 3 && d.xi_f[1] == 0.0f;
    void (*kA)(Dev, int) = mid0 ? k_dmd32_dens<NT, 3> : k_dmd32_dens<NT, 0>;
    void (*kB)(Dev, int, int, int, int) = mid0 ? k_dmd32_force<NT, 3> : k_dmd32_force<NT, 0>;
    const int rA = resident_blocks((const void*)kA, smA), rB = resident_blocks((const void*)kB, smB);
    if (rA == 0 || rB == 0) return cudaErrorInvalidConfiguration;
    const int gA = pair_grid(d.npairs, rA, d.tune_bps), gB = pair_grid(d.npairs, rB, d.tune_bps2);
    const int g2 = div_up(d.natms, kFFBlock), g0 = div_up(std::max(d.nall, 1), kFFBlock);
    if (!d.srec || !d.dE32 || !d.facc) return cudaErrorInvalidValue;
    if (evs) cudaEventRecord(evs[0], st);
    // the density pass's warps each test K chunks of 32 listed pairs and own a
    // region of K batches of the in-cut list
    const int W = gA * kFFWarps;
    const int K = (int)std::max(1LL, (d.npairs + (long long)gA * kFFBlock - 1) / ((long long)gA * kFFBlock));
    if ((long long)W * K * 32 > d.icut_cap || W > dmd32_icut_warps()) return cudaErrorInvalidValue;
    k_dmd32_prep<NT><<<g0, kFFBlock, 0, st>>>(d);
    kA<<<gA, kFFBlock, smA, st>>>(d, K);
    if (evs) cudaEventRecord(evs[1], st);
    k_dmd32_embed<NT><<<g2, kFFBlock, 0, st>>>(d, 0);
    if (evs) cudaEventRecord(evs[2], st);
    kB<<<gB, kFFBlock, smB, st>>>(d, st_clc, g2, W, K);
    k_dmd32_fmerge<NT><<<g2, kFFBlock, 0, st>>>(d);
    if (evs) cudaEventRecord(evs[3], st);
    *nb = g2 + gB;
    return cudaGetLastError();
}

template <int NT>
cudaError_t dmd32_fill_nt(const Dev& d, cudaStream_t st)
{
    constexpr int NC = NT * (NT + 1) / 2;
    if (!d.pkS || !d.prf) return cudaErrorInvalidValue;
    if (d.npairs == 0) return cudaSuccess;
    const size_t sm = (size_t)(NT * NT + NC) * d.nrS * sizeof(float4);
    const bool mid0 = d.nq == 3 && d.xi_f[1] == 0.0f;
    void (*kf)(Dev) = mid0 ? k_dmd32_fill<NT, 3> : k_dmd32_fill<NT, 0>;
    const int r = resident_blocks((const void*)kf, sm);
    if (r == 0) return cudaErrorInvalidConfiguration;
    kf<<<pair_grid(d.npairs, r, 0), kFFBlock, sm, st>>>(d);
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

cudaError_t launch_dmd32_pair_values(const Dev& d, cudaStream_t st)
{
    switch (d.nt) {
    case 1: return dmd32_fill_nt<1>(d, st);
    case 2: return dmd32_fill_nt<2>(d, st);
    case 3: return dmd32_fill_nt<3>(d, st);
    case 4: return dmd32_fill_nt<4>(d, st);
    default: return cudaErrorInvalidValue;
    }
}

int dmd32_icut_warps() { return num_sms() * kMaxPassBlocksPerSM * kFFWarps; }

long long dmd32_icut_capacity(long long maxp)
{
    // every warp of the density pass pads its last batch to 32 entries
    return maxp + 32LL * num_sms() * kMaxPassBlocksPerSM * kFFWarps;
}

}  // namespace mg
