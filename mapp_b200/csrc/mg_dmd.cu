// Diffusive-MD free energy, forces and chemical potentials
// (ForceField_DMD_I / DMD_II / DMD: ff_dmd_I.cpp:88-668, 2138-2674;
// ff_dmd_II.cpp:2151-2630; ff_dmd.cpp:2221-2606), plain FP64 form.
//
// Work layout as in mg_eam.cu: one warp per owned site i, lanes over i's half
// list; i-side sums by warp shuffles, j-side sums by FP64 atomics on owned j.
// Per-pair results of the force pass live in SoA blocks of the pair scratch
// `pr` (pair slot i*maxnb+k), in the reference's slot order
// (rho slot b*nt+a for species pair (a,b) = type2rho[a][b]; phi slot COMP(a,b)):
//   block 0        rho           [nt*nt]
//   block nt^2     drho_dr       [nt*nt]
//   block 2nt^2    drho_dalpha   [nt*nt]
//   block 3nt^2    phi           [nc]     nc = nt(nt+1)/2
//   block 3nt^2+nc dphi_dr, then dphi_dalpha
// Slots the reference would leave untouched (pair beyond the smeared cut,
// alpha outside (alpha_min, alpha_max), no node inside the table) are written
// as zero, so results never depend on earlier calls.
#include "mg_reduce.cuh"
#include "mg_dmd_common.cuh"

namespace mg {

namespace {

// ---- force_calc pass 1 (ff_dmd_I.cpp:156-320) ----------------------------
// One thread per half pair of the compact pair list (pairs sorted by i), so
// every lane carries work however many neighbours a site has; the i-side sums
// of a warp are segmented shuffles finished by one atomic per site.  Per-pair
// results are streamed to the pair scratch at the pair's compact index.
#ifndef MG_DMD_MINB
#define MG_DMD_MINB 3
#endif
#ifndef MG_DMD_PACK
#define MG_DMD_PACK true
#endif

template <int NT, int NQ>
__global__ void __launch_bounds__(kFFBlock, MG_DMD_MINB) k_dmd_pass1(Dev d, int row0)
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
        double Ei[NT];
#pragma unroll
        for (int a = 0; a < NT; a++) Ei[a] = 0.0;
        const bool act = valid && site_active(d, i);
        double epair = 0.0;
        if (act) {
            int j = d.pair_j[p];
            double4 xi = d.pos[i], xj = d.pos[j];
            double ai[NT], ci[NT], aj[NT], cj[NT], Ej[NT];
#pragma unroll
            for (int a = 0; a < NT; a++) {
                ai[a] = d.alpha[(size_t)i * NT + a];
                ci[a] = d.c[(size_t)i * NT + a];
                aj[a] = d.alpha[(size_t)j * NT + a];
                cj[a] = d.c[(size_t)j * NT + a];
                Ej[a] = 0.0;
            }
            double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
            double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
            bool own_j = j < d.natms;
            bool in_cut = rsq < d.cut_sq_mod;
            double r_inv = rsqrt(rsq);
            double r = rsq * r_inv;
            double w = own_j ? 0.5 : 0.25;
            double* out = d.pr + p;
#pragma unroll
            for (int a = 0; a < NT; a++)
#pragma unroll
                for (int b = 0; b < NT; b++) {
                    const int rs = b * NT + a, ps = comp_idx(a, b);
                    double g0 = 0, gdr = 0, gda = 0, f0 = 0, fdr = 0, fda = 0;
                    bool hit = false;
                    if (in_cut) {
                        double alpha = (ai[a] * aj[b]) / (ai[a] + aj[b]);
                        hit = (a >= b) ? smear<true, true, NQ, MG_DMD_PACK>(d, rs, ps, r, r_inv, rsq, alpha, g0, gdr,
                                                                            gda, f0, fdr, fda, a * NT + b)
                                       : smear<false, true, NQ, MG_DMD_PACK>(d, rs, ps, r, r_inv, rsq, alpha, g0, gdr,
                                                                             gda, f0, fdr, fda, a * NT + b);
                    }
                    if (!hit) g0 = gdr = gda = f0 = fdr = fda = 0.0;
                    __stcs(out + (S::RHO + rs) * mp, g0);
                    __stcs(out + (S::DRR + rs) * mp, gdr);
                    __stcs(out + (S::DRA + rs) * mp, gda);
                    if (a >= b) {
                        __stcs(out + (S::PHI + ps) * mp, f0);
                        __stcs(out + (S::DPR + ps) * mp, fdr);
                        __stcs(out + (S::DPA + ps) * mp, fda);
                        epair += w * (cj[b] * ci[a] + cj[a] * ci[b]) * f0;
                    }
                    Ei[a] += g0 * cj[b];
                    Ej[b] += g0 * ci[a];
                }
            if (own_j && in_cut) {
#pragma unroll
                for (int b = 0; b < NT; b++)
                    if (Ej[b] != 0.0) atomicAdd(&d.E[(size_t)j * NT + b], Ej[b]);
            }
        }
        Seg sg = seg_of(i);
#pragma unroll
        for (int a = 0; a < NT; a++) {
            double t = seg_sum(Ei[a], sg);
            if (valid && lane == sg.first && t != 0.0) atomicAdd(&d.E[(size_t)i * NT + a], t);
        }
        if (d.site_cell) cell_energy_add(d, valid ? i : -1, epair);
        else acc[0] += epair;
    }
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// ---- per-site embedding, entropy and alpha terms (ff_dmd_I.cpp:322-351) ---
// One thread per (site, species), so that twice as many warps hide the
// table gather and the logarithms as with one thread per site.
template <int NT>
__global__ void __launch_bounds__(kFFBlock) k_dmd_embed(Dev d, int with_force, int row0)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = idx / NT, a = idx - (idx / NT) * NT;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    double e = 0.0;
    if (i < d.natms && site_active(d, i)) {
        double tmp0, tmp1;
        embed_F(d, a, d.E[(size_t)idx], tmp0, tmp1, nullptr);
        const double ca = d.c[(size_t)idx], al = d.alpha[(size_t)idx];
        d.E[(size_t)idx] = tmp0;
        if (with_force) d.dE[(size_t)idx] = tmp1;
        e += ca * tmp0;
        e += d.kbT * calc_ent(ca);
        e += 1.5 * d.kbT * ca * log(al) + ca * d.c0[a];
        if (with_force) {
            // with forces this kernel starts the site's force row (no memset
            // before the call): zero position terms and the alpha entropy
            // term, to which pass 2 adds the pair terms
            double* fi = d.f + (size_t)i * d.x_dim;
            if (a == 0) fi[0] = fi[1] = fi[2] = 0.0;
            fi[3 + a] = 0.0 - 1.5 * d.kbT * ca / al;
        }
    }
    if (d.site_cell) cell_energy_add(d, i < d.natms ? i : -1, e);
    else acc[0] += e;
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// ---- force_calc pass 2 (ff_dmd_I.cpp:357-436) ----------------------------
// One thread per compact pair: the 14 stored derivatives of a pair are read
// with coalesced streaming loads; i-side forces by segmented shuffles.
template <int NT>
__global__ void __launch_bounds__(kFFBlock, MG_DMD_MINB) k_dmd_pass2(Dev d, int st_clc, int row0)
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
        double fi[3 + NT];
#pragma unroll
        for (int q = 0; q < 3 + NT; q++) fi[q] = 0.0;
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
            const double* in = d.pr + p;
            double drr[NT * NT], dra[NT * NT], dpr[S::NC], dpa[S::NC];
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
            double ai[NT], ci[NT], dEi[NT], aj[NT], cj[NT], dEj[NT], fj[NT];
#pragma unroll
            for (int a = 0; a < NT; a++) {
                ai[a] = d.alpha[(size_t)i * NT + a];
                ci[a] = d.c[(size_t)i * NT + a];
                dEi[a] = d.dE[(size_t)i * NT + a];
                aj[a] = d.alpha[(size_t)j * NT + a];
                cj[a] = d.c[(size_t)j * NT + a];
                dEj[a] = d.dE[(size_t)oj * NT + a];
                fj[a] = 0.0;
            }
            double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
            double r_inv = rsqrt(dx0 * dx0 + dx1 * dx1 + dx2 * dx2);
            bool own_j = j < d.natms;
            double fsum = 0.0;
#pragma unroll
            for (int a = 0; a < NT; a++)
#pragma unroll
                for (int b = 0; b < NT; b++) {
                    const int ab = a * NT + b, ba = b * NT + a, ps = comp_idx(a, b);
                    double cc = ci[a] * cj[b];
                    double fpair = -(drr[ab] * dEi[a] + drr[ba] * dEj[b] + dpr[ps]) * cc * r_inv;
                    double sa = ai[a] + aj[b];
                    double apair = -(dra[ab] * dEi[a] + dra[ba] * dEj[b] + dpa[ps]) * cc / (sa * sa);
                    fsum += fpair;
                    fi[3 + a] += apair * aj[b] * aj[b];
                    fj[b] += apair * ai[a] * ai[a];
                }
            fi[0] = dx0 * fsum;
            fi[1] = dx1 * fsum;
            fi[2] = dx2 * fsum;
            if (st_clc) {
                double wf = (own_j ? 1.0 : 0.5) * fsum;
                acc[1] -= wf * dx0 * dx0;
                acc[2] -= wf * dx1 * dx1;
                acc[3] -= wf * dx2 * dx2;
                acc[4] -= wf * dx1 * dx2;
                acc[5] -= wf * dx2 * dx0;
                acc[6] -= wf * dx0 * dx1;
            }
            if (own_j) {
                double* fjp = d.f + (size_t)j * d.x_dim;
                if (fsum != 0.0) {
                    atomicAdd(fjp + 0, -dx0 * fsum);
                    atomicAdd(fjp + 1, -dx1 * fsum);
                    atomicAdd(fjp + 2, -dx2 * fsum);
                }
#pragma unroll
                for (int b = 0; b < NT; b++)
                    if (fj[b] != 0.0) atomicAdd(fjp + 3 + b, fj[b]);
            }
        }
        Seg sg = seg_of(i);
#pragma unroll
        for (int q = 0; q < 3 + NT; q++) {
            double t = seg_sum(fi[q], sg);
            if (valid && lane == sg.first && t != 0.0) atomicAdd(d.f + (size_t)i * d.x_dim + q, t);
        }
    }
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// ---- energy_calc pass (ff_dmd_I.cpp:489-633): species pairs b >= a only --
// One thread per compact pair like force pass 1, values only (no derivatives,
// nothing stored per pair); the arithmetic of a pair is the reference's
// (r = sqrt(rsq), r_inv = 1 / r).
template <int NT, int NQ>
__global__ void __launch_bounds__(kFFBlock, MG_DMD_MINB) k_dmd_energy_pass(Dev d, int row0)
{
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (long long base = (long long)blockIdx.x * blockDim.x + threadIdx.x - lane; base < d.npairs; base += stride) {
        const long long p = base + lane;
        const bool valid = p < d.npairs;
        const int i = valid ? d.pair_i[p] : -1;
        double Ei[NT];
#pragma unroll
        for (int a = 0; a < NT; a++) Ei[a] = 0.0;
        if (valid) {
            const int j = d.pair_j[p];
            const double4 xi = d.pos[i], xj = d.pos[j];
            const double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
            const double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
            if (rsq < d.cut_sq_mod) {
                double ai[NT], ci[NT], aj[NT], cj[NT], Ej[NT];
#pragma unroll
                for (int a = 0; a < NT; a++) {
                    ai[a] = d.alpha[(size_t)i * NT + a];
                    ci[a] = d.c[(size_t)i * NT + a];
                    aj[a] = d.alpha[(size_t)j * NT + a];
                    cj[a] = d.c[(size_t)j * NT + a];
                    Ej[a] = 0.0;
                }
                const bool own_j = j < d.natms;
                const double r = sqrt(rsq);
                const double r_inv = 1.0 / r;
                const double w = own_j ? 0.5 : 0.25;
#pragma unroll
                for (int a = 0; a < NT; a++)
#pragma unroll
                    for (int b = a; b < NT; b++) {
                        const int rs = b * NT + a, ps = comp_idx(a, b);
                        const double alpha = (ai[a] * aj[b]) / (ai[a] + aj[b]);
                        double g0 = 0, f0 = 0, u0, u1, u2, u3;
                        const bool hit =
                            (a == b) ? smear<true, false, NQ>(d, rs, ps, r, r_inv, rsq, alpha, g0, u0, u1, f0, u2, u3)
                                     : smear<false, false, NQ>(d, rs, ps, r, r_inv, rsq, alpha, g0, u0, u1, f0, u2, u3);
                        if (hit) {
                            Ei[a] += g0 * cj[b];
                            Ej[b] += g0 * ci[a];
                            if (a == b) acc[0] += w * (cj[b] * ci[a] + cj[a] * ci[b]) * f0;
                        }
                    }
                if (own_j) {
#pragma unroll
                    for (int b = 0; b < NT; b++)
                        if (Ej[b] != 0.0) atomicAdd(&d.E[(size_t)j * NT + b], Ej[b]);
                }
            }
        }
        const Seg sg = seg_of(i);
#pragma unroll
        for (int a = 0; a < NT; a++) {
            const double t = seg_sum(Ei[a], sg);
            if (valid && lane == sg.first && t != 0.0) atomicAdd(&d.E[(size_t)i * NT + a], t);
        }
    }
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// ---- create_2nd_neigh_lst (ff_dmd_I.cpp:2138-2217) ------------------------
__global__ void __launch_bounds__(kFFBlock) k_dmd_crd(Dev d)
{
    int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (i >= d.natms) return;
    double4 xi = d.pos[i];
    int nn = d.nnb[i];
    unsigned lt = (1u << lane) - 1u;
    int cnt = 0;
    for (int k0 = 0; k0 < nn; k0 += 32) {
        int k = k0 + lane;
        bool ok = false;
        int j = 0;
        if (k < nn) {
            j = d.nbr[(size_t)i * d.maxnb + k];
            double4 xj = d.pos[j];
            double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
            double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
            ok = rsq < d.rsq_crd;
        }
        unsigned m = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            int s = cnt + __popc(m & lt);
            if (s < d.maxcrd) d.crdl[(size_t)i * d.maxcrd + s] = j;
            if (j < d.natms) atomicAdd(&d.crd[j], 1);
        }
        cnt += __popc(m);
    }
    if (lane == 0) {
        d.ncrd[i] = min(cnt, d.maxcrd);
        atomicAdd(&d.crd[i], cnt);
        if (cnt > d.maxcrd) {
            d.status[2] = 1;
            atomicMax(&d.status[3], cnt);
        }
    }
}

__global__ void k_crd_ghosts(Dev d)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < d.nph) d.crd[d.natms + k] = d.crd[d.root[d.natms + k]];
}

// ---- c_d_calc / calc_g shared passes -------------------------------------
// Each site's list is walked by an aligned group of lanes: the neighbour
// list (about 42 entries per site at the bench density) by 16 lanes, the
// r_crd sub-list (about 6, its half of the 12 first neighbours) by 8, so that
// few lanes idle; the group's sums close with group_sum.
#ifndef MG_NBR_LANES
#define MG_NBR_LANES 16
#endif
#ifndef MG_CRD_LANES
#define MG_CRD_LANES 8
#endif
constexpr int kNbrLanes = MG_NBR_LANES;
constexpr int kCrdLanes = MG_CRD_LANES;
// E from the stored per-pair densities (ff_dmd_I.cpp:2273-2292).
template <int NT, typename P, int G>
__global__ void __launch_bounds__(kFFBlock) k_mu_E(Dev d)
{
    int i = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    int lane = threadIdx.x & (G - 1);
    if (i >= d.natms) return;
    const PairVals<NT, P> pv(d);
    double ci[NT], Ei[NT];
#pragma unroll
    for (int a = 0; a < NT; a++) {
        ci[a] = d.c[(size_t)i * NT + a];
        Ei[a] = 0.0;
    }
    int nn = d.act_on ? d.nact[i] : d.nnb[i];
    for (int k = lane; k < nn; k += G) {
        const long long slot = (d.act_on ? (long long)d.act_off[i] : (long long)d.poff[i]) + k;
        const int j = d.act_on ? d.act_pj[slot] : d.pair_j[slot];
        double cj[NT], Ej[NT];
#pragma unroll
        for (int b = 0; b < NT; b++) {
            cj[b] = d.c[(size_t)j * NT + b];
            Ej[b] = 0.0;
        }
#pragma unroll
        for (int a = 0; a < NT; a++)
#pragma unroll
            for (int b = 0; b < NT; b++) {
                Ei[a] += cj[b] * pv.rho(a * NT + b, slot);
                Ej[b] += ci[a] * pv.rho(b * NT + a, slot);
            }
        if (j < d.natms) {
#pragma unroll
            for (int b = 0; b < NT; b++)
                if (Ej[b] != 0.0) atomicAdd(&d.E[(size_t)j * NT + b], Ej[b]);
        }
    }
#pragma unroll
    for (int a = 0; a < NT; a++) {
        double s = group_sum<G>(Ei[a]);
        if (lane == 0) atomicAdd(&d.E[(size_t)i * NT + a], s);
    }
}

// n = E = F(E), dE = F'(E) (and ddE) per owned site (ff_dmd_I.cpp:2294-2314, 2472-2494).
template <int NT>
__global__ void k_mu_embed(Dev d, int with_dd)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= d.natms * NT) return;
    int a = idx % NT;
    double tmp0, tmp1, dd;
    embed_F(d, a, d.E[idx], tmp0, tmp1, with_dd ? &dd : nullptr);
    d.n[idx] = d.E[idx] = tmp0;
    d.dE[idx] = tmp1;
    if (with_dd) d.ddE[idx] = dd;
}

// Value of dE at the reference's flat index q = atom + species (the
// dE[jatm+jtype] indexing of ff_dmd_I.cpp:2336,2339), ghost entries read from
// their owner.
template <int NT>
__device__ __forceinline__ double dE_flat(const Dev& d, int q)
{
    int atom = q / NT, sp = q - atom * NT;
    return d.dE[(size_t)owner(d, atom) * NT + sp];
}

// chemical-potential pair sums (ff_dmd_I.cpp:2320-2345).
template <int NT, typename P, int G>
__global__ void __launch_bounds__(kFFBlock) k_mu_npairs(Dev d)
{
    using S = Slots<NT>;
    int i = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    int lane = threadIdx.x & (G - 1);
    if (i >= d.natms) return;
    const PairVals<NT, P> pv(d);
    double ci[NT], ni[NT], dEi_q[NT];
#pragma unroll
    for (int a = 0; a < NT; a++) {
        ci[a] = d.c[(size_t)i * NT + a];
        ni[a] = 0.0;
        dEi_q[a] = dE_flat<NT>(d, i + a);
    }
    int nn = d.act_on ? d.nact[i] : d.nnb[i];
    for (int k = lane; k < nn; k += G) {
        const long long slot = (d.act_on ? (long long)d.act_off[i] : (long long)d.poff[i]) + k;
        const int j = d.act_on ? d.act_pj[slot] : d.pair_j[slot];
        double cj[NT], nj[NT], dEj_q[NT];
#pragma unroll
        for (int b = 0; b < NT; b++) {
            cj[b] = d.c[(size_t)j * NT + b];
            nj[b] = 0.0;
            dEj_q[b] = dE_flat<NT>(d, j + b);
        }
#pragma unroll
        for (int a = 0; a < NT; a++)
#pragma unroll
            for (int b = 0; b < NT; b++) {
                double ph = pv.phi(comp_idx(a, b), slot);
                ni[a] += cj[b] * (pv.rho(b * NT + a, slot) * dEj_q[b] + ph);
                nj[b] += ci[a] * (pv.rho(a * NT + b, slot) * dEi_q[a] + ph);
            }
        if (j < d.natms) {
#pragma unroll
            for (int b = 0; b < NT; b++)
                if (nj[b] != 0.0) atomicAdd(&d.n[(size_t)j * NT + b], nj[b]);
        }
    }
#pragma unroll
    for (int a = 0; a < NT; a++) {
        double s = group_sum<G>(ni[a]);
        if (lane == 0) atomicAdd(&d.n[(size_t)i * NT + a], s);
    }
}

// per-site finalisation of n; mode as in the oracle:
//   0 c_d_calc DMD_I/DMD, 1 c_d_calc DMD_II, 2 calc_g DMD_I/DMD, 3 calc_g DMD_II
template <int NT>
__device__ __forceinline__ void mu_nfinal(const Dev& d, int idx, int mode)
{
    int a = idx % NT;
    double la = d.alpha[idx];
    double v = d.n[idx];
    if (mode == 0) {
        v += d.c0[a] + 1.5 * d.kbT * log(la);
        v *= d.beta;
    } else if (mode == 1) {
        v += d.c0[a] + 1.5 * d.kbT * log(la);
    } else if (mode == 2) {
        v += d.c0[a];
        v *= d.beta;
        v += 1.5 * log(la);
    } else {
        v += d.c0[a];
        v += 1.5 * d.kbT * log(la);
    }
    d.n[idx] = v;
}

template <int NT>
__global__ void k_mu_nfinal(Dev d, int mode)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < d.natms * NT) mu_nfinal<NT>(d, idx, mode);
}

// jump-rate term of one crd pair and species (ff_dmd_I.cpp:2372-2376,
// ff_dmd.cpp:2371-2376, ff_dmd_II.cpp:2314-2322)
__device__ __forceinline__ double rate_sij(const Dev& d, double ni, double nj, double ci, double cj)
{
    if (d.style == STYLE_DMD_II) {
        double mt = (ni > nj ? ni : nj) + 0.5;
        double exp_fi = exp(d.beta * (ni - mt));
        double exp_fj = exp(d.beta * (nj - mt));
        return cj * (1.0 - ci) * exp_fj - ci * (1.0 - cj) * exp_fi;
    }
    double Mat = (d.style == STYLE_DMD ? 5.2 : 0.4) * d.beta;
    double tmp0, tmp1;
    if (d.style == STYLE_DMD) {
        tmp0 = exp(ni + Mat);
        tmp1 = exp(nj + Mat);
    } else {
        tmp0 = exp(0.5 * (ni - nj) + Mat);
        tmp1 = exp(0.5 * (nj - ni) + Mat);
    }
    return (1.0 - ci) * cj * tmp1 - (1.0 - cj) * ci * tmp0;
}

// c_d over the r_crd sub-list (ff_dmd_I.cpp:2361-2382).
template <int NT, int G>
__global__ void __launch_bounds__(kFFBlock) k_cd_rates(Dev d)
{
    int i = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    int lane = threadIdx.x & (G - 1);
    if (i >= d.natms) return;
    double ni[NT], ci[NT], cdi[NT];
#pragma unroll
    for (int a = 0; a < NT; a++) {
        ni[a] = d.n[(size_t)i * NT + a];
        ci[a] = d.c[(size_t)i * NT + a];
        cdi[a] = 0.0;
    }
    int nc = d.ncrd[i];
    for (int k = lane; k < nc; k += G) {
        int j = d.crdl[(size_t)i * d.maxcrd + k];
        int oj = owner(d, j);
#pragma unroll
        for (int a = 0; a < NT; a++) {
            double s = rate_sij(d, ni[a], d.n[(size_t)oj * NT + a], ci[a], d.c[(size_t)j * NT + a]);
            cdi[a] += s;
            if (j < d.natms) atomicAdd(&d.c_d[(size_t)j * NT + a], -s);
        }
    }
#pragma unroll
    for (int a = 0; a < NT; a++) {
        double s = group_sum<G>(cdi[a]);
        if (lane == 0) atomicAdd(&d.c_d[(size_t)i * NT + a], s);
    }
}

// calc_g: s = 2(c + a) then the rate terms (ff_dmd_I.cpp:2537-2564,
// ff_dmd_II.cpp:2471-2511); block partial of sum s^2 computed in k_g_cost.
// (with calc_g's finalisation of n, which needs nothing from other sites)
template <int NT>
__global__ void k_g_sinit(Dev d, int mode)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= d.natms * NT) return;
    mu_nfinal<NT>(d, idx, mode);
    d.s[idx] = 2.0 * (d.c[idx] + d.a_in[idx]);
    if (d.style == STYLE_DMD_II) d.c_d[idx] = 0.0;
}

template <int NT, int G>
__global__ void __launch_bounds__(kFFBlock) k_g_srates(Dev d, double alpha)
{
    if (d.g_alpha) alpha = *d.g_alpha;
    int i = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    int lane = threadIdx.x & (G - 1);
    if (i >= d.natms) return;
    double ni[NT], ci[NT], si[NT], cdi[NT];
#pragma unroll
    for (int a = 0; a < NT; a++) {
        ni[a] = d.n[(size_t)i * NT + a];
        ci[a] = d.c[(size_t)i * NT + a];
        si[a] = cdi[a] = 0.0;
    }
    bool II = d.style == STYLE_DMD_II;
    int nc = d.ncrd[i];
    for (int k = lane; k < nc; k += G) {
        int j = d.crdl[(size_t)i * d.maxcrd + k];
        int oj = owner(d, j);
#pragma unroll
        for (int a = 0; a < NT; a++) {
            double sij = rate_sij(d, ni[a], d.n[(size_t)oj * NT + a], ci[a], d.c[(size_t)j * NT + a]);
            // DMD_I / DMD: s_ij = -2 alpha * (rate); DMD_II: s -= 2 alpha s_ij, c_d += s_ij
            double ds = -2.0 * alpha * sij;
            si[a] += ds;
            if (II) cdi[a] += sij;
            if (j < d.natms) {
                atomicAdd(&d.s[(size_t)j * NT + a], -ds);
                if (II) atomicAdd(&d.c_d[(size_t)j * NT + a], -sij);
            }
        }
    }
#pragma unroll
    for (int a = 0; a < NT; a++) {
        double s = group_sum<G>(si[a]);
        if (lane == 0) atomicAdd(&d.s[(size_t)i * NT + a], s);
        if (II) {
            double c2 = group_sum<G>(cdi[a]);
            if (lane == 0) atomicAdd(&d.c_d[(size_t)i * NT + a], c2);
        }
    }
}

template <int NT>
__global__ void __launch_bounds__(kFFBlock) k_g_cost(Dev d, int row0, int chk)
{
    if (d.g_chk) chk = *d.g_chk;
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    if (idx < d.natms * NT) {
        double s = d.s[idx];
        acc[0] = s * s;
        // the cost-only call leaves g zeroed, as the reference's does
        // (g cleared at ff_dmd_I.cpp:2444-2445, return before the g terms)
        d.g[idx] = chk ? 0.0 : -s;
        d.t[idx] = 0.0;
        d.v[idx] = 0.0;
    }
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// t and the first g terms over the crd sub-list (ff_dmd_I.cpp:2582-2608,
// ff_dmd.cpp:2582-2605, ff_dmd_II.cpp:2529-2564).
template <int NT, int G>
__global__ void __launch_bounds__(kFFBlock) k_g_trates(Dev d, double alpha)
{
    if (d.g_chk && *d.g_chk) return;  // cost-only call: no g terms
    if (d.g_alpha) alpha = *d.g_alpha;
    int i = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    int lane = threadIdx.x & (G - 1);
    if (i >= d.natms) return;
    double ni[NT], ci[NT], si[NT], ti[NT], gi[NT];
#pragma unroll
    for (int a = 0; a < NT; a++) {
        ni[a] = d.n[(size_t)i * NT + a];
        ci[a] = d.c[(size_t)i * NT + a];
        si[a] = d.s[(size_t)i * NT + a];
        ti[a] = gi[a] = 0.0;
    }
    int nc = d.ncrd[i];
    for (int k = lane; k < nc; k += G) {
        int j = d.crdl[(size_t)i * d.maxcrd + k];
        int oj = owner(d, j);
        bool own_j = j < d.natms;
#pragma unroll
        for (int a = 0; a < NT; a++) {
            double nj = d.n[(size_t)oj * NT + a], cj = d.c[(size_t)j * NT + a], sj = d.s[(size_t)oj * NT + a];
            double dt_i, dt_j, dg_i, dg_j;
            double ds = si[a] - sj;
            if (d.style == STYLE_DMD_II) {
                double mt = (ni[a] > nj ? ni[a] : nj) + 0.5;
                double exp_fi = exp(d.beta * (ni[a] - mt)), exp_fj = exp(d.beta * (nj - mt));
                double tmpi = ci[a] * (1.0 - cj), tmpj = cj * (1.0 - ci[a]);
                double dmi = ni[a] > nj ? 1.0 : 0.0, dmj = nj > ni[a] ? 1.0 : 0.0;
                dt_i = (tmpi * exp_fi + dmi * (tmpj * exp_fj - tmpi * exp_fi)) * ds;
                dt_j = (tmpj * exp_fj + dmj * (tmpi * exp_fi - tmpj * exp_fj)) * ds;
                dg_i = -alpha * ((1.0 - cj) * exp_fi + cj * exp_fj) * ds;
                dg_j = alpha * ((1.0 - ci[a]) * exp_fj + ci[a] * exp_fi) * ds;
            } else if (d.style == STYLE_DMD) {
                double Mat = 5.2 * d.beta;
                double tmp0 = ds * exp(Mat + ni[a]), tmp1 = ds * exp(Mat + nj);
                dt_i = ci[a] * tmp0 * (1.0 - cj);
                dt_j = cj * tmp1 * (1.0 - ci[a]);
                dg_i = -alpha * (tmp0 * (1.0 - cj) + tmp1 * cj);
                dg_j = alpha * (tmp1 * (1.0 - ci[a]) + ci[a] * tmp0);
            } else {
                double Mat = 0.4 * d.beta;
                double tmp0 = exp(0.5 * (ni[a] - nj) + Mat) * ds, tmp1 = exp(0.5 * (nj - ni[a]) + Mat) * ds;
                double t_ij = 0.5 * (ci[a] * (1.0 - cj) * tmp0 + cj * (1.0 - ci[a]) * tmp1);
                dt_i = t_ij;
                dt_j = t_ij;
                dg_i = -alpha * (tmp0 * (1.0 - cj) + tmp1 * cj);
                dg_j = alpha * (tmp1 * (1.0 - ci[a]) + ci[a] * tmp0);
            }
            ti[a] += dt_i;
            gi[a] += dg_i;
            if (own_j) {
                atomicAdd(&d.t[(size_t)j * NT + a], -dt_j);
                atomicAdd(&d.g[(size_t)j * NT + a], dg_j);
            }
        }
    }
#pragma unroll
    for (int a = 0; a < NT; a++) {
        double s = group_sum<G>(ti[a]), g = group_sum<G>(gi[a]);
        if (lane == 0) {
            atomicAdd(&d.t[(size_t)i * NT + a], s);
            atomicAdd(&d.g[(size_t)i * NT + a], g);
        }
    }
}

// v and the t-weighted g terms over the full list (ff_dmd_I.cpp:2612-2644).
template <int NT, typename P, int G>
__global__ void __launch_bounds__(kFFBlock) k_g_vpass(Dev d, double alpha)
{
    if (d.g_chk && *d.g_chk) return;  // cost-only call: no g terms
    if (d.g_alpha) alpha = *d.g_alpha;
    using S = Slots<NT>;
    int i = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    int lane = threadIdx.x & (G - 1);
    if (i >= d.natms) return;
    const PairVals<NT, P> pv(d);
    double dEi[NT], ti[NT], vi[NT], gi[NT];
#pragma unroll
    for (int a = 0; a < NT; a++) {
        dEi[a] = d.dE[(size_t)i * NT + a];
        ti[a] = d.t[(size_t)i * NT + a];
        vi[a] = gi[a] = 0.0;
    }
    double ba = d.beta * alpha;
    int nn = d.act_on ? d.nact[i] : d.nnb[i];
    for (int k = lane; k < nn; k += G) {
        const long long slot = (d.act_on ? (long long)d.act_off[i] : (long long)d.poff[i]) + k;
        const int j = d.act_on ? d.act_pj[slot] : d.pair_j[slot];
        int oj = owner(d, j);
        double dEj[NT], tj[NT], vj[NT], gj[NT];
#pragma unroll
        for (int b = 0; b < NT; b++) {
            dEj[b] = d.dE[(size_t)oj * NT + b];
            tj[b] = d.t[(size_t)oj * NT + b];
            vj[b] = gj[b] = 0.0;
        }
#pragma unroll
        for (int a = 0; a < NT; a++)
#pragma unroll
            for (int b = 0; b < NT; b++) {
                double r_ab = pv.rho(a * NT + b, slot);  // type2rho[jtype][itype]
                double r_ba = pv.rho(b * NT + a, slot);  // type2rho[itype][jtype]
                double tmp0 = pv.phi(comp_idx(b, a), slot) + r_ab * dEi[a] + r_ba * dEj[b];
                tmp0 *= ba;
                vi[a] += r_ab * tj[b];
                gi[a] += tmp0 * tj[b];
                vj[b] += r_ba * ti[a];
                gj[b] += tmp0 * ti[a];
            }
        if (j < d.natms) {
#pragma unroll
            for (int b = 0; b < NT; b++) {
                if (vj[b] != 0.0) atomicAdd(&d.v[(size_t)j * NT + b], vj[b]);
                if (gj[b] != 0.0) atomicAdd(&d.g[(size_t)j * NT + b], gj[b]);
            }
        }
    }
#pragma unroll
    for (int a = 0; a < NT; a++) {
        double s = group_sum<G>(vi[a]), g = group_sum<G>(gi[a]);
        if (lane == 0) {
            atomicAdd(&d.v[(size_t)i * NT + a], s);
            atomicAdd(&d.g[(size_t)i * NT + a], g);
        }
    }
}

// last g terms with ddE (ff_dmd_I.cpp:2649-2670).
template <int NT, typename P, int G>
__global__ void __launch_bounds__(kFFBlock) k_g_last(Dev d, double alpha)
{
    if (d.g_chk && *d.g_chk) return;  // cost-only call: no g terms
    if (d.g_alpha) alpha = *d.g_alpha;
    int i = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    int lane = threadIdx.x & (G - 1);
    if (i >= d.natms) return;
    const PairVals<NT, P> pv(d);
    double wi[NT], gi[NT];
    double ab = alpha * d.beta;
#pragma unroll
    for (int a = 0; a < NT; a++) {
        size_t q = (size_t)i * NT + a;
        wi[a] = d.ddE[q] * d.c[q] * d.v[q];
        gi[a] = 0.0;
    }
    int nn = d.act_on ? d.nact[i] : d.nnb[i];
    for (int k = lane; k < nn; k += G) {
        const long long slot = (d.act_on ? (long long)d.act_off[i] : (long long)d.poff[i]) + k;
        const int j = d.act_on ? d.act_pj[slot] : d.pair_j[slot];
        int oj = owner(d, j);
        double wj[NT], gj[NT];
#pragma unroll
        for (int b = 0; b < NT; b++) {
            size_t q = (size_t)oj * NT + b;
            wj[b] = d.ddE[q] * d.c[(size_t)j * NT + b] * d.v[q];
            gj[b] = 0.0;
        }
#pragma unroll
        for (int a = 0; a < NT; a++)
#pragma unroll
            for (int b = 0; b < NT; b++) {
                gi[a] += ab * pv.rho(b * NT + a, slot) * wj[b];
                gj[b] += ab * pv.rho(a * NT + b, slot) * wi[a];
            }
        if (j < d.natms) {
#pragma unroll
            for (int b = 0; b < NT; b++)
                if (gj[b] != 0.0) atomicAdd(&d.g[(size_t)j * NT + b], gj[b]);
        }
    }
#pragma unroll
    for (int a = 0; a < NT; a++) {
        double g = group_sum<G>(gi[a]);
        if (lane == 0) atomicAdd(&d.g[(size_t)i * NT + a], g);
    }
}

// the active sublist (Dev::act_*): a listed pair is active when any of its
// stored densities or pair energies (the only per-pair values c_d_calc and
// calc_g read) is non-zero; an inactive pair adds exact zeros there.
// Pass 1 counts each owned site's active pairs (nact, with nact[natms] = 0 so
// that the scan's last element is the total); pass 2, after the scan into
// act_off, copies their partners and values to the CSR arrays.
template <int NT>
__device__ __forceinline__ bool pair_active(const Dev& d, long long slot)
{
    using S = Slots<NT>;
    bool on = false;
#pragma unroll
    for (int q = 0; q < NT * NT; q++) on |= d.pr[(size_t)(S::RHO + q) * d.maxp + slot] != 0.0;
#pragma unroll
    for (int q = 0; q < S::NC; q++) on |= d.pr[(size_t)(S::PHI + q) * d.maxp + slot] != 0.0;
    return on;
}

template <int NT>
__global__ void k_active_count(Dev d)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) d.nact[d.natms] = 0;
    if (i >= d.natms) return;
    const int nn = d.nnb[i];
    int m = 0;
    for (int k = 0; k < nn; k++) m += pair_active<NT>(d, (long long)d.poff[i] + k) ? 1 : 0;
    d.nact[i] = m;
}

template <int NT>
__global__ void k_active_fill(Dev d)
{
    using S = Slots<NT>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.natms) return;
    const int nn = d.nnb[i];
    long long o = d.act_off[i];
    for (int k = 0; k < nn; k++) {
        const long long slot = (long long)d.poff[i] + k;
        if (!pair_active<NT>(d, slot)) continue;
        d.act_pj[o] = d.pair_j[slot];
#pragma unroll
        for (int q = 0; q < NT * NT; q++) d.act_pv[(size_t)q * d.act_cap + o] = d.pr[(size_t)(S::RHO + q) * d.maxp + slot];
#pragma unroll
        for (int q = 0; q < S::NC; q++)
            d.act_pv[(size_t)(NT * NT + q) * d.act_cap + o] = d.pr[(size_t)(S::PHI + q) * d.maxp + slot];
        o++;
    }
}

template <int NT>
cudaError_t dmd_force_nt(const Dev& d, int st_clc, int* nb, cudaStream_t st, cudaEvent_t* evs)
{
    int g1 = persistent_grid(d.npairs, d.tune_bps > 0 ? d.tune_bps : MG_DMD_MINB), g2 = div_up(d.natms * NT, kFFBlock);
    int g3 = persistent_grid(d.npairs, d.tune_bps2 > 0 ? d.tune_bps2 : MG_DMD_MINB);
    if (evs) cudaEventRecord(evs[0], st);
    if (d.nq == 3) k_dmd_pass1<NT, 3><<<g1, kFFBlock, 0, st>>>(d, 0);
    else k_dmd_pass1<NT, 0><<<g1, kFFBlock, 0, st>>>(d, 0);
    if (evs) cudaEventRecord(evs[1], st);
    k_dmd_embed<NT><<<g2, kFFBlock, 0, st>>>(d, 1, g1);
    if (evs) cudaEventRecord(evs[2], st);
    k_dmd_pass2<NT><<<g3, kFFBlock, 0, st>>>(d, st_clc, g1 + g2);
    if (evs) cudaEventRecord(evs[3], st);
    *nb = g1 + g2 + g3;
    return cudaGetLastError();
}

template <int NT>
cudaError_t dmd_energy_nt(const Dev& d, int* nb, cudaStream_t st)
{
    int g1 = persistent_grid(d.npairs, MG_DMD_MINB), g2 = div_up(d.natms * NT, kFFBlock);
    if (d.nq == 3) k_dmd_energy_pass<NT, 3><<<g1, kFFBlock, 0, st>>>(d, 0);
    else k_dmd_energy_pass<NT, 0><<<g1, kFFBlock, 0, st>>>(d, 0);
    k_dmd_embed<NT><<<g2, kFFBlock, 0, st>>>(d, 0, g1);
    *nb = g1 + g2;
    return cudaGetLastError();
}

template <int NT, typename P>
cudaError_t dmd_cdot_ntp(const Dev& d, cudaStream_t st)
{
    int gw = div_up((long long)d.natms * kNbrLanes, kFFBlock), gc = div_up((long long)d.natms * kCrdLanes, kFFBlock);
    int gs = div_up((long long)d.natms * NT, kFFBlock);
    k_mu_E<NT, P, kNbrLanes><<<gw, kFFBlock, 0, st>>>(d);
    k_mu_embed<NT><<<gs, kFFBlock, 0, st>>>(d, 0);
    k_mu_npairs<NT, P, kNbrLanes><<<gw, kFFBlock, 0, st>>>(d);
    k_mu_nfinal<NT><<<gs, kFFBlock, 0, st>>>(d, d.style == STYLE_DMD_II ? 1 : 0);
    k_cd_rates<NT, kCrdLanes><<<gc, kFFBlock, 0, st>>>(d);
    return cudaGetLastError();
}

template <int NT>
cudaError_t dmd_cdot_nt(const Dev& d, cudaStream_t st)
{
    return d.form != 0 ? dmd_cdot_ntp<NT, float>(d, st) : dmd_cdot_ntp<NT, double>(d, st);
}

template <int NT, typename P>
cudaError_t dmd_calc_g_ntp(const Dev& d, int chk, double alpha, int* nb, cudaStream_t st)
{
    int gw = div_up((long long)d.natms * kNbrLanes, kFFBlock), gc = div_up((long long)d.natms * kCrdLanes, kFFBlock);
    int gs = div_up((long long)d.natms * NT, kFFBlock);
    k_mu_E<NT, P, kNbrLanes><<<gw, kFFBlock, 0, st>>>(d);
    k_mu_embed<NT><<<gs, kFFBlock, 0, st>>>(d, 1);
    k_mu_npairs<NT, P, kNbrLanes><<<gw, kFFBlock, 0, st>>>(d);
    k_g_sinit<NT><<<gs, kFFBlock, 0, st>>>(d, d.style == STYLE_DMD_II ? 3 : 2);
    k_g_srates<NT, kCrdLanes><<<gc, kFFBlock, 0, st>>>(d, alpha);
    k_g_cost<NT><<<gs, kFFBlock, 0, st>>>(d, 0, chk);
    *nb = gs;
    if (!chk || d.g_chk) {
        k_g_trates<NT, kCrdLanes><<<gc, kFFBlock, 0, st>>>(d, alpha);
        k_g_vpass<NT, P, kNbrLanes><<<gw, kFFBlock, 0, st>>>(d, alpha);
        k_g_last<NT, P, kNbrLanes><<<gw, kFFBlock, 0, st>>>(d, alpha);
    }
    return cudaGetLastError();
}

template <int NT>
cudaError_t dmd_calc_g_nt(const Dev& d, int chk, double alpha, int* nb, cudaStream_t st)
{
    return d.form != 0 ? dmd_calc_g_ntp<NT, float>(d, chk, alpha, nb, st)
                       : dmd_calc_g_ntp<NT, double>(d, chk, alpha, nb, st);
}

}  // namespace

cudaError_t launch_dmd_force(const Dev& d, int st_clc, int* nb, cudaStream_t st, cudaEvent_t* evs)
{
    switch (d.nt) {
    case 1: return dmd_force_nt<1>(d, st_clc, nb, st, evs);
    case 2: return dmd_force_nt<2>(d, st_clc, nb, st, evs);
    case 3: return dmd_force_nt<3>(d, st_clc, nb, st, evs);
    case 4: return dmd_force_nt<4>(d, st_clc, nb, st, evs);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dmd_energy(const Dev& d, int* nb, cudaStream_t st)
{
    switch (d.nt) {
    case 1: return dmd_energy_nt<1>(d, nb, st);
    case 2: return dmd_energy_nt<2>(d, nb, st);
    case 3: return dmd_energy_nt<3>(d, nb, st);
    case 4: return dmd_energy_nt<4>(d, nb, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dmd_crd(const Dev& d, cudaStream_t st)
{
    if (d.natms) k_dmd_crd<<<div_up((long long)d.natms * 32, kFFBlock), kFFBlock, 0, st>>>(d);
    if (d.nph) k_crd_ghosts<<<div_up(d.nph, kFFBlock), kFFBlock, 0, st>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_dmd_cdot(const Dev& d, cudaStream_t st)
{
    switch (d.nt) {
    case 1: return dmd_cdot_nt<1>(d, st);
    case 2: return dmd_cdot_nt<2>(d, st);
    case 3: return dmd_cdot_nt<3>(d, st);
    case 4: return dmd_cdot_nt<4>(d, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_active_count(const Dev& d, cudaStream_t st)
{
    const int g = div_up(d.natms + 1, kFFBlock);
    switch (d.nt) {
    case 1: k_active_count<1><<<g, kFFBlock, 0, st>>>(d); break;
    case 2: k_active_count<2><<<g, kFFBlock, 0, st>>>(d); break;
    case 3: k_active_count<3><<<g, kFFBlock, 0, st>>>(d); break;
    case 4: k_active_count<4><<<g, kFFBlock, 0, st>>>(d); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_active_fill(const Dev& d, cudaStream_t st)
{
    const int g = div_up(d.natms, kFFBlock);
    switch (d.nt) {
    case 1: k_active_fill<1><<<g, kFFBlock, 0, st>>>(d); break;
    case 2: k_active_fill<2><<<g, kFFBlock, 0, st>>>(d); break;
    case 3: k_active_fill<3><<<g, kFFBlock, 0, st>>>(d); break;
    case 4: k_active_fill<4><<<g, kFFBlock, 0, st>>>(d); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_dmd_calc_g(const Dev& d, int chk, double alpha, int* nb, cudaStream_t st)
{
    switch (d.nt) {
    case 1: return dmd_calc_g_nt<1>(d, chk, alpha, nb, st);
    case 2: return dmd_calc_g_nt<2>(d, chk, alpha, nb, st);
    case 3: return dmd_calc_g_nt<3>(d, chk, alpha, nb, st);
    case 4: return dmd_calc_g_nt<4>(d, chk, alpha, nb, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace mg
