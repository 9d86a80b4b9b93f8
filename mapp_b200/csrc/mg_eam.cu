// Tabulated EAM (ff_eam.cpp:44-356) and analytic Finnis-Sinclair
// (ff_fs.cpp:379-684) force / energy kernels.
//
// Layout of work: one warp per owned atom i, lanes stride over i's half list.
// i-side sums (density, force) are warp-shuffle reductions finished with one
// atomic per warp; j-side contributions are FP64 atomics on j (owned j only,
// as in the reference: ghost j receive nothing and their pair energy and
// virial count one half).  Energy and virial go to per-block partial rows
// reduced deterministically at the end.
//
// Pass 1 stores -drho/dr / r for both sides of every pair (pair slot
// i*maxnb+k) exactly like drhoi_dr / drhoj_dr (ff_eam.cpp:172-173); pass 2
// reads F'(rho) of a ghost j from its owner (the ghost refresh
// atoms->update(rho_n), ff_eam.cpp:194, fused into the load).
#include "mg_reduce.cuh"

namespace mg {

namespace {

__device__ __forceinline__ int owner(const Dev& d, int j) { return j < d.natms ? j : d.root[j]; }

// One knot row of a spline table (8 doubles: c0..c3 of the value, c4..c6 of
// the derivative, one pad) as two 32-byte read-only loads.
struct Row8 {
    double4 v, dv;
};
__device__ __forceinline__ Row8 row8(const double* __restrict__ row)
{
    Row8 r;
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(r.v.x), "=d"(r.v.y), "=d"(r.v.z), "=d"(r.v.w) : "l"(row));
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
        : "=d"(r.dv.x), "=d"(r.dv.y), "=d"(r.dv.z), "=d"(r.dv.w)
        : "l"(row + 4));
    return r;
}

// Resident blocks per SM the EAM pass 1 is compiled for (64 registers a
// thread at 4): a small system's warps then fit one wave.
#ifndef MG_EAM_MINB
#define MG_EAM_MINB 4
#endif

// EAM pass 1 (ff_eam.cpp:95-177).  energy_only skips forces and stored
// derivatives (ForceField_eam::energy_calc, ff_eam.cpp:297-338).
template <bool kEnergyOnly>
__global__ void __launch_bounds__(kFFBlock, MG_EAM_MINB) k_eam_pass1(Dev d, int st_clc, int row0)
{
    int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    if (i < d.natms) {
        double4 xi = d.pos[i];
        int ti = d.type[i];
        int nt = d.nt;
        double rho_i = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
        int nn = d.nnb[i];
        for (int k = lane; k < nn; k += 32) {
            long long slot = (long long)i * d.maxnb + k;
            int j = d.nbr[slot];
            int tj = d.type[j];
            double4 xj = d.pos[j];
            double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
            double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
            double pi_ = 0.0, pj_ = 0.0;
            if (rsq < d.cut_sq) {
                double r = sqrt(rsq);
                double r_inv = 1.0 / r;
                double p = r * d.dr_inv;
                int m = min((int)p, d.nr - 2);
                p -= m;
                p = fmin(p, 1.0);
                const Row8 cf = row8(d.rhoT + ((size_t)(ti * nt + tj) * d.nr + m) * 8);
                double rho_iv = ((cf.v.w * p + cf.v.z) * p + cf.v.y) * p + cf.v.x;
                double drho_i = (cf.dv.z * p + cf.dv.y) * p + cf.dv.x;
                // the j-side density row is the same row when the species agree
                const Row8 cg = tj == ti ? cf : row8(d.rhoT + ((size_t)(tj * nt + ti) * d.nr + m) * 8);
                double rho_jv = ((cg.v.w * p + cg.v.z) * p + cg.v.y) * p + cg.v.x;
                double drho_j = (cg.dv.z * p + cg.dv.y) * p + cg.dv.x;
                const Row8 ch = row8(d.phiT + ((size_t)comp_idx(ti, tj) * d.nr + m) * 8);
                double z2 = ((ch.v.w * p + ch.v.z) * p + ch.v.y) * p + ch.v.x;
                double phi = z2 * r_inv;
                rho_i += rho_iv;
                bool own_j = j < d.natms;
                if (own_j) atomicAdd(&d.rho[j], rho_jv);
                double w = own_j ? 1.0 : 0.5;
                acc[0] += w * phi;
                if (!kEnergyOnly) {
                    double z2p = (ch.dv.z * p + ch.dv.y) * p + ch.dv.x;
                    double dphi = z2p * r_inv - phi * r_inv;
                    double fpair = -dphi * r_inv;
                    fx += fpair * dx0;
                    fy += fpair * dx1;
                    fz += fpair * dx2;
                    if (own_j) {
                        double* fj = d.f + (size_t)j * 3;
                        atomicAdd(fj + 0, -fpair * dx0);
                        atomicAdd(fj + 1, -fpair * dx1);
                        atomicAdd(fj + 2, -fpair * dx2);
                    }
                    if (st_clc) {
                        double wf = w * fpair;
                        acc[1] -= wf * dx0 * dx0;
                        acc[2] -= wf * dx1 * dx1;
                        acc[3] -= wf * dx2 * dx2;
                        acc[4] -= wf * dx1 * dx2;
                        acc[5] -= wf * dx2 * dx0;
                        acc[6] -= wf * dx0 * dx1;
                    }
                    pi_ = -drho_i * r_inv;
                    pj_ = -drho_j * r_inv;
                }
            }
            if (!kEnergyOnly) {
                d.pr[slot] = pi_;
                d.pr[d.maxp + slot] = pj_;
            }
        }
        rho_i = warp_sum(rho_i);
        if (!kEnergyOnly) {
            fx = warp_sum(fx);
            fy = warp_sum(fy);
            fz = warp_sum(fz);
        }
        if (lane == 0) {
            atomicAdd(&d.rho[i], rho_i);
            if (!kEnergyOnly) {
                atomicAdd(d.f + (size_t)i * 3 + 0, fx);
                atomicAdd(d.f + (size_t)i * 3 + 1, fy);
                atomicAdd(d.f + (size_t)i * 3 + 2, fz);
            }
        }
    }
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// Embedding energy F(rho) and F'(rho) per owned atom (ff_eam.cpp:178-190);
// the index clamp uses nr-2 like the reference (ff_eam.cpp:180).
template <bool kEnergyOnly>
__global__ void __launch_bounds__(kFFBlock) k_eam_embed(Dev d, int row0)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    if (i < d.natms) {
        double rv = d.rho[i];
        double p = rv * d.drho_inv;
        int m = max(0, min((int)p, d.nr - 2));  // lower clamp: never index before the table
        p -= m;
        p = fmin(p, 1.0);
        const double* cf = d.FT + ((size_t)d.type[i] * (d.nrho + 1) + m) * d.Fw;
        double tmp1 = (cf[6] * p + cf[5]) * p + cf[4];
        double tmp0 = ((cf[3] * p + cf[2]) * p + cf[1]) * p + cf[0];
        if (rv > d.rho_max) tmp0 += tmp1 * (rv - d.rho_max);
        acc[0] = tmp0;
        if (!kEnergyOnly) d.rho[i] = tmp1;
    }
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// EAM / FS pass 2: embedding forces from the stored pair derivatives
// (ff_eam.cpp:196-250, ff_fs.cpp:531-588).
__global__ void __launch_bounds__(kFFBlock) k_embed_pass2(Dev d, int st_clc, int row0)
{
    int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    if (i < d.natms) {
        double4 xi = d.pos[i];
        double dFi = d.rho[i];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        int nn = d.nnb[i];
        for (int k = lane; k < nn; k += 32) {
            long long slot = (long long)i * d.maxnb + k;
            double pi_ = d.pr[slot], pj_ = d.pr[d.maxp + slot];
            if (pi_ != 0.0 || pj_ != 0.0) {
                int j = d.nbr[slot];
                double4 xj = d.pos[j];
                double fpair = dFi * pi_ + d.rho[owner(d, j)] * pj_;
                double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
                fx += dx0 * fpair;
                fy += dx1 * fpair;
                fz += dx2 * fpair;
                bool own_j = j < d.natms;
                if (own_j) {
                    double* fj = d.f + (size_t)j * 3;
                    atomicAdd(fj + 0, -dx0 * fpair);
                    atomicAdd(fj + 1, -dx1 * fpair);
                    atomicAdd(fj + 2, -dx2 * fpair);
                }
                if (st_clc) {
                    double wf = (own_j ? 1.0 : 0.5) * fpair;
                    acc[1] -= wf * dx0 * dx0;
                    acc[2] -= wf * dx1 * dx1;
                    acc[3] -= wf * dx2 * dx2;
                    acc[4] -= wf * dx1 * dx2;
                    acc[5] -= wf * dx2 * dx0;
                    acc[6] -= wf * dx0 * dx1;
                }
            }
        }
        fx = warp_sum(fx);
        fy = warp_sum(fy);
        fz = warp_sum(fz);
        if (lane == 0) {
            atomicAdd(d.f + (size_t)i * 3 + 0, fx);
            atomicAdd(d.f + (size_t)i * 3 + 1, fy);
            atomicAdd(d.f + (size_t)i * 3 + 2, fz);
        }
    }
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// Analytic FS pass 1 (ff_fs.cpp:424-527).
template <bool kEnergyOnly>
__global__ void __launch_bounds__(kFFBlock) k_fs_pass1(Dev d, int st_clc, int row0)
{
    int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    if (i < d.natms) {
        double4 xi = d.pos[i];
        int ti = d.type[i];
        double rho_i = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
        int nn = d.nnb[i];
        for (int k = lane; k < nn; k += 32) {
            long long slot = (long long)i * d.maxnb + k;
            int j = d.nbr[slot];
            int tj = d.type[j];
            int cs = comp_idx(ti, tj);
            double pi_ = 0.0, pj_ = 0.0;
            if (d.fs_chk[cs]) {
                double4 xj = d.pos[j];
                double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
                double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
                if (rsq < d.fs_cut_sq[cs]) {
                    double r = sqrt(rsq);
                    double r_inv = 1.0 / r;
                    bool own_j = j < d.natms;
                    double w = own_j ? 1.0 : 0.5;
                    if (r < d.fs_cut_rho[cs]) {
                        double dr_ = r - d.fs_cut_rho[cs];
                        rho_i += dr_ * dr_ * (d.fst1[tj][ti] + d.fst2[tj][ti] * dr_);
                        if (own_j) atomicAdd(&d.rho[j], dr_ * dr_ * (d.fst1[ti][tj] + d.fst2[ti][tj] * dr_));
                        pi_ = -r_inv * dr_ * (d.fst1[tj][ti] + 1.5 * d.fst2[tj][ti] * dr_);
                        pj_ = -r_inv * dr_ * (d.fst1[ti][tj] + 1.5 * d.fst2[ti][tj] * dr_);
                    }
                    if (r < d.fs_cut_phi[cs]) {
                        double dp = r - d.fs_cut_phi[cs];
                        double poly = d.fsk1[cs] + d.fsk2[cs] * r + d.fsk3[cs] * rsq;
                        acc[0] += w * (dp * dp * poly);
                        if (!kEnergyOnly) {
                            double pc = 2.0 * dp * poly + dp * dp * (d.fsk2[cs] + 2.0 * d.fsk3[cs] * r);
                            pc *= -r_inv;
                            fx += dx0 * pc;
                            fy += dx1 * pc;
                            fz += dx2 * pc;
                            if (own_j) {
                                double* fj = d.f + (size_t)j * 3;
                                atomicAdd(fj + 0, -dx0 * pc);
                                atomicAdd(fj + 1, -dx1 * pc);
                                atomicAdd(fj + 2, -dx2 * pc);
                            }
                            if (st_clc) {
                                double wf = w * pc;
                                acc[1] -= wf * dx0 * dx0;
                                acc[2] -= wf * dx1 * dx1;
                                acc[3] -= wf * dx2 * dx2;
                                acc[4] -= wf * dx1 * dx2;
                                acc[5] -= wf * dx2 * dx0;
                                acc[6] -= wf * dx0 * dx1;
                            }
                        }
                    }
                }
            }
            if (!kEnergyOnly) {
                d.pr[slot] = pi_;
                d.pr[d.maxp + slot] = pj_;
            }
        }
        rho_i = warp_sum(rho_i);
        if (!kEnergyOnly) {
            fx = warp_sum(fx);
            fy = warp_sum(fy);
            fz = warp_sum(fz);
        }
        if (lane == 0) {
            atomicAdd(&d.rho[i], rho_i);
            if (!kEnergyOnly) {
                atomicAdd(d.f + (size_t)i * 3 + 0, fx);
                atomicAdd(d.f + (size_t)i * 3 + 1, fy);
                atomicAdd(d.f + (size_t)i * 3 + 2, fz);
            }
        }
    }
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

// FS embedding: F = -A sqrt(rho), stores 2 F'(rho) = -A / sqrt(rho) (ff_fs.cpp:524-526).
template <bool kEnergyOnly>
__global__ void __launch_bounds__(kFFBlock) k_fs_embed(Dev d, int row0)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    if (i < d.natms) {
        double rs = sqrt(d.rho[i]);
        double A = d.fsA[d.type[i]];
        acc[0] = -(A * rs);
        if (!kEnergyOnly) d.rho[i] = -A / rs;
    }
    block_partials<7>(acc, d.partial, row0 + blockIdx.x);
}

}  // namespace

cudaError_t launch_eam_force(const Dev& d, int st_clc, int* nblocks_out, cudaStream_t st)
{
    int g1 = div_up((long long)d.natms * 32, kFFBlock), g2 = div_up(d.natms, kFFBlock);
    k_eam_pass1<false><<<g1, kFFBlock, 0, st>>>(d, st_clc, 0);
    k_eam_embed<false><<<g2, kFFBlock, 0, st>>>(d, g1);
    k_embed_pass2<<<g1, kFFBlock, 0, st>>>(d, st_clc, g1 + g2);
    *nblocks_out = 2 * g1 + g2;
    return cudaGetLastError();
}

cudaError_t launch_eam_energy(const Dev& d, int* nblocks_out, cudaStream_t st)
{
    int g1 = div_up((long long)d.natms * 32, kFFBlock), g2 = div_up(d.natms, kFFBlock);
    k_eam_pass1<true><<<g1, kFFBlock, 0, st>>>(d, 0, 0);
    k_eam_embed<true><<<g2, kFFBlock, 0, st>>>(d, g1);
    *nblocks_out = g1 + g2;
    return cudaGetLastError();
}

cudaError_t launch_fs_force(const Dev& d, int st_clc, int* nblocks_out, cudaStream_t st)
{
    int g1 = div_up((long long)d.natms * 32, kFFBlock), g2 = div_up(d.natms, kFFBlock);
    k_fs_pass1<false><<<g1, kFFBlock, 0, st>>>(d, st_clc, 0);
    k_fs_embed<false><<<g2, kFFBlock, 0, st>>>(d, g1);
    k_embed_pass2<<<g1, kFFBlock, 0, st>>>(d, st_clc, g1 + g2);
    *nblocks_out = 2 * g1 + g2;
    return cudaGetLastError();
}

cudaError_t launch_fs_energy(const Dev& d, int* nblocks_out, cudaStream_t st)
{
    int g1 = div_up((long long)d.natms * 32, kFFBlock), g2 = div_up(d.natms, kFFBlock);
    k_fs_pass1<true><<<g1, kFFBlock, 0, st>>>(d, 0, 0);
    k_fs_embed<true><<<g2, kFFBlock, 0, st>>>(d, g1);
    *nblocks_out = g1 + g2;
    return cudaGetLastError();
}

}  // namespace mg
