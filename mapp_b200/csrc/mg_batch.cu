// Batched form: many independent periodic DMD cells relaxed by L-BFGS
// together on one GPU.
//
// Layout.  The cells are concatenated into one system: all owned sites first
// (cell by cell), then all ghosts (cell by cell), and one compact pair list
// whose indices point into that numbering.  The force kernels of the plain
// and precision forms run on it unchanged except for two batch hooks: pairs
// and sites of stopped cells are skipped, and energies are summed per cell
// (Dev::site_cell / cell_active / cell_E).  A ghost keeps its owner and the
// fixed image shift x_ghost - x_owner of its cell, so refreshing ghosts after
// a move is one add per ghost.
//
// Solver.  Each cell runs Min_LBFGS::run (min_l-bfgs.cpp:616-773) with
// LineSearch_BackTrack::line_min (line_search.cpp:223-342) as a state machine
// in k_lbfgs_step, one CTA per cell: after every force evaluation the cell
// either accepts its trial point (history update, two-loop recursion, new
// direction, first trial of the next line search), halves its step, or
// stops.  The line search takes its energies from the force pass, so an
// accepted trial already has its forces.  Dot products, Armijo tests and
// energies are FP64.
//
// Launch.  One iteration (ghost refresh, zeroing, the three force passes, the
// L-BFGS step, the loop test) is captured once as the body of a conditional
// WHILE node; a relaxation is one graph launch, and the loop test ends it
// when no cell is left running or the iteration budget is spent.  When a
// cell's trial point leaves its neighbour list's skin (the rule of
// Atoms::update_0, atoms.cpp:1800-1818) the cell pauses; after the launch the
// host rebuilds the lists of every cell and launches again.
//
// Autotuning.  The blocks per SM of the two pair passes and the threads per
// cell of the L-BFGS step are timed on the batch itself and the choice is
// kept in a cache keyed by the batch's shape.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include <cooperative_groups.h>

#include "../../include/mapp_b200.h"
#include "mg_reduce.cuh"

using namespace mg;

namespace {

constexpr int kBMaxM = 8;

// line_search.h:7 codes; kRunning while the cell is active
enum { kRunning = 0, kDownhill = 1, kGrad0 = 2, kAlphaMin = 3, kMaxIter = 4, kTolerance = 5 };
enum { PH_FIRST = 0, PH_TRIAL = 1, PH_DONE = 2, PH_PAUSED = 3 };

struct CellState {
    int phase, code, k_it, head, iter, halvings, nevals, pad;
    double E_curr, fh, alpha_m, ratio, ls_alpha_min, max_f;
    double rho[kBMaxM];
    unsigned long long t_done;
};

struct BatchParams {
    int m, max_iter, max_halvings;
    int cg;  // 1: Min_CG's Polak-Ribiere direction instead of the L-BFGS two-loop
    double fmax_tol, energy_tol, skin_sq;
};

struct BatchView {
    CellState* st;
    const int* base;   // first owned site of each cell
    const int* nat;    // owned sites of each cell
    unsigned char* active;
    double *h, *x0, *f0, *s, *y;
    const double4* pos0;  // owned positions at the last list build
    size_t vstride;       // natms_total * x_dim
    int ncells;
    unsigned long long* t0;
    int* budget;
    long long* iters;
    // whole-GPU step of a single cell (CS = 0): barrier [count, generation],
    // per-CTA partials [2][kMaxGridCtas], and a wait-timeout flag
    unsigned int* gbar;
    double* gpart;
    int* gerr;
    unsigned long long wait_ns;  // a grid-barrier wait gives up after this long
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// x component q of owned site i: position (q < 3) or alpha of species q - 3
__device__ __forceinline__ double xget(const Dev& d, int i, int q)
{
    if (q < 3) return reinterpret_cast<const double*>(d.pos)[(size_t)i * 4 + q];
    return d.alpha[(size_t)i * d.nt + (q - 3)];
}
__device__ __forceinline__ void xset(const Dev& d, int i, int q, double v)
{
    if (q < 3) reinterpret_cast<double*>(d.pos)[(size_t)i * 4 + q] = v;
    else d.alpha[(size_t)i * d.nt + (q - 3)] = v;
}

// block-wide sum / max / min, the result in every thread (fixed order, so
// every thread and every run gets the same value)
template <int OP>
__device__ __forceinline__ double block_red(double v, double* sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double t = __shfl_xor_sync(0xffffffffu, v, o);
        v = OP == 0 ? v + t : (OP == 1 ? fmax(v, t) : fmin(v, t));
    }
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = sh[0];
    for (int k = 1; k < nw; k++) r = OP == 0 ? r + sh[k] : (OP == 1 ? fmax(r, sh[k]) : fmin(r, sh[k]));
    return r;
}

// A cell's L-BFGS step runs on a thread-block cluster of CS CTAs (one CTA when
// CS = 1), or, for a batch of one cell, on the whole GPU (CS = 0: one CTA per
// SM, launched cooperatively so that all are resident).  Element e of the
// cell's vectors belongs to thread e mod (CTAs * T) in every loop; reductions
// combine the CTAs' block results in CTA order -- through distributed shared
// memory in a cluster, through a global array after a grid barrier on the
// whole GPU -- so every thread gets the same value.
constexpr int kMaxGridCtas = 1024;
constexpr double kGridWaitS = 2.0;  // default: a barrier wait gives up after 2 s (mg_batch_set_limits)

struct RedCtx {
    double* sh;    // shared [32]
    double* slot;  // shared, one double (cluster mode)
    int* par;      // shared, which half of gpart the next reduction uses (grid mode)
    unsigned int* gbar;
    double* gpart;
    int* gerr;
    unsigned long long wait_ns;
};

template <int CS>
__device__ __forceinline__ int nctas() { return CS == 0 ? (int)gridDim.x : CS; }
template <int CS>
__device__ __forceinline__ int cell_idx() { return CS == 0 ? 0 : (int)blockIdx.x / CS; }
template <int CS>
__device__ __forceinline__ int rank_idx() { return CS == 0 ? (int)blockIdx.x : (int)blockIdx.x % CS; }

// Grid barrier of the whole-GPU step (sense by generation count).  A wait
// that outlasts R.wait_ns, or sees another CTA's timeout, sets *gerr and
// returns, so a stuck barrier ends the launch instead of hanging it: the
// loop test then stops the relaxation, which returns MG_ERR_TIMEOUT.  Every
// index the step uses comes from the cell's state as the launch read it, so
// the work a CTA still does after a failed wait stays in bounds.
__device__ __forceinline__ void grid_sync(const RedCtx& R)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = R.gbar + 1;
        const unsigned int g = *gen;
        __threadfence();
        if (atomicAdd(R.gbar, 1u) == gridDim.x - 1) {
            atomicExch(R.gbar, 0u);
            __threadfence();
            atomicAdd(R.gbar + 1, 1u);
        } else {
            const unsigned long long t_start = global_ns();
            while (*gen == g) {
                if (*(volatile int*)R.gerr) break;
                if (global_ns() - t_start >= R.wait_ns) {
                    atomicExch(R.gerr, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

template <int CS>
__device__ __forceinline__ void phase_sync(const RedCtx& R)
{
    if (CS == 0) grid_sync(R);
    else if (CS == 1) __syncthreads();
    else cooperative_groups::this_cluster().sync();
}

template <int OP>
__device__ __forceinline__ double red_op(double a, double b)
{
    return OP == 0 ? a + b : (OP == 1 ? fmax(a, b) : fmin(a, b));
}

template <int CS, int OP>
__device__ __forceinline__ double cred(double v, const RedCtx& R)
{
    double b = block_red<OP>(v, R.sh);
    if (CS == 1) return b;
    if (CS == 0) {
        double* buf = R.gpart + (size_t)(*R.par) * kMaxGridCtas;
        if (threadIdx.x == 0) buf[blockIdx.x] = b;
        grid_sync(R);
        if (threadIdx.x < 32) {
            double a = OP == 0 ? 0.0 : (OP == 1 ? -INFINITY : INFINITY);
            for (int k = threadIdx.x; k < (int)gridDim.x; k += 32) a = red_op<OP>(a, __ldcg(buf + k));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a = red_op<OP>(a, __shfl_xor_sync(0xffffffffu, a, o));
            if (threadIdx.x == 0) {
                R.sh[0] = a;
                *R.par ^= 1;
            }
        }
        __syncthreads();
        const double r = R.sh[0];
        __syncthreads();
        return r;
    }
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    if (threadIdx.x == 0) *R.slot = b;
    cl.sync();
    double r = *cl.map_shared_rank(R.slot, 0);
#pragma unroll
    for (int k = 1; k < CS; k++) r = red_op<OP>(r, *cl.map_shared_rank(R.slot, k));
    cl.sync();  // no CTA overwrites its slot before every CTA has read it
    return r;
}

// x = x0 + a h over the cell; returns the largest squared displacement of a
// site from its position at the last list build
template <int CS>
__device__ double set_trial(const Dev& d, const BatchView& B, int base, int nat, double a, const RedCtx& R, int t0,
                           int ts)
{
    const int xd = d.x_dim;
    const double* x0 = B.x0 + (size_t)base * xd;
    const double* h = B.h + (size_t)base * xd;
    double dmax = 0.0;
    phase_sync<CS>(R);
    for (int k = t0; k < nat; k += ts) {
        const int i = base + k;
        for (int q = 0; q < xd; q++) xset(d, i, q, x0[(size_t)k * xd + q] + a * h[(size_t)k * xd + q]);
        const double4 p = d.pos[i], p0 = B.pos0[i];
        const double dx = p.x - p0.x, dy = p.y - p0.y, dz = p.z - p0.z;
        dmax = fmax(dmax, dx * dx + dy * dy + dz * dz);
    }
    return cred<CS, 1>(dmax, R);
}

// One L-BFGS step of every running cell, after the force evaluation of its
// current point (d.f, d.cell_E).  Min_LBFGS::run non-box branch
// (min_l-bfgs.cpp:616-773) with LineSearch_BackTrack::line_min, DMD branch
// (line_search.cpp:223-342), unrolled into phases.
template <int CS>
__global__ void __launch_bounds__(1024) k_lbfgs_step(Dev d, BatchView B, BatchParams P)
{
    __shared__ double sh[32];
    __shared__ double slot_sh;
    __shared__ int par_sh;
    if (threadIdx.x == 0) par_sh = 0;
    __syncthreads();
    const RedCtx R{sh, &slot_sh, &par_sh, B.gbar, B.gpart, B.gerr, B.wait_ns};
    const int c = cell_idx<CS>(), rank = rank_idx<CS>();
    const int t0 = rank * blockDim.x + threadIdx.x, ts = nctas<CS>() * blockDim.x;
    CellState* S = B.st + c;
    const int phase = S->phase;
    if (phase == PH_DONE || phase == PH_PAUSED) return;
    const int xd = d.x_dim, nt = d.nt, base = B.base[c], nat = B.nat[c], n = nat * xd;
    const size_t vb = (size_t)base * xd;
    double* f = d.f + vb;
    double* h = B.h + vb;
    double* x0 = B.x0 + vb;
    double* f0 = B.f0 + vb;
    const double E_new = d.cell_E[c];
    double E_curr = S->E_curr, fh = S->fh, alpha_m = S->alpha_m, ratio = S->ratio, ls_alpha_min = S->ls_alpha_min;
    double max_f = S->max_f;
    int k_it = S->k_it, head = S->head, iter = S->iter, halvings = S->halvings, nevals = S->nevals + 1;
    double rho[kBMaxM];
#pragma unroll
    for (int k = 0; k < kBMaxM; k++) rho[k] = S->rho[k];
    int code = kRunning, next = PH_TRIAL;
    bool new_dir = false;
    double cg_beta = 0.0;  // CG: the ratio of this step's direction update

    if (phase == PH_FIRST) {
        // Min_LBFGS::init: the first force_calc gives curr_energy
        E_curr = E_new;
        ratio = 1.0;
        k_it = 0;
        head = 0;
        iter = 0;
        ls_alpha_min = 0.0;
        new_dir = true;
    } else {
        const double ideal = E_curr - alpha_m * 0.4 * fh;
        if (E_new <= ideal) {
            // accepted (line_search.cpp:320-326), then min_l-bfgs.cpp:680-758
            const double E_prev = E_curr;
            E_curr = E_new;
            double fm = 0.0;
            for (int e = t0; e < n; e += ts) fm = fmax(fm, fabs(f[e]));
            max_f = cred<CS, 1>(fm, R);
            if (E_prev - E_curr < P.energy_tol) code = kTolerance;
            else if (iter == P.max_iter) code = kMaxIter;
            else if (P.fmax_tol > 0.0 && max_f < P.fmax_tol) code = kTolerance;
            if (code == kRunning && P.cg) {
                // Min_CG::run after its force_calc (min_cg.cpp:526-558): f.f,
                // f.f0, the Polak-Ribiere ratio; ratio keeps f0.f0 between steps
                double ff = 0.0, ff0 = 0.0;
                for (int e = t0; e < n; e += ts) {
                    ff += f[e] * f[e];
                    ff0 += f[e] * f0[e];
                }
                ff = cred<CS, 0>(ff, R);
                ff0 = cred<CS, 0>(ff0, R);
                cg_beta = (ff - ff0) / ratio;
                ratio = ff;
                iter++;
                new_dir = true;
            } else if (code == kRunning) {
                int slot;
                if (k_it == P.m) {
                    slot = head;
                    head = (head + 1) % P.m;
                } else {
                    slot = (head + k_it) % P.m;
                    k_it++;
                }
                double* sv = B.s + (size_t)slot * B.vstride + vb;
                double* yv = B.y + (size_t)slot * B.vstride + vb;
                double in1 = 0.0, in2 = 0.0;
                for (int e = t0; e < n; e += ts) {
                    const double sv_e = alpha_m * h[e], yv_e = f[e] - f0[e];
                    sv[e] = sv_e;
                    yv[e] = yv_e;
                    in1 += sv_e * yv_e;
                    in2 += yv_e * yv_e;
                }
                in1 = cred<CS, 0>(in1, R);
                in2 = cred<CS, 0>(in2, R);
                ratio = -in1 / in2;
                rho[slot] = 1.0 / in1;
                iter++;
                new_dir = true;
            }
        } else {
            alpha_m *= 0.5;
            halvings++;
            if (alpha_m <= ls_alpha_min || (P.max_halvings > 0 && halvings >= P.max_halvings)) {
                // energy(0): back to x0, whose forces and energy are f0 and E_curr
                phase_sync<CS>(R);
                for (int k = t0; k < nat; k += ts)
                    for (int q = 0; q < xd; q++) xset(d, base + k, q, x0[(size_t)k * xd + q]);
                for (int e = t0; e < n; e += ts) f[e] = f0[e];
                code = kAlphaMin;
            } else if (set_trial<CS>(d, B, base, nat, alpha_m, R, t0, ts) > P.skin_sq) {
                next = PH_PAUSED;
            }
        }
    }

    if (new_dir && P.cg) {
        // Min_CG: h = f at the start (f0.f0 = f.f kept in ratio), else
        // h = beta h + f with h.f < 0 falling back to h = f; then x_prev = x,
        // f_prev = f and f0.f0 == 0 ends the run (min_cg.cpp:452-481, 546-558)
        phase_sync<CS>(R);
        if (phase == PH_FIRST) {
            double ff = 0.0;
            for (int e = t0; e < n; e += ts) {
                h[e] = f[e];
                ff += f[e] * f[e];
            }
            ratio = cred<CS, 0>(ff, R);
        } else {
            double fhv = 0.0;
            for (int e = t0; e < n; e += ts) {
                double he = h[e] * cg_beta;
                he += f[e];
                h[e] = he;
                fhv += he * f[e];
            }
            fhv = cred<CS, 0>(fhv, R);
            if (fhv < 0.0)
                for (int e = t0; e < n; e += ts) h[e] = f[e];
        }
        for (int k = t0; k < nat; k += ts)
            for (int q = 0; q < xd; q++) x0[(size_t)k * xd + q] = xget(d, base + k, q);
        for (int e = t0; e < n; e += ts) f0[e] = f[e];
        if (ratio == 0.0) {
            code = kGrad0;
            new_dir = false;
        }
    } else if (new_dir) {
        // h = f, x_prev = x, f_prev = f, then the two-loop recursion
        phase_sync<CS>(R);
        for (int k = t0; k < nat; k += ts)
            for (int q = 0; q < xd; q++) x0[(size_t)k * xd + q] = xget(d, base + k, q);
        for (int e = t0; e < n; e += ts) {
            h[e] = f[e];
            f0[e] = f[e];
        }
        double al[kBMaxM];
        for (int i = k_it - 1; i > -1; i--) {
            const int slot = (head + i) % P.m;
            const double* sv = B.s + (size_t)slot * B.vstride + vb;
            const double* yv = B.y + (size_t)slot * B.vstride + vb;
            double in = 0.0;
            for (int e = t0; e < n; e += ts) in += h[e] * sv[e];
            al[i] = cred<CS, 0>(in, R) * rho[slot];
            for (int e = t0; e < n; e += ts) h[e] -= al[i] * yv[e];
        }
        for (int e = t0; e < n; e += ts) h[e] *= ratio;
        for (int i = 0; i < k_it; i++) {
            const int slot = (head + i) % P.m;
            const double* sv = B.s + (size_t)slot * B.vstride + vb;
            const double* yv = B.y + (size_t)slot * B.vstride + vb;
            double in = 0.0;
            for (int e = t0; e < n; e += ts) in += h[e] * yv[e];
            const double be = cred<CS, 0>(in, R) * rho[slot];
            for (int e = t0; e < n; e += ts) h[e] -= (be + al[i]) * sv[e];
        }
    }
    if (new_dir) {
        // line_min: alpha_min from the smallest alpha coordinate, |h| = 1,
        // downhill test, first step min(1, max|h|)
        double mn = INFINITY;
        for (int k = t0; k < nat; k += ts)
            for (int t = 0; t < nt; t++) mn = fmin(mn, d.alpha[(size_t)(base + k) * nt + t]);
        mn = cred<CS, 2>(mn, R) * 0.99;
        ls_alpha_min = fmin(ls_alpha_min, mn);
        double hh = 0.0;
        for (int e = t0; e < n; e += ts) hh += h[e] * h[e];
        hh = 1.0 / sqrt(cred<CS, 0>(hh, R));
        double fhl = 0.0, mh = 0.0;
        for (int e = t0; e < n; e += ts) {
            h[e] *= hh;
            fhl += f[e] * h[e];
            mh = fmax(mh, fabs(h[e]));
        }
        fh = cred<CS, 0>(fhl, R);
        mh = cred<CS, 1>(mh, R);
        if (fh <= 0) code = kDownhill;
        else if (mh == 0) code = kGrad0;
        else {
            alpha_m = fmin(1.0, mh);
            halvings = 0;
            if (alpha_m <= ls_alpha_min) code = kAlphaMin;
            else if (set_trial<CS>(d, B, base, nat, alpha_m, R, t0, ts) > P.skin_sq) next = PH_PAUSED;
        }
    }
    if (code != kRunning) next = PH_DONE;
    phase_sync<CS>(R);  // every CTA of the cluster has read the state before it changes
    if (rank == 0 && threadIdx.x == 0) {
        S->phase = next;
        S->code = code;
        S->k_it = k_it;
        S->head = head;
        S->iter = iter;
        S->halvings = halvings;
        S->nevals = nevals;
        S->E_curr = E_curr;
        S->fh = fh;
        S->alpha_m = alpha_m;
        S->ratio = ratio;
        S->ls_alpha_min = ls_alpha_min;
        S->max_f = max_f;
        for (int k = 0; k < kBMaxM; k++) S->rho[k] = rho[k];
        if (next == PH_DONE) S->t_done = global_ns() - *B.t0;
        B.active[c] = next == PH_TRIAL ? 1 : 0;
    }
}

// Loop test of the while node: continue while a cell is running and the
// iteration budget lasts.
__global__ void k_loop_test(BatchView B, cudaGraphConditionalHandle handle)
{
    __shared__ int sh_n;
    if (threadIdx.x == 0) sh_n = 0;
    __syncthreads();
    int n = 0;
    for (int c = threadIdx.x; c < B.ncells; c += blockDim.x) n += B.active[c];
    atomicAdd(&sh_n, n);
    __syncthreads();
    if (threadIdx.x == 0) {
        int left = --(*B.budget);
        (*B.iters)++;
        cudaGraphSetConditional(handle, (sh_n > 0 && left > 0 && *B.gerr == 0) ? 1u : 0u);
    }
}

__global__ void k_stamp(unsigned long long* t0) { *t0 = global_ns(); }

// forces and densities of the running cells' sites to zero (a stopped cell
// keeps the forces of its final point)
__global__ void k_zero_active(Dev d)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.natms || !d.cell_active[d.site_cell[i]]) return;
    for (int q = 0; q < d.x_dim; q++) d.f[(size_t)i * d.x_dim + q] = 0.0;
    for (int t = 0; t < d.nt; t++) d.E[(size_t)i * d.nt + t] = 0.0;
}

// ghosts of running cells from their owners (position + image shift, alpha)
__global__ void k_refresh_ghosts(Dev d, const double* __restrict__ shift, const unsigned char* __restrict__ active)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.nph) return;
    const int g = d.natms + (int)k, o = d.root[g];
    if (!active[d.site_cell[o]]) return;
    const double4 po = d.pos[o];
    double4 pg = d.pos[g];
    pg.x = po.x + shift[3 * k];
    pg.y = po.y + shift[3 * k + 1];
    pg.z = po.z + shift[3 * k + 2];
    d.pos[g] = pg;
    for (int t = 0; t < d.nt; t++) d.alpha[(size_t)g * d.nt + t] = d.alpha[(size_t)o * d.nt + t];
}

// one built cell of the builder system into the batch numbering
struct GatherDst {
    double4* pos;
    double4* pos0;
    double* alpha;
    double* c;
    int* root;
    int* site_cell;
    double* shift;
    int* pair_i;
    int* pair_j;
    int natms_total;
};

__global__ void k_gather_cell(Dev s, GatherDst D, int cell, int obase, int gbase, long long pbase)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nt = s.nt;
    if (k < s.nall) {
        const int src = (int)k;
        const bool owned = src < s.natms;
        const int dst = owned ? obase + src : D.natms_total + gbase + (src - s.natms);
        const double4 p = s.pos[src];
        D.pos[dst] = p;
        for (int t = 0; t < nt; t++) {
            D.alpha[(size_t)dst * nt + t] = s.alpha[(size_t)src * nt + t];
            D.c[(size_t)dst * nt + t] = s.c[(size_t)src * nt + t];
        }
        if (owned) {
            D.site_cell[dst] = cell;
            D.pos0[dst] = p;
        } else {
            const int o = s.root[src];
            const double4 po = s.pos[o];
            D.root[dst] = obase + o;
            const size_t gk = (size_t)(dst - D.natms_total);
            D.shift[3 * gk] = p.x - po.x;
            D.shift[3 * gk + 1] = p.y - po.y;
            D.shift[3 * gk + 2] = p.z - po.z;
        }
    }
    if (k < s.npairs) {
        D.pair_i[pbase + k] = obase + s.pair_i[k];
        const int j = s.pair_j[k];
        D.pair_j[pbase + k] = j < s.natms ? obase + j : D.natms_total + gbase + (j - s.natms);
    }
}

// Probe for the autotuner: the reductions of a full two-loop step
// (2m + 4 cluster dot products over the cell's vectors), nothing written but
// one value per cell.
template <int CS>
__global__ void __launch_bounds__(1024) k_lbfgs_probe(Dev d, BatchView B, int m, double* out)
{
    __shared__ double sh[32];
    __shared__ double slot_sh;
    __shared__ int par_sh;
    if (threadIdx.x == 0) par_sh = 0;
    __syncthreads();
    const RedCtx R{sh, &slot_sh, &par_sh, B.gbar, B.gpart, B.gerr, B.wait_ns};
    const int c = cell_idx<CS>(), rank = rank_idx<CS>();
    const int t0 = rank * blockDim.x + threadIdx.x, ts = nctas<CS>() * blockDim.x;
    const int xd = d.x_dim, n = B.nat[c] * xd;
    const size_t vb = (size_t)B.base[c] * xd;
    double acc = 0.0;
    for (int r = 0; r < 2 * m + 4; r++) {
        const double* a = (r < 2 * m ? (r & 1 ? B.y : B.s) + (size_t)(r >> 1) * B.vstride : B.h) + vb;
        double in = 0.0;
        for (int e = t0; e < n; e += ts) in += a[e] * d.f[vb + e];
        acc += cred<CS, 0>(in, R);
    }
    if (rank == 0 && threadIdx.x == 0) out[c] = acc;
}

// launch of a per-cell kernel on clusters of cs CTAs (cs = 1: plain launch;
// cs = 0: one cell on one CTA per SM, cooperative so that all are resident)
template <class... A>
cudaError_t launch_cells(void (*kern)(A...), int cs, int ncells, int threads, cudaStream_t st, A... args)
{
    if (cs == 0) {
        if (ncells != 1) return cudaErrorInvalidValue;
        int per_sm = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)std::min(num_sms(), kMaxGridCtas), 1, 1);
        cfg.blockDim = dim3((unsigned)threads, 1, 1);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, kern, args...);
    }
    if (cs == 1) {
        kern<<<ncells, threads, 0, st>>>(args...);
        return cudaGetLastError();
    }
    if (cs > 8) cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(ncells * cs), 1, 1);
    cfg.blockDim = dim3((unsigned)threads, 1, 1);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

cudaError_t launch_step(int cs, int ncells, int threads, cudaStream_t st, const Dev& d, const BatchView& B,
                        const BatchParams& P)
{
    switch (cs) {
    case 0: return launch_cells(k_lbfgs_step<0>, 0, ncells, threads, st, d, B, P);
    case 1: return launch_cells(k_lbfgs_step<1>, 1, ncells, threads, st, d, B, P);
    case 2: return launch_cells(k_lbfgs_step<2>, 2, ncells, threads, st, d, B, P);
    case 4: return launch_cells(k_lbfgs_step<4>, 4, ncells, threads, st, d, B, P);
    case 8: return launch_cells(k_lbfgs_step<8>, 8, ncells, threads, st, d, B, P);
    case 16: return launch_cells(k_lbfgs_step<16>, 16, ncells, threads, st, d, B, P);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_probe(int cs, int ncells, int threads, cudaStream_t st, const Dev& d, const BatchView& B, int m,
                         double* out)
{
    switch (cs) {
    case 0: return launch_cells(k_lbfgs_probe<0>, 0, ncells, threads, st, d, B, m, out);
    case 1: return launch_cells(k_lbfgs_probe<1>, 1, ncells, threads, st, d, B, m, out);
    case 2: return launch_cells(k_lbfgs_probe<2>, 2, ncells, threads, st, d, B, m, out);
    case 4: return launch_cells(k_lbfgs_probe<4>, 4, ncells, threads, st, d, B, m, out);
    case 8: return launch_cells(k_lbfgs_probe<8>, 8, ncells, threads, st, d, B, m, out);
    case 16: return launch_cells(k_lbfgs_probe<16>, 16, ncells, threads, st, d, B, m, out);
    default: return cudaErrorInvalidValue;
    }
}

// ---- host ------------------------------------------------------------------

int bfail(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return internal_fail(code, buf);
}

#define BCU(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) return bfail(MG_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                            __FILE__, __LINE__);                                         \
    } while (0)

#define BCHK(call)         \
    do {                   \
        int r_ = (call);   \
        if (r_) return r_; \
    } while (0)

// device array with capacity; grow() keeps the first `keep` elements
template <class T>
struct DArr {
    T* p = nullptr;
    size_t cap = 0;
    int grow(size_t need, size_t keep, cudaStream_t st)
    {
        if (need <= cap) return MG_OK;
        size_t n = std::max(need, cap + cap / 2 + 1024);
        T* q = nullptr;
        cudaError_t e = cudaMalloc((void**)&q, n * sizeof(T));
        if (e != cudaSuccess) return bfail(MG_ERR_CAPACITY, "cudaMalloc of %zu bytes failed", n * sizeof(T));
        if (p && keep) {
            BCU(cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, st));
            BCU(cudaStreamSynchronize(st));
        }
        if (p) cudaFree(p);
        p = q;
        cap = n;
        return MG_OK;
    }
    int exact(size_t need)
    {
        if (need <= cap) return MG_OK;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc((void**)&p, (need ? need : 1) * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            return bfail(MG_ERR_CAPACITY, "cudaMalloc of %zu bytes failed", need * sizeof(T));
        }
        cap = need;
        return MG_OK;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

struct HostCell {
    int natms;
    double H[9], B[9];          // box and its inverse as the builder computed it
    std::vector<double> x_in;   // natms * x_dim as given (fractional, then alpha)
    std::vector<double> x;      // the same for the next build (after a rebuild: current state)
    std::vector<double> c;
};

std::mutex g_tune_mu;
std::map<std::string, std::vector<int>> g_tune_mem;

}  // namespace

struct mg_batch {
    mg_system* builder = nullptr;
    int device = 0, nt = 0, xd = 0, form = MG_FORM_FP64;
    int m = 5, max_iter = 10000, max_halvings = 60, cg = 0;
    double fmax_tol = 1e-5, energy_tol = 1e-8, skin = 0.5;
    int autotune = 0;
    std::string cache_path;
    // failure limits (mg_batch_set_limits): iteration budget of one launch
    // (0: from max_iter and max_halvings) and the grid-barrier wait
    long long iter_budget = 0;
    double wait_s = kGridWaitS;
    std::vector<HostCell> cells;
    cudaStream_t st = nullptr;
    // batch numbering
    bool built = false;
    int natms_total = 0, nghost_total = 0;
    long long npairs_total = 0;
    std::vector<int> h_base, h_nat;
    Dev bd{};
    DArr<double4> pos, pos0;
    DArr<double> alpha, c, shift, f, E, dE, pr, partial, cell_E, vec, probe_out;
    DArr<float> prf;
    DArr<int4> icut;       // the precision form's in-cut pair list (two int4 per pair)
    DArr<float4> srec;     // and its per-site FP32 records
    DArr<float> dE32, facc;
    DArr<unsigned> icut_n;
    DArr<int> root, site_cell, pair_i, pair_j, base, nat;
    DArr<unsigned char> active;
    DArr<CellState> state;
    DArr<unsigned long long> t0;
    DArr<int> budget;
    DArr<long long> iters;
    DArr<unsigned int> gbar;  // whole-GPU step: barrier words
    DArr<double> gpart;       // whole-GPU step: per-CTA partials
    DArr<int> gerr;           // whole-GPU step: a barrier wait timed out
    // launch shapes
    int bps1 = 0, bps2 = 0, lbt = 256, lcs = 1;  // pass grids, L-BFGS threads per CTA and CTAs per cell
    bool tuned = false, from_cache = false;
    double tune_ms = 0, build_ms = 0;
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
};

namespace {

BatchView view(mg_batch* b)
{
    BatchView v;
    v.st = b->state.p;
    v.base = b->base.p;
    v.nat = b->nat.p;
    v.active = b->active.p;
    const size_t vs = (size_t)b->natms_total * b->xd;
    v.h = b->vec.p;
    v.x0 = v.h + vs;
    v.f0 = v.x0 + vs;
    v.s = v.f0 + vs;
    v.y = v.s + (size_t)b->m * vs;
    v.pos0 = b->pos0.p;
    v.vstride = vs;
    v.ncells = (int)b->cells.size();
    v.t0 = b->t0.p;
    v.budget = b->budget.p;
    v.iters = b->iters.p;
    v.gbar = b->gbar.p;
    v.gpart = b->gpart.p;
    v.gerr = b->gerr.p;
    v.wait_ns = (unsigned long long)(b->wait_s * 1e9);
    return v;
}

BatchParams params(mg_batch* b)
{
    BatchParams P;
    P.m = b->m;
    P.cg = b->cg;
    P.max_iter = b->max_iter;
    P.max_halvings = b->max_halvings;
    P.fmax_tol = b->fmax_tol;
    P.energy_tol = b->energy_tol;
    P.skin_sq = b->skin * b->skin;
    return P;
}

// fractional coordinates of Cartesian x in a lower-triangular box (x2s,
// atoms.cpp:1869-1897), wrapped into [0, 1)
void x2s_host(const double* B, const double* x, double* s)
{
    for (int j = 0; j < 3; j++) {
        double v = x[j] * B[3 * j + j];
        for (int k = j + 1; k < 3; k++) v += B[3 * k + j] * x[k];
        while (v < 0.0) v++;
        while (v >= 1.0) v--;
        s[j] = v;
    }
}

// ghosts and lists of every cell with the builder, gathered into the batch
int build_all(mg_batch* b)
{
    auto t_start = std::chrono::steady_clock::now();
    const int ncells = (int)b->cells.size(), nt = b->nt;
    mg_system* sb = b->builder;
    cudaStream_t bst = system_stream(sb);
    b->natms_total = 0;
    b->h_base.assign(ncells, 0);
    b->h_nat.assign(ncells, 0);
    for (int c = 0; c < ncells; c++) {
        b->h_base[c] = b->natms_total;
        b->h_nat[c] = b->cells[c].natms;
        b->natms_total += b->cells[c].natms;
    }
    const int NT = b->natms_total;
    // owned part has a fixed size; the ghost part and the pair list grow
    size_t ghost_cap = 0;
    long long pair_fill = 0;
    int ghost_fill = 0;
    BCHK(b->pos.grow((size_t)NT + 1, 0, bst));
    BCHK(b->pos0.exact((size_t)NT + 1));
    BCHK(b->alpha.grow((size_t)(NT + 1) * nt, 0, bst));
    BCHK(b->c.grow((size_t)(NT + 1) * nt, 0, bst));
    BCHK(b->root.grow((size_t)NT + 1, 0, bst));
    BCHK(b->site_cell.exact((size_t)NT + 1));
    // largest cells first, so the builder's buffers reach their final size at once
    std::vector<int> order(ncells);
    for (int c = 0; c < ncells; c++) order[c] = c;
    std::stable_sort(order.begin(), order.end(),
                     [&](int u, int v) { return b->cells[u].natms > b->cells[v].natms; });
    for (int c : order) {
        HostCell& hc = b->cells[c];
        BCHK(mg_atoms_set_box(sb, hc.H));
        system_shape(sb, nullptr, nullptr, nullptr, nullptr, hc.B);
        BCHK(mg_atoms_set(sb, hc.natms, hc.x.data(), nullptr, hc.c.data()));
        BCHK(mg_ff_init(sb));
        const Dev& d = system_dev(sb);
        const int nph = d.nph;
        const long long np = d.npairs;
        const size_t nall_need = (size_t)NT + ghost_fill + nph + 1;
        const size_t keep = (size_t)NT + ghost_fill;
        BCHK(b->pos.grow(nall_need, keep, bst));
        BCHK(b->alpha.grow(nall_need * nt, keep * nt, bst));
        BCHK(b->c.grow(nall_need * nt, keep * nt, bst));
        BCHK(b->root.grow(nall_need, keep, bst));
        if ((size_t)(ghost_fill + nph) + 1 > ghost_cap) {
            BCHK(b->shift.grow(3 * ((size_t)ghost_fill + nph + 1), 3 * (size_t)ghost_fill, bst));
            ghost_cap = b->shift.cap / 3;
        }
        BCHK(b->pair_i.grow((size_t)(pair_fill + np + 1), (size_t)pair_fill, bst));
        BCHK(b->pair_j.grow((size_t)(pair_fill + np + 1), (size_t)pair_fill, bst));
        GatherDst D;
        D.pos = b->pos.p;
        D.pos0 = b->pos0.p;
        D.alpha = b->alpha.p;
        D.c = b->c.p;
        D.root = b->root.p;
        D.site_cell = b->site_cell.p;
        D.shift = b->shift.p;
        D.pair_i = b->pair_i.p;
        D.pair_j = b->pair_j.p;
        D.natms_total = NT;
        const long long work = std::max<long long>((long long)d.nall, np);
        if (work > 0)
            k_gather_cell<<<(unsigned)div_up(work, 256), 256, 0, bst>>>(d, D, c, b->h_base[c], ghost_fill, pair_fill);
        BCU(cudaGetLastError());
        ghost_fill += nph;
        pair_fill += np;
    }
    BCU(cudaStreamSynchronize(bst));
    b->nghost_total = ghost_fill;
    b->npairs_total = pair_fill;
    const size_t nall = (size_t)NT + ghost_fill;
    // per-evaluation arrays
    BCHK(b->f.exact((size_t)NT * b->xd));
    BCHK(b->E.exact(nall * nt));
    BCHK(b->dE.exact(nall * nt));
    const int nblk = 3 * nt * nt + 3 * nt * (nt + 1) / 2;
    const size_t maxp = (size_t)pair_fill + 1;
    if (b->form == MG_FORM_FP32) {
        BCHK(b->icut.exact((size_t)dmd32_icut_capacity((long long)maxp) * 2));
        BCHK(b->icut_n.exact((size_t)dmd32_icut_warps()));
        BCHK(b->srec.exact(nall * kSiteRec));
        BCHK(b->dE32.exact(nall * nt));
        BCHK(b->facc.exact((size_t)NT * 8));
    } else
        BCHK(b->pr.exact(maxp * nblk));
    // pass 1 and pass 2 at one thread per pair at most, the embedding at one per (site, species)
    const long long rows = 2LL * div_up(pair_fill, kFFBlock) + div_up((long long)NT * nt, kFFBlock) + 64;
    BCHK(b->partial.exact((size_t)rows * 8));
    BCHK(b->cell_E.exact((size_t)ncells));
    BCHK(b->active.exact((size_t)ncells));
    BCHK(b->base.exact((size_t)ncells));
    BCHK(b->nat.exact((size_t)ncells));
    BCU(cudaMemcpy(b->base.p, b->h_base.data(), ncells * sizeof(int), cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->nat.p, b->h_nat.data(), ncells * sizeof(int), cudaMemcpyHostToDevice));
    // batch view of the system: the builder's tables and constants, batch arrays
    Dev bd = system_dev(sb);
    bd.natms = NT;
    bd.nph = ghost_fill;
    bd.nall = (int)nall;
    bd.pos = b->pos.p;
    bd.alpha = b->alpha.p;
    bd.c = b->c.p;
    bd.root = b->root.p;
    bd.pair_i = b->pair_i.p;
    bd.pair_j = b->pair_j.p;
    bd.npairs = pair_fill;
    bd.maxp = (long long)maxp;
    bd.f = b->f.p;
    bd.E = b->E.p;
    bd.dE = b->dE.p;
    bd.pr = b->pr.p;
    bd.prf = nullptr;
    bd.icut = b->icut.p;
    bd.icut_n = b->icut_n.p;
    bd.icut_cap = (long long)b->icut.cap / 2;
    bd.srec = b->srec.p;
    bd.dE32 = b->dE32.p;
    bd.facc = b->facc.p;
    bd.partial = b->partial.p;
    bd.form = b->form;
    bd.site_cell = b->site_cell.p;
    bd.cell_active = b->active.p;
    bd.cell_E = b->cell_E.p;
    bd.tune_bps = b->bps1;
    bd.tune_bps2 = b->bps2;
    // unused by the force passes in a batch
    bd.nbr = nullptr;
    bd.nnb = nullptr;
    bd.poff = nullptr;
    bd.pos0 = nullptr;
    bd.sfr = nullptr;
    b->bd = bd;
    b->built = true;
    b->build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    return MG_OK;
}

// one iteration of the device loop on stream st (captured into the body)
int enqueue_iteration(mg_batch* b, cudaGraphConditionalHandle handle, bool with_step)
{
    Dev& d = b->bd;
    cudaStream_t st = b->st;
    if (d.nph > 0) k_refresh_ghosts<<<(unsigned)div_up(d.nph, 256), 256, 0, st>>>(d, b->shift.p, b->active.p);
    if (d.natms > 0) k_zero_active<<<(unsigned)div_up(d.natms, 256), 256, 0, st>>>(d);
    BCU(cudaMemsetAsync(d.cell_E, 0, b->cells.size() * sizeof(double), st));
    int rows = 0;
    if (d.npairs > 0) {
        if (b->form == MG_FORM_FP32) BCU(launch_dmd_force_f32(d, 0, &rows, st, nullptr));
        else BCU(launch_dmd_force(d, 0, &rows, st, nullptr));
    }
    if (with_step) {
        BCU(launch_step(b->lcs, (int)b->cells.size(), b->lbt, st, d, view(b), params(b)));
        k_loop_test<<<1, 256, 0, st>>>(view(b), handle);
        BCU(cudaGetLastError());
    }
    return MG_OK;
}

void destroy_graph(mg_batch* b)
{
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
}

int capture_graph(mg_batch* b)
{
    destroy_graph(b);
    BCU(cudaGraphCreate(&b->graph, 0));
    cudaGraphConditionalHandle handle;
    BCU(cudaGraphConditionalHandleCreate(&handle, b->graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    BCU(cudaGraphAddNode(&node, b->graph, nullptr, 0, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    BCU(cudaStreamBeginCaptureToGraph(b->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    int rc = enqueue_iteration(b, handle, true);
    cudaGraph_t out = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->st, &out);
    if (rc) return rc;
    BCU(e);
    BCU(cudaGraphInstantiate(&b->gexec, b->graph, 0));
    return MG_OK;
}

std::string tune_key(mg_batch* b)
{
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, b->device);
    const Dev& d = b->bd;
    std::ostringstream k;
    k << prop.name << "|sm" << prop.multiProcessorCount << "|form" << b->form << "|nt" << d.nt << "|nq" << d.nq
      << "|cells" << b->cells.size() << "|sites" << b->natms_total << "|pairs~"
      << (int)std::lround(4.0 * std::log2((double)std::max<long long>(b->npairs_total, 1))) << "|m" << b->m;
    return k.str();
}

bool cache_lookup(mg_batch* b, const std::string& key, std::vector<int>& v)
{
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune_mem.find(key);
    if (it != g_tune_mem.end()) {
        v = it->second;
        return true;
    }
    if (b->cache_path.empty()) return false;
    std::ifstream in(b->cache_path);
    std::string line;
    while (std::getline(in, line)) {
        size_t tab = line.find('\t');
        if (tab == std::string::npos || line.compare(0, tab, key) != 0 || tab != key.size()) continue;
        std::istringstream is(line.substr(tab + 1));
        std::vector<int> w(4, 1);
        if (is >> w[0] >> w[1] >> w[2]) {
            if (!(is >> w[3])) w[3] = 1;
            v = w;
            g_tune_mem[key] = w;
            return true;
        }
    }
    return false;
}

void cache_store(mg_batch* b, const std::string& key, const std::vector<int>& v)
{
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune_mem[key] = v;
    if (b->cache_path.empty()) return;
    std::ofstream out(b->cache_path, std::ios::app);
    out << key << '\t' << v[0] << ' ' << v[1] << ' ' << v[2] << ' ' << v[3] << '\n';
}

// time `reps` force evaluations (all cells active) with the current shapes
int time_force(mg_batch* b, int reps, float* ms)
{
    cudaEvent_t e0, e1;
    BCU(cudaEventCreate(&e0));
    BCU(cudaEventCreate(&e1));
    b->bd.tune_bps = b->bps1;
    b->bd.tune_bps2 = b->bps2;
    BCHK(enqueue_iteration(b, 0, false));  // warm-up
    BCU(cudaEventRecord(e0, b->st));
    for (int r = 0; r < reps; r++) BCHK(enqueue_iteration(b, 0, false));
    BCU(cudaEventRecord(e1, b->st));
    BCU(cudaEventSynchronize(e1));
    BCU(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return MG_OK;
}

// time the probe at (threads, cs); a shape the device cannot launch (cluster
// too large for a GPC) reports an infinite time
int time_probe(mg_batch* b, int threads, int cs, int reps, float* ms)
{
    const int nc = (int)b->cells.size();
    if (launch_probe(cs, nc, threads, b->st, b->bd, view(b), b->m, b->probe_out.p) != cudaSuccess) {
        cudaGetLastError();
        *ms = 1e30f;
        return MG_OK;
    }
    cudaEvent_t e0, e1;
    BCU(cudaEventCreate(&e0));
    BCU(cudaEventCreate(&e1));
    BCU(cudaEventRecord(e0, b->st));
    for (int r = 0; r < reps; r++) BCU(launch_probe(cs, nc, threads, b->st, b->bd, view(b), b->m, b->probe_out.p));
    BCU(cudaEventRecord(e1, b->st));
    BCU(cudaEventSynchronize(e1));
    BCU(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return MG_OK;
}

// Coordinate search over the pass-1 and pass-2 blocks per SM, then the
// threads per cell of the L-BFGS step; the choice is cached by batch shape.
int autotune(mg_batch* b)
{
    const std::string key = tune_key(b);
    std::vector<int> v;
    b->from_cache = false;
    if (cache_lookup(b, key, v)) {
        b->bps1 = v[0];
        b->bps2 = v[1];
        b->lbt = v[2];
        b->lcs = v[3];
        b->from_cache = true;
        b->tune_ms = 0;
        return MG_OK;
    }
    auto t_start = std::chrono::steady_clock::now();
    BCHK(b->probe_out.exact(b->cells.size()));
    const int cand[] = {2, 3, 4, 6, 8};
    float best = 1e30f, ms = 0;
    int best1 = 3, best2 = 3;
    b->bps2 = 3;
    for (int c1 : cand) {
        b->bps1 = c1;
        BCHK(time_force(b, 3, &ms));
        if (ms < best) {
            best = ms;
            best1 = c1;
        }
    }
    b->bps1 = best1;
    best = 1e30f;
    for (int c2 : cand) {
        b->bps2 = c2;
        BCHK(time_force(b, 3, &ms));
        if (ms < best) {
            best = ms;
            best2 = c2;
        }
    }
    b->bps2 = best2;
    // threads per CTA x CTAs per cell (a thread-block cluster)
    const int tc[][2] = {{128, 1}, {256, 1}, {512, 1}, {1024, 1}, {512, 2}, {1024, 2}, {1024, 4}, {1024, 8}, {1024, 16}};
    best = 1e30f;
    int bestt = 256, bestc = 1;
    std::vector<std::array<int, 2>> shapes;
    for (const auto& t : tc) shapes.push_back({t[0], t[1]});
    if (b->cells.size() == 1) shapes.push_back({1024, 0});  // one cell: also the whole GPU
    for (const auto& t : shapes) {
        BCHK(time_probe(b, t[0], t[1], 5, &ms));
        if (ms < best) {
            best = ms;
            bestt = t[0];
            bestc = t[1];
        }
    }
    b->lbt = bestt;
    b->lcs = bestc;
    b->tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    cache_store(b, key, {b->bps1, b->bps2, b->lbt, b->lcs});
    return MG_OK;
}

int check_batch(mg_batch* b)
{
    if (!b) return bfail(MG_ERR_ARG, "null mg_batch");
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(MG_ERR_CUDA, "cudaSetDevice(%d) failed", b->device);
    return MG_OK;
}

}  // namespace

extern "C" {

int mg_batch_create(mg_system* builder, mg_batch** out)
{
    if (!builder || !out) return bfail(MG_ERR_ARG, "null builder or output pointer");
    int style = -1, nt = 0, xd = 0, form = 0;
    double Bx[9];
    system_shape(builder, &style, &nt, &xd, &form, Bx);
    if (style != STYLE_DMD_I && style != STYLE_DMD_II && style != STYLE_DMD)
        return bfail(MG_ERR_STATE, "the batched form needs a DMD system with ff_coef done as builder");
    mg_batch* b = new mg_batch();
    b->builder = builder;
    b->device = system_device(builder);
    b->nt = nt;
    b->xd = xd;
    b->skin = 0.5;
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return bfail(MG_ERR_CUDA, "could not create the batch stream");
    }
    *out = b;
    return MG_OK;
}

int mg_batch_destroy(mg_batch* b)
{
    if (!b) return MG_OK;
    cudaSetDevice(b->device);
    destroy_graph(b);
    b->pos.release();
    b->pos0.release();
    b->alpha.release();
    b->c.release();
    b->shift.release();
    b->f.release();
    b->E.release();
    b->dE.release();
    b->pr.release();
    b->prf.release();
    b->icut.release();
    b->srec.release();
    b->dE32.release();
    b->facc.release();
    b->icut_n.release();
    b->partial.release();
    b->cell_E.release();
    b->vec.release();
    b->probe_out.release();
    b->root.release();
    b->site_cell.release();
    b->pair_i.release();
    b->pair_j.release();
    b->base.release();
    b->nat.release();
    b->active.release();
    b->state.release();
    b->t0.release();
    b->budget.release();
    b->iters.release();
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
    return MG_OK;
}

int mg_batch_add_cell(mg_batch* b, int natms, const double* H, const double* x_frac, const double* c, int* index)
{
    BCHK(check_batch(b));
    if (natms < 1 || !H || !x_frac || !c) return bfail(MG_ERR_ARG, "need natms >= 1 and non-null H, x_frac, c");
    HostCell hc;
    hc.natms = natms;
    memcpy(hc.H, H, sizeof(hc.H));
    hc.x_in.assign(x_frac, x_frac + (size_t)natms * b->xd);
    hc.x = hc.x_in;
    hc.c.assign(c, c + (size_t)natms * b->nt);
    b->cells.push_back(std::move(hc));
    b->built = false;
    destroy_graph(b);
    if (index) *index = (int)b->cells.size() - 1;
    return MG_OK;
}

int mg_batch_set_params(mg_batch* b, int m, int max_iter, double fmax_tol, double energy_tol, int max_halvings)
{
    BCHK(check_batch(b));
    if (m < 1 || m > kBMaxM) return bfail(MG_ERR_ARG, "history m must be 1..%d", kBMaxM);
    if (max_iter < 1 || max_halvings < 0 || !(fmax_tol >= 0.0) || !(energy_tol > 0.0))
        return bfail(MG_ERR_ARG, "need max_iter >= 1, max_halvings >= 0, fmax_tol >= 0, energy_tol > 0");
    b->m = m;
    b->max_iter = max_iter;
    b->fmax_tol = fmax_tol;
    b->energy_tol = energy_tol;
    b->max_halvings = max_halvings;
    destroy_graph(b);
    return MG_OK;
}

int mg_batch_set_method(mg_batch* b, int method)
{
    BCHK(check_batch(b));
    if (method != MG_MIN_LBFGS && method != MG_MIN_CG) return bfail(MG_ERR_ARG, "method must be MG_MIN_LBFGS or MG_MIN_CG");
    if ((method == MG_MIN_CG) != (b->cg != 0)) {
        b->cg = method == MG_MIN_CG;
        destroy_graph(b);
    }
    return MG_OK;
}

int mg_batch_set_form(mg_batch* b, int form)
{
    BCHK(check_batch(b));
    if (form != MG_FORM_FP64 && form != MG_FORM_FP32)
        return bfail(MG_ERR_UNSUPPORTED, "the batched form runs the FP64 or the FP32 force passes");
    if (form != b->form) {
        b->form = form;
        b->built = false;
        b->tuned = false;
        destroy_graph(b);
    }
    return MG_OK;
}

int mg_batch_set_tuning(mg_batch* b, int autotune_on, const char* cache_path)
{
    BCHK(check_batch(b));
    b->autotune = autotune_on ? 1 : 0;
    b->cache_path = cache_path ? cache_path : "";
    b->tuned = false;
    if (!autotune_on) {
        b->bps1 = b->bps2 = 0;
        b->lbt = 256;
        b->lcs = 1;
    }
    destroy_graph(b);
    return MG_OK;
}

int mg_batch_set_launch(mg_batch* b, int bps1, int bps2, int lbfgs_threads, int lbfgs_cluster)
{
    BCHK(check_batch(b));
    const bool ok_t = lbfgs_threads >= 32 && lbfgs_threads <= 1024 && lbfgs_threads % 32 == 0;
    const bool ok_c = lbfgs_cluster == 1 || lbfgs_cluster == 2 || lbfgs_cluster == 4 || lbfgs_cluster == 8 ||
                      lbfgs_cluster == 16 || lbfgs_cluster == MG_LAUNCH_WHOLE_GPU;
    if (bps1 < 0 || bps2 < 0 || !ok_t || !ok_c)
        return bfail(MG_ERR_ARG, "need bps >= 0, 32..1024 threads (multiple of 32), cluster 1, 2, 4, 8, 16 or "
                                 "MG_LAUNCH_WHOLE_GPU");
    if (lbfgs_cluster == MG_LAUNCH_WHOLE_GPU && b->cells.size() > 1)
        return bfail(MG_ERR_ARG, "the whole-GPU step takes a batch of one cell");
    if (lbfgs_cluster == MG_LAUNCH_WHOLE_GPU) lbfgs_cluster = 0;
    b->autotune = 0;
    b->tuned = false;
    b->bps1 = bps1;
    b->bps2 = bps2;
    b->lbt = lbfgs_threads;
    b->lcs = lbfgs_cluster;
    destroy_graph(b);
    return MG_OK;
}

int mg_batch_set_limits(mg_batch* b, long long iteration_budget, double barrier_wait_s)
{
    BCHK(check_batch(b));
    if (iteration_budget < 0 || !(barrier_wait_s >= 0.0) || barrier_wait_s > 3600.0)
        return bfail(MG_ERR_ARG, "need iteration_budget >= 0 and 0 <= barrier_wait_s <= 3600");
    b->iter_budget = iteration_budget;
    b->wait_s = barrier_wait_s;
    destroy_graph(b);
    return MG_OK;
}

int mg_batch_relax(mg_batch* b, mg_batch_stats* stats)
{
    MG_NVTX("mg_batch_relax");
    BCHK(check_batch(b));
    const int ncells = (int)b->cells.size();
    if (ncells == 0) return bfail(MG_ERR_STATE, "no cells in the batch");
    b->build_ms = 0;
    b->tune_ms = 0;
    for (HostCell& hc : b->cells) hc.x = hc.x_in;
    // the builder's skin decides the list cut and the rebuild rule
    b->skin = system_skin(b->builder);
    BCHK(build_all(b));
    // solver state
    const size_t vs = (size_t)b->natms_total * b->xd;
    BCHK(b->vec.exact(vs * (3 + 2 * (size_t)b->m)));
    BCHK(b->state.exact((size_t)ncells));
    BCHK(b->t0.exact(1));
    BCHK(b->budget.exact(1));
    BCHK(b->iters.exact(1));
    BCHK(b->gbar.exact(2));
    BCHK(b->gpart.exact(2 * (size_t)kMaxGridCtas));
    BCHK(b->gerr.exact(1));
    BCU(cudaMemsetAsync(b->gbar.p, 0, 2 * sizeof(unsigned int), b->st));
    BCU(cudaMemsetAsync(b->gerr.p, 0, sizeof(int), b->st));
    BCU(cudaMemsetAsync(b->vec.p, 0, vs * (3 + 2 * (size_t)b->m) * sizeof(double), b->st));
    BCU(cudaMemsetAsync(b->state.p, 0, ncells * sizeof(CellState), b->st));
    BCU(cudaMemsetAsync(b->active.p, 1, ncells, b->st));
    BCU(cudaMemsetAsync(b->iters.p, 0, sizeof(long long), b->st));
    if (b->autotune && !b->tuned) {
        BCHK(autotune(b));
        b->tuned = true;
    }
    b->bd.tune_bps = b->bps1;
    b->bd.tune_bps2 = b->bps2;
    BCHK(capture_graph(b));
    // iteration budget of one launch: every cell's iterations and halvings, bounded
    const long long per_cell = (long long)(b->max_iter + 2) * (long long)(b->max_halvings > 0 ? b->max_halvings + 1 : 64);
    long long bud = std::min<long long>(per_cell + 8, 1LL << 30);
    if (b->iter_budget > 0) bud = std::min(bud, b->iter_budget);
    const int budget = (int)bud;
    int rounds = 0;
    auto t_start = std::chrono::steady_clock::now();
    k_stamp<<<1, 1, 0, b->st>>>(b->t0.p);
    std::vector<CellState> hs(ncells);
    for (;;) {
        BCU(cudaMemcpyAsync(b->budget.p, &budget, sizeof(int), cudaMemcpyHostToDevice, b->st));
        BCU(cudaGraphLaunch(b->gexec, b->st));
        BCU(cudaMemcpyAsync(hs.data(), b->state.p, ncells * sizeof(CellState), cudaMemcpyDeviceToHost, b->st));
        int gerr_h = 0;
        BCU(cudaMemcpyAsync(&gerr_h, b->gerr.p, sizeof(int), cudaMemcpyDeviceToHost, b->st));
        BCU(cudaStreamSynchronize(b->st));
        if (gerr_h) return bfail(MG_ERR_TIMEOUT, "a grid barrier of the whole-GPU step timed out");
        int paused = 0, running = 0;
        for (const CellState& s : hs) {
            paused += s.phase == PH_PAUSED;
            running += s.phase == PH_FIRST || s.phase == PH_TRIAL;
        }
        if (running > 0 && paused == 0) return bfail(MG_ERR_TIMEOUT, "iteration budget spent with %d cells running", running);
        if (paused == 0) break;
        // list rebuild: every cell from its current positions (x2s into the
        // cell, as update_0 does before Neighbor::create_list)
        rounds++;
        if (rounds > 1000) return bfail(MG_ERR_TIMEOUT, "more than 1000 list rebuild rounds");
        std::vector<double4> hp(b->natms_total);
        std::vector<double> ha((size_t)b->natms_total * b->nt);
        BCU(cudaMemcpyAsync(hp.data(), b->pos.p, hp.size() * sizeof(double4), cudaMemcpyDeviceToHost, b->st));
        BCU(cudaMemcpyAsync(ha.data(), b->alpha.p, ha.size() * sizeof(double), cudaMemcpyDeviceToHost, b->st));
        BCU(cudaStreamSynchronize(b->st));
        for (int c = 0; c < ncells; c++) {
            HostCell& hc = b->cells[c];
            for (int k = 0; k < hc.natms; k++) {
                const double4 p = hp[(size_t)b->h_base[c] + k];
                const double xv[3] = {p.x, p.y, p.z};
                x2s_host(hc.B, xv, hc.x.data() + (size_t)k * b->xd);
                for (int t = 0; t < b->nt; t++)
                    hc.x[(size_t)k * b->xd + 3 + t] = ha[((size_t)b->h_base[c] + k) * b->nt + t];
            }
        }
        BCHK(build_all(b));
        for (CellState& s : hs)
            if (s.phase == PH_PAUSED) s.phase = PH_TRIAL;
        std::vector<unsigned char> act(ncells);
        for (int c = 0; c < ncells; c++) act[c] = hs[c].phase == PH_TRIAL || hs[c].phase == PH_FIRST;
        BCU(cudaMemcpyAsync(b->state.p, hs.data(), ncells * sizeof(CellState), cudaMemcpyHostToDevice, b->st));
        BCU(cudaMemcpyAsync(b->active.p, act.data(), ncells, cudaMemcpyHostToDevice, b->st));
        BCHK(capture_graph(b));
    }
    const double relax_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    if (stats) {
        long long it = 0;
        BCU(cudaMemcpy(&it, b->iters.p, sizeof(long long), cudaMemcpyDeviceToHost));
        memset(stats, 0, sizeof(*stats));
        stats->relax_ms = relax_ms;
        stats->build_ms = b->build_ms;
        stats->tune_ms = b->tune_ms;
        stats->iterations = it;
        long long ev = 0;
        int conv = 0;
        for (const CellState& s : hs) {
            ev += s.nevals;
            conv += s.code == kTolerance && b->fmax_tol > 0.0 && s.max_f < b->fmax_tol;
        }
        stats->evaluations = ev;
        stats->rebuild_rounds = rounds;
        stats->converged = conv;
        stats->bps1 = b->bps1;
        stats->bps2 = b->bps2;
        stats->lbfgs_threads = b->lbt;
        stats->lbfgs_cluster = b->lcs == 0 ? MG_LAUNCH_WHOLE_GPU : b->lcs;
        stats->from_cache = b->from_cache ? 1 : 0;
    }
    return MG_OK;
}

int mg_batch_cell_result(mg_batch* b, int cell, double* x, double* f, mg_cell_result* r)
{
    BCHK(check_batch(b));
    if (!b->built || !b->state.p) return bfail(MG_ERR_STATE, "mg_batch_relax first");
    if (cell < 0 || cell >= (int)b->cells.size()) return bfail(MG_ERR_ARG, "cell %d out of range", cell);
    const int nat = b->h_nat[cell], base = b->h_base[cell], xd = b->xd, nt = b->nt;
    if (x) {
        std::vector<double4> hp(nat);
        std::vector<double> ha((size_t)nat * nt);
        BCU(cudaMemcpy(hp.data(), b->pos.p + base, nat * sizeof(double4), cudaMemcpyDeviceToHost));
        BCU(cudaMemcpy(ha.data(), b->alpha.p + (size_t)base * nt, ha.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int k = 0; k < nat; k++) {
            x[(size_t)k * xd + 0] = hp[k].x;
            x[(size_t)k * xd + 1] = hp[k].y;
            x[(size_t)k * xd + 2] = hp[k].z;
            for (int t = 0; t < nt; t++) x[(size_t)k * xd + 3 + t] = ha[(size_t)k * nt + t];
        }
    }
    if (f) BCU(cudaMemcpy(f, b->f.p + (size_t)base * xd, (size_t)nat * xd * sizeof(double), cudaMemcpyDeviceToHost));
    if (r) {
        CellState s;
        BCU(cudaMemcpy(&s, b->state.p + cell, sizeof(CellState), cudaMemcpyDeviceToHost));
        r->energy = s.E_curr;
        r->max_f = s.max_f;
        r->t_ms = s.t_done * 1e-6;
        r->code = s.code;
        r->iterations = s.iter;
        r->evaluations = s.nevals;
        r->natms = nat;
    }
    return MG_OK;
}

static int min_single(mg_system* s, int method, int m, int max_iter, double fmax_tol, double energy_tol,
                      int max_halvings, int lbfgs_cluster, mg_cell_result* r, mg_batch_stats* stats)
{
    if (!s) return bfail(MG_ERR_ARG, "null mg_system");
    int style = -1, nt = 0, xd = 0, form = 0;
    double B[9], H[9];
    system_shape(s, &style, &nt, &xd, &form, B);
    system_box(s, H);
    const int natms = system_natms(s);
    if (natms < 1) return bfail(MG_ERR_STATE, "the device minimiser needs an initialised system with sites");
    if (form != MG_FORM_FP64 && form != MG_FORM_FP32)
        return bfail(MG_ERR_UNSUPPORTED, "the device minimiser runs the FP64 or FP32 force passes");
    // the current state as one cell: fractional positions (x2s) and alpha, c
    std::vector<double> x((size_t)natms * xd), xs((size_t)natms * xd), c((size_t)natms * nt);
    BCHK(mg_atoms_get_x(s, x.data()));
    BCU(cudaMemcpy(c.data(), system_dev(s).c, c.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int k = 0; k < natms; k++) {
        x2s_host(B, x.data() + (size_t)k * xd, xs.data() + (size_t)k * xd);
        for (int t = 0; t < nt; t++) xs[(size_t)k * xd + 3 + t] = x[(size_t)k * xd + 3 + t];
    }
    mg_batch* b = nullptr;
    BCHK(mg_batch_create(s, &b));
    struct Guard {
        mg_batch* b;
        ~Guard() { mg_batch_destroy(b); }
    } guard{b};
    BCHK(mg_batch_add_cell(b, natms, H, xs.data(), c.data(), nullptr));
    BCHK(mg_batch_set_params(b, m, max_iter, fmax_tol, energy_tol, max_halvings));
    BCHK(mg_batch_set_method(b, method));
    BCHK(mg_batch_set_form(b, form));
    if (lbfgs_cluster != 0) BCHK(mg_batch_set_launch(b, 0, 0, 1024, lbfgs_cluster));
    else BCHK(mg_batch_set_tuning(b, 1, nullptr));
    BCHK(mg_batch_relax(b, stats));
    mg_cell_result res;
    BCHK(mg_batch_cell_result(b, 0, x.data(), nullptr, &res));
    if (r) *r = res;
    // the system takes the final state (ghosts and lists rebuilt from it)
    for (int k = 0; k < natms; k++) {
        x2s_host(B, x.data() + (size_t)k * xd, xs.data() + (size_t)k * xd);
        for (int t = 0; t < nt; t++) xs[(size_t)k * xd + 3 + t] = x[(size_t)k * xd + 3 + t];
    }
    BCHK(mg_atoms_set(s, natms, xs.data(), nullptr, c.data()));
    BCHK(mg_ff_init(s));
    return MG_OK;
}

int mg_min_lbfgs(mg_system* s, int m, int max_iter, double fmax_tol, double energy_tol, int max_halvings,
                 int lbfgs_cluster, mg_cell_result* r, mg_batch_stats* stats)
{
    MG_NVTX("mg_min_lbfgs");
    return min_single(s, MG_MIN_LBFGS, m, max_iter, fmax_tol, energy_tol, max_halvings, lbfgs_cluster, r, stats);
}

int mg_min_cg(mg_system* s, int max_iter, double fmax_tol, double energy_tol, int max_halvings, int cluster,
              mg_cell_result* r, mg_batch_stats* stats)
{
    MG_NVTX("mg_min_cg");
    return min_single(s, MG_MIN_CG, 1, max_iter, fmax_tol, energy_tol, max_halvings, cluster, r, stats);
}

}  // extern "C"
