// Adams and BDF clocks on the device: Clock_Adams (clock_adams.cpp) and
// Clock_BDF (clock_bdf.cpp) for a DMD system, with every concentration-sized
// vector resident in HBM.
//
// The reference keeps a, g, g0, c0, h and the c_d history on the host and
// loops over them between calc_g calls, which in a GPU build would move every
// vector across the boundary tens of times per step.  Here the vector work is
// a handful of kernels over the natms * nt concentrations (forming a, the
// predictor, the conjugate-gradient direction, the box-constrained step
// bound) and the force field's own calc_g / c_d_calc kernels.  A solve's line
// searches run on the device as one conditional graph (k_bs_*), steered by
// the reference's scalar control flow evaluated there; the step-size and
// order control of the BDF clock stays on the host, one synchronisation per
// solve.  Dot products and minima are deterministic: per-block partials
// reduced in a fixed order by the last block to finish.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "mg_internal.h"
#include "../../include/mapp_b200.h"

namespace mg {

namespace {

constexpr int kCkBlock = 256;
constexpr int kMaxOrder = 6;

// slots of the device scalar block
enum { SC_RATIO = 0, SC_GG0 = 1, SC_GG = 2, SC_GH = 3, SC_GAMMA = 4, SC_G0G0 = 5, SC_A = 6, SC_B = 7, SC_COUNT = 8 };

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

struct CkView {
    double* c;      // owned then ghost concentrations (the system's)
    const double* c_d;
    const double* g;
    double* a;      // calc_g's input (the system's a_in)
    double* g0;
    double* c0;
    double* h;
    double* part;   // per-block partial rows, 8 doubles each
    double* sc;     // scalars
    unsigned int* counter;
    int n, nblocks;
    const int* root;  // ghost -> owning site (the system's)
    int natms, nph, nt;
};

// Block reduction of NV values, then the fixed-order reduction of all block
// rows by the last block; bit k of MINMASK selects the minimum instead of the
// sum for value k.  Returns true in the last block, where tot holds the
// results in every thread.
template <int NV, unsigned MINMASK>
__device__ bool reduce_last(double (&v)[NV], const CkView& V, double (&tot)[NV])
{
    __shared__ double sh[kCkBlock / 32][NV];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        const bool mn = (MINMASK >> k) & 1u;
        double a = v[k];
        for (int o = 16; o > 0; o >>= 1) {
            double b = __shfl_down_sync(0xffffffffu, a, o);
            a = mn ? fmin(a, b) : a + b;
        }
        if (lane == 0) sh[w][k] = a;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        const bool mn = (MINMASK >> threadIdx.x) & 1u;
        double a = sh[0][threadIdx.x];
        for (int j = 1; j < kCkBlock / 32; j++) a = mn ? fmin(a, sh[j][threadIdx.x]) : a + sh[j][threadIdx.x];
        V.part[(size_t)blockIdx.x * 8 + threadIdx.x] = a;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(V.counter, 1u) == (unsigned)(V.nblocks - 1);
    __syncthreads();
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        const bool mn = (MINMASK >> k) & 1u;
        double a = mn ? 1.0 : 0.0;
        for (int b = threadIdx.x; b < V.nblocks; b += kCkBlock) {
            double x = __ldcg(V.part + (size_t)b * 8 + k);
            a = mn ? fmin(a, x) : a + x;
        }
        for (int o = 16; o > 0; o >>= 1) {
            double b = __shfl_down_sync(0xffffffffu, a, o);
            a = mn ? fmin(a, b) : a + b;
        }
        if (lane == 0) sh[w][k] = a;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        const bool mn = (MINMASK >> k) & 1u;
        double a = sh[0][k];
        for (int j = 1; j < kCkBlock / 32; j++) a = mn ? fmin(a, sh[j][k]) : a + sh[j][k];
        tot[k] = a;
    }
    if (threadIdx.x == 0) *V.counter = 0u;
    return true;
}

// the box bound of a step c -> c + s d (clock_adams.cpp:269-276, 302-313):
// the largest fraction of the step that keeps c inside [0, 1]
__device__ __forceinline__ double box_bound(double c, double t, double cur)
{
    if (t > 1.0) return fmin(ddiv(dsub(1.0, c), dsub(t, c)), cur);
    if (t < 0.0) return fmin(ddiv(dsub(c, 0.0), dsub(c, t)), cur);
    return cur;
}

struct History {
    const double* y[kMaxOrder];
    double coef[kMaxOrder];  // delta_t * beta[j + 1]
    int m;
};

// a = -c - sum_j (delta_t beta[j+1]) y_j (clock_adams.cpp:205-213)
__global__ void __launch_bounds__(kCkBlock) k_ck_form_a(CkView V, History Y)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    if (i >= V.n) return;
    double a = -V.c[i];
    for (int j = 0; j < Y.m; j++) a = dsub(a, dmul(Y.coef[j], Y.y[j][i]));
    V.a[i] = a;
}

// the predictor's bound: min over i of the fraction of c_d dt that keeps c in [0, 1]
__global__ void __launch_bounds__(kCkBlock) k_ck_predict_bound(CkView V, double dt)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    double v[1] = {1.0};
    if (i < V.n) v[0] = box_bound(V.c[i], dadd(dmul(V.c_d[i], dt), V.c[i]), 1.0);
    double tot[1];
    if (reduce_last<1, 1u>(v, V, tot) && threadIdx.x == 0) V.sc[SC_RATIO] = tot[0];
}

// c += c_d dt ratio (clock_adams.cpp:277-283)
__global__ void __launch_bounds__(kCkBlock) k_ck_predict(CkView V, double dt)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    if (i >= V.n) return;
    const double r = V.sc[SC_RATIO];
    V.c[i] = dadd(V.c[i], dmul(dmul(V.c_d[i], dt), r));
}

// g.g0 and g.g after the line search (clock_adams.cpp:340-352)
__global__ void __launch_bounds__(kCkBlock) k_ck_dots(CkView V)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < V.n) {
        const double gi = V.g[i];
        v[0] = dmul(gi, V.g0[i]);
        v[1] = dmul(gi, gi);
    }
    double tot[2];
    if (reduce_last<2, 0u>(v, V, tot) && threadIdx.x == 0) {
        V.sc[SC_GG0] = tot[0];
        V.sc[SC_GG] = tot[1];
    }
}

// the first direction h = g with g.g, fused with the start of the first
// conjugate-gradient iteration (g0 = g, c0 = c and the box bound along h):
// clock_adams.cpp:287-314, clock_bdf.cpp:727-759
__global__ void __launch_bounds__(kCkBlock) k_ck_first_dir(CkView V)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    double v[2] = {0.0, 1.0};
    if (i < V.n) {
        const double gi = V.g[i], ci = V.c[i];
        V.h[i] = gi;
        V.g0[i] = gi;
        V.c0[i] = ci;
        v[0] = dmul(gi, gi);
        v[1] = box_bound(ci, dadd(ci, gi), 1.0);
    }
    double tot[2];
    if (reduce_last<2, 2u>(v, V, tot) && threadIdx.x == 0) {
        V.sc[SC_G0G0] = tot[0];
        V.sc[SC_GAMMA] = tot[1];
    }
}

// ---- BDF clock (clock_bdf.cpp) ---------------------------------------------

constexpr int kMaxBdfOrder = 12;

struct BdfVecs {
    double* y_0;
    double* e_n;
    double* dy;
};

// the interpolation's history terms (clock_bdf.cpp:345-352): alpha_y[j] and
// beta * dalpha_y[j] against y[j]
struct BdfHist {
    const double* y[kMaxBdfOrder];
    double ay[kMaxBdfOrder];
    double bdy[kMaxBdfOrder];
    int q;
};

// Clock_BDF::interpolate's vector part (clock_bdf.cpp:343-360): the predictor
// y_0 and calc_g's a; SC_A receives -1 when some y_0 leaves [0, 1], else 1
__global__ void __launch_bounds__(kCkBlock) k_bdf_interp(CkView V, BdfVecs B, BdfHist Y, double b_dady0, double ady0)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    double v[1] = {1.0};
    if (i < V.n) {
        const double dyi = B.dy[i];
        double a = dmul(b_dady0, dyi), y0 = dmul(ady0, dyi);
        for (int j = 0; j < Y.q; j++) {
            const double yj = Y.y[j][i];
            a = dadd(a, dmul(Y.bdy[j], yj));
            y0 = dadd(y0, dmul(Y.ay[j], yj));
        }
        V.a[i] = dsub(a, y0);
        B.y_0[i] = y0;
        if (y0 < 0.0 || y0 > 1.0) v[0] = -1.0;
    }
    double tot[1];
    if (reduce_last<1, 1u>(v, V, tot) && threadIdx.x == 0) V.sc[SC_A] = tot[0];
}

// the bound of the explicit predictor step y[0] + dy del_t (clock_bdf.cpp:
// 706-714)
__global__ void __launch_bounds__(kCkBlock) k_bdf_predict_bound(CkView V, const double* y0, const double* dy, double dt)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    double v[1] = {1.0};
    if (i < V.n) v[0] = box_bound(y0[i], dadd(dmul(dy[i], dt), y0[i]), 1.0);
    double tot[1];
    if (reduce_last<1, 1u>(v, V, tot) && threadIdx.x == 0) V.sc[SC_RATIO] = tot[0];
}

// c = y[0] + dy del_t ratio (clock_bdf.cpp:716-717)
__global__ void __launch_bounds__(kCkBlock) k_bdf_predict(CkView V, const double* y0, const double* dy, double dt)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    if (i >= V.n) return;
    V.c[i] = dadd(y0[i], dmul(dmul(dy[i], dt), V.sc[SC_RATIO]));
}

// the step's error sums (clock_bdf.cpp:856-863) and the domain check
// (clock_bdf.cpp:876-878): sum (y_0 - c)^2, sum c_d^2, count of c outside [0, 1]
__global__ void __launch_bounds__(kCkBlock) k_bdf_err(CkView V, BdfVecs B)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    if (i < V.n) {
        const double ci = V.c[i], t = dsub(B.y_0[i], ci), cd = V.c_d[i];
        v[0] = dmul(t, t);
        v[1] = dmul(cd, cd);
        v[2] = (ci < 0.0 || ci > 1.0) ? 1.0 : 0.0;
    }
    double tot[3];
    if (reduce_last<3, 0u>(v, V, tot) && threadIdx.x == 0) {
        V.sc[SC_GG0] = tot[0];
        V.sc[SC_GG] = tot[1];
        V.sc[SC_GH] = tot[2];
    }
}

struct BdfHiLo {
    const double* y[kMaxBdfOrder];
    double lwr[kMaxBdfOrder];
    double q_n, hi_pre, lwr_y, lwr_dy, c1_c0;
    int hi, lo, m;
};

// Clock_BDF::hi_lo_err_est's vector part (clock_bdf.cpp:436-464): the
// higher- and lower-order error sums, then e_n = c - y_0
__global__ void __launch_bounds__(kCkBlock) k_bdf_hilo(CkView V, BdfVecs B, BdfHiLo P)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < V.n) {
        const double ci = V.c[i], y0 = B.y_0[i];
        if (P.hi) {
            const double t = dmul(dsub(dsub(ci, y0), dmul(P.q_n, B.e_n[i])), P.hi_pre);
            v[0] = dmul(t, t);
        }
        if (P.lo) {
            double t = dmul(P.lwr_y, ci);
            t = dadd(t, dmul(P.lwr_dy, V.c_d[i]));
            for (int j = 0; j < P.m; j++) t = dadd(t, dmul(P.lwr[j], P.y[j][i]));
            t = dmul(t, P.c1_c0);
            v[1] = dmul(t, t);
        }
        B.e_n[i] = dsub(ci, y0);
    }
    double tot[2];
    if (reduce_last<2, 0u>(v, V, tot) && threadIdx.x == 0) {
        V.sc[SC_GG0] = tot[0];
        V.sc[SC_GG] = tot[1];
    }
}

// ---- the clocks' line searches, steered on the device ------------------------
// The conjugate-gradient iterations of Clock_BDF::solve (clock_bdf.cpp:
// 727-828) and Clock_Adams::solve (clock_adams.cpp:316-365) run as one CUDA
// graph: a conditional WHILE node whose body is one calc_g with its step
// set-up and its decision, so a solve synchronises with the host once instead
// of once per calc_g. The scalar control (Armijo test, step reduction, restore
// of c0, direction update) is the reference's, evaluated by one thread in the
// same order of operations (explicitly rounded: no contraction into fused
// multiply-adds), so the device takes the steps the host loop took. The two
// solves differ in three places: the BDF clock starts a line search at
// 0.9 min(0.99, bound), the Adams clock at the bound; the BDF clock's trials
// take the full calc_g and a failed search restores c0, the Adams clock's
// trials take the cost only and every line search ends with a full calc_g at
// the last point; the BDF clock updates the direction after a successful
// search only, the Adams clock after every search.
struct SolveDev {
    double tol, min_gamma, gamma_red, slope;  // the cost tolerance, and the options
    double alpha;                             // calc_g's alpha
    double curr_cost, cost, g0_g0, g_h, bound, max_gamma, g_g, g_g0, ratio;
    int max_iter, iter, chk;
    int adams;      // Clock_Adams::solve's variant of the loop
    int mode;       // the body's calc_g: 0 at a trial point, 1 after restoring c0 (BDF),
                    // 2 the full calc_g at the last point after a line search (Adams)
    int calc_chk;   // calc_g's chk argument for the body (read by the g kernels)
    int line_done;  // the line search ended with this calc_g
    int need_next;  // a direction update follows (the line search succeeded)
    int copy_hg;    // h = g (the updated direction pointed uphill)
    int overrun;    // the iteration guard ended the loop
    long long n_calc_g;
};

// more body iterations than max_iter line searches of at most
// log(min_gamma) / log(gamma_red) trials each can take: a guard against a
// loop that does not end, reported as MG_ERR_TIMEOUT
constexpr long long kBsGuard = 100000;

// the top of the outer loop: its test, then the next line search's start;
// true when a calc_g follows, false when the solve is over
__device__ bool bs_outer_top(SolveDev& S)
{
    for (;;) {
        if (!(S.curr_cost > S.tol && S.iter < S.max_iter && S.max_gamma > S.min_gamma)) return false;
        if (S.adams) {
            S.max_gamma = S.bound;
        } else {
            // min(0.99, the box bounds along h) (clock_bdf.cpp:744-759)
            const double gamma = S.bound < 0.99 ? S.bound : 0.99;
            S.max_gamma = dmul(gamma, 0.9);
        }
        S.chk = 1;
        S.cost = S.curr_cost;
        if (S.max_gamma > S.min_gamma) {
            S.mode = 0;
            S.calc_chk = S.adams ? 1 : 0;
            return true;
        }
        if (S.adams) {
            // an empty line search still ends with the full calc_g
            S.mode = 2;
            S.calc_chk = 0;
            return true;
        }
        S.iter++;  // an empty line search: chk stays 1, no direction update
    }
}

// after the first calc_g and the first direction (k_ck_first_dir)
__global__ void k_bs_init(SolveDev* S, const double* red_out, const double* sc, cudaGraphConditionalHandle h)
{
    if (threadIdx.x) return;
    S->curr_cost = dmul(red_out[0], 0.25);
    S->g0_g0 = sc[SC_G0G0];
    S->g_h = S->g0_g0;
    S->bound = sc[SC_GAMMA];
    S->max_gamma = 1.0;
    S->iter = 0;
    S->n_calc_g = 0;
    S->overrun = 0;
    cudaGraphSetConditional(h, bs_outer_top(*S) ? 1u : 0u);
}

// the body's point: c0 + max_gamma h, or c0 itself after a failed line
// search; ghosts from their owners (what the reference's refresh copies)
__global__ void __launch_bounds__(kCkBlock) k_bs_trial(CkView V, const SolveDev* S)
{
    if (S->mode == 2) return;  // the full calc_g at the last point
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    const bool restore = S->mode == 1;
    const double gamma = S->max_gamma;
    if (i < V.n) {
        V.c[i] = restore ? V.c0[i] : dadd(V.c0[i], dmul(gamma, V.h[i]));
        return;
    }
    const int k = i - V.n;
    if (k >= V.nph * V.nt) return;
    const int gq = k / V.nt, a = k - gq * V.nt;
    const size_t o = (size_t)V.root[V.natms + gq] * V.nt + a;
    V.c[(size_t)(V.natms + gq) * V.nt + a] = restore ? V.c0[o] : dadd(V.c0[o], dmul(gamma, V.h[o]));
}

// the Armijo test of the body's calc_g and the step reduction
// (clock_bdf.cpp:760-806)
__global__ void k_bs_post(SolveDev* S, const double* red_out, const double* sc)
{
    if (threadIdx.x) return;
    S->n_calc_g++;
    S->curr_cost = dmul(red_out[0], 0.25);
    S->g_g0 = sc[SC_GG0];
    S->g_g = sc[SC_GG];
    S->need_next = 0;
    S->line_done = 1;
    if (S->adams) {
        if (S->mode == 0) {
            const double ideal = dsub(S->cost, dmul(dmul(S->slope, S->max_gamma), S->g_h));
            if (S->curr_cost < ideal) S->chk = 0;
            S->max_gamma = dmul(S->max_gamma, S->gamma_red);
            // the search goes on, or the full calc_g at this point follows
            S->mode = (S->chk && S->max_gamma > S->min_gamma) ? 0 : 2;
            S->calc_chk = S->mode == 0 ? 1 : 0;
            S->line_done = 0;
            return;
        }
        // after the full calc_g: the direction update, whatever the search gave
        S->ratio = ddiv(dsub(S->g_g, S->g_g0), S->g0_g0);
        S->g0_g0 = S->g_g;
        S->need_next = 1;
        return;
    }
    if (S->mode == 0) {
        const double ideal = dsub(S->cost, dmul(dmul(S->slope, S->max_gamma), S->g_h));
        if (S->curr_cost < ideal) S->chk = 0;
        S->max_gamma = dmul(S->max_gamma, S->gamma_red);
        if (S->max_gamma <= S->min_gamma) {
            // restore c0 and take the cost there (calc_g with chk = 1)
            S->mode = 1;
            S->calc_chk = 1;
            S->line_done = 0;
            return;
        }
        if (S->chk) {
            S->calc_chk = 0;
            S->line_done = 0;
            return;
        }
    }
    if (S->chk == 0) {
        S->ratio = ddiv(dsub(S->g_g, S->g_g0), S->g0_g0);
        S->g0_g0 = S->g_g;
        S->need_next = 1;
    }
}

// the direction update h = h ratio + g with h.g (clock_adams.cpp:356-366,
// clock_bdf.cpp:810-828), fused with the start of the next iteration: g0 = g,
// c0 = c, and the box bounds along the new h and along g (the direction
// restarts from g when h.g < 0); only when the body's post step asked for it
__global__ void __launch_bounds__(kCkBlock) k_bs_next_dir(CkView V, const SolveDev* S)
{
    if (!S->need_next) return;
    const double ratio = S->ratio;
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    double v[3] = {0.0, 1.0, 1.0};
    if (i < V.n) {
        const double gi = V.g[i], ci = V.c[i];
        const double hi = dadd(dmul(V.h[i], ratio), gi);
        V.h[i] = hi;
        V.g0[i] = gi;
        V.c0[i] = ci;
        v[0] = dmul(hi, gi);
        v[1] = box_bound(ci, dadd(ci, hi), 1.0);
        v[2] = box_bound(ci, dadd(ci, gi), 1.0);
    }
    double tot[3];
    if (reduce_last<3, 6u>(v, V, tot) && threadIdx.x == 0) {
        V.sc[SC_GH] = tot[0];
        V.sc[SC_GAMMA] = tot[1];
        V.sc[SC_B] = tot[2];
    }
}

// the end of an outer iteration: h.g, the step bounds, the restart from g
// when h.g < 0 (clock_bdf.cpp:810-828), then the outer loop's test
__global__ void k_bs_fin(SolveDev* S, const double* sc, cudaGraphConditionalHandle h)
{
    if (threadIdx.x) return;
    bool go = true;
    S->copy_hg = 0;
    if (S->line_done) {
        if (S->need_next) {
            S->g_h = sc[SC_GH];
            S->bound = sc[SC_GAMMA];
            if (S->g_h < 0.0) {
                S->copy_hg = 1;
                S->g_h = S->g_g;
                S->bound = sc[SC_B];
            }
        }
        S->iter++;
        go = bs_outer_top(*S);
    }
    if (go && S->n_calc_g >= kBsGuard) {
        S->overrun = 1;
        go = false;
    }
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

__global__ void __launch_bounds__(kCkBlock) k_bs_copy(CkView V, const SolveDev* S)
{
    if (!S->copy_hg) return;
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    if (i < V.n) V.h[i] = V.g[i];
}

constexpr double kBeta[6][6] = {
    {1.0, 0, 0, 0, 0, 0},
    {1.0 / 2.0, 1.0 / 2.0, 0, 0, 0, 0},
    {5.0 / 12.0, 8.0 / 12.0, -1.0 / 12.0, 0, 0, 0},
    {9.0 / 24.0, 19.0 / 24.0, -5.0 / 24.0, 1.0 / 24.0, 0, 0},
    {251.0 / 720.0, 646.0 / 720.0, -264.0 / 720.0, 106.0 / 720.0, -19.0 / 720.0, 0},
    {475.0 / 1440.0, 1427.0 / 1440.0, -798.0 / 1440.0, 482.0 / 1440.0, -173.0 / 1440.0, 27.0 / 1440.0}};

int ck_fail(cudaError_t e, const char* what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return internal_fail(MG_ERR_CUDA, m.c_str());
}

#define KCU(call)                                          \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return ck_fail(e_, #call);  \
    } while (0)
#define KCHK(call)                  \
    do {                            \
        int r_ = (call);            \
        if (r_ != MG_OK) return r_; \
    } while (0)

struct Clock {
    mg_system* s = nullptr;
    cudaStream_t st = nullptr;
    CkView V{};
    std::vector<double*> y;
    double* block = nullptr;  // one allocation for every vector and the scalars
    long long n_calc_g = 0;
    // the scalars and the line search's final state as the host reads them,
    // in page-locked memory: the copies are asynchronous, so one
    // synchronisation brings both (a copy into pageable memory would block
    // the host by itself, one more round trip per step)
    struct HostOut {
        double sc[SC_COUNT];
        SolveDev r;
    };
    HostOut* hout = nullptr;
    double* host_sc = nullptr;
    // the line search's graph (captured once per run) and its device state
    SolveDev* S_dev = nullptr;
    cudaGraph_t ls_graph = nullptr;
    cudaGraphExec_t ls_exec = nullptr;
    ~Clock()
    {
        if (ls_exec) cudaGraphExecDestroy(ls_exec);
        if (ls_graph) cudaGraphDestroy(ls_graph);
        cudaFree(S_dev);
        cudaFree(block);
        if (hout) cudaFreeHost(hout);
    }

    int grid() const { return V.nblocks; }
    int trial_grid() const { return div_up(V.n + V.nph * V.nt, kCkBlock); }

    // one iteration of the line search: the point, calc_g (chk and alpha from
    // the device state), the dot products, the Armijo test, the direction
    // update, the outer loop's test
    int enqueue_ls_body(cudaGraphConditionalHandle h)
    {
        k_bs_trial<<<trial_grid(), kCkBlock, 0, st>>>(V, S_dev);
        KCU(cudaGetLastError());
        int rows = 0;
        KCHK(system_enqueue_calc_g_dev(s, &S_dev->calc_chk, &S_dev->alpha, &rows));
        k_ck_dots<<<grid(), kCkBlock, 0, st>>>(V);
        k_bs_post<<<1, 32, 0, st>>>(S_dev, system_red_out(s), V.sc);
        k_bs_next_dir<<<grid(), kCkBlock, 0, st>>>(V, S_dev);
        k_bs_fin<<<1, 32, 0, st>>>(S_dev, V.sc, h);
        k_bs_copy<<<grid(), kCkBlock, 0, st>>>(V, S_dev);
        KCU(cudaGetLastError());
        return MG_OK;
    }

    // graph: k_bs_init, then WHILE (condition set by k_bs_init and k_bs_fin)
    int build_ls_graph()
    {
        KCU(cudaMalloc(&S_dev, sizeof(SolveDev)));
        KCU(cudaMallocHost((void**)&hout, sizeof(HostOut)));
        host_sc = hout->sc;
        KCU(cudaGraphCreate(&ls_graph, 0));
        cudaGraphConditionalHandle h;
        KCU(cudaGraphConditionalHandleCreate(&h, ls_graph, 0, cudaGraphCondAssignDefault));
        SolveDev* S = S_dev;
        const double* red = system_red_out(s);
        const double* sc = V.sc;
        void* args[] = {&S, &red, &sc, &h};
        cudaKernelNodeParams kp = {};
        kp.func = (void*)k_bs_init;
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(32);
        kp.sharedMemBytes = 0;
        kp.kernelParams = args;
        cudaGraphNode_t init;
        KCU(cudaGraphAddKernelNode(&init, ls_graph, nullptr, 0, &kp));
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        KCU(cudaGraphAddNode(&node, ls_graph, &init, 1, &np));
        cudaGraph_t body = np.conditional.phGraph_out[0];
        KCU(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        const int rc = enqueue_ls_body(h);
        cudaGraph_t out = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &out);
        if (rc != MG_OK) return rc;
        KCU(e);
        KCU(cudaGraphInstantiate(&ls_exec, ls_graph, 0));
        return MG_OK;
    }

    int refresh_c()
    {
        KCU(launch_refresh_c(system_dev(s), st));
        return MG_OK;
    }

    int read_scalars()
    {
        KCU(cudaMemcpyAsync(host_sc, V.sc, SC_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st));
        KCU(cudaStreamSynchronize(st));
        return MG_OK;
    }

    // Clock_Adams::solve (clock_adams.cpp:246-365): the first calc_g, c_d, the
    // bounded predictor and the first direction are enqueued, then the line
    // searches run as one graph launch (k_bs_*, the Adams variant), and the
    // final cost comes back in one synchronisation
    int solve(double delta_t, double bet, double* out_cost)
    {
        const double alpha = delta_t * bet;
        int rows = 0;
        KCHK(system_enqueue_calc_g(s, 0, alpha, &rows));
        n_calc_g++;
        KCHK(system_enqueue_c_d(s));
        k_ck_predict_bound<<<grid(), kCkBlock, 0, st>>>(V, delta_t);
        k_ck_predict<<<grid(), kCkBlock, 0, st>>>(V, delta_t);
        KCU(cudaGetLastError());
        KCHK(refresh_c());
        // h = g, and the first iteration's g0, c0 and step bound with it
        k_ck_first_dir<<<grid(), kCkBlock, 0, st>>>(V);
        KCU(cudaGetLastError());
        SolveDev hs{};
        hs.tol = 1.0e-8;
        hs.min_gamma = 1.0e-16;
        hs.gamma_red = 0.8;
        hs.slope = 0.4;
        hs.alpha = alpha;
        hs.max_iter = 50;
        hs.adams = 1;
        KCU(cudaMemcpyAsync(S_dev, &hs, sizeof(SolveDev), cudaMemcpyHostToDevice, st));
        KCU(cudaGraphLaunch(ls_exec, st));
        KCU(cudaMemcpyAsync(&hout->r, S_dev, sizeof(SolveDev), cudaMemcpyDeviceToHost, st));
        KCU(cudaStreamSynchronize(st));
        const SolveDev& r = hout->r;
        n_calc_g += r.n_calc_g;
        if (r.overrun) return internal_fail(MG_ERR_TIMEOUT, "Adams clock: the line search did not end");
        *out_cost = r.curr_cost;
        return MG_OK;
    }
};

// Clock_BDF's run (clock_bdf.cpp:479-675) over the device vectors: the
// interpolation coefficients, error prefactors and step/order control are
// scalar host work on the time history, exactly as the reference computes
// them; the vectors y_0, e_n, dy and the history y[0..max_order) stay on the
// device.
struct Bdf {
    Clock* ck = nullptr;
    mg_bdf_opts p{};
    int n = 0, dof_tot = 0, hi_ord_avail = 0, lo_ord_avail = 0;
    BdfVecs B{};
    std::vector<double*> y;  // y[0] newest; rotated by pointer as the reference does
    std::vector<double> t;
    double alpha_y[kMaxBdfOrder + 1], dalpha_y[kMaxBdfOrder + 1], lwr_alpha[kMaxBdfOrder + 1];
    double alpha_dy_0 = 0, dalpha_dy_0 = 0, beta = 0, err = 0, lo_err = 0, hi_err = 0, eq_ratio = 0;

    int grid() const { return ck->V.nblocks; }

    // Clock_BDF::interpolate (clock_bdf.cpp:295-368) -> 1 or -1
    int interpolate(double del_t, int q, int* ret)
    {
        double tmp0, tmp1, c0 = 1.0, c1 = 0.0, c2 = 0.0, c3, t_new = t[0] + del_t;
        for (int i = 1; i < q; i++) {
            tmp0 = (t_new - t[0]) / (t[i] - t[0]);
            tmp1 = tmp0 * tmp0;
            for (int j = 1; j < q; j++)
                if (i != j) tmp1 *= (t_new - t[j]) / (t[i] - t[j]);
            alpha_y[i] = tmp1;
            c0 *= (t_new - t[i]) / (t[0] - t[i]);
            c1 += 1.0 / (t[0] - t[i]);
            c2 += 1.0 / (t_new - t[i]);
        }
        alpha_y[0] = (1.0 - (t_new - t[0]) * c1) * c0;
        alpha_dy_0 = c0 * (t_new - t[0]);
        c3 = 2.0 / (t_new - t[0]);
        dalpha_dy_0 = alpha_dy_0 * (c2 + 0.5 * c3);
        dalpha_y[0] = c0 * (c2 - c1 + (t_new - t[0]) * c1 * c2);
        for (int i = 1; i < q; i++) dalpha_y[i] = alpha_y[i] * (c2 + c3 - 1.0 / (t_new - t[i]));
        tmp0 = 0.0;
        for (int i = 0; i < q; i++) tmp0 += 1.0 / (double)(i + 1);
        beta = del_t / tmp0;
        BdfHist H{};
        H.q = q;
        for (int j = 0; j < q; j++) {
            H.y[j] = y[j];
            H.ay[j] = alpha_y[j];
            H.bdy[j] = beta * dalpha_y[j];
        }
        k_bdf_interp<<<grid(), kCkBlock, 0, ck->st>>>(ck->V, B, H, beta * dalpha_dy_0, alpha_dy_0);
        KCU(cudaGetLastError());
        KCHK(ck->read_scalars());
        *ret = ck->host_sc[SC_A] < 0.0 ? -1 : 1;
        return MG_OK;
    }

    // Clock_BDF::solve (clock_bdf.cpp:677-884); *out = the cost ratio.  The
    // predictor, the first calc_g and the first direction are enqueued, then
    // the line search runs as one graph launch (k_bs_*), and the error sums
    // come back with its state in one synchronisation.  The error estimate
    // there reads an uninitialised local curr_t (clock_bdf.cpp:838-854) which
    // the reference built with gcc -O2 evaluates as 0.0; so does this.
    int solve(double del_t, int q, double* out)
    {
        const mg_bdf_opts& o = p;
        k_bdf_predict_bound<<<grid(), kCkBlock, 0, ck->st>>>(ck->V, y[0], B.dy, del_t);
        k_bdf_predict<<<grid(), kCkBlock, 0, ck->st>>>(ck->V, y[0], B.dy, del_t);
        KCU(cudaGetLastError());
        KCHK(ck->refresh_c());
        int rows = 0;
        KCHK(system_enqueue_calc_g(ck->s, 0, beta, &rows));
        ck->n_calc_g++;
        // h = g, and the first iteration's g0, c0 and step bound with it
        k_ck_first_dir<<<grid(), kCkBlock, 0, ck->st>>>(ck->V);
        KCU(cudaGetLastError());
        SolveDev hs{};
        hs.tol = o.m_tol * (double)dof_tot;
        hs.min_gamma = o.min_gamma;
        hs.gamma_red = o.gamma_red;
        hs.slope = o.slope;
        hs.alpha = beta;
        hs.max_iter = o.max_iter;
        KCU(cudaMemcpyAsync(ck->S_dev, &hs, sizeof(SolveDev), cudaMemcpyHostToDevice, ck->st));
        KCU(cudaGraphLaunch(ck->ls_exec, ck->st));
        k_bdf_err<<<grid(), kCkBlock, 0, ck->st>>>(ck->V, B);
        KCU(cudaGetLastError());
        // the line search's state and the error sums in one synchronisation
        KCU(cudaMemcpyAsync(&ck->hout->r, ck->S_dev, sizeof(SolveDev), cudaMemcpyDeviceToHost, ck->st));
        KCHK(ck->read_scalars());
        const SolveDev& r = ck->hout->r;
        ck->n_calc_g += r.n_calc_g;
        if (r.overrun) return internal_fail(MG_ERR_TIMEOUT, "BDF clock: the line search did not end");
        const double curr_cost = r.curr_cost;
        double a_1 = 1.0, curr_t = 0.0, l1_q = 0.0, err_pre_fac;
        for (int i = 0; i < q; i++) {
            l1_q += 1.0 / (curr_t - t[i]);
            if (i != 0) a_1 *= (curr_t - t[i]) / (t[0] - t[i]);
        }
        err_pre_fac = -1.0 / (l1_q * (1.0 + a_1));
        eq_ratio = sqrt(ck->host_sc[SC_GG] / (double)dof_tot) / o.e_tol;
        err = sqrt(ck->host_sc[SC_GG0] / ((double)dof_tot * o.a_tol));
        err *= fabs(err_pre_fac);
        if (ck->host_sc[SC_GH] != 0.0) return internal_fail(MG_ERR_DOMAIN, "c exceeded the domain");
        *out = curr_cost / (o.m_tol * (double)dof_tot);
        return MG_OK;
    }

    // Clock_BDF::hi_lo_err_est (clock_bdf.cpp:372-476)
    int hi_lo(double del_t, int q)
    {
        double curr_t = t[0] + del_t, c0 = 0.0, c1 = 1.0, tmp0;
        double a_0 = 1.0, a_1 = 1.0, l1_q = 0.0, hi_a_0, hi_a_1, hi_l1_q, lo_err_pre_fac;
        BdfHiLo P{};
        P.q_n = 1.0;
        P.hi_pre = 1.0;
        for (int i = 0; i < q; i++) {
            l1_q += 1.0 / (curr_t - t[i]);
            a_0 *= curr_t - t[i];
            if (i != 0) a_1 *= (curr_t - t[i]) / (t[0] - t[i]);
        }
        if (hi_ord_avail) {
            hi_a_0 = hi_a_1 = 1.0;
            for (int i = 0; i < q; i++) {
                hi_a_0 *= t[0] - t[i + 1];
                if (i != 0) hi_a_1 *= (t[0] - t[i + 1]) / (t[1] - t[i + 1]);
            }
            P.q_n = (a_0 / hi_a_0) * (1.0 + a_1) / (1.0 + hi_a_1) * (del_t / (t[0] - t[1]));
            hi_l1_q = l1_q + 1.0 / (curr_t - t[q]);
            P.hi_pre = -(curr_t - t[q]) / (q + 2);
            P.hi_pre *= 1.0 / (hi_l1_q * (1.0 + a_1) * del_t * del_t);
        }
        if (lo_ord_avail) {
            lo_err_pre_fac = -del_t * a_0 / (curr_t - t[q - 1]);
            c0 = 0.0;
            c1 = 1.0;
            for (int i = 0; i < q - 1; i++) {
                tmp0 = 1.0 / (curr_t - t[i]);
                c0 += tmp0;
                c1 *= tmp0;
                lwr_alpha[i] = tmp0 * tmp0;
                for (int j = 0; j < q - 1; j++)
                    if (i != j) lwr_alpha[i] *= 1.0 / (t[i] - t[j]);
                lwr_alpha[i] *= lo_err_pre_fac;
            }
            P.lwr_dy = c1 * lo_err_pre_fac;
            P.lwr_y = -c0 * c1 * lo_err_pre_fac;
            P.c1_c0 = c1 / c0;
            P.m = q - 1;
            for (int j = 0; j < q - 1; j++) {
                P.lwr[j] = lwr_alpha[j];
                P.y[j] = y[j];
            }
        }
        P.hi = hi_ord_avail;
        P.lo = lo_ord_avail;
        k_bdf_hilo<<<grid(), kCkBlock, 0, ck->st>>>(ck->V, B, P);
        KCU(cudaGetLastError());
        // the error sums only steer an order change: with neither order
        // available the host has nothing to read (the kernel still updates
        // e_n), so the step goes on without a synchronisation
        if (!hi_ord_avail && !lo_ord_avail) return MG_OK;
        KCHK(ck->read_scalars());
        lo_err = sqrt(ck->host_sc[SC_GG] / ((double)dof_tot * p.a_tol));
        hi_err = sqrt(ck->host_sc[SC_GG0] / ((double)dof_tot * p.a_tol));
        return MG_OK;
    }
};

int bdf_check(const mg_bdf_opts& o)
{
    const char* m = nullptr;
    if (o.min_gamma <= 0.0) m = "min_gamma should be larger than zero";
    else if (o.gamma_red <= 0.0 || o.gamma_red >= 1.0) m = "gamma_red should be between zero and one";
    else if (o.slope <= 0.0 || o.slope >= 1.0) m = "slope should be between zero and one";
    else if (o.max_iter <= 0) m = "max_iter should be larger than zero";
    else if (o.max_order <= 0) m = "max_order should be larger than zero";
    else if (o.m_tol <= 0.0) m = "m_tol should be larger than zero";
    else if (o.a_tol <= 0.0) m = "a_tol should be larger than zero";
    else if (o.e_tol < 0.0) m = "e_tol should be larger than zero";
    else if (o.min_del_t <= 0.0) m = "min_del_t should be larger than zero";
    else if (o.max_del_t <= 0.0) m = "max_del_t should be larger than zero";
    else if (o.min_del_t >= o.max_del_t) m = "max_del_t should be larger than min_del_t";
    else if (o.initial_del_t == 0.0) m = "initial_del_t should be larger than zero";
    if (m) return internal_fail(MG_ERR_ARG, m);
    if (o.max_order > kMaxBdfOrder) return internal_fail(MG_ERR_UNSUPPORTED, "max_order above 12");
    return MG_OK;
}

// the clock's set-up shared by the Adams and BDF clocks: DMD style in the
// plain form, then Clock::init's crd list and force_calc(1), which fills the
// per-pair buffers c_d_calc and calc_g read
int clock_setup(mg_system* s, const char* what)
{
    KCHK(system_check_ready(s));
    int style = -1, nt = 0, x_dim = 0, form = 0;
    system_shape(s, &style, &nt, &x_dim, &form, nullptr);
    if (style != STYLE_DMD_I && style != STYLE_DMD_II && style != STYLE_DMD) {
        std::string m = std::string("the ") + what + " clock integrates DMD concentrations";
        return internal_fail(MG_ERR_UNSUPPORTED, m.c_str());
    }
    if (form != MG_FORM_FP64) {
        std::string m = std::string("the ") + what + " clock runs calc_g in the plain FP64 form";
        return internal_fail(MG_ERR_UNSUPPORTED, m.c_str());
    }
    return MG_OK;
}

// the clocks keep positions and lists fixed, so calc_g and c_d_calc may walk
// the active-pair sublist for the whole run; switched off again on every exit
struct ActivePairs {
    mg_system* s;
    explicit ActivePairs(mg_system* sys) : s(sys) {}
    ~ActivePairs() { system_set_active_pairs(s, false); }
};

int clock_force_init(mg_system* s)
{
    int style = -1, nt = 0, x_dim = 0, form = 0;
    system_shape(s, &style, &nt, &x_dim, &form, nullptr);
    const int natms = system_natms(s);
    KCHK(mg_ff_create_2nd_neigh_lst(s));
    double* fdev = nullptr;
    KCU(cudaMalloc(&fdev, ((size_t)natms * x_dim + 1) * sizeof(double)));
    double en[7];
    int rc = mg_ff_force_calc(s, 1, fdev, en);
    cudaFree(fdev);
    if (rc != MG_OK) return rc;
    return system_set_active_pairs(s, true);
}

}  // namespace

}  // namespace mg

using namespace mg;

extern "C" int mg_clock_adams(mg_system* s, int order, int nsteps, double delta_t, double* err, long long* n_calc_g)
{
    MG_NVTX("mg_clock_adams");
    KCHK(clock_setup(s, "Adams"));
    int style = -1, nt = 0, x_dim = 0, form = 0;
    system_shape(s, &style, &nt, &x_dim, &form, nullptr);
    if (order < 1 || order > 6) {
        char msg[96];
        snprintf(msg, sizeof(msg), "BDF cannot operate with order: %d", order);  // the reference's text
        return internal_fail(MG_ERR_ARG, msg);
    }
    if (nsteps < 0 || !(delta_t > 0.0)) return internal_fail(MG_ERR_ARG, "steps >= 0 and delta_t > 0 are required");
    const int natms = system_natms(s);
    Clock ck;
    ck.s = s;
    ck.st = system_stream(s);
    ActivePairs active(s);
    KCHK(clock_force_init(s));
    const int n = natms * nt;
    if (n == 0 || nsteps == 0) {
        if (n_calc_g) *n_calc_g = 0;
        return MG_OK;
    }
    const int m = order > 1 ? order - 1 : 0;
    const int nblocks = div_up(n, kCkBlock);
    size_t vec = ((size_t)n + 31) / 32 * 32;
    size_t total = vec * (3 + m) + (size_t)nblocks * 8 + SC_COUNT + 8;
    KCU(cudaMalloc(&ck.block, total * sizeof(double)));
    Dev& d = system_dev(s);
    ck.V.c = d.c;
    ck.V.c_d = d.c_d;
    ck.V.g = d.g;
    ck.V.a = d.a_in;
    ck.V.g0 = ck.block;
    ck.V.c0 = ck.block + vec;
    ck.V.h = ck.block + 2 * vec;
    for (int j = 0; j < m; j++) ck.y.push_back(ck.block + (3 + j) * vec);
    ck.V.part = ck.block + (3 + m) * vec;
    ck.V.sc = ck.V.part + (size_t)nblocks * 8;
    ck.V.counter = reinterpret_cast<unsigned int*>(ck.V.sc + SC_COUNT);
    ck.V.n = n;
    ck.V.nblocks = nblocks;
    ck.V.root = d.root;
    ck.V.natms = natms;
    ck.V.nph = d.nph;
    ck.V.nt = nt;
    KCU(cudaMemsetAsync(ck.V.counter, 0, 8 * sizeof(double), ck.st));
    KCHK(ck.build_ls_graph());
    const double* beta = kBeta[order - 1];
    std::vector<int> slot(m);
    for (int j = 0; j < m; j++) slot[j] = j;
    for (int istep = 0; istep < nsteps; istep++) {
        History Y{};
        double bet = 1.0;
        if (istep >= order) {
            Y.m = m;
            for (int j = 0; j < m; j++) {
                Y.y[j] = ck.y[slot[j]];
                Y.coef[j] = delta_t * beta[j + 1];
            }
            bet = beta[0];
        }
        k_ck_form_a<<<nblocks, kCkBlock, 0, ck.st>>>(ck.V, Y);
        KCU(cudaGetLastError());
        double cur = 0.0;
        KCHK(ck.solve(delta_t, bet, &cur));
        if (err) err[istep] = cur;
        if (m > 0) {
            int last = slot[m - 1];
            for (int i = m - 1; i > 0; i--) slot[i] = slot[i - 1];
            slot[0] = last;
            KCU(cudaMemcpyAsync(ck.y[slot[0]], d.c_d, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, ck.st));
        }
    }
    KCU(cudaStreamSynchronize(ck.st));
    if (n_calc_g) *n_calc_g = ck.n_calc_g;
    return MG_OK;
}

extern "C" void mg_bdf_defaults(mg_bdf_opts* o)
{
    if (!o) return;
    // Clock_BDF's constructor defaults (clock_bdf.cpp:14-24)
    o->max_order = 6;
    o->max_iter = 50;
    o->min_gamma = 1.0e-10;
    o->gamma_red = 0.8;
    o->slope = 0.4;
    o->m_tol = 1.0e-10;
    o->a_tol = 1.0e-6;
    o->e_tol = 0.0;
    o->min_del_t = 1.0e-12;
    o->max_del_t = 1.0e4;
    o->initial_del_t = -1.0;
}

extern "C" int mg_clock_bdf(mg_system* s, int nsteps, const mg_bdf_opts* opts, double* hist, int* steps_taken,
                            long long* n_calc_g)
{
    MG_NVTX("mg_clock_bdf");
    KCHK(clock_setup(s, "BDF"));
    if (nsteps <= 0) return internal_fail(MG_ERR_ARG, "no of steps should be greater than zero");
    mg_bdf_opts o;
    mg_bdf_defaults(&o);
    if (opts) o = *opts;
    KCHK(bdf_check(o));
    int style = -1, nt = 0, x_dim = 0, form = 0;
    system_shape(s, &style, &nt, &x_dim, &form, nullptr);
    const int natms = system_natms(s);
    Clock ck;
    ck.s = s;
    ck.st = system_stream(s);
    // Clock_BDF::init (clock_bdf.cpp:201-275)
    ActivePairs active(s);
    KCHK(clock_force_init(s));
    const int n = natms * nt;
    if (steps_taken) *steps_taken = 0;
    if (n_calc_g) *n_calc_g = 0;
    if (n == 0) return MG_OK;
    const int mo = o.max_order, nblocks = div_up(n, kCkBlock);
    const size_t vec = ((size_t)n + 31) / 32 * 32;
    const size_t total = vec * (6 + mo) + (size_t)nblocks * 8 + SC_COUNT + 8;
    KCU(cudaMalloc(&ck.block, total * sizeof(double)));
    Dev& d = system_dev(s);
    ck.V.c = d.c;
    ck.V.c_d = d.c_d;
    ck.V.g = d.g;
    ck.V.a = d.a_in;
    ck.V.g0 = ck.block;
    ck.V.c0 = ck.block + vec;
    ck.V.h = ck.block + 2 * vec;
    Bdf b;
    b.ck = &ck;
    b.p = o;
    b.n = n;
    b.dof_tot = n;
    b.B.y_0 = ck.block + 3 * vec;
    b.B.e_n = ck.block + 4 * vec;
    b.B.dy = ck.block + 5 * vec;
    for (int j = 0; j < mo; j++) b.y.push_back(ck.block + (6 + j) * vec);
    b.t.assign(mo + 1, 0.0);
    ck.V.part = ck.block + (6 + mo) * vec;
    ck.V.sc = ck.V.part + (size_t)nblocks * 8;
    ck.V.counter = reinterpret_cast<unsigned int*>(ck.V.sc + SC_COUNT);
    ck.V.n = n;
    ck.V.nblocks = nblocks;
    ck.V.root = d.root;
    ck.V.natms = natms;
    ck.V.nph = d.nph;
    ck.V.nt = nt;
    KCU(cudaMemsetAsync(ck.block, 0, total * sizeof(double), ck.st));
    KCHK(ck.build_ls_graph());
    KCHK(system_enqueue_c_d(s));
    const size_t bytes = (size_t)n * sizeof(double);
    double initial_del_t = o.initial_del_t;
    if (initial_del_t < 0.0) {
        // y_0 is still zero: the error kernel's second sum is sum c_d^2
        k_bdf_err<<<nblocks, kCkBlock, 0, ck.st>>>(ck.V, b.B);
        KCU(cudaGetLastError());
        KCHK(ck.read_scalars());
        double sum = sqrt(ck.host_sc[SC_GG] / (double)n);
        initial_del_t = o.a_tol / sum > o.min_del_t ? o.a_tol / sum : o.min_del_t;
        initial_del_t = initial_del_t < o.max_del_t ? initial_del_t : o.max_del_t;
    }
    KCU(cudaMemcpyAsync(b.y[0], d.c, bytes, cudaMemcpyDeviceToDevice, ck.st));
    KCU(cudaMemcpyAsync(b.B.dy, d.c_d, bytes, cudaMemcpyDeviceToDevice, ck.st));
    // Clock_BDF::run (clock_bdf.cpp:479-675); the reference's retry loops on a
    // predictor outside [0, 1] have no bound, these give up after 100000 tries
    const long kMaxRetries = 100000;
    double del_t = initial_del_t, del_t_tmp, err1, ratio = 1.0, cost = 0.0, lo_ratio, hi_ratio;
    int ord = 1, chk = 1, const_stp = 0, istep = 0;
    long guard = 0;
    b.eq_ratio = 1.0;
    while (b.eq_ratio >= 1.0 && istep < nsteps) {
        KCHK(b.interpolate(del_t, ord, &chk));
        while (chk == -1) {
            if (++guard > kMaxRetries) return internal_fail(MG_ERR_DOMAIN, "the predictor stays outside [0, 1]");
            // at min_del_t the clamped retry repeats the same interpolation:
            // the reference would loop for ever
            if (del_t == o.min_del_t)
                return internal_fail(MG_ERR_DOMAIN, "the predictor leaves [0, 1] even at min_del_t");
            del_t *= 0.8;
            del_t = del_t > o.min_del_t ? del_t : o.min_del_t;
            KCHK(b.interpolate(del_t, ord, &chk));
        }
        KCHK(b.solve(del_t, ord, &cost));
        double tried = del_t;
        while (b.err >= 1.0 || cost >= 1.0) {
            if (++guard > kMaxRetries) return internal_fail(MG_ERR_DOMAIN, "the step size does not settle");
            err1 = b.err > cost ? b.err : cost;
            ratio = pow(0.5 / err1, 1.0 / (double)(ord + 1));
            if (ratio < 0.5) ratio = 0.5;
            else if (ratio > 0.9) ratio = 0.9;
            del_t_tmp = del_t * ratio;
            del_t = del_t_tmp < o.min_del_t ? o.min_del_t : del_t_tmp;
            KCHK(b.interpolate(del_t, ord, &chk));
            while (chk == -1) {
                if (++guard > kMaxRetries) return internal_fail(MG_ERR_DOMAIN, "the predictor stays outside [0, 1]");
                del_t *= 0.8;
                KCHK(b.interpolate(del_t, ord, &chk));
            }
            // a retry at the step size just tried repeats that solve exactly:
            // the reference would loop for ever
            if (del_t == tried) return internal_fail(MG_ERR_DOMAIN, "the step cannot shrink below min_del_t");
            tried = del_t;
            KCHK(b.solve(del_t, ord, &cost));
        }
        double* tmp_y = b.y[mo - 1];
        for (int i = mo - 1; i > 0; i--) {
            b.t[i] = b.t[i - 1];
            b.y[i] = b.y[i - 1];
        }
        b.y[0] = tmp_y;
        b.t[0] += del_t;
        KCU(cudaMemcpyAsync(b.y[0], d.c, bytes, cudaMemcpyDeviceToDevice, ck.st));
        KCU(cudaMemcpyAsync(b.B.dy, d.c_d, bytes, cudaMemcpyDeviceToDevice, ck.st));
        b.lo_ord_avail = (ord != 1 && const_stp > ord + 1) ? 1 : 0;
        b.hi_ord_avail = ((ord < mo && istep != 0) && const_stp > ord + 1) ? 1 : 0;
        KCHK(b.hi_lo(del_t, ord));
        if (hist) {
            hist[3 * istep] = del_t;
            hist[3 * istep + 1] = ord;
            hist[3 * istep + 2] = b.t[0];
        }
        if (b.hi_ord_avail && b.lo_ord_avail) {
            lo_ratio = pow(0.5 / b.lo_err, 1.0 / (double)ord);
            hi_ratio = pow(0.5 / b.hi_err, 1.0 / (double)(ord + 2));
            ratio = pow(0.5 / b.err, 1.0 / (double)(ord + 1));
            if (hi_ratio > lo_ratio && hi_ratio > ratio) {
                ord++;
                ratio = hi_ratio;
            } else if (lo_ratio > hi_ratio && lo_ratio > ratio) {
                ord--;
                ratio = lo_ratio;
            }
        } else if (b.hi_ord_avail == 1 && b.lo_ord_avail == 0) {
            hi_ratio = pow(0.5 / b.hi_err, 1.0 / (double)(ord + 2));
            ratio = pow(0.5 / b.err, 1.0 / (double)(ord + 1));
            if (hi_ratio > ratio) {
                ord++;
                ratio = hi_ratio;
            }
        } else if (b.hi_ord_avail == 0 && b.lo_ord_avail == 1) {
            lo_ratio = pow(0.5 / b.lo_err, 1.0 / (double)ord);
            ratio = pow(0.5 / b.err, 1.0 / (double)(ord + 1));
            if (lo_ratio > ratio) {
                ord--;
                ratio = lo_ratio;
            }
        } else
            ratio = pow(0.5 / b.err, 1.0 / (double)(ord + 1));
        if (ratio >= 2.0) {
            ratio = 2.0;
            const_stp = 0;
        } else if (ratio <= 0.5) {
            ratio = 0.5;
            const_stp = 0;
        } else {
            ratio = 1.0;
            const_stp++;
        }
        del_t_tmp = ratio * del_t;
        if (del_t_tmp > o.max_del_t) del_t = o.max_del_t;
        else if (del_t_tmp < o.min_del_t) del_t = o.min_del_t;
        else del_t = del_t_tmp;
        istep++;
    }
    KCU(cudaStreamSynchronize(ck.st));
    if (steps_taken) *steps_taken = istep;
    if (n_calc_g) *n_calc_g = ck.n_calc_g;
    return MG_OK;
}
