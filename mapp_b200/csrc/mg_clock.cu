// Adams clock on the device: Clock_Adams (clock_adams.cpp) for a DMD system,
// with every concentration-sized vector resident in HBM.
//
// The reference keeps a, g, g0, c0, h and the c_d history on the host and
// loops over them between calc_g calls, which in a GPU build would move every
// vector across the boundary tens of times per step.  Here the vector work is
// a handful of kernels over the natms * nt concentrations (forming a, the
// predictor, the conjugate-gradient direction, the box-constrained step
// bound) and the force field's own calc_g / c_d_calc kernels; only the scalars
// that steer the solve (costs, dot products, step bounds) come back to the
// host, which runs the reference's control flow on them unchanged.  Dot
// products and minima are deterministic: per-block partials reduced in a
// fixed order by the last block to finish.
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
enum { SC_RATIO = 0, SC_GG0 = 1, SC_GG = 2, SC_GH = 3, SC_GAMMA = 4, SC_G0G0 = 5, SC_COUNT = 8 };

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
};

// Block reduction of NV values, then the fixed-order reduction of all block
// rows by the last block; MIN selects minima instead of sums.  Returns true
// in the last block, where tot holds the result in every thread.
template <int NV, bool MIN>
__device__ bool reduce_last(double (&v)[NV], const CkView& V, double (&tot)[NV])
{
    __shared__ double sh[kCkBlock / 32][NV];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double a = v[k];
        for (int o = 16; o > 0; o >>= 1) {
            double b = __shfl_down_sync(0xffffffffu, a, o);
            a = MIN ? fmin(a, b) : a + b;
        }
        if (lane == 0) sh[w][k] = a;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double a = sh[0][threadIdx.x];
        for (int j = 1; j < kCkBlock / 32; j++) a = MIN ? fmin(a, sh[j][threadIdx.x]) : a + sh[j][threadIdx.x];
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
        double a = MIN ? 1.0 : 0.0;
        for (int b = threadIdx.x; b < V.nblocks; b += kCkBlock) {
            double x = __ldcg(V.part + (size_t)b * 8 + k);
            a = MIN ? fmin(a, x) : a + x;
        }
        for (int o = 16; o > 0; o >>= 1) {
            double b = __shfl_down_sync(0xffffffffu, a, o);
            a = MIN ? fmin(a, b) : a + b;
        }
        if (lane == 0) sh[w][k] = a;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double a = sh[0][k];
        for (int j = 1; j < kCkBlock / 32; j++) a = MIN ? fmin(a, sh[j][k]) : a + sh[j][k];
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
    if (reduce_last<1, true>(v, V, tot) && threadIdx.x == 0) V.sc[SC_RATIO] = tot[0];
}

// c += c_d dt ratio; then h = g and g.g (clock_adams.cpp:277-290)
__global__ void __launch_bounds__(kCkBlock) k_ck_predict(CkView V, double dt)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    if (i >= V.n) return;
    const double r = V.sc[SC_RATIO];
    V.c[i] = dadd(V.c[i], dmul(dmul(V.c_d[i], dt), r));
}

__global__ void __launch_bounds__(kCkBlock) k_ck_h_from_g(CkView V)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    double v[1] = {0.0};
    if (i < V.n) {
        const double gi = V.g[i];
        V.h[i] = gi;
        v[0] = dmul(gi, gi);
    }
    double tot[1];
    if (reduce_last<1, false>(v, V, tot) && threadIdx.x == 0) V.sc[SC_G0G0] = tot[0];
}

// start of a conjugate-gradient iteration: g0 = g, c0 = c, and the step bound
// gamma along h (clock_adams.cpp:296-314)
__global__ void __launch_bounds__(kCkBlock) k_ck_begin(CkView V)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    double v[1] = {1.0};
    if (i < V.n) {
        const double ci = V.c[i], hi = V.h[i];
        V.g0[i] = V.g[i];
        V.c0[i] = ci;
        v[0] = box_bound(ci, dadd(ci, hi), 1.0);
    }
    double tot[1];
    if (reduce_last<1, true>(v, V, tot) && threadIdx.x == 0) V.sc[SC_GAMMA] = tot[0];
}

// trial point c = c0 + gamma h (clock_adams.cpp:322-323)
__global__ void __launch_bounds__(kCkBlock) k_ck_trial(CkView V, double gamma)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    if (i < V.n) V.c[i] = dadd(V.c0[i], dmul(gamma, V.h[i]));
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
    if (reduce_last<2, false>(v, V, tot) && threadIdx.x == 0) {
        V.sc[SC_GG0] = tot[0];
        V.sc[SC_GG] = tot[1];
    }
}

// h = h ratio + g and h.g (clock_adams.cpp:356-366)
__global__ void __launch_bounds__(kCkBlock) k_ck_direction(CkView V, double ratio)
{
    const int i = blockIdx.x * kCkBlock + threadIdx.x;
    double v[1] = {0.0};
    if (i < V.n) {
        const double gi = V.g[i];
        const double hi = dadd(dmul(V.h[i], ratio), gi);
        V.h[i] = hi;
        v[0] = dmul(hi, gi);
    }
    double tot[1];
    if (reduce_last<1, false>(v, V, tot) && threadIdx.x == 0) V.sc[SC_GH] = tot[0];
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
    double host_sc[SC_COUNT];
    ~Clock() { cudaFree(block); }

    int grid() const { return V.nblocks; }

    // calc_g(chk, alpha, a, g) -> cost (one synchronisation)
    int calc_g(int chk, double alpha, double* cost, bool with_dots = false)
    {
        int rows = 0;
        KCHK(system_enqueue_calc_g(s, chk, alpha, &rows));
        n_calc_g++;
        if (with_dots) {
            k_ck_dots<<<grid(), kCkBlock, 0, st>>>(V);
            KCU(cudaGetLastError());
        }
        double r[1];
        KCU(cudaMemcpyAsync(r, system_red_out(s), sizeof(double), cudaMemcpyDeviceToHost, st));
        if (with_dots) KCU(cudaMemcpyAsync(host_sc, V.sc, SC_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st));
        KCU(cudaStreamSynchronize(st));
        *cost = r[0] * 0.25;
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

    // Clock_Adams::solve (clock_adams.cpp:246-365)
    int solve(double delta_t, double bet, double* out_cost)
    {
        const double min_gamma = 1.0e-16, slope = 0.4, gamma_red = 0.8, alpha = delta_t * bet;
        double max_gamma = 1.0, ratio, g0_g0, g_g, g_g0, g_h, curr_cost, ideal_cost, cost;
        int chk;
        KCHK(calc_g(0, alpha, &curr_cost));
        KCHK(system_enqueue_c_d(s));
        k_ck_predict_bound<<<grid(), kCkBlock, 0, st>>>(V, delta_t);
        k_ck_predict<<<grid(), kCkBlock, 0, st>>>(V, delta_t);
        KCU(cudaGetLastError());
        KCHK(refresh_c());
        k_ck_h_from_g<<<grid(), kCkBlock, 0, st>>>(V);
        KCU(cudaGetLastError());
        KCHK(read_scalars());
        g0_g0 = host_sc[SC_G0G0];
        g_h = g0_g0;
        int iter = 0;
        while (curr_cost > 1.0e-8 && iter < 50 && max_gamma > min_gamma) {
            k_ck_begin<<<grid(), kCkBlock, 0, st>>>(V);
            KCU(cudaGetLastError());
            KCHK(read_scalars());
            max_gamma = host_sc[SC_GAMMA];
            chk = 1;
            cost = curr_cost;
            while (chk && max_gamma > min_gamma) {
                k_ck_trial<<<grid(), kCkBlock, 0, st>>>(V, max_gamma);
                KCU(cudaGetLastError());
                KCHK(refresh_c());
                KCHK(calc_g(1, alpha, &curr_cost));
                ideal_cost = cost - slope * max_gamma * g_h;
                if (curr_cost < ideal_cost) chk = 0;
                max_gamma *= gamma_red;
                // the reference restores c0 when max_gamma <= 0, which the
                // positive factor gamma_red never reaches
            }
            KCHK(calc_g(0, alpha, &curr_cost, true));
            g_g0 = host_sc[SC_GG0];
            g_g = host_sc[SC_GG];
            ratio = (g_g - g_g0) / g0_g0;
            g0_g0 = g_g;
            k_ck_direction<<<grid(), kCkBlock, 0, st>>>(V, ratio);
            KCU(cudaGetLastError());
            KCHK(read_scalars());
            g_h = host_sc[SC_GH];
            if (g_h < 0.0) {
                KCU(cudaMemcpyAsync(V.h, V.g, (size_t)V.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
                g_h = g_g;
            }
            iter++;
        }
        *out_cost = curr_cost;
        return MG_OK;
    }
};

}  // namespace

}  // namespace mg

using namespace mg;

extern "C" int mg_clock_adams(mg_system* s, int order, int nsteps, double delta_t, double* err, long long* n_calc_g)
{
    KCHK(system_check_ready(s));
    int style = -1, nt = 0, x_dim = 0, form = 0;
    system_shape(s, &style, &nt, &x_dim, &form, nullptr);
    if (style != STYLE_DMD_I && style != STYLE_DMD_II && style != STYLE_DMD)
        return internal_fail(MG_ERR_UNSUPPORTED, "the Adams clock integrates DMD concentrations");
    if (form != MG_FORM_FP64) return internal_fail(MG_ERR_UNSUPPORTED, "the Adams clock runs calc_g in the plain FP64 form");
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
    // Clock_Adams::init after the set-up: the crd list and force_calc(1), which
    // fills the per-pair buffers c_d_calc and calc_g read
    KCHK(mg_ff_create_2nd_neigh_lst(s));
    {
        double* fdev = nullptr;
        KCU(cudaMalloc(&fdev, ((size_t)natms * x_dim + 1) * sizeof(double)));
        double en[7];
        int rc = mg_ff_force_calc(s, 1, fdev, en);
        cudaFree(fdev);
        if (rc != MG_OK) return rc;
    }
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
    KCU(cudaMemsetAsync(ck.V.counter, 0, 8 * sizeof(double), ck.st));
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
