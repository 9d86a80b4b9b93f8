// Nose-Hoover NVT molecular dynamics on the device: MD_NH without a barostat
// and without a "dof" vector (md_nh.cpp:385-683, 865-1035), driving the EAM /
// FS force path of one system.
//
// One step of the reference is
//   update_NH_T(dt/2)  update_x_d(dt/2)  update_x(dt)  update_0
//   zero_f  force_calc  update_x_d(dt/2)  update_NH_T(dt/2)
// and here it is five kernels per step, all but the rebuild on the device:
//   k_md_kick_drift   x_d *= the two pending thermostat factors, x_d += f dt/2m,
//                     x_u = x + x_d dt, and the mean displacement (last block)
//   k_md_center       x = x_u - mean for owned atoms and ghosts, the skin test
//                     against x_0, zero f and rho; sets the loop condition
//   force passes      the library's EAM / FS kernels
//   k_md_kick2        x_d += f dt/2m, kinetic tensor; the last block runs the
//                     chain for the end of this step and the start of the next
// The steps between two list rebuilds run as one CUDA graph with a while node;
// a step whose skin test fails leaves the loop after k_md_center, the host
// rebuilds the ghosts and the list (the rebuild branch of Atoms::update_0) and
// relaunches.  The chain rescale of x_d (update_NH_T's last loop) is folded
// into the next kernel that touches x_d, applied factor by factor in the same
// order.  update_x_d's kinetic tensor of the first half kick only feeds the
// reference's thermo output and is not formed.
//
// Every per-atom operation uses round-to-nearest intrinsics in the reference's
// order; the sums over atoms (kinetic tensor, mean displacement) are
// deterministic block partials reduced in a fixed order by the last block.
#include <cmath>
#include <cstring>
#include <vector>

#include "mg_internal.h"
#include "../../include/mapp_b200.h"

namespace mg {

namespace {

constexpr int kMdBlock = 256;
constexpr int kMaxEta = 16;

struct NhConst {
    double mass[kMaxTypes];
    double dt, dt2, boltz, t_tar, t_freq, ke_tar, sq_skin, inv_n;
    int no_dof, no_it, no_ch, nsteps, nblocks_own, nblocks_all;
};

struct NhState {
    double eta_m[kMaxEta], eta_d[kMaxEta], eta_dd[kMaxEta];
    double ke_curr[6], ke_cur, t_cur;
    double fac_a, fac_b;  // pending x_d factors: end of the last step, start of the next
    double ave[3];        // mean displacement of the step being built
    int step, rebuild, done, pad;
    unsigned int count[3];  // last-block counters of the three reducing kernels
};

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// a species' mass, selected without indexing the parameter struct dynamically
// (which would copy it to local memory)
__device__ __forceinline__ double mass_of(const NhConst& C, int t)
{
    static_assert(kMaxTypes == 4, "mass_of selects among four species");
    return t == 0 ? C.mass[0] : t == 1 ? C.mass[1] : t == 2 ? C.mass[2] : C.mass[3];
}

// MD_NH::update_NH_T (md_nh.cpp:965-1035) on the state; returns velfac
__device__ double nh_chain(NhState* S, const NhConst& C, double dlt)
{
    const int nc = C.no_ch;
    double* em = S->eta_m;
    double* ed = S->eta_d;
    double* edd = S->eta_dd;
    for (int i = 0; i < nc; i++) em[i] = ddiv(dmul(C.boltz, C.t_tar), dmul(C.t_freq, C.t_freq));
    em[0] = dmul(em[0], (double)C.no_dof);
    double dltm = dmul(dlt, ddiv(1.0, (double)C.no_it));
    double dltm2 = dmul(0.5, dltm), dltm4 = dmul(0.25, dltm), velfac = 1.0, exfac;
    edd[0] = ddiv(dsub(S->ke_cur, C.ke_tar), em[0]);
    for (int it = 0; it < C.no_it; it++) {
        exfac = 1.0;
        for (int ich = nc - 1; ich > -1; ich--) {
            ed[ich] = dmul(ed[ich], exfac);
            ed[ich] = dadd(ed[ich], dmul(edd[ich], dltm2));
            ed[ich] = dmul(ed[ich], exfac);
            exfac = exp(dmul(-dltm4, ed[ich]));
        }
        exfac = exp(dmul(-dltm, ed[0]));
        velfac = dmul(velfac, exfac);
        double e2 = dmul(exfac, exfac);
        S->t_cur = dmul(S->t_cur, e2);
        S->ke_cur = dmul(S->ke_cur, e2);
        for (int k = 0; k < 6; k++) S->ke_curr[k] = dmul(S->ke_curr[k], e2);
        exfac = exp(dmul(-dltm4, ed[1]));
        ed[0] = dmul(ed[0], exfac);
        edd[0] = ddiv(dsub(S->ke_cur, C.ke_tar), em[0]);
        ed[0] = dadd(ed[0], dmul(edd[0], dltm2));
        ed[0] = dmul(ed[0], exfac);
        for (int ich = 1; ich < nc; ich++) {
            exfac = ich == nc - 1 ? 1.0 : exp(dmul(-dltm4, ed[ich + 1]));
            ed[ich] = dmul(ed[ich], exfac);
            edd[ich] = ddiv(dsub(dmul(dmul(em[ich - 1], ed[ich - 1]), ed[ich - 1]), dmul(C.boltz, C.t_tar)), em[ich]);
            ed[ich] = dadd(ed[ich], dmul(edd[ich], dltm2));
            ed[ich] = dmul(ed[ich], exfac);
        }
    }
    return velfac;
}

// Block sum of NV values per thread into part[blockIdx][0..NV), then, in the
// last block to finish, the fixed-order sum of all block rows into tot[0..NV).
// Returns true in the last block (tot valid in every thread of it).
template <int NV>
__device__ bool last_block_sum(double (&v)[NV], double* __restrict__ part, unsigned int* counter, int nblocks,
                               double (&tot)[NV])
{
    __shared__ double sh[kMdBlock / 32][NV];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double a = v[k];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) sh[w][k] = a;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double a = 0.0;
        for (int j = 0; j < kMdBlock / 32; j++) a += sh[j][threadIdx.x];
        part[(size_t)blockIdx.x * 8 + threadIdx.x] = a;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == (unsigned)(nblocks - 1);
    __syncthreads();
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double a = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += kMdBlock) a += __ldcg(part + (size_t)b * 8 + k);
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) sh[w][k] = a;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double a = 0.0;
        for (int j = 0; j < kMdBlock / 32; j++) a += sh[j][k];
        tot[k] = a;
    }
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

// start of the very first step: the thermostat's first half step
__global__ void k_md_begin(NhState* S, NhConst C)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        S->fac_a = 1.0;
        S->fac_b = nh_chain(S, C, C.dt2);
    }
}

// update_NH_T's rescale (both pending factors), update_x_d(dt/2), update_x(dt)
// before the mean is removed (md_nh.cpp:885-898)
__global__ void __launch_bounds__(kMdBlock) k_md_kick_drift(Dev d, NhConst C, NhState* S, double4* __restrict__ xd,
                                                            double4* __restrict__ xu, double* __restrict__ part)
{
    if (S->done) return;
    const int i = blockIdx.x * kMdBlock + threadIdx.x;
    const double fa = S->fac_a, fb = S->fac_b;
    double v3[3] = {0.0, 0.0, 0.0};
    if (i < d.natms) {
        double4 v = xd[i];
        const double m = mass_of(C, d.type[i]);
        const double* f = d.f + (size_t)i * 3;
        v.x = dadd(dmul(dmul(v.x, fa), fb), ddiv(dmul(f[0], C.dt2), m));
        v.y = dadd(dmul(dmul(v.y, fa), fb), ddiv(dmul(f[1], C.dt2), m));
        v.z = dadd(dmul(dmul(v.z, fa), fb), ddiv(dmul(f[2], C.dt2), m));
        xd[i] = v;
        double4 p = d.pos[i];
        v3[0] = dmul(v.x, C.dt);
        v3[1] = dmul(v.y, C.dt);
        v3[2] = dmul(v.z, C.dt);
        xu[i] = make_double4(dadd(p.x, v3[0]), dadd(p.y, v3[1]), dadd(p.z, v3[2]), 0.0);
    }
    double tot[3];
    if (last_block_sum<3>(v3, part, &S->count[0], C.nblocks_own, tot) && threadIdx.x == 0) {
        for (int k = 0; k < 3; k++) S->ave[k] = dmul(tot[k], C.inv_n);
        S->fac_a = 1.0;
        S->fac_b = 1.0;
    }
}

// the mean removed from owned atoms and ghosts (a ghost is its root's centred
// position moved along its chain), the skin test of Atoms::update_0 against
// x_0, and force_calc's zeroing of f and rho.  The last block sets the while
// node's condition: go on unless a rebuild is due or the run is over.
__global__ void __launch_bounds__(kMdBlock) k_md_center(Dev d, NhConst C, NhState* S,
                                                        const double4* __restrict__ xu,
                                                        cudaGraphConditionalHandle handle, int set_cond)
{
    __shared__ bool last;
    if (S->done) {
        if (set_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(handle, 0u);
        return;
    }
    const int i = blockIdx.x * kMdBlock + threadIdx.x;
    const double a0 = S->ave[0], a1 = S->ave[1], a2 = S->ave[2];
    if (i < d.natms) {
        double4 u = xu[i];
        double4 p = make_double4(dsub(u.x, a0), dsub(u.y, a1), dsub(u.z, a2), 0.0);
        d.pos[i] = p;
        double4 q = d.pos0[i];
        double dx0 = dsub(p.x, q.x), dx1 = dsub(p.y, q.y), dx2 = dsub(p.z, q.z);
        double sq = dadd(dadd(dmul(dx0, dx0), dmul(dx1, dx1)), dmul(dx2, dx2));
        if (sq > C.sq_skin) atomicOr(&S->rebuild, 1);
        double* f = d.f + (size_t)i * 3;
        f[0] = 0.0;
        f[1] = 0.0;
        f[2] = 0.0;
        d.rho[i] = 0.0;
    } else if (i < d.natms + d.nph) {
        int r = d.root[i];
        double4 u = xu[r];
        double4 p = make_double4(dsub(u.x, a0), dsub(u.y, a1), dsub(u.z, a2), 0.0);
        d.pos[i] = ghost_image(d, d.gchain[i], p);
    }
    if (!set_cond) return;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&S->count[1], 1u) == (unsigned)(C.nblocks_all - 1);
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        S->count[1] = 0u;
        cudaGraphSetConditional(handle, atomicAdd(&S->rebuild, 0) ? 0u : 1u);
    }
}

// update_x_d(dt/2) with its kinetic tensor (md_nh.cpp:903-961); the last block
// finishes the step: update_NH_T(dt/2), and, unless the run is over, the next
// step's opening update_NH_T(dt/2)
__global__ void __launch_bounds__(kMdBlock) k_md_kick2(Dev d, NhConst C, NhState* S, double4* __restrict__ xd,
                                                       double* __restrict__ part)
{
    const int i = blockIdx.x * kMdBlock + threadIdx.x;
    double t[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < d.natms) {
        double4 v = xd[i];
        const double m = mass_of(C, d.type[i]);
        const double* f = d.f + (size_t)i * 3;
        v.x = dadd(v.x, ddiv(dmul(f[0], C.dt2), m));
        v.y = dadd(v.y, ddiv(dmul(f[1], C.dt2), m));
        v.z = dadd(v.z, ddiv(dmul(f[2], C.dt2), m));
        xd[i] = v;
        t[0] = dmul(dmul(m, v.x), v.x);
        t[1] = dmul(dmul(m, v.y), v.y);
        t[2] = dmul(dmul(m, v.z), v.z);
        t[3] = dmul(dmul(m, v.y), v.z);
        t[4] = dmul(dmul(m, v.x), v.z);
        t[5] = dmul(dmul(m, v.x), v.y);
    }
    double tot[6];
    if (last_block_sum<6>(t, part, &S->count[2], C.nblocks_own, tot) && threadIdx.x == 0) {
        for (int k = 0; k < 6; k++) S->ke_curr[k] = tot[k];
        S->ke_cur = dadd(dadd(tot[0], tot[1]), tot[2]);
        S->t_cur = ddiv(S->ke_cur, dmul(C.boltz, (double)C.no_dof));
        S->fac_a = nh_chain(S, C, C.dt2);
        S->step += 1;
        if (S->step < C.nsteps) {
            S->fac_b = nh_chain(S, C, C.dt2);
        } else {
            S->fac_b = 1.0;
            S->done = 1;
        }
    }
}

// the last step's pending rescale
__global__ void k_md_finish(Dev d, NhState* S, double4* __restrict__ xd)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.natms) return;
    const double fa = S->fac_a;
    double4 v = xd[i];
    xd[i] = make_double4(dmul(v.x, fa), dmul(v.y, fa), dmul(v.z, fa), 0.0);
}

// Random (rand_engine.cpp:35-74): Park-Miller by Schrage's factorisation and
// the polar Gaussian caching its second value; host side, run once per create_vel
struct Rng {
    int seed, cached;
    double reserved;
    double uniform()
    {
        int first = seed / 127773, second = seed % 127773;
        int rnd = 16807 * second - 2836 * first;
        seed = rnd > 0 ? rnd : rnd + 2147483647;
        return seed * 1.0 / 2147483647;
    }
    double gaussian()
    {
        if (!cached) {
            double u = 0.0, v = 0.0, s = 1.0;
            while (s >= 1.0) {
                u = 2.0 * uniform() - 1.0;
                v = 2.0 * uniform() - 1.0;
                s = u * u + v * v;
            }
            double q = std::sqrt(-2.0 * std::log(s) / s);
            cached = 1;
            reserved = v * q;
            return u * q;
        }
        cached = 0;
        return reserved;
    }
};

struct Buffers {
    double4* xd = nullptr;
    double4* xu = nullptr;
    double* part = nullptr;
    NhState* S = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~Buffers()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        cudaFree(xd);
        cudaFree(xu);
        cudaFree(part);
        cudaFree(S);
    }
};

int cuda_fail(cudaError_t e, const char* what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return internal_fail(MG_ERR_CUDA, m.c_str());
}

#define MCU(call)                                          \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)
#define MCHK(call)            \
    do {                              \
        int r_ = (call);              \
        if (r_ != MG_OK) return r_;   \
    } while (0)

// the loop body: force passes, second half kick and chain, the next step's
// first half kick, drift and centring (which decides the loop condition)
int enqueue_body(mg_system* s, const NhConst& C, Buffers& b, cudaGraphConditionalHandle h)
{
    cudaStream_t st = system_stream(s);
    const Dev& d = system_dev(s);
    int rows = 0;
    MCHK(system_enqueue_force(s, 0, 0, &rows));  // f and rho were zeroed by k_md_center
    k_md_kick2<<<C.nblocks_own, kMdBlock, 0, st>>>(d, C, b.S, b.xd, b.part);
    k_md_kick_drift<<<C.nblocks_own, kMdBlock, 0, st>>>(d, C, b.S, b.xd, b.xu, b.part);
    k_md_center<<<C.nblocks_all, kMdBlock, 0, st>>>(d, C, b.S, b.xu, h, 1);
    MCU(cudaGetLastError());
    return MG_OK;
}

int capture_loop(mg_system* s, const NhConst& C, Buffers& b)
{
    if (b.exec) cudaGraphExecDestroy(b.exec);
    if (b.graph) cudaGraphDestroy(b.graph);
    b.exec = nullptr;
    b.graph = nullptr;
    cudaStream_t st = system_stream(s);
    MCU(cudaGraphCreate(&b.graph, 0));
    cudaGraphConditionalHandle h;
    MCU(cudaGraphConditionalHandleCreate(&h, b.graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    MCU(cudaGraphAddNode(&node, b.graph, nullptr, 0, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    MCU(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    int rc = enqueue_body(s, C, b, h);
    cudaGraph_t out = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &out);
    if (rc != MG_OK) return rc;
    MCU(e);
    MCU(cudaGraphInstantiate(&b.exec, b.graph, 0));
    return MG_OK;
}

}  // namespace

}  // namespace mg

using namespace mg;

extern "C" int mg_md_nh(mg_system* s, double t_tar, double t_period, int eta_iteration, int eta_chains, double dt,
                        double boltz, int seed, const double* xd_in, int nsteps, double* xd_out, double* thermo,
                        int* rebuilds_out)
{
    MG_NVTX("mg_md_nh");
    MCHK(system_check_ready(s));
    int style = -1, nt = 0, x_dim = 0, form = 0;
    system_shape(s, &style, &nt, &x_dim, &form, nullptr);
    if (style != STYLE_EAM && style != STYLE_FS)
        return internal_fail(MG_ERR_UNSUPPORTED, "md nh drives the MD-mode (EAM / FS) force fields");
    if (!(t_tar > 0.0) || !(t_period > 0.0) || !(dt > 0.0) || !(boltz > 0.0) || nsteps < 0)
        return internal_fail(MG_ERR_ARG, "temperature, period, time step and boltzmann must be > 0, steps >= 0");
    if (eta_iteration < 1 || eta_chains < 3 || eta_chains > kMaxEta)
        return internal_fail(MG_ERR_ARG, "eta_iteration >= 1 and 3 <= eta_chains <= 16");
    if (seed <= 0 && !xd_in) return internal_fail(MG_ERR_ARG, "initial velocities or a create_vel seed are required");
    const int natms = system_natms(s);
    if (natms < 2) return internal_fail(MG_ERR_ARG, "md nh needs at least two atoms (3N - 3 degrees of freedom)");
    Dev& d0 = system_dev(s);
    std::vector<int> type(natms);
    cudaStream_t st = system_stream(s);
    MCU(cudaMemcpyAsync(type.data(), d0.type, natms * sizeof(int), cudaMemcpyDeviceToHost, st));
    MCU(cudaStreamSynchronize(st));
    double mass[kMaxTypes] = {0, 0, 0, 0};
    system_masses(s, mass);
    for (int t = 0; t < nt; t++)
        if (!(mass[t] > 0.0)) return internal_fail(MG_ERR_STATE, "every species needs a positive mass");

    // init: velocities (create_vel or init_vel, md_nh.cpp:1211-1341), serially on the host
    const int no_dof = natms * 3 - 3;
    std::vector<double> v((size_t)natms * 3);
    if (seed > 0) {
        Rng r{seed, 0, 0.0};
        for (int i = 0; i < natms; i++)
            for (int k = 0; k < 3; k++) v[3 * i + k] = r.gaussian() / (std::sqrt(mass[type[i]]));
    } else {
        bool dev = false;
        cudaPointerAttributes pa;
        if (cudaPointerGetAttributes(&pa, xd_in) == cudaSuccess && pa.type == cudaMemoryTypeDevice) dev = true;
        cudaGetLastError();
        MCU(cudaMemcpy(v.data(), xd_in, v.size() * sizeof(double), dev ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
    }
    NhState S;
    memset(&S, 0, sizeof(S));
    {
        double t6[6] = {0, 0, 0, 0, 0, 0};
        for (int i = 0; i < natms; i++) {
            double m = mass[type[i]];
            const double* x = &v[3 * i];
            t6[0] += m * x[0] * x[0];
            t6[1] += m * x[1] * x[1];
            t6[2] += m * x[2] * x[2];
            t6[3] += m * x[1] * x[2];
            t6[4] += m * x[0] * x[2];
            t6[5] += m * x[0] * x[1];
        }
        for (int k = 0; k < 6; k++) S.ke_curr[k] = t6[k];
        S.ke_cur = S.ke_curr[0] + S.ke_curr[1] + S.ke_curr[2];
        S.t_cur = S.ke_cur / (boltz * no_dof);
        if (seed <= 0 && S.ke_cur == 0)
            return internal_fail(MG_ERR_ARG, "initial velocities are zero: give velocities or a create_vel seed");
        double ke_des = (boltz * no_dof) * t_tar;
        double factor = std::sqrt(ke_des / S.ke_cur);
        double facsq = seed > 0 ? ke_des / S.ke_cur : factor * factor;
        for (double& x : v) x *= factor;
        for (int k = 0; k < 6; k++) S.ke_curr[k] *= facsq;
        S.ke_cur *= facsq;
        S.t_cur *= facsq;
    }
    NhConst C;
    memset(&C, 0, sizeof(C));
    for (int t = 0; t < kMaxTypes; t++) C.mass[t] = mass[t];
    C.dt = dt;
    C.dt2 = 0.5 * dt;
    C.boltz = boltz;
    C.t_tar = t_tar;
    C.t_freq = 1.0 / t_period;
    C.ke_tar = t_tar * boltz * no_dof;
    C.sq_skin = system_skin(s) * system_skin(s);
    C.inv_n = 1.0 / natms;
    C.no_dof = no_dof;
    C.no_it = eta_iteration;
    C.no_ch = eta_chains;
    C.nsteps = nsteps;
    C.nblocks_own = div_up(natms, kMdBlock);
    for (int i = 0; i < eta_chains; i++) S.eta_m[i] = boltz * t_tar / (C.t_freq * C.t_freq);
    S.eta_m[0] *= no_dof;
    for (int i = 1; i < eta_chains; i++)
        S.eta_dd[i] = (S.eta_m[i - 1] * S.eta_d[i - 1] * S.eta_d[i - 1] - boltz * t_tar) / S.eta_m[i];
    S.fac_a = S.fac_b = 1.0;
    S.done = nsteps == 0;

    Buffers b;
    MCU(cudaMalloc(&b.xd, (size_t)natms * sizeof(double4)));
    MCU(cudaMalloc(&b.xu, (size_t)natms * sizeof(double4)));
    MCU(cudaMalloc(&b.part, (size_t)C.nblocks_own * 8 * sizeof(double)));
    MCU(cudaMalloc(&b.S, sizeof(NhState)));
    {
        std::vector<double4> v4(natms);
        for (int i = 0; i < natms; i++) v4[i] = make_double4(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.0);
        MCU(cudaMemcpyAsync(b.xd, v4.data(), natms * sizeof(double4), cudaMemcpyHostToDevice, st));
        MCU(cudaMemcpyAsync(b.S, &S, sizeof(NhState), cudaMemcpyHostToDevice, st));
        MCU(cudaStreamSynchronize(st));
    }
    // init's force_calc, then x_0 = 0 (MD_NH::init never stores x_0, so the first
    // update_0 compares against the reader's unset x_0, taken as zero)
    int rows = 0;
    MCHK(system_enqueue_force(s, 1, 1, &rows));
    MCU(cudaMemsetAsync(system_dev(s).pos0, 0, (size_t)natms * sizeof(double4), st));
    int rebuilds = 0;
    if (nsteps > 0) {
        {
            const Dev& d = system_dev(s);
            C.nblocks_all = div_up((long long)d.natms + d.nph, kMdBlock);
            k_md_begin<<<1, 32, 0, st>>>(b.S, C);
            k_md_kick_drift<<<C.nblocks_own, kMdBlock, 0, st>>>(d, C, b.S, b.xd, b.xu, b.part);
            k_md_center<<<C.nblocks_all, kMdBlock, 0, st>>>(d, C, b.S, b.xu, cudaGraphConditionalHandle{}, 0);
            MCU(cudaGetLastError());
        }
        bool need_capture = true;
        for (;;) {
            int fl[2];  // rebuild, done
            MCU(cudaMemcpyAsync(fl, &b.S->rebuild, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
            MCU(cudaStreamSynchronize(st));
            if (fl[1]) break;
            if (fl[0]) {
                MCHK(system_rebuild(s));
                rebuilds++;
                const Dev& d = system_dev(s);
                MCU(cudaMemsetAsync(d.f, 0, (size_t)natms * 3 * sizeof(double), st));
                MCU(cudaMemsetAsync(d.rho, 0, (size_t)natms * sizeof(double), st));
                MCU(cudaMemsetAsync(&b.S->rebuild, 0, sizeof(int), st));
                C.nblocks_all = div_up((long long)d.natms + d.nph, kMdBlock);
                need_capture = true;
            }
            if (need_capture) {
                MCHK(capture_loop(s, C, b));
                need_capture = false;
            }
            MCU(cudaGraphLaunch(b.exec, st));
        }
        k_md_finish<<<C.nblocks_own, kMdBlock, 0, st>>>(system_dev(s), b.S, b.xd);
        MCU(cudaGetLastError());
        // the thermo pass of the last step: force_calc(1) at the final positions
        MCHK(system_enqueue_force(s, 1, 1, &rows));
    }
    MCU(launch_reduce_partials(system_dev(s), rows, 7, system_red_out(s), st));
    double en[8] = {0};
    MCU(cudaMemcpyAsync(en, system_red_out(s), 7 * sizeof(double), cudaMemcpyDeviceToHost, st));
    MCU(cudaMemcpyAsync(&S, b.S, sizeof(NhState), cudaMemcpyDeviceToHost, st));
    std::vector<double4> v4(natms);
    MCU(cudaMemcpyAsync(v4.data(), b.xd, natms * sizeof(double4), cudaMemcpyDeviceToHost, st));
    MCU(cudaStreamSynchronize(st));
    if (xd_out)
        for (int i = 0; i < natms; i++) {
            xd_out[3 * i] = v4[i].x;
            xd_out[3 * i + 1] = v4[i].y;
            xd_out[3 * i + 2] = v4[i].z;
        }
    if (thermo) {
        for (int k = 0; k < 7; k++) thermo[k] = en[k];
        thermo[7] = S.ke_cur;
        thermo[8] = S.t_cur;
        for (int i = 0; i < eta_chains; i++) thermo[9 + i] = S.eta_d[i];
    }
    if (rebuilds_out) *rebuilds_out = rebuilds;
    return MG_OK;
}
