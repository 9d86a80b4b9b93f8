// Host side of the mapp_b200 C ABI: potential readers, spline construction,
// cut-offs, ghost / neighbour-list rebuild orchestration and the ForceField
// entry points.  Numbers that decide list membership (B, cut_ph_s, cut_sk_sq,
// table coefficients) are computed here in plain IEEE double in the
// reference's operation order, so they equal the reference's bit for bit.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mapp_b200.h"
#include "mg_internal.h"
#include "mg_reduce.cuh"

using namespace mg;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CU(call)                                                                                        \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return fail(MG_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                           __FILE__, __LINE__);                                         \
    } while (0)

#define CHK(call)             \
    do {                      \
        int r_ = (call);      \
        if (r_) return r_;    \
    } while (0)

template <class T>
int dalloc(T** p, size_t n)
{
    if (*p) cudaFree(*p);
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(MG_ERR_CAPACITY, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
    }
    return MG_OK;
}

// grow keeping the first `keep` elements
template <class T>
int dgrow(T** p, size_t n, size_t keep, cudaStream_t st)
{
    T* q = nullptr;
    cudaError_t e = cudaMalloc((void**)&q, (n ? n : 1) * sizeof(T));
    if (e != cudaSuccess) return fail(MG_ERR_CAPACITY, "cudaMalloc of %zu bytes failed", n * sizeof(T));
    if (*p && keep) {
        e = cudaMemcpyAsync(q, *p, keep * sizeof(T), cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return fail(MG_ERR_CUDA, "grow copy: %s", cudaGetErrorString(e));
        cudaStreamSynchronize(st);
    }
    if (*p) cudaFree(*p);
    *p = q;
    return MG_OK;
}

// where a caller's pointer lives: 0 pageable host memory (a device-to-host
// copy into it blocks the host until the stream has drained), 1 page-locked
// host memory, 2 device (or managed) memory
int ptr_kind(const void* p)
{
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return 2;
    return a.type == cudaMemoryTypeHost ? 1 : 0;
}

bool is_device_ptr(const void* p) { return ptr_kind(p) == 2; }

// ---- splines: interpolate (ff_eam.cpp:1323-1352) and interpolate_m
// (ff_dmd_I.cpp:1794-1836), on rows of `w` doubles ---------------------------
void spline_cubic(int n, double delta, double* s, int w)
{
    auto S = [&](int i, int k) -> double& { return s[(size_t)i * w + k]; };
    S(0, 1) = S(1, 0) - S(0, 0);
    S(1, 1) = 0.5 * (S(2, 0) - S(0, 0));
    S(n - 2, 1) = 0.5 * (S(n - 1, 0) - S(n - 3, 0));
    S(n - 1, 1) = S(n - 1, 0) - S(n - 2, 0);
    for (int i = 2; i < n - 2; i++) S(i, 1) = ((S(i - 2, 0) - S(i + 2, 0)) + 8.0 * (S(i + 1, 0) - S(i - 1, 0))) / 12.0;
    for (int i = 0; i < n - 1; i++) {
        S(i, 2) = 3.0 * (S(i + 1, 0) - S(i, 0)) - 2.0 * S(i, 1) - S(i + 1, 1);
        S(i, 3) = S(i, 1) + S(i + 1, 1) - 2.0 * (S(i + 1, 0) - S(i, 0));
    }
    S(n - 1, 2) = 0.0;
    S(n - 1, 3) = 0.0;
}

void spline7(int n, double delta, double* s, int w)
{
    spline_cubic(n, delta, s, w);
    for (int i = 0; i < n; i++) {
        s[(size_t)i * w + 4] = s[(size_t)i * w + 1] / delta;
        s[(size_t)i * w + 5] = 2.0 * s[(size_t)i * w + 2] / delta;
        s[(size_t)i * w + 6] = 3.0 * s[(size_t)i * w + 3] / delta;
    }
}

void spline9(int n, double delta, double* s, int w)
{
    spline_cubic(n, delta, s, w);
    auto S = [&](int i, int k) -> double& { return s[(size_t)i * w + k]; };
    for (int i = 0; i < n - 1; i++) S(i, 4) = (S(i + 1, 2) - S(i, 2)) / 6.0 - 0.5 * S(i, 3);
    S(n - 1, 4) = 0.0;
    for (int i = 0; i < n; i++) {
        S(i, 5) = S(i, 1) / delta;
        S(i, 6) = 2.0 * S(i, 2) / delta;
        S(i, 7) = 3.0 * S(i, 3) / delta;
        S(i, 8) = 4.0 * S(i, 4) / delta;
    }
}

// Gauss-Hermite nodes and weights for weight exp(-x^2), by Newton iteration on
// the orthonormal Hermite recurrence (Golub-Welsch initial guesses as in the
// classical "gauher" routine), long double, ascending order.
void gauss_hermite(int n, double* x_out, double* w_out)
{
    const long double pim4 = 0.7511255444649425L;
    long double x[kMaxQuad], w[kMaxQuad], z = 0, z1, p1, p2, p3, pp = 0;
    int m = (n + 1) / 2;
    for (int i = 0; i < m; i++) {
        if (i == 0) z = sqrtl((long double)(2 * n + 1)) - 1.85575L * powl((long double)(2 * n + 1), -0.16667L);
        else if (i == 1) z -= 1.14L * powl((long double)n, 0.426L) / z;
        else if (i == 2) z = 1.86L * z - 0.86L * x[0];
        else if (i == 3) z = 1.91L * z - 0.91L * x[1];
        else z = 2.0L * z - x[i - 2];
        for (int it = 0; it < 100; it++) {
            p1 = pim4;
            p2 = 0.0L;
            for (int j = 0; j < n; j++) {
                p3 = p2;
                p2 = p1;
                p1 = z * sqrtl(2.0L / (j + 1)) * p2 - sqrtl((long double)j / (j + 1)) * p3;
            }
            pp = sqrtl(2.0L * n) * p2;
            z1 = z;
            z = z1 - p1 / pp;
            if (fabsl(z - z1) <= 1e-19L * fabsl(z)) break;
        }
        x[i] = z;
        x[n - 1 - i] = -z;
        w[i] = 2.0L / (pp * pp);
        w[n - 1 - i] = w[i];
    }
    if (n % 2 == 1) x[m - 1] = 0.0L;
    for (int i = 0; i < n; i++) {
        x_out[i] = (double)x[n - 1 - i];
        w_out[i] = (double)w[n - 1 - i];
    }
}

// whitespace tokens of a line up to a '#' (MAPP::parse_line, MAPP.cpp:468-521)
std::vector<std::string> tokens(const std::string& line)
{
    std::vector<std::string> out;
    std::string s = line.substr(0, line.find('#'));
    std::istringstream is(s);
    std::string t;
    while (is >> t) out.push_back(t);
    return out;
}

}  // namespace

int mg::internal_fail(int code, const char* msg) { return fail(code, "%s", msg); }
const char* mg::internal_last_error() { return g_err.c_str(); }

struct mg_system {
    int style = 0, form = MG_FORM_FP64, device = 0, nt = 0, x_dim = 3, dmd = 0;
    std::vector<std::string> names;
    std::vector<double> masses;
    bool types_set = false, box_set = false, atoms_set = false, coef_set = false, initialized = false;
    double H[3][3] = {{0}}, B[3][3] = {{0}}, skin = 0.5;
    int natms = 0;
    // tables (host, built by coef)
    int nr = 0, nrho = 0;
    double dr = 0, drho = 0;
    std::vector<double> rhoT, phiT, FT;  // device layouts
    int Fw = 7;
    // FS analytic
    std::vector<double> fsA, fst1, fst2, fs_cut_rho, fs_cut_phi, fsk1, fsk2, fsk3;
    std::vector<int> fs_chk;
    // DMD
    double rsq_crd = 0, alpha_min = 0, alpha_max = 0, T = 0;
    int nq = 0;
    double xi[kMaxQuad], w0[kMaxQuad];
    // derived box/bins
    int comm_need[3] = {1, 1, 1};
    double tot_cut_ph = 0;
    // device
    Dev d;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    // a second stream of the library's own for the copy of a final per-site
    // array (forces, g) to the caller while the main stream reduces the
    // totals; ev_fork / ev_join order it after the producing kernels and
    // before the call returns
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool side_pending = false;
    // a copy into pageable or device memory is not moved to the side stream:
    // it is queued on the main stream by join_side
    struct {
        void* dst;
        const void* src;
        size_t bytes;
    } deferred{nullptr, nullptr, 0};
    size_t cap = 0;          // per-atom capacity (owned + ghost)
    int cap_bins = 0;
    void* scan_tmp = nullptr;
    size_t scan_tmp_bytes = 0;
    double* stage = nullptr;  // device staging for host arrays
    size_t stage_cap = 0;
    size_t act_cap = 0;   // capacity of the active-pair sublist (entries)
    size_t nact_cap = 0;  // and of its per-site counts and offsets (sites + 1)
    // one device block of 8 doubles (the reduced totals) followed by the 8
    // status words, d.status pointing into it, so that one copy reads both
    double* red_out = nullptr;
    // Page-locked host block for the small results the entry points read back.
    // A copy into pageable memory blocks the host until the stream has
    // drained, so a pageable read of a total before the force copy would leave
    // the GPU idle for a host round trip; into this block every copy is
    // asynchronous and the one synchronisation at the end of a call covers them
    // all.  Its first two members mirror the device block above.
    struct HostPin {
        double tot[8];
        int status[8];
        GhostCtl gc;
        int count;
    };
    HostPin* hp = nullptr;
    double* d_rhoT = nullptr;
    double* d_phiT = nullptr;
    double* d_FT = nullptr;
    float* d_pkT = nullptr;
    double* d_pk64 = nullptr;
    float* d_pkS = nullptr;
    int* cursor = nullptr;
    int crd_built = 0;
    int npair_blocks = 2;
    long long npairs = 0;
    long long pair_cap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t evk[4] = {nullptr, nullptr, nullptr, nullptr};
    // device timing (mg_set_timing): 0 none, 1 (default) the whole call of
    // each entry point, 2 also the kernels of the DMD force call; every event
    // costs the call about 3 us at 32000 sites.  A phase time below zero, and
    // t_k_valid false, mean the last call took none
    int timing = 1;
    bool t_k_valid = false;
    // learned form
    MlpState mlp{};
    bool mlp_ready = false;
    float* mlp_loss = nullptr;
    int mlp_loss_n = 0;
    unsigned long long mlp_calls = 0;
    bool skin_pending = false;  // update_x's skin test not yet read (status[7])
    // the value update_x's skin test writes to status[7] when some site moved
    // more than the skin: a new one per update_x, so the word needs no reset
    int skin_gen = 0;
    GhostCtl* gctl = nullptr;  // device control of the ghost passes (two, ping-pong)
    unsigned* gtiles = nullptr;  // look-back words of the ghost passes (two halves)
    int gtiles_cap = 0;
    double t_list = 0, t_force = 0, t_energy = 0, t_cd = 0, t_g = 0;
    double t_k[3] = {0, 0, 0};  // DMD force: pass 1, embedding, pass 2
    long long partial_rows = 0;
    bool tables_uploaded = false;  // device tables match the last ff_coef
    // the last force_calc ran in the precision form, which stores no per-pair
    // values; c_d_calc and calc_g have them written first (ensure_pair_values)
    bool prf_stale = false;
    size_t owned_cap = 0, nbr_cap = 0, crdl_cap = 0;  // element capacities of the per-owned-site, ELL and crd buffers
};

namespace {

int rebuild(mg_system* s);

// the argument check of every entry point, without settling a pending skin
// test (update_x, update_c and force_calc take care of it themselves)
int check_sys_nores(mg_system* s)
{
    if (!s) return fail(MG_ERR_ARG, "null mg_system");
    if (cudaSetDevice(s->device) != cudaSuccess) return fail(MG_ERR_CUDA, "cudaSetDevice(%d) failed", s->device);
    s->deferred.dst = nullptr;  // (a failed call's copy into pageable memory is dropped)
    if (s->side_pending) {
        // a call that failed between its side copy and the join: nothing
        // queued from here on may overwrite the array that copy reads
        s->side_pending = false;
        if (cudaStreamWaitEvent(s->st, s->ev_join, 0) != cudaSuccess) return fail(MG_ERR_CUDA, "stream join failed");
    }
    return MG_OK;
}

// update_x called without asking whether it rebuilt leaves its skin test on
// the device (status[7]); the next entry point that reads positions, ghosts or
// lists settles it first: the flag is read and, when some site moved more than
// the skin since the last build, the list is rebuilt, as update_0 would have
int resolve_skin(mg_system* s)
{
    if (!s->skin_pending) return MG_OK;
    s->skin_pending = false;
    CU(cudaMemcpyAsync(&s->hp->status[7], s->d.status + 7, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    if (s->hp->status[7] == s->skin_gen) {
        CU(launch_x2s(s->d, s->st));
        CHK(rebuild(s));
    }
    return MG_OK;
}

int check_sys(mg_system* s)
{
    CHK(check_sys_nores(s));
    return resolve_skin(s);
}

int stage_in(mg_system* s, const void* src, size_t bytes, const void** dev_out)
{
    if (is_device_ptr(src)) {
        *dev_out = src;
        return MG_OK;
    }
    if (bytes > s->stage_cap) {
        CHK(dalloc((char**)&s->stage, bytes));
        s->stage_cap = bytes;
    }
    CU(cudaMemcpyAsync(s->stage, src, bytes, cudaMemcpyHostToDevice, s->st));
    *dev_out = s->stage;
    return MG_OK;
}

int copy_out(mg_system* s, void* dst, const void* dev_src, size_t bytes)
{
    if (!dst || !bytes) return MG_OK;
    cudaMemcpyKind k = is_device_ptr(dst) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CU(cudaMemcpyAsync(dst, dev_src, bytes, k, s->st));
    return MG_OK;
}

// copy_out of an array that is final at this point of the main stream: into
// page-locked host memory it runs on the side stream, so it overlaps what the
// main stream queues next (the reduction of the totals), and join_side makes
// the main stream wait for it.  Into pageable memory (a copy that blocks the
// host) or device memory (a copy of about a microsecond, nothing to hide) it
// runs on the main stream, from join_side.
int copy_out_side(mg_system* s, void* dst, const void* dev_src, size_t bytes)
{
    if (!dst || !bytes) return MG_OK;
    const int kind = ptr_kind(dst);
    if (kind != 1) {
        s->deferred.dst = dst;
        s->deferred.src = dev_src;
        s->deferred.bytes = bytes;
        return MG_OK;
    }
    const cudaMemcpyKind k = cudaMemcpyDeviceToHost;
    CU(cudaEventRecord(s->ev_fork, s->st));
    CU(cudaStreamWaitEvent(s->side, s->ev_fork, 0));
    CU(cudaMemcpyAsync(dst, dev_src, bytes, k, s->side));
    CU(cudaEventRecord(s->ev_join, s->side));
    s->side_pending = true;
    return MG_OK;
}

int join_side(mg_system* s)
{
    if (s->deferred.dst) {
        void* dst = s->deferred.dst;
        s->deferred.dst = nullptr;
        CHK(copy_out(s, dst, s->deferred.src, s->deferred.bytes));
    }
    if (!s->side_pending) return MG_OK;
    s->side_pending = false;
    CU(cudaStreamWaitEvent(s->st, s->ev_join, 0));
    return MG_OK;
}

int ensure_partials(mg_system* s, long long rows)
{
    if (rows <= s->partial_rows) return MG_OK;
    long long n = rows + rows / 4 + 64;
    CHK(dalloc(&s->d.partial, (size_t)n * 8));
    s->partial_rows = n;
    return MG_OK;
}

// per-atom arrays (owned + ghost), keeping rebuild inputs
int ensure_atoms(mg_system* s, size_t need, size_t keep)
{
    if (need <= s->cap) return MG_OK;
    size_t cap = need + need / 2 + 1024;
    int nt = s->nt;
    Dev& d = s->d;
    CHK(dgrow(&d.sfr, cap, keep, s->st));
    CHK(dgrow(&d.alpha, cap * nt, keep * nt, s->st));
    if (s->dmd) CHK(dgrow(&d.c, cap * nt, keep * nt, s->st));
    else CHK(dgrow(&d.type, cap, keep, s->st));
    CHK(dgrow(&d.root, cap, keep, s->st));
    CHK(dgrow(&d.gchain, cap, keep, s->st));
    CHK(dgrow(&d.pos, cap, keep, s->st));
    CHK(dalloc(&d.bin, cap));
    CHK(dalloc(&d.cell_pos, cap));
    CHK(dalloc(&d.rho, cap));
    CHK(dalloc(&d.E, cap * nt));
    CHK(dalloc(&d.dE, cap * nt));
    CHK(dalloc(&d.ddE, cap * nt));
    CHK(dalloc(&d.n, cap * nt));
    CHK(dalloc(&d.s, cap * nt));
    CHK(dalloc(&d.t, cap * nt));
    CHK(dalloc(&d.v, cap * nt));
    CHK(dalloc(&d.crd, cap));
    if (s->dmd) {
        CHK(dalloc(&d.srec, cap * kSiteRec));
        CHK(dalloc(&d.dE32, cap * nt));
        CHK(dalloc(&d.facc, cap * 8));
    }
    size_t tb = scan_temp_bytes((int)cap);
    if (tb > s->scan_tmp_bytes) {
        CHK(dalloc((char**)&s->scan_tmp, tb));
        s->scan_tmp_bytes = tb;
    }
    s->cap = cap;
    return MG_OK;
}

// ELL list storage; EAM / FS keep their two per-pair derivatives in ELL slots
int ensure_pairs(mg_system* s, int maxnb)
{
    Dev& d = s->d;
    size_t np = (size_t)s->natms * maxnb;
    if (np > s->nbr_cap) {
        size_t cap = np + np / 4 + 1024;
        CHK(dalloc(&d.nbr, cap));
        if (!s->dmd) CHK(dalloc(&d.pr, cap * s->npair_blocks));
        s->nbr_cap = cap;
    }
    d.maxnb = maxnb;
    if (!s->dmd) d.maxp = (long long)np;
    return MG_OK;
}

// compact pair list and (DMD) per-pair scratch for npairs pairs
int ensure_compact(mg_system* s, long long npairs)
{
    Dev& d = s->d;
    if (npairs <= s->pair_cap) return MG_OK;
    long long cap = npairs + npairs / 5 + 1024;
    CHK(dalloc(&d.pair_i, (size_t)cap));
    CHK(dalloc(&d.pair_j, (size_t)cap));
    if (s->dmd) {
        CHK(dalloc(&d.pr, (size_t)cap * s->npair_blocks));
        CHK(dalloc(&d.prf, (size_t)cap * s->npair_blocks));
        d.maxp = cap;
        d.icut_cap = dmd32_icut_capacity(cap);
        CHK(dalloc(&d.icut, (size_t)d.icut_cap * 2));
        if (!d.icut_n) CHK(dalloc(&d.icut_n, (size_t)dmd32_icut_warps()));
    }
    s->pair_cap = cap;
    return MG_OK;
}

void fill_dev_scalars(mg_system* s)
{
    Dev& d = s->d;
    d.natms = s->natms;
    d.nt = s->nt;
    d.x_dim = s->x_dim;
    d.style = s->style;
    d.form = s->form;
    memcpy(d.H, s->H, sizeof(d.H));
    memcpy(d.B, s->B, sizeof(d.B));
}

// ForceField::init cut-offs (ff_eam.cpp:360-371, ff_fs.cpp:339-352,
// ff_dmd_I.cpp:672-682) and Atoms::set_ph (atoms.cpp:249-278); returns ph_cut.
void compute_cutoffs(mg_system* s)
{
    Dev& d = s->d;
    double skin = s->skin, ph_cut = 0.0;
    int nt = s->nt, ncomp = nt * (nt + 1) / 2;
    if (s->style == STYLE_EAM) {
        for (int i = 0; i < ncomp; i++) d.cut_sk_sq[i] = d.cut_sq + (skin) * (skin) + 2 * sqrt(d.cut_sq) * (skin);
        ph_cut = sqrt(d.cut_sq);
    } else if (s->style == STYLE_FS) {
        for (int i = 0; i < ncomp; i++)
            if (d.fs_chk[i]) {
                double a = d.fs_cut_phi[i] * d.fs_cut_phi[i], b = d.fs_cut_rho[i] * d.fs_cut_rho[i];
                d.fs_cut_sq[i] = a > b ? a : b;
                d.cut_sk_sq[i] = d.fs_cut_sq[i] + (skin) * (skin) + 2 * sqrt(d.fs_cut_sq[i]) * (skin);
                double c = sqrt(d.fs_cut_sq[i]);
                ph_cut = ph_cut > c ? ph_cut : c;
            } else {
                d.fs_cut_sq[i] = 0.0;
                d.cut_sk_sq[i] = 0.0;
            }
    } else {
        for (int i = 0; i < ncomp; i++)
            d.cut_sk_sq[i] = d.cut_sq_mod + (skin) * (skin) + 2.0 * sqrt(d.cut_sq_mod) * (skin);
        ph_cut = sqrt(d.cut_sq_mod);
    }
    s->tot_cut_ph = ph_cut + skin;
    for (int i = 0; i < 3; i++) {
        double tmp = 0.0;
        for (int j = i; j < 3; j++) tmp += s->B[j][i] * s->B[j][i];
        d.cut_ph_s[i] = s->tot_cut_ph * sqrt(tmp);
    }
    for (int i = 0; i < 3; i++) {
        d.s_ph_hi[i] = 1.0 - d.cut_ph_s[i];
        d.s_ph_lo[i] = 0.0 + d.cut_ph_s[i];
    }
    for (int i = 0; i < 3; i++) s->comm_need[i] = (int)(d.cut_ph_s[i] / (1.0 - 0.0)) + 1;
    // Neighbor::create_bin_list (neighbor.cpp:311-330)
    d.tot_bin = 1;
    for (int i = 0; i < 3; i++) {
        d.grid[i] = (int)((2.0 * d.cut_ph_s[i] + 1.0 - 0.0) / d.cut_ph_s[i]) + 1;
        d.tot_bin *= d.grid[i];
    }
    for (int i = 0; i < 3; i++) {
        int no = 1;
        for (int j = 0; j < i; j++) no *= d.grid[j];
        d.denom[i] = no;
    }
}

// Atoms::ph_setup (atoms.cpp:317-372), then binning, s2x and the half list.
// Expects d.sfr (owned, fractional) and root/gchain of owned atoms set.
int rebuild(mg_system* s)
{
    Dev& d = s->d;
    cudaStream_t st = s->st;
    CU(cudaEventRecord(s->ev0, st));
    int natms = s->natms, nph = 0;
    fill_dev_scalars(s);
    if (!s->gctl) CHK(dalloc(&s->gctl, 2));
    // The ghost passes run back to back on the device (bounds and counts in
    // GhostCtl, one launch per pass), and so do binning and the half list,
    // which read the ghost count from the device. One synchronisation reads
    // the ghost count, the list's overflow word and the pair count; ghosts that
    // did not fit the arrays make them grow and the build run again, a list
    // overflow makes the per-atom list capacity grow and the list run again.
    int np_h = 0;
    for (int attempt = 0;; attempt++) {
        const int cap = (int)s->cap, nt_tiles = ghost_tiles(cap);
        // the tile words of both halves, then the two tickets: one memset
        if (2 * nt_tiles + 2 > s->gtiles_cap) {
            CHK(dalloc(&s->gtiles, (size_t)2 * nt_tiles + 2));
            s->gtiles_cap = 2 * nt_tiles + 2;
        }
        int* gticket = reinterpret_cast<int*>(s->gtiles + 2 * nt_tiles);
        CU(cudaMemsetAsync(d.status, 0, 8 * sizeof(int), st));
        CU(cudaMemsetAsync(s->gtiles, 0, ((size_t)2 * nt_tiles + 2) * sizeof(unsigned), st));
        CU(launch_ghost_init(d, s->gctl, st));
        int cur = 0;
        for (int dim = 0; dim < 3; dim++)
            for (int dir = 0; dir < 2; dir++)
                for (int pass = 0; pass < s->comm_need[dim]; pass++) {
                    const int next_mode = pass + 1 < s->comm_need[dim] ? 0 : (dir == 0 ? 1 : 2);
                    CU(launch_ghost_pass(d, s->gctl + cur, s->gctl + (cur ^ 1), s->gtiles + cur * nt_tiles,
                                         s->gtiles + (cur ^ 1) * nt_tiles, gticket + cur, gticket + (cur ^ 1),
                                         cap, dim, dir, next_mode, st));
                    cur ^= 1;
                }
        const GhostCtl* gfin = s->gctl + cur;
        // bins
        if (d.tot_bin + 1 > s->cap_bins) {
            CHK(dalloc(&d.cell_count, 2 * ((size_t)d.tot_bin + 1)));
            CHK(dalloc(&d.cell_start, d.tot_bin + 1));
            s->cap_bins = d.tot_bin + 1;
            size_t tb = scan_temp_bytes(d.tot_bin + 1);
            if (tb > s->scan_tmp_bytes) {
                CHK(dalloc((char**)&s->scan_tmp, tb));
                s->scan_tmp_bytes = tb;
            }
        }
        // the fill cursors sit right after this build's counts (the allocation
        // holds two arrays of cap_bins), so one memset zeroes both
        s->cursor = d.cell_count + d.tot_bin + 1;
        CU(cudaMemsetAsync(d.cell_count, 0, 2 * ((size_t)d.tot_bin + 1) * sizeof(int), st));
        CU(launch_bin_and_s2x(d, gfin, cap, st));
        CU(launch_exclusive_scan(d.cell_count, d.cell_start, d.tot_bin + 1, s->scan_tmp, s->scan_tmp_bytes, st));
        CU(launch_cell_fill(d, s->cursor, gfin, cap, st));
        // half list, then the scan of the per-atom counts
        bool regrow_ghosts = false;
        for (int attempt_nb = 0;; attempt_nb++) {
            const GhostCtl& gc = s->hp->gc;
            const int* st_h = s->hp->status;
            // (the list kernel zeroes nnb[natms], the scan's last element)
            if (attempt_nb) CU(cudaMemsetAsync(d.status, 0, 2 * sizeof(int), st));
            CU(launch_neigh(d, st));
            CU(launch_exclusive_scan(d.nnb, d.poff, natms + 1, s->scan_tmp, s->scan_tmp_bytes, st));
            CU(cudaMemcpyAsync(&s->hp->gc, gfin, sizeof(GhostCtl), cudaMemcpyDeviceToHost, st));
            CU(cudaMemcpyAsync(s->hp->status, d.status, 8 * sizeof(int), cudaMemcpyDeviceToHost, st));
            CU(cudaMemcpyAsync(&s->hp->count, d.poff + natms, sizeof(int), cudaMemcpyDeviceToHost, st));
            CU(cudaStreamSynchronize(st));
            np_h = s->hp->count;
            if (st_h[4])
                return fail(MG_ERR_CAPACITY, "ghost image chain deeper than %d swaps (box too small for the cut-off)",
                            kMaxChain);
            if (st_h[6]) return fail(MG_ERR_TIMEOUT, "ghost build: a compaction wait ran out");
            if (gc.over > 0) {
                if (attempt == 4) return fail(MG_ERR_CAPACITY, "ghost arrays could not be grown to fit");
                // the owned atoms are kept; every ghost is rebuilt
                CHK(ensure_atoms(s, (size_t)natms + (size_t)gc.nph + (size_t)gc.over + s->cap / 2, natms));
                regrow_ghosts = true;
                break;
            }
            nph = gc.nph;
            if (!st_h[0]) break;
            if (attempt_nb == 3) return fail(MG_ERR_CAPACITY, "neighbour list capacity could not be met");
            CHK(ensure_pairs(s, st_h[1] + 16));
        }
        if (!regrow_ghosts) break;
    }
    d.nph = nph;
    d.nall = natms + nph;
    // compact CSR pair list (pairs sorted by i)
    CHK(ensure_compact(s, np_h));
    // partial rows: every launcher's grid is at most one block per 256 pairs (or
    // 4 * SMs for the persistent learned-form pass) plus per-atom grids
    CHK(ensure_partials(s, 2LL * div_up((long long)np_h, kFFBlock) + 2LL * div_up((long long)natms * 32, kFFBlock) +
                               div_up((long long)natms * s->nt, kFFBlock) + 4LL * num_sms() + 64));
    d.npairs = np_h;
    CU(launch_pairs_compact(d, st));
    CU(launch_store_x0(d, st));
    s->crd_built = 0;
    CU(cudaEventRecord(s->ev1, st));
    CU(cudaEventSynchronize(s->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    s->t_list = ms;
    return MG_OK;
}

// ---- potential readers -----------------------------------------------------

int read_all(const char* path, std::vector<std::string>& lines)
{
    std::ifstream in(path);
    if (!in) return fail(MG_ERR_FILE, "file %s not found", path);
    std::string ln;
    while (std::getline(in, ln)) lines.push_back(ln);
    return MG_OK;
}

// setfl / FS table files (ff_eam.cpp:674-879, 883-1108; ff_dmd_I.cpp:1300-1548):
// four lines (the 4th lists the file's elements), "Nrho drho Nr dr cut", one
// element header line, then the values.
int read_tables(mg_system* s, const char* path, bool fs_layout)
{
    std::vector<std::string> lines;
    CHK(read_all(path, lines));
    if (lines.size() < 6) return fail(MG_ERR_FORMAT, "eam potential file ended immaturely");
    std::vector<std::string> el = tokens(lines[3]);
    int nt = s->nt;
    if ((int)el.size() < 2 || (int)el.size() - 1 < nt) return fail(MG_ERR_FORMAT, "wrong format in eam potential file");
    int tot = (int)el.size() - 1;
    std::vector<int> fe(nt);
    for (int a = 0; a < nt; a++) {
        int k = 0;
        while (k < tot && el[k + 1] != s->names[a]) k++;
        if (k == tot) return fail(MG_ERR_FORMAT, "atom type not found in eam file");
        fe[a] = k;
    }
    std::vector<std::string> h = tokens(lines[4]);
    if (h.size() != 5) return fail(MG_ERR_FORMAT, "wrong format in eam potential file");
    int nrho = atoi(h[0].c_str()), nr = atoi(h[2].c_str());
    double drho = atof(h[1].c_str()), dr = atof(h[3].c_str());
    if (nr < 5 || nrho < 5) return fail(MG_ERR_FORMAT, "table sizes too small (nr=%d nrho=%d)", nr, nrho);
    std::vector<double> v;
    size_t need = fs_layout ? (size_t)tot * nrho + (size_t)tot * tot * nr + (size_t)tot * (tot + 1) / 2 * nr
                            : (size_t)tot * (nrho + nr) + (size_t)tot * (tot + 1) / 2 * nr;
    v.reserve(need);
    for (size_t li = 6; li < lines.size() && v.size() < need; li++)
        for (const std::string& t : tokens(lines[li])) v.push_back(strtod(t.c_str(), nullptr));
    if (v.size() < need) return fail(MG_ERR_FORMAT, "eam potential file ended immaturely");
    s->nr = nr;
    s->nrho = nrho;
    s->dr = dr;
    s->drho = drho;
    s->Fw = s->dmd ? 9 : 7;
    int ncomp = nt * (nt + 1) / 2;
    s->FT.assign((size_t)nt * (nrho + 1) * s->Fw, 0.0);
    s->rhoT.assign((size_t)nt * nt * nr * 8, 0.0);
    s->phiT.assign((size_t)ncomp * nr * 8, 0.0);
    // offsets of each file element's blocks
    size_t per_el = fs_layout ? (size_t)nrho + (size_t)tot * nr : (size_t)nrho + nr;
    size_t phi0 = per_el * tot;
    auto phi_off = [&](int e1, int e2) {  // e1 >= e2
        return phi0 + ((size_t)e1 * (e1 + 1) / 2 + e2) * nr;
    };
    for (int a = 0; a < nt; a++) {
        const double* Fsrc = v.data() + per_el * fe[a];
        double* Fd = s->FT.data() + (size_t)a * (nrho + 1) * s->Fw;
        for (int k = 0; k < nrho; k++) Fd[(size_t)k * s->Fw] = Fsrc[k];
        if (s->dmd) spline9(nrho, drho, Fd, s->Fw);
        else spline7(nrho, drho, Fd, s->Fw);
    }
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++) {
            // density slot b*nt+a: FS block [a][b]; setfl: the source element's
            // single density, aliased to every slot of that element
            const double* src = fs_layout ? v.data() + per_el * fe[a] + nrho + (size_t)fe[b] * nr
                                          : v.data() + per_el * fe[a] + nrho;
            double* dst = s->rhoT.data() + (size_t)(b * nt + a) * nr * 8;
            for (int k = 0; k < nr; k++) dst[(size_t)k * 8] = src[k];
            spline7(nr, dr, dst, 8);
        }
    for (int a = 0; a < nt; a++)
        for (int b = 0; b <= a; b++) {
            int e1 = fe[a] > fe[b] ? fe[a] : fe[b], e2 = fe[a] > fe[b] ? fe[b] : fe[a];
            const double* src = v.data() + phi_off(e1, e2);
            double* dst = s->phiT.data() + (size_t)comp_idx(a, b) * nr * 8;
            for (int k = 0; k < nr; k++) dst[(size_t)k * 8] = src[k];
            spline7(nr, dr, dst, 8);
        }
    return MG_OK;
}

// the 4-point Lagrange interpolation of ForceField_eam::set_funcfl
// (ff_eam.cpp:565-580); tab[0] = 0 and the value at grid index m is tab[m + 1]
double lagrange4(const std::vector<double>& tab, int n_src, double d_src, double x)
{
    const double sixth = 1.0 / 6.0;
    double p = x / d_src + 1.0;
    int k = static_cast<int>(p);
    k = k < n_src - 2 ? k : n_src - 2;
    k = k > 2 ? k : 2;
    p -= k;
    p = p < 2.0 ? p : 2.0;
    double c1 = -sixth * p * (p - 1.0) * (p - 2.0);
    double c2 = 0.5 * (p * p - 1.0) * (p - 2.0);
    double c3 = -0.5 * p * (p + 1.0) * (p - 2.0);
    double c4 = sixth * p * (p * p - 1.0);
    return c1 * tab[k - 1] + c2 * tab[k] + c3 * tab[k + 1] + c4 * tab[k + 2];
}

// funcfl files, one per type (ForceField_eam::set_funcfl, ff_eam.cpp:433-670):
// a comment line, "Z mass a lattice", "nrho drho nr dr cut", then F, Z(r) and
// rho(r).  The tables are regridded onto nr = int(max_r / max_dr + 0.5) points
// of max_dr; nrho comes from the same r expression (ff_eam.cpp:547-548); the
// pair term is 27.2 * 0.529 * Z_i Z_j.  For more than one type the reference
// writes type i's density to slot i*(i+1) (ff_eam.cpp:583), which it never
// allocated; here every slot b*nt+a holds type a's density, as for setfl.
int read_funcfl(mg_system* s, int nfiles, const char* const* files)
{
    const int nt = s->nt;
    if (nfiles != nt) return fail(MG_ERR_ARG, "no of types and number of files should be equal in eam");
    std::vector<int> nrs(nt), nrhos(nt);
    std::vector<double> drs(nt), drhos(nt);
    std::vector<std::vector<double>> tF(nt), tZ(nt), tR(nt);
    for (int t = 0; t < nt; t++) {
        std::vector<std::string> lines;
        CHK(read_all(files[t], lines));
        if (lines.size() < 3) return fail(MG_ERR_FORMAT, "eam potential file ended immaturely");
        std::vector<std::string> h = tokens(lines[2]);
        if (h.size() != 5) return fail(MG_ERR_FORMAT, "wrong line in eam file: %s", lines[2].c_str());
        nrhos[t] = atoi(h[0].c_str());
        drhos[t] = atof(h[1].c_str());
        nrs[t] = atoi(h[2].c_str());
        drs[t] = atof(h[3].c_str());
        if (nrs[t] < 5 || nrhos[t] < 5 || !(drs[t] > 0.0) || !(drhos[t] > 0.0))
            return fail(MG_ERR_FORMAT, "table sizes too small (nr=%d nrho=%d)", nrs[t], nrhos[t]);
        const size_t tot = (size_t)nrhos[t] + 2 * (size_t)nrs[t];
        std::vector<double> v;
        v.reserve(tot);
        for (size_t li = 3; li < lines.size() && v.size() < tot; li++) {
            std::vector<std::string> tk = tokens(lines[li]);
            if (v.size() + tk.size() > tot) return fail(MG_ERR_FORMAT, "eam potential file ended immaturely");
            for (const std::string& x : tk) v.push_back(atof(x.c_str()));
        }
        if (v.size() < tot) return fail(MG_ERR_FORMAT, "eam potential file ended immaturely");
        tF[t].assign(1, 0.0);
        tF[t].insert(tF[t].end(), v.begin(), v.begin() + nrhos[t]);
        tZ[t].assign(1, 0.0);
        tZ[t].insert(tZ[t].end(), v.begin() + nrhos[t], v.begin() + nrhos[t] + nrs[t]);
        tR[t].assign(1, 0.0);
        tR[t].insert(tR[t].end(), v.begin() + nrhos[t] + nrs[t], v.end());
    }
    double maxr = 0.0, maxrho = 0.0, maxdr = 0.0, maxdrho = 0.0;
    for (int t = 0; t < nt; t++) {
        double r = static_cast<double>(nrs[t] - 1) * drs[t], rh = static_cast<double>(nrhos[t] - 1) * drhos[t];
        maxr = maxr > r ? maxr : r;
        maxrho = maxrho > rh ? maxrho : rh;
        maxdr = maxdr > drs[t] ? maxdr : drs[t];
        maxdrho = maxdrho > drhos[t] ? maxdrho : drhos[t];
    }
    const int nr = static_cast<int>(maxr / maxdr + 0.5), nrho = static_cast<int>(maxr / maxdr + 0.5);
    const double dr = maxdr, drho = maxdrho;
    if (nr < 5 || nrho < 5) return fail(MG_ERR_FORMAT, "table sizes too small (nr=%d nrho=%d)", nr, nrho);
    s->nr = nr;
    s->nrho = nrho;
    s->dr = dr;
    s->drho = drho;
    s->Fw = 7;
    const int ncomp = nt * (nt + 1) / 2;
    s->FT.assign((size_t)nt * (nrho + 1) * s->Fw, 0.0);
    s->rhoT.assign((size_t)nt * nt * nr * 8, 0.0);
    s->phiT.assign((size_t)ncomp * nr * 8, 0.0);
    for (int a = 0; a < nt; a++) {
        double* Fd = s->FT.data() + (size_t)a * (nrho + 1) * s->Fw;
        for (int j = 0; j < nrho; j++) Fd[(size_t)j * s->Fw] = lagrange4(tF[a], nrhos[a], drhos[a], static_cast<double>(j) * drho);
        spline7(nrho, drho, Fd, s->Fw);
    }
    for (int a = 0; a < nt; a++) {
        std::vector<double> col(nr);
        for (int j = 0; j < nr; j++) col[j] = lagrange4(tR[a], nrs[a], drs[a], static_cast<double>(j) * dr);
        for (int b = 0; b < nt; b++) {
            double* dst = s->rhoT.data() + (size_t)(b * nt + a) * nr * 8;
            for (int j = 0; j < nr; j++) dst[(size_t)j * 8] = col[j];
            spline7(nr, dr, dst, 8);
        }
    }
    for (int a = 0; a < nt; a++)
        for (int b = a; b < nt; b++) {
            double* dst = s->phiT.data() + (size_t)comp_idx(a, b) * nr * 8;
            for (int j = 0; j < nr; j++) {
                double r = static_cast<double>(j) * dr;
                double t0 = lagrange4(tZ[a], nrs[a], drs[a], r), t1 = lagrange4(tZ[b], nrs[b], drs[b], r);
                dst[(size_t)j * 8] = 27.2 * 0.529 * t0 * t1;
            }
            spline7(nr, dr, dst, 8);
        }
    return MG_OK;
}

// analytic FS coefficient file (ff_fs.cpp:113-335)
int read_fs_coeffs(mg_system* s, const char* path)
{
    std::vector<std::string> lines;
    CHK(read_all(path, lines));
    std::vector<std::vector<std::string>> rows;
    for (const std::string& l : lines) {
        std::vector<std::string> t = tokens(l);
        if (!t.empty()) rows.push_back(t);
    }
    int nt = s->nt;
    size_t r = 0;
    if (rows.empty() || (int)rows[0].size() != nt)
        return fail(MG_ERR_FORMAT, "number of types represented and forcefield do not match");
    std::vector<int> types(nt);
    for (int i = 0; i < nt; i++) {
        int k = 0;
        while (k < nt && s->names[k] != rows[0][i]) k++;
        if (k == nt) return fail(MG_ERR_FORMAT, "atom type %s not found", rows[0][i].c_str());
        types[i] = k;
    }
    r = 1;
    Dev& d = s->d;
    for (int i = 0; i < nt; i++, r++) {
        if (r >= rows.size() || rows[r].size() != 1) return fail(MG_ERR_FORMAT, "Wrong format in the force filed file");
        d.fsA[types[i]] = atof(rows[r][0].c_str());
    }
    for (int i = 0; i < nt; i++)
        for (int j = 0; j < nt; j++, r++) {
            if (r >= rows.size() || rows[r].size() != 2) return fail(MG_ERR_FORMAT, "Wrong format in the force filed file");
            d.fst1[types[i]][types[j]] = atof(rows[r][0].c_str());
            d.fst2[types[i]][types[j]] = atof(rows[r][1].c_str());
        }
    for (int q = 0; q < 16; q++) d.fs_chk[q] = 0;
    for (int i = 0; i < nt; i++)
        for (int j = i; j < nt; j++, r++) {
            if (r >= rows.size() || rows[r].size() != 5) return fail(MG_ERR_FORMAT, "Wrong format in the force filed file");
            int c = comp_idx(types[i], types[j]);
            d.fs_cut_rho[c] = atof(rows[r][0].c_str());
            d.fs_cut_phi[c] = atof(rows[r][1].c_str());
            d.fsk1[c] = atof(rows[r][2].c_str());
            d.fsk2[c] = atof(rows[r][3].c_str());
            d.fsk3[c] = atof(rows[r][4].c_str());
            d.fs_chk[c] = 1;
        }
    return MG_OK;
}

int upload_tables(mg_system* s)
{
    Dev& d = s->d;
    if (s->style == STYLE_FS || s->tables_uploaded) return MG_OK;
    CHK(dalloc(&s->d_rhoT, s->rhoT.size()));
    CHK(dalloc(&s->d_phiT, s->phiT.size()));
    CHK(dalloc(&s->d_FT, s->FT.size()));
    CU(cudaMemcpy(s->d_rhoT, s->rhoT.data(), s->rhoT.size() * 8, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(s->d_phiT, s->phiT.data(), s->phiT.size() * 8, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(s->d_FT, s->FT.data(), s->FT.size() * 8, cudaMemcpyHostToDevice));
    d.rhoT = s->d_rhoT;
    d.phiT = s->d_phiT;
    d.FT = s->d_FT;
    if (s->dmd) {
        // precision form: {rho c0..c3 of slot b*nt+a, phi c0..c3 of COMP(a,b)} per (a,b) and knot
        int nt = s->nt, nr = s->nr;
        std::vector<float> pk((size_t)nt * nt * nr * 8, 0.0f);
        for (int a = 0; a < nt; a++)
            for (int b = 0; b < nt; b++)
                for (int m = 0; m < nr; m++) {
                    float* dst = pk.data() + (((size_t)(a * nt + b) * nr + m) * 8);
                    const double* rr = s->rhoT.data() + ((size_t)(b * nt + a) * nr + m) * 8;
                    for (int k = 0; k < 4; k++) dst[k] = (float)rr[k];
                    if (a >= b) {
                        const double* pp = s->phiT.data() + ((size_t)comp_idx(a, b) * nr + m) * 8;
                        for (int k = 0; k < 4; k++) dst[4 + k] = (float)pp[k];
                    }
                }
        CHK(dalloc(&s->d_pkT, pk.size()));
        CU(cudaMemcpy(s->d_pkT, pk.data(), pk.size() * sizeof(float), cudaMemcpyHostToDevice));
        d.pkT = reinterpret_cast<const float4*>(s->d_pkT);
        // plain form: the same pairing, coefficients copied unchanged
        std::vector<double> pk64((size_t)nt * nt * nr * 8, 0.0);
        for (int a = 0; a < nt; a++)
            for (int b = 0; b < nt; b++)
                for (int m = 0; m < nr; m++) {
                    double* dst = pk64.data() + (((size_t)(a * nt + b) * nr + m) * 8);
                    const double* rr = s->rhoT.data() + ((size_t)(b * nt + a) * nr + m) * 8;
                    for (int k = 0; k < 4; k++) dst[k] = rr[k];
                    if (a >= b) {
                        const double* pp = s->phiT.data() + ((size_t)comp_idx(a, b) * nr + m) * 8;
                        for (int k = 0; k < 4; k++) dst[4 + k] = pp[k];
                    }
                }
        CHK(dalloc(&s->d_pk64, pk64.size()));
        CU(cudaMemcpy(s->d_pk64, pk64.data(), pk64.size() * sizeof(double), cudaMemcpyHostToDevice));
        d.pk64 = s->d_pk64;
        // The precision form's shared-memory table: kSplitKnots knots over
        // [0, rc], each interval the cubic Hermite piece through the fine
        // spline's value and slope at its ends (fine interpolant evaluated as in
        // the force kernels, index clamp nr-2 and p <= 1), and a last row of
        // zeros for |x| >= rc.  The reference's node test, xi_q inside
        // ((r - rc) sqrt(alpha), (r + rc) sqrt(alpha)) (ff_dmd_I.cpp:198), is
        // |r - xi_q / sqrt(alpha)| < rc, so a node it rejects reads the zero row
        // and adds an exact zero without a test.  For the decaying rho and r*phi
        // of these tables the resampling error is below FP32 rounding already at
        // 256 knots.
        const int K = kSplitKnots, ncomp = nt * (nt + 1) / 2;
        const double rc = (nr - 1) * s->dr, hc = rc / (K - 1);
        auto fine = [&](const double* slot, double r, double& v, double& dv) {
            double pp = r * (1.0 / s->dr);
            int m = std::min((int)pp, nr - 2);
            double p = std::min(pp - m, 1.0);
            const double* c = slot + (size_t)m * 8;
            v = ((c[3] * p + c[2]) * p + c[1]) * p + c[0];
            dv = ((3.0 * c[3] * p + 2.0 * c[2]) * p + c[1]) * (1.0 / s->dr);
        };
        auto resample = [&](const double* slot, float* dst) {
            for (int k = 0; k < K - 1; k++) {
                double v0, d0, v1, d1;
                fine(slot, k * hc, v0, d0);
                fine(slot, std::min((k + 1) * hc, rc), v1, d1);
                d0 *= hc;
                d1 *= hc;
                float* o = dst + (size_t)k * 4;
                o[0] = (float)v0;
                o[1] = (float)d0;
                o[2] = (float)(3.0 * (v1 - v0) - 2.0 * d0 - d1);
                o[3] = (float)(2.0 * (v0 - v1) + d0 + d1);
            }
            float* o = dst + (size_t)(K - 1) * 4;
            o[0] = o[1] = o[2] = o[3] = 0.0f;
        };
        std::vector<float> ps((size_t)(nt * nt + ncomp) * K * 4, 0.0f);
        for (int a = 0; a < nt; a++)
            for (int b = 0; b < nt; b++)
                resample(s->rhoT.data() + (size_t)(b * nt + a) * nr * 8, ps.data() + (size_t)(a * nt + b) * K * 4);
        for (int q = 0; q < ncomp; q++)
            resample(s->phiT.data() + (size_t)q * nr * 8, ps.data() + (size_t)(nt * nt + q) * K * 4);
        CHK(dalloc(&s->d_pkS, ps.size()));
        CU(cudaMemcpy(s->d_pkS, ps.data(), ps.size() * sizeof(float), cudaMemcpyHostToDevice));
        d.pkS = reinterpret_cast<const float4*>(s->d_pkS);
        d.nrS = K;
        d.drS_inv = (float)(1.0 / hc);
    }
    d.Fw = s->Fw;
    d.nr = s->nr;
    d.nrho = s->nrho;
    d.dr = s->dr;
    d.drho = s->drho;
    d.dr_inv = 1.0 / s->dr;
    d.drho_inv = 1.0 / s->drho;
    s->tables_uploaded = true;
    return MG_OK;
}

// c_d_calc and calc_g read the per-pair densities and pair energies of the last
// force_calc; the precision form's force call does not store them, so they are
// written here, once, before the first reader (at the current positions: every
// caller of the boundary runs these at the positions of its last force_calc)
int ensure_pair_values(mg_system* s)
{
    if (!s->prf_stale || s->form != MG_FORM_FP32) return MG_OK;
    fill_dev_scalars(s);
    CU(launch_dmd32_pair_values(s->d, s->st));
    s->prf_stale = false;
    return MG_OK;
}

int timed_begin(mg_system* s)
{
    if (s->timing > 0) CU(cudaEventRecord(s->ev0, s->st));
    return MG_OK;
}

// marks the end of the timed work; the caller reads the time with
// timed_read after its own stream synchronisation, so that the result copies
// queue behind the kernels without a host round trip between them
int timed_end(mg_system* s)
{
    if (s->timing > 0) CU(cudaEventRecord(s->ev1, s->st));
    return MG_OK;
}

int timed_read(mg_system* s, double* slot)
{
    if (s->timing <= 0) {
        *slot = -1.0;
        return MG_OK;
    }
    CU(cudaEventSynchronize(s->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    *slot = ms;
    return MG_OK;
}

}  // namespace

// ============================================================================
extern "C" {

const char* mg_last_error(void) { return g_err.c_str(); }

int mg_version(void) { return 100; }

int mg_create(const char* style, int device, mg_system** out)
{
    if (!style || !out) return fail(MG_ERR_ARG, "null argument");
    int st;
    if (!strcmp(style, "EAM")) st = STYLE_EAM;
    else if (!strcmp(style, "FS")) st = STYLE_FS;
    else if (!strcmp(style, "DMD_I")) st = STYLE_DMD_I;
    else if (!strcmp(style, "DMD_II")) st = STYLE_DMD_II;
    else if (!strcmp(style, "DMD")) st = STYLE_DMD;
    else return fail(MG_ERR_ARG, "unknown forcefield: %s", style);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(MG_ERR_CUDA, "no CUDA device available: the mapp_b200 library has no CPU path");
    }
    if (device < 0 || device >= ndev) return fail(MG_ERR_ARG, "device %d out of range", device);
    mg_system* s = new mg_system();
    s->style = st;
    s->dmd = st >= STYLE_DMD_I;
    s->device = device;
    s->mlp.act = MG_MLP_ACT_SPLIT;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete s;
        return fail(MG_ERR_CUDA, "cudaSetDevice failed");
    }
    if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete s;
        return fail(MG_ERR_CUDA, "cudaStreamCreate failed");
    }
    s->own_stream = true;
    cudaEventCreate(&s->ev0);
    cudaEventCreate(&s->ev1);
    for (int k = 0; k < 4; k++) cudaEventCreate(&s->evk[k]);
    memset(&s->d, 0, sizeof(Dev));
    int r = MG_OK;
    if (cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        r = fail(MG_ERR_CUDA, "side stream creation failed");
    }
    if (!r) r = dalloc(&s->red_out, 12);  // 8 totals, then 8 ints of status
    if (!r) {
        s->d.status = reinterpret_cast<int*>(s->red_out + 8);
        if (cudaMallocHost((void**)&s->hp, sizeof(mg_system::HostPin)) != cudaSuccess) {
            cudaGetLastError();
            s->hp = nullptr;
            r = fail(MG_ERR_CAPACITY, "cudaMallocHost of the result block failed");
        } else
            memset(s->hp, 0, sizeof(mg_system::HostPin));
    }
    if (r) {
        if (s->red_out) cudaFree(s->red_out);
        for (int k = 0; k < 4; k++) cudaEventDestroy(s->evk[k]);
        cudaEventDestroy(s->ev0);
        cudaEventDestroy(s->ev1);
        if (s->ev_fork) cudaEventDestroy(s->ev_fork);
        if (s->ev_join) cudaEventDestroy(s->ev_join);
        if (s->side) cudaStreamDestroy(s->side);
        cudaStreamDestroy(s->st);
        delete s;
        return r;
    }
    *out = s;
    return MG_OK;
}

int mg_destroy(mg_system* s)
{
    if (!s) return MG_OK;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->st);
    if (s->side) cudaStreamSynchronize(s->side);
    Dev& d = s->d;
    void* ptrs[] = {d.prf, s->d_pkT, s->d_pk64, s->d_pkS, d.icut, d.icut_n, d.srec, d.dE32, d.facc, d.poff, d.pair_i, d.pair_j, d.pos, d.sfr, d.pos0, d.alpha, d.c, d.type, d.root, d.gchain, d.bin, d.cell_start,
                    d.cell_count, d.cell_pos, d.nbr, d.nnb, d.crdl, d.ncrd, d.crd, d.f, d.rho, d.E,
                    d.dE, d.ddE, d.n, d.s, d.t, d.v, d.c_d, d.a_in, d.g, d.pr, d.partial, d.act_pj, d.act_pv, d.act_off, d.nact,
                    s->scan_tmp, s->stage, s->red_out, s->d_rhoT, s->d_phiT, s->d_FT, s->gctl, s->gtiles};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    void* mptrs[] = {s->mlp.par, s->mlp.wbf, s->mlp.m, s->mlp.v, s->mlp.gpart, s->mlp.audit, s->mlp_loss,
                     s->mlp.row_in, s->mlp.row_id, s->mlp.row_r, s->mlp.row_n, s->mlp.audit_rows};
    for (void* p : mptrs)
        if (p) cudaFree(p);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    for (int k = 0; k < 4; k++)
        if (s->evk[k]) cudaEventDestroy(s->evk[k]);
    if (s->own_stream && s->st) cudaStreamDestroy(s->st);
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    if (s->ev_join) cudaEventDestroy(s->ev_join);
    if (s->side) cudaStreamDestroy(s->side);
    if (s->hp) cudaFreeHost(s->hp);
    delete s;
    return MG_OK;
}

int mg_set_stream(mg_system* s, void* stream)
{
    CHK(check_sys(s));
    cudaStreamSynchronize(s->st);
    if (s->own_stream && s->st) cudaStreamDestroy(s->st);
    s->st = (cudaStream_t)stream;
    s->own_stream = false;
    return MG_OK;
}

int mg_set_form(mg_system* s, int form)
{
    CHK(check_sys(s));
    if (form == MG_FORM_FP32 && !s->dmd)
        return fail(MG_ERR_UNSUPPORTED, "the FP32 precision form is implemented for the DMD styles");
    if (form == MG_FORM_MLP && (!s->dmd || s->nt > 2))
        return fail(MG_ERR_UNSUPPORTED, "the learned form is implemented for the DMD styles with one or two species");
    if (form == MG_FORM_MLP && !s->mlp_ready)
        return fail(MG_ERR_STATE, "the learned form needs mg_mlp_init (and normally mg_mlp_train) first");
    if (form != MG_FORM_FP64 && form != MG_FORM_FP32 && form != MG_FORM_MLP)
        return fail(MG_ERR_UNSUPPORTED, "form %d is not available", form);
    s->form = form;
    s->d.form = form;
    return MG_OK;
}

int mg_atoms_set_types(mg_system* s, int ntypes, const char* const* names, const double* masses)
{
    CHK(check_sys(s));
    if (ntypes < 1 || ntypes > kMaxTypes) return fail(MG_ERR_ARG, "ntypes must be 1..%d", kMaxTypes);
    if (!names || !masses) return fail(MG_ERR_ARG, "null names / masses");
    s->nt = ntypes;
    s->names.clear();
    s->masses.clear();
    for (int i = 0; i < ntypes; i++) {
        if (!names[i]) return fail(MG_ERR_ARG, "null type name");
        if (masses[i] <= 0.0) return fail(MG_ERR_ARG, "mass cannot be zero");
        s->names.push_back(names[i]);
        s->masses.push_back(masses[i]);
    }
    s->x_dim = s->dmd ? 3 + ntypes : 3;
    s->types_set = true;
    return MG_OK;
}

int mg_atoms_set_box(mg_system* s, const double* H)
{
    CHK(check_sys(s));
    if (!H) return fail(MG_ERR_ARG, "null H");
    double A[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) A[i][j] = s->H[i][j] = H[i * 3 + j];
    for (int i = 0; i < 3; i++)
        for (int j = i + 1; j < 3; j++)
            if (A[i][j] != 0.0) return fail(MG_ERR_ARG, "H must be lower triangular (Atoms::H convention)");
    // M3INV (init.h:72-85)
    double (*Bm)[3] = s->B;
    Bm[0][0] = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    Bm[1][1] = A[2][2] * A[0][0] - A[2][0] * A[0][2];
    Bm[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
    Bm[1][0] = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    Bm[2][1] = A[2][0] * A[0][1] - A[2][1] * A[0][0];
    Bm[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
    Bm[2][0] = A[1][0] * A[2][1] - A[2][0] * A[1][1];
    Bm[0][1] = A[2][1] * A[0][2] - A[0][1] * A[2][2];
    Bm[1][2] = A[0][2] * A[1][0] - A[1][2] * A[0][0];
    double det = A[0][0] * Bm[0][0] + A[0][1] * Bm[1][0] + A[0][2] * Bm[2][0];
    if (det == 0.0) return fail(MG_ERR_ARG, "H determinant is zero");
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Bm[i][j] /= det;
    s->box_set = true;
    return MG_OK;
}

int mg_atoms_set_skin(mg_system* s, double skin)
{
    CHK(check_sys(s));
    if (!(skin >= 0.0)) return fail(MG_ERR_ARG, "skin cannot be negative");
    s->skin = skin;
    return MG_OK;
}

int mg_atoms_set(mg_system* s, int natms, const double* x, const int* type, const double* c)
{
    CHK(check_sys(s));
    if (!s->types_set) return fail(MG_ERR_STATE, "atom types must be set before atoms");
    if (natms < 0) return fail(MG_ERR_ARG, "natms < 0");
    if (natms > 0 && !x) return fail(MG_ERR_ARG, "null x");
    if (natms > 0 && s->dmd && !c) return fail(MG_ERR_ARG, "DMD needs c");
    if (natms > 0 && !s->dmd && !type) return fail(MG_ERR_ARG, "EAM/FS need type");
    s->natms = natms;
    Dev& d = s->d;
    fill_dev_scalars(s);
    // Buffers keep their capacity from one call to the next, so a system that
    // is loaded with many configurations of different sizes (the batched form's
    // builder) allocates for the largest once.
    size_t cap0 = (size_t)natms * 4 + 1024;
    CHK(ensure_atoms(s, cap0, 0));
    if ((size_t)natms + 1 > s->owned_cap) {
        size_t oc = (size_t)natms + natms / 4 + 64;
        CHK(dalloc(&d.pos0, oc));
        CHK(dalloc(&d.nnb, oc + 1));
        CHK(dalloc(&d.poff, oc + 1));
        CHK(dalloc(&d.ncrd, oc));
        CHK(dalloc(&d.f, oc * s->x_dim));
        CHK(dalloc(&d.c_d, oc * s->nt));
        CHK(dalloc(&d.a_in, oc * s->nt));
        CHK(dalloc(&d.g, oc * s->nt));
        s->owned_cap = oc;
    }
    s->npair_blocks = s->dmd ? 3 * s->nt * s->nt + 3 * (s->nt * (s->nt + 1) / 2) : 2;
    CHK(ensure_pairs(s, std::max(d.maxnb, s->dmd ? 96 : 64)));
    d.maxcrd = std::max(d.maxcrd, 32);
    if ((size_t)natms * d.maxcrd > s->crdl_cap) {
        s->crdl_cap = (size_t)natms * d.maxcrd + 1024;
        CHK(dalloc(&d.crdl, s->crdl_cap));
    }
    if (natms) {
        const void* dx = nullptr;
        CHK(stage_in(s, x, (size_t)natms * s->x_dim * sizeof(double), &dx));
        CU(launch_split_x(d, (const double*)dx, 1, s->st));
        if (s->dmd) {
            CU(cudaMemcpyAsync(d.c, c, (size_t)natms * s->nt * sizeof(double),
                               is_device_ptr(c) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s->st));
        } else {
            CU(cudaMemcpyAsync(d.type, type, (size_t)natms * sizeof(int),
                               is_device_ptr(type) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s->st));
        }
        CU(cudaStreamSynchronize(s->st));
    }
    s->atoms_set = true;
    s->initialized = false;
    return MG_OK;
}

int mg_ff_coef(mg_system* s, int narg, const char* const* arg)
{
    CHK(check_sys(s));
    if (!s->types_set) return fail(MG_ERR_STATE, "atom types must be set before ff_coef");
    Dev& d = s->d;
    if (s->style == STYLE_EAM) {
        if (narg < 3) return fail(MG_ERR_ARG, "wrong coeff command for eam Force Field");
        if (!strcmp(arg[1], "FS")) {
            if (narg != 3) return fail(MG_ERR_ARG, "one file is needed for eam");
            CHK(read_tables(s, arg[2], true));
        } else if (!strcmp(arg[1], "SetFL")) {
            if (narg != 3) return fail(MG_ERR_ARG, "one file is needed for eam");
            CHK(read_tables(s, arg[2], false));
        } else if (!strcmp(arg[1], "FuncFL")) {
            CHK(read_funcfl(s, narg - 2, arg + 2));
        } else
            return fail(MG_ERR_ARG, "wrong coeff command for eam Force Field");
        // ff_eam.cpp:424-425
        d.cut_sq = (s->nr - 1.0) * (s->nr - 1.0) * s->dr * s->dr;
        d.rho_max = (s->nrho - 1.0) * s->drho;
    } else if (s->style == STYLE_FS) {
        if (narg != 2) return fail(MG_ERR_ARG, "wrong coeff command for Finnis-Sinclair Force Field");
        CHK(read_fs_coeffs(s, arg[1]));
    } else {
        if (narg < 8) return fail(MG_ERR_ARG, "wrong coeff command for eam Force Field");
        double kb = 8.617332478e-5, hbar = 6.5821192815e-16;
        d.rsq_crd = atof(arg[1]);
        d.rsq_crd *= d.rsq_crd;
        int n = atoi(arg[2]);
        if (n < 1 || n > kMaxQuad) return fail(MG_ERR_ARG, "n should be between 1 and 14");
        s->nq = n;
        d.nq = n;
        gauss_hermite(n, d.xi, d.w0);
        for (int i = 0; i < n; i++) {
            d.w1[i] = d.w0[i] * d.xi[i];
            d.w2[i] = d.w0[i] * d.xi[i] * d.xi[i];
            d.xi_f[i] = (float)d.xi[i];
            d.w0_f[i] = (float)d.w0[i];
            d.w1_f[i] = (float)d.w1[i];
            d.w2_f[i] = (float)d.w2[i];
        }
        d.alpha_min = atof(arg[3]);
        d.alpha_max = atof(arg[4]);
        double T = atof(arg[5]);
        if (!strcmp(arg[6], "FS")) {
            if (narg != 8) return fail(MG_ERR_ARG, "one file is needed for eam");
            CHK(read_tables(s, arg[7], true));
        } else if (!strcmp(arg[6], "SetFL") || !strcmp(arg[6], "FuncFL")) {
            return fail(MG_ERR_UNSUPPORTED, "DMD styles read FS tables (got %s)", arg[6]);
        } else
            return fail(MG_ERR_ARG, "wrong coeff command for eam Force Field");
        for (int i = 0; i < s->nt; i++) {
            double mass = s->masses[i];
            mass *= 1.0364269184093291236e-28;
            double deb_l = hbar * hbar * 2.0 / (mass * kb * T);
            d.c0[i] = 1.5 * kb * T * (log(deb_l) - 1.0);
        }
        d.kbT = kb * T;
        d.beta = 1.0 / d.kbT;
        if (d.alpha_min == 0.0) return fail(MG_ERR_ARG, "minimum alpha cannot be zero");
        d.rc = (static_cast<double>(s->nr) - 1.0) * s->dr;
        d.rho_max = (static_cast<double>(s->nrho) - 1.0) * s->drho;
        d.cut_sq = d.rc * d.rc;
        double mod_rc = d.rc + d.xi[n - 1] / sqrt(d.alpha_min);
        d.cut_sq_mod = mod_rc * mod_rc;
    }
    s->coef_set = true;
    s->tables_uploaded = false;
    s->initialized = false;
    return MG_OK;
}

int mg_ff_init(mg_system* s)
{
    MG_NVTX("mg_ff_init");
    CHK(check_sys(s));
    if (!s->types_set || !s->box_set || !s->atoms_set || !s->coef_set)
        return fail(MG_ERR_STATE, "types, box, atoms and ff_coef must be set before init");
    CHK(upload_tables(s));
    fill_dev_scalars(s);
    compute_cutoffs(s);
    if (s->natms == 0) {  // an empty system: no ghosts, no pairs, zero energy and forces
        s->d.nph = 0;
        s->d.nall = 0;
        s->d.npairs = 0;
        s->npairs = 0;
        s->initialized = true;
        return MG_OK;
    }
    // owned atoms: root / chain identity, s already in d.sfr
    {
        std::vector<int> root(s->natms);
        for (int i = 0; i < s->natms; i++) root[i] = i;
        if (s->natms) {
            CU(cudaMemcpyAsync(s->d.root, root.data(), s->natms * sizeof(int), cudaMemcpyHostToDevice, s->st));
            CU(cudaMemsetAsync(s->d.gchain, 0, s->natms * sizeof(unsigned long long), s->st));
        }
        CU(cudaStreamSynchronize(s->st));
    }
    CHK(ensure_partials(s, 2LL * div_up((long long)s->natms * 32, kFFBlock) + div_up((long long)s->natms * 4, kFFBlock) + 8));
    CHK(rebuild(s));
    s->initialized = true;
    return MG_OK;
}

int mg_atoms_update_x(mg_system* s, const double* x, int* rebuilt)
{
    MG_NVTX("mg_atoms_update_x");
    CHK(check_sys_nores(s));
    if (!s->initialized) return fail(MG_ERR_STATE, "init must run before update_0");
    CHK(resolve_skin(s));  // an earlier update_x whose test nothing has read yet
    if (s->natms == 0) {
        if (rebuilt) *rebuilt = 0;
        return MG_OK;
    }
    Dev& d = s->d;
    const void* dx = nullptr;
    CHK(stage_in(s, x, (size_t)s->natms * s->x_dim * sizeof(double), &dx));
    // new x, the skin test and the ghost refresh in one launch (the refresh
    // runs before the flag is known: it only writes the ghost slots, which a
    // rebuild recreates anyway)
    s->skin_gen = s->skin_gen % 0x7ffffffe + 1;
    CU(launch_update_x(d, (const double*)dx, s->skin * s->skin, d.status + 7, s->skin_gen, s->st));
    if (!rebuilt) {
        // nobody asked: the test is settled by the next entry point that needs
        // the lists, so the host does not wait here (force_calc reads it
        // with its results)
        s->skin_pending = true;
        return MG_OK;
    }
    CU(cudaMemcpyAsync(&s->hp->status[7], d.status + 7, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    const int flag = s->hp->status[7] == s->skin_gen;
    if (flag) {
        CU(launch_x2s(d, s->st));
        CHK(rebuild(s));
    }
    *rebuilt = flag;
    return MG_OK;
}

int mg_atoms_update_c(mg_system* s, const double* c)
{
    MG_NVTX("mg_atoms_update_c");
    // (a pending skin test may stay pending: a rebuild copies the new c to
    // the ghosts it makes)
    CHK(check_sys_nores(s));
    if (!s->dmd) return fail(MG_ERR_UNSUPPORTED, "c exists only in DMD mode");
    if (!s->initialized) return fail(MG_ERR_STATE, "init must run first");
    if (s->natms == 0) return MG_OK;
    size_t bytes = (size_t)s->natms * s->nt * sizeof(double);
    CU(cudaMemcpyAsync(s->d.c, c, bytes, is_device_ptr(c) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s->st));
    CU(launch_refresh_c(s->d, s->st));
    return MG_OK;
}

int mg_atoms_get_x(mg_system* s, double* x)
{
    CHK(check_sys(s));
    if (!x) return fail(MG_ERR_ARG, "null x");
    if (s->natms == 0) return MG_OK;
    size_t bytes = (size_t)s->natms * s->x_dim * sizeof(double);
    if (bytes > s->stage_cap) {
        CHK(dalloc((char**)&s->stage, bytes));
        s->stage_cap = bytes;
    }
    CU(launch_merge_x(s->d, s->stage, 0, s->natms, s->st));
    CHK(copy_out(s, x, s->stage, bytes));
    CU(cudaStreamSynchronize(s->st));
    return MG_OK;
}

int mg_atoms_get_ghosts(mg_system* s, double* x, int* owner)
{
    CHK(check_sys(s));
    int nph = s->d.nph;
    if (x && nph) {
        size_t bytes = (size_t)nph * s->x_dim * sizeof(double);
        if (bytes > s->stage_cap) {
            CHK(dalloc((char**)&s->stage, bytes));
            s->stage_cap = bytes;
        }
        CU(launch_merge_x(s->d, s->stage, s->natms, nph, s->st));
        CHK(copy_out(s, x, s->stage, bytes));
    }
    if (owner && nph) CHK(copy_out(s, owner, s->d.root + s->natms, (size_t)nph * sizeof(int)));
    CU(cudaStreamSynchronize(s->st));
    return MG_OK;
}

int mg_ff_force_calc(mg_system* s, int st_clc, double* f, double* en_st)
{
    MG_NVTX("mg_ff_force_calc");
    CHK(check_sys_nores(s));
    // with update_x's skin test pending the force is computed on the current
    // list and the test read with the results; if some site moved more than
    // the skin, the list is rebuilt and the force computed again
    const bool speculative = s->skin_pending;
    if (!s->initialized) return fail(MG_ERR_STATE, "force_calc before init");
    if (s->natms == 0) {
        if (en_st)
            for (int i = 0; i < (st_clc ? 7 : 1); i++) en_st[i] = 0.0;
        return MG_OK;
    }
    Dev& d = s->d;
    fill_dev_scalars(s);
    cudaEvent_t* evk = s->timing >= 2 ? s->evk : nullptr;
    CHK(timed_begin(s));
    // the precision form's first kernel zeroes f and E itself
    const bool f32 = s->dmd && s->form == MG_FORM_FP32;
    // (and the plain DMD form's embedding kernel writes f's first terms)
    if (!f32 && !(s->dmd && s->form == MG_FORM_FP64))
        CU(cudaMemsetAsync(d.f, 0, (size_t)s->natms * s->x_dim * sizeof(double), s->st));
    int rows = 0;
    if (s->style == STYLE_EAM || s->style == STYLE_FS) {
        CU(cudaMemsetAsync(d.rho, 0, (size_t)s->natms * sizeof(double), s->st));
        CU(s->style == STYLE_EAM ? launch_eam_force(d, st_clc, &rows, s->st) : launch_fs_force(d, st_clc, &rows, s->st));
    } else {
        if (!f32) CU(cudaMemsetAsync(d.E, 0, (size_t)s->natms * s->nt * sizeof(double), s->st));
        if (f32) {
            CU(launch_dmd_force_f32(d, st_clc, &rows, s->st, evk));
            s->prf_stale = true;
        } else if (s->form == MG_FORM_MLP) {
            // the network-row list holds every row of the list at most
            const long long need = d.npairs * s->nt * s->nt;
            if (need > s->mlp.row_cap) {
                const long long cap = need + need / 5 + 1024;
                CHK(dalloc(&s->mlp.row_in, (size_t)cap));
                CHK(dalloc(&s->mlp.row_id, (size_t)cap));
                CHK(dalloc(&s->mlp.row_r, (size_t)cap));
                // the hashed 1% audit: 2% plus a margin holds any realistic draw;
                // rows beyond the capacity are not audited
                const long long acap = cap / 50 + 4096;
                CHK(dalloc(&s->mlp.audit_rows, (size_t)acap));
                s->mlp.row_cap = cap;
                s->mlp.audit_cap = acap;
            }
            CU(cudaMemsetAsync(s->mlp.audit, 0, 16 * sizeof(float), s->st));
            CU(cudaMemsetAsync(d.status + 5, 0, sizeof(int), s->st));
            CU(launch_dmd_force_mlp(d, s->mlp, 0x51ed270b3a5d4e1ull + 0x9e37ull * (++s->mlp_calls), st_clc, &rows,
                                    s->st, evk));
            s->prf_stale = false;
        } else
            CU(launch_dmd_force(d, st_clc, &rows, s->st, evk));
    }
    // the forces are final: their copy runs beside the reduction of the
    // totals, which are read with every status word in one more copy; all
    // asynchronous, one synchronisation
    CHK(copy_out_side(s, f, d.f, (size_t)s->natms * s->x_dim * sizeof(double)));
    CU(launch_reduce_partials(d, rows, 7, s->red_out, s->st));
    CHK(timed_end(s));
    CU(cudaMemcpyAsync(s->hp, s->red_out, 8 * sizeof(double) + 8 * sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CHK(join_side(s));
    CU(cudaStreamSynchronize(s->st));
    const double* tot = s->hp->tot;
    const int icut_over = s->dmd && s->form == MG_FORM_FP32 ? s->hp->status[4] : 0;
    const int tc_timeout = s->dmd && s->form == MG_FORM_MLP ? s->hp->status[5] : 0;
    if (speculative) {
        s->skin_pending = false;
        if (s->hp->status[7] == s->skin_gen) {
            CU(launch_x2s(d, s->st));
            CHK(rebuild(s));
            return mg_ff_force_calc(s, st_clc, f, en_st);
        }
    }
    if (icut_over) return fail(MG_ERR_CAPACITY, "precision form: in-cut pair list overflow");
    if (tc_timeout) return fail(MG_ERR_TIMEOUT, "learned form: a tensor-core wait ran out");
    CHK(timed_read(s, &s->t_force));
    s->t_k_valid = s->dmd && evk;
    if (s->t_k_valid)
        for (int k = 0; k < 3; k++) {
            float ms = 0;
            CU(cudaEventElapsedTime(&ms, s->evk[k], s->evk[k + 1]));
            s->t_k[k] = ms;
        }
    if (en_st) {
        if (st_clc)
            for (int i = 0; i < 7; i++) en_st[i] = tot[i];
        else
            en_st[0] = tot[0];
    }
    return MG_OK;
}

int mg_ff_energy_calc(mg_system* s, double* energy)
{
    MG_NVTX("mg_ff_energy_calc");
    CHK(check_sys(s));
    if (!s->initialized) return fail(MG_ERR_STATE, "energy_calc before init");
    if (s->natms == 0) {
        if (energy) *energy = 0.0;
        return MG_OK;
    }
    Dev& d = s->d;
    CHK(timed_begin(s));
    int rows = 0;
    if (s->style == STYLE_EAM || s->style == STYLE_FS) {
        CU(cudaMemsetAsync(d.rho, 0, (size_t)s->natms * sizeof(double), s->st));
        CU(s->style == STYLE_EAM ? launch_eam_energy(d, &rows, s->st) : launch_fs_energy(d, &rows, s->st));
    } else {
        CU(cudaMemsetAsync(d.E, 0, (size_t)s->natms * s->nt * sizeof(double), s->st));
        CU(launch_dmd_energy(d, &rows, s->st));
    }
    CU(launch_reduce_partials(d, rows, 1, s->red_out, s->st));
    CHK(timed_end(s));
    CU(cudaMemcpyAsync(s->hp->tot, s->red_out, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    CHK(timed_read(s, &s->t_energy));
    if (energy) *energy = s->hp->tot[0];
    return MG_OK;
}

int mg_ff_create_2nd_neigh_lst(mg_system* s)
{
    MG_NVTX("mg_ff_create_2nd_neigh_lst");
    CHK(check_sys(s));
    if (!s->dmd) return MG_OK;  // empty in EAM / FS (ff_eam.h:61)
    if (!s->initialized) return fail(MG_ERR_STATE, "create_2nd_neigh_lst before init");
    if (s->natms == 0) {
        s->crd_built = 1;
        return MG_OK;
    }
    Dev& d = s->d;
    for (int attempt = 0; attempt < 4; attempt++) {
        CU(cudaMemsetAsync(d.crd, 0, (size_t)d.nall * sizeof(int), s->st));
        CU(cudaMemsetAsync(d.status, 0, 8 * sizeof(int), s->st));
        CU(launch_dmd_crd(d, s->st));
        const int* st_h = s->hp->status;
        CU(cudaMemcpyAsync(s->hp->status, d.status, 8 * sizeof(int), cudaMemcpyDeviceToHost, s->st));
        CU(cudaStreamSynchronize(s->st));
        if (!st_h[2]) break;
        d.maxcrd = st_h[3] + 8;
        if ((size_t)s->natms * d.maxcrd > s->crdl_cap) {
            s->crdl_cap = (size_t)s->natms * d.maxcrd + 1024;
            CHK(dalloc(&d.crdl, s->crdl_cap));
        }
        if (attempt == 3) return fail(MG_ERR_CAPACITY, "coordination list capacity could not be met");
    }
    s->crd_built = 1;
    return MG_OK;
}

int mg_ff_c_d_calc(mg_system* s, double* c_d)
{
    MG_NVTX("mg_ff_c_d_calc");
    CHK(check_sys(s));
    if (!s->dmd) return MG_OK;
    if (!s->crd_built) return fail(MG_ERR_STATE, "create_2nd_neigh_lst must run before c_d_calc");
    if (s->natms == 0) return MG_OK;
    Dev& d = s->d;
    size_t bytes = (size_t)s->natms * s->nt * sizeof(double);
    CHK(timed_begin(s));
    CHK(ensure_pair_values(s));
    CU(cudaMemsetAsync(d.E, 0, bytes, s->st));
    CU(cudaMemsetAsync(d.c_d, 0, bytes, s->st));
    CU(launch_dmd_cdot(d, s->st));
    CHK(timed_end(s));
    CHK(copy_out(s, c_d, d.c_d, bytes));
    CU(cudaStreamSynchronize(s->st));
    CHK(timed_read(s, &s->t_cd));
    return MG_OK;
}

int mg_ff_calc_g(mg_system* s, int chk, double alpha, const double* a, double* g, double* cost)
{
    MG_NVTX("mg_ff_calc_g");
    CHK(check_sys(s));
    if (!s->dmd) {
        if (cost) *cost = 0.0;  // ff_eam.h:62 returns 0
        return MG_OK;
    }
    if (!s->crd_built) return fail(MG_ERR_STATE, "create_2nd_neigh_lst must run before calc_g");
    if (!a && s->natms) return fail(MG_ERR_ARG, "null a");
    if (s->natms == 0) {
        if (cost) *cost = 0.0;
        return MG_OK;
    }
    Dev& d = s->d;
    size_t bytes = (size_t)s->natms * s->nt * sizeof(double);
    CU(cudaMemcpyAsync(d.a_in, a, bytes, is_device_ptr(a) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s->st));
    CHK(timed_begin(s));
    CHK(ensure_pair_values(s));
    CU(cudaMemsetAsync(d.E, 0, bytes, s->st));
    int rows = 0;
    CU(launch_dmd_calc_g(d, chk, alpha, &rows, s->st));
    CHK(copy_out_side(s, g, d.g, bytes));
    CU(launch_reduce_partials(d, rows, 1, s->red_out, s->st));
    CHK(timed_end(s));
    CU(cudaMemcpyAsync(s->hp->tot, s->red_out, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CHK(join_side(s));
    CU(cudaStreamSynchronize(s->st));
    CHK(timed_read(s, &s->t_g));
    if (cost) *cost = s->hp->tot[0] * 0.25;
    return MG_OK;
}

int mg_ff_fin(mg_system* s)
{
    CHK(check_sys(s));
    Dev& d = s->d;
    cudaStreamSynchronize(s->st);
    if (d.pr) cudaFree(d.pr);
    d.pr = nullptr;
    d.maxp = 0;
    if (s->dmd) s->pair_cap = 0;
    else s->nbr_cap = 0;  // EAM / FS keep their pair derivatives beside the ELL list
    s->initialized = false;
    s->crd_built = 0;
    return MG_OK;
}

int mg_neighbor_create_list(mg_system* s)
{
    MG_NVTX("mg_neighbor_create_list");
    CHK(check_sys(s));
    if (!s->initialized) return fail(MG_ERR_STATE, "init must run first");
    if (s->natms == 0) return MG_OK;
    CU(launch_x2s(s->d, s->st));
    return rebuild(s);
}

int mg_neighbor_counts(mg_system* s, int* natms, int* natms_ph, long long* no_pairs)
{
    CHK(check_sys(s));
    if (natms) *natms = s->natms;
    if (natms_ph) *natms_ph = s->d.nph;
    if (no_pairs) {
        std::vector<int> n(s->natms);
        if (s->natms) CU(cudaMemcpy(n.data(), s->d.nnb, s->natms * sizeof(int), cudaMemcpyDeviceToHost));
        long long t = 0;
        for (int v : n) t += v;
        *no_pairs = t;
    }
    return MG_OK;
}

int mg_neighbor_get_list(mg_system* s, int* sizes, int* pairs)
{
    CHK(check_sys(s));
    int natms = s->natms, maxnb = s->d.maxnb;
    std::vector<int> n(natms), all((size_t)natms * maxnb);
    if (natms) {
        CU(cudaMemcpy(n.data(), s->d.nnb, natms * sizeof(int), cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(all.data(), s->d.nbr, all.size() * sizeof(int), cudaMemcpyDeviceToHost));
    }
    long long off = 0;
    for (int i = 0; i < natms; i++) {
        if (sizes) sizes[i] = n[i];
        if (pairs) memcpy(pairs + off, all.data() + (size_t)i * maxnb, n[i] * sizeof(int));
        off += n[i];
    }
    return MG_OK;
}

int mg_get_vector(mg_system* s, const char* name, double* out)
{
    CHK(check_sys(s));
    if (!name || !out) return fail(MG_ERR_ARG, "null argument");
    Dev& d = s->d;
    int nt = s->nt;
    const double* src = nullptr;
    size_t count = 0;
    if (!strcmp(name, "E")) src = d.E, count = (size_t)s->natms * nt;
    else if (!strcmp(name, "dE")) src = d.dE, count = (size_t)s->natms * nt;
    else if (!strcmp(name, "ddE")) src = d.ddE, count = (size_t)s->natms * nt;
    else if (!strcmp(name, "n")) src = d.n, count = (size_t)s->natms * nt;
    else if (!strcmp(name, "c_d")) src = d.c_d, count = (size_t)s->natms * nt;
    else if (!strcmp(name, "c") && s->dmd) src = d.c, count = (size_t)s->natms * nt;
    else if (!strcmp(name, "rho")) src = d.rho, count = (size_t)s->natms;
    else return fail(MG_ERR_ARG, "unknown vector %s", name);
    CHK(copy_out(s, out, src, count * sizeof(double)));
    CU(cudaStreamSynchronize(s->st));
    return MG_OK;
}

int mg_get_int_vector(mg_system* s, const char* name, int* out)
{
    CHK(check_sys(s));
    if (!name || !out) return fail(MG_ERR_ARG, "null argument");
    if (!strcmp(name, "crd")) {
        CHK(copy_out(s, out, s->d.crd, (size_t)s->d.nall * sizeof(int)));
        CU(cudaStreamSynchronize(s->st));
        return MG_OK;
    }
    return fail(MG_ERR_ARG, "unknown vector %s", name);
}

int mg_last_time(mg_system* s, const char* phase, double* ms)
{
    CHK(check_sys(s));
    if (!phase || !ms) return fail(MG_ERR_ARG, "null argument");
    if (!strcmp(phase, "list")) *ms = s->t_list;
    else if (!strcmp(phase, "force")) *ms = s->t_force;
    else if (!strcmp(phase, "energy")) *ms = s->t_energy;
    else if (!strcmp(phase, "c_d")) *ms = s->t_cd;
    else if (!strcmp(phase, "calc_g")) *ms = s->t_g;
    else if (!strncmp(phase, "force.", 6)) {
        int k = !strcmp(phase, "force.pass1") ? 0 : !strcmp(phase, "force.embed") ? 1 : !strcmp(phase, "force.pass2") ? 2 : -1;
        if (k < 0) return fail(MG_ERR_ARG, "unknown phase %s", phase);
        if (!s->t_k_valid)
            return fail(MG_ERR_STATE, "%s: the last force_calc took no per-kernel times (mg_set_timing level 2)",
                        phase);
        *ms = s->t_k[k];
    } else
        return fail(MG_ERR_ARG, "unknown phase %s", phase);
    if (*ms < 0.0) return fail(MG_ERR_STATE, "%s: the last call was not timed (mg_set_timing level 0)", phase);
    return MG_OK;
}

int mg_set_timing(mg_system* s, int level)
{
    CHK(check_sys(s));
    if (level < 0 || level > 2) return fail(MG_ERR_ARG, "timing level %d is not 0, 1 or 2", level);
    s->timing = level;
    return MG_OK;
}

// ---- learned form ------------------------------------------------------------
static unsigned short f2bf(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    uint32_t r = 0x7fffu + ((u >> 16) & 1u);
    return (unsigned short)((u + r) >> 16);
}

static int mlp_upload_params(mg_system* s, const std::vector<float>& par)
{
    std::vector<unsigned short> bf(par.size());
    for (size_t k = 0; k < par.size(); k++) bf[k] = f2bf(par[k]);
    CU(cudaMemcpy(s->mlp.par, par.data(), par.size() * sizeof(float), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(s->mlp.wbf, bf.data(), bf.size() * sizeof(unsigned short), cudaMemcpyHostToDevice));
    return MG_OK;
}

int mg_mlp_nparam(void) { return mlp_nparam(); }

int mg_mlp_set_activation(mg_system* s, int act)
{
    CHK(check_sys(s));
    if (act != MG_MLP_ACT_POLY && act != MG_MLP_ACT_TANH && act != MG_MLP_ACT_SPLIT)
        return fail(MG_ERR_ARG, "unknown activation %d", act);
    s->mlp.act = act;
    return MG_OK;
}

int mg_mlp_init(mg_system* s, double r_lo, double r_hi, double w_lo, double w_hi, unsigned long long seed)
{
    CHK(check_sys(s));
    if (!s->dmd || !s->coef_set) return fail(MG_ERR_STATE, "the learned form needs a DMD style with ff_coef done");
    if (s->nt > 2) return fail(MG_ERR_UNSUPPORTED, "the learned form is implemented for one or two species");
    if (!(r_hi > r_lo) || !(w_hi > w_lo) || w_lo <= 0.0) return fail(MG_ERR_ARG, "bad training box");
    if (!s->d_rhoT) CHK(upload_tables(s));
    int np = mlp_nparam(), npart = mlp_npart();
    MlpState& M = s->mlp;
    CHK(dalloc(&M.par, np));
    CHK(dalloc((unsigned short**)&M.wbf, np));
    CHK(dalloc(&M.m, np));
    CHK(dalloc(&M.v, np));
    CHK(dalloc(&M.gpart, (size_t)npart * 4096));  // up to 4096 tiles of 64 rows per step
    CHK(dalloc(&M.audit, 16));
    if (!M.row_n) CHK(dalloc(&M.row_n, 4));
    CU(cudaMemset(M.m, 0, np * sizeof(float)));
    CU(cudaMemset(M.v, 0, np * sizeof(float)));
    M.box.r_lo = (float)r_lo;
    M.box.r_hi = (float)r_hi;
    M.box.w_lo = (float)w_lo;
    M.box.w_hi = (float)w_hi;
    for (int q = 0; q < 6; q++) {
        M.out_mean[q] = 0.f;
        M.out_scale[q] = 1.f;
    }
    // weights U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from a splitmix64 stream; biases
    // and the padding rows / columns zero
    std::vector<float> par(np, 0.0f);
    unsigned long long st = seed;
    auto next = [&]() {
        st += 0x9e3779b97f4a7c15ull;
        unsigned long long z = st;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    const int H = 64;
    auto fill = [&](int off, int rows, int cols, int real_rows, int real_cols, int fan_in) {
        double bnd = 1.0 / sqrt((double)fan_in);
        for (int r = 0; r < rows; r++)
            for (int c = 0; c < cols; c++) {
                double u = next();
                par[off + r * cols + c] = (r < real_rows && c < real_cols) ? (float)((2.0 * u - 1.0) * bnd) : 0.0f;
            }
    };
    fill(0, 16, H, 4, H, 4);
    fill(16 * H + H, H, H, H, H, H);
    fill(16 * H + H + H * H + H, H, H, H, H, H);
    fill(16 * H + H + 2 * (H * H + H), H, 8, H, 6, H);
    CHK(mlp_upload_params(s, par));
    s->mlp_ready = true;
    return MG_OK;
}

int mg_mlp_state(mg_system* s, float* par_out, const float* par_in, float* scaling_out, const float* scaling_in)
{
    CHK(check_sys(s));
    if (!s->mlp_ready) return fail(MG_ERR_STATE, "mg_mlp_init first");
    int np = mlp_nparam();
    if (par_in) {
        std::vector<float> par(par_in, par_in + np);
        CHK(mlp_upload_params(s, par));
    }
    if (scaling_in)
        for (int q = 0; q < 6; q++) {
            s->mlp.out_mean[q] = scaling_in[q];
            s->mlp.out_scale[q] = scaling_in[6 + q];
        }
    if (par_out) CU(cudaMemcpy(par_out, s->mlp.par, np * sizeof(float), cudaMemcpyDeviceToHost));
    if (scaling_out)
        for (int q = 0; q < 6; q++) {
            scaling_out[q] = s->mlp.out_mean[q];
            scaling_out[6 + q] = s->mlp.out_scale[q];
        }
    return MG_OK;
}

int mg_mlp_train(mg_system* s, long long nsamples, int steps, int batch, double lr, unsigned long long seed,
                 double* final_loss)
{
    MG_NVTX("mg_mlp_train");
    CHK(check_sys(s));
    if (!s->mlp_ready) return fail(MG_ERR_STATE, "mg_mlp_init first");
    if (nsamples < 64 || steps < 1 || batch < 64 || batch % 64 || batch / 64 > 4096)
        return fail(MG_ERR_ARG, "need nsamples >= 64, steps >= 1, batch a multiple of 64 up to 262144");
    if (nsamples > (1LL << 31) - 1) return fail(MG_ERR_ARG, "too many samples");
    int n = (int)nsamples;
    float *X = nullptr, *Y = nullptr;
    CHK(dalloc(&X, (size_t)n * 4));
    CHK(dalloc(&Y, (size_t)n * 6));
    fill_dev_scalars(s);
    CU(launch_mlp_labels(s->d, s->mlp.box, seed, n, X, Y, s->st));
    // output standardisation from the labels
    std::vector<float> yh((size_t)n * 6);
    CU(cudaMemcpyAsync(yh.data(), Y, yh.size() * sizeof(float), cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    for (int q = 0; q < 6; q++) {
        double m = 0, m2 = 0;
        for (int k = 0; k < n; k++) {
            double v = yh[(size_t)k * 6 + q];
            m += v;
            m2 += v * v;
        }
        m /= n;
        double var = m2 / n - m * m;
        s->mlp.out_mean[q] = (float)m;
        s->mlp.out_scale[q] = (float)(var > 1e-30 ? sqrt(var) : 1.0);
    }
    if (s->mlp_loss_n < steps) {
        CHK(dalloc(&s->mlp_loss, steps));
        s->mlp_loss_n = steps;
    }
    for (int t = 0; t < steps; t++)
        CU(launch_mlp_train_step(s->mlp, X, Y, n, batch, seed, t, steps, (float)lr, 0, nullptr, s->mlp_loss, s->st));
    float last = 0.f;
    CU(cudaMemcpyAsync(&last, s->mlp_loss + steps - 1, sizeof(float), cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    cudaFree(X);
    cudaFree(Y);
    if (final_loss) *final_loss = last;
    return MG_OK;
}

int mg_mlp_loss_history(mg_system* s, int n, float* out)
{
    CHK(check_sys(s));
    if (n > s->mlp_loss_n) return fail(MG_ERR_ARG, "history holds %d steps", s->mlp_loss_n);
    if (n > 0) CU(cudaMemcpy(out, s->mlp_loss, n * sizeof(float), cudaMemcpyDeviceToHost));
    return MG_OK;
}

int mg_mlp_eval(mg_system* s, int n, const float* x, float* y)
{
    CHK(check_sys(s));
    if (!s->mlp_ready) return fail(MG_ERR_STATE, "mg_mlp_init first");
    if (n < 1 || !x || !y) return fail(MG_ERR_ARG, "need n >= 1 and non-null x, y");
    float *X = nullptr, *Y = nullptr;
    CHK(dalloc(&X, (size_t)n * 4));
    CHK(dalloc(&Y, (size_t)n * 6));
    CU(cudaMemcpy(X, x, (size_t)n * 4 * sizeof(float), cudaMemcpyDefault));
    CU(launch_mlp_eval(s->mlp, X, n, Y, s->st));
    CU(cudaMemcpyAsync(y, Y, (size_t)n * 6 * sizeof(float), cudaMemcpyDefault, s->st));
    CU(cudaStreamSynchronize(s->st));
    cudaFree(X);
    cudaFree(Y);
    return MG_OK;
}

int mg_mlp_grad(mg_system* s, int n, const float* x, const float* y, float* grad, double* loss)
{
    CHK(check_sys(s));
    if (!s->mlp_ready) return fail(MG_ERR_STATE, "mg_mlp_init first");
    if (n < 64 || n % 64 || n / 64 > 4096) return fail(MG_ERR_ARG, "n must be a multiple of 64");
    float *X = nullptr, *Y = nullptr, *G = nullptr, *L = nullptr;
    CHK(dalloc(&X, (size_t)n * 4));
    CHK(dalloc(&Y, (size_t)n * 6));
    CHK(dalloc(&G, (size_t)mlp_nparam()));
    CHK(dalloc(&L, 1));
    CU(cudaMemcpy(X, x, (size_t)n * 4 * sizeof(float), cudaMemcpyDefault));
    CU(cudaMemcpy(Y, y, (size_t)n * 6 * sizeof(float), cudaMemcpyDefault));
    CU(launch_mlp_train_step(s->mlp, X, Y, n, n, 0, 0, 1, 0.0f, 1, G, L, s->st));
    CU(cudaMemcpyAsync(grad, G, mlp_nparam() * sizeof(float), cudaMemcpyDefault, s->st));
    float l = 0;
    CU(cudaMemcpyAsync(&l, L, sizeof(float), cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    if (loss) *loss = l;
    cudaFree(X);
    cudaFree(Y);
    cudaFree(G);
    cudaFree(L);
    return MG_OK;
}

int mg_mlp_audit(mg_system* s, double* max_err, long long* counts)
{
    CHK(check_sys(s));
    if (!s->mlp_ready) return fail(MG_ERR_STATE, "mg_mlp_init first");
    float a[16];
    CU(cudaMemcpy(a, s->mlp.audit, sizeof(a), cudaMemcpyDeviceToHost));
    if (max_err)
        for (int q = 0; q < 6; q++) max_err[q] = a[q];
    if (counts) {
        unsigned long long c[2];
        memcpy(&c[0], a + 6, 8);
        memcpy(&c[1], a + 8, 8);
        counts[0] = (long long)c[0];
        counts[1] = (long long)c[1];
    }
    return MG_OK;
}

}  // extern "C"

// ---- accessors for the batched form ---------------------------------------
Dev& mg::system_dev(mg_system* s) { return s->d; }
cudaStream_t mg::system_stream(mg_system* s) { return s->st; }
int mg::system_device(mg_system* s) { return s->device; }
void mg::system_shape(mg_system* s, int* style, int* nt, int* x_dim, int* form, double* B_out)
{
    if (style) *style = s->coef_set ? s->style : -1;
    if (nt) *nt = s->nt;
    if (x_dim) *x_dim = s->x_dim;
    if (form) *form = s->form;
    if (B_out)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) B_out[3 * i + j] = s->B[i][j];
}
double mg::system_skin(mg_system* s) { return s->skin; }
void mg::system_box(mg_system* s, double* H_out)
{
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) H_out[3 * i + j] = s->H[i][j];
}
int mg::system_natms(mg_system* s) { return s->natms; }
int mg::system_check_ready(mg_system* s)
{
    CHK(check_sys(s));
    if (!s->initialized) return fail(MG_ERR_STATE, "ff_init must run first");
    return MG_OK;
}
void mg::system_masses(mg_system* s, double* out)
{
    for (int t = 0; t < s->nt; t++) out[t] = t < (int)s->masses.size() ? s->masses[t] : 0.0;
}
int mg::system_rebuild(mg_system* s)
{
    if (s->natms == 0) return MG_OK;
    CU(launch_x2s(s->d, s->st));
    return rebuild(s);
}
int mg::system_enqueue_force(mg_system* s, int st_clc, int zero, int* rows)
{
    if (s->style != STYLE_EAM && s->style != STYLE_FS)
        return fail(MG_ERR_UNSUPPORTED, "the device MD loop drives EAM / FS force fields");
    Dev& d = s->d;
    if (zero) {
        CU(cudaMemsetAsync(d.f, 0, (size_t)s->natms * s->x_dim * sizeof(double), s->st));
        CU(cudaMemsetAsync(d.rho, 0, (size_t)s->natms * sizeof(double), s->st));
    }
    CU(s->style == STYLE_EAM ? launch_eam_force(d, st_clc, rows, s->st) : launch_fs_force(d, st_clc, rows, s->st));
    return MG_OK;
}
double* mg::system_red_out(mg_system* s) { return s->red_out; }
int mg::system_enqueue_calc_g(mg_system* s, int chk, double alpha, int* rows)
{
    if (!s->dmd) return fail(MG_ERR_UNSUPPORTED, "calc_g needs a DMD force field");
    if (!s->crd_built) return fail(MG_ERR_STATE, "create_2nd_neigh_lst must run before calc_g");
    CHK(ensure_pair_values(s));
    Dev& d = s->d;
    CU(cudaMemsetAsync(d.E, 0, (size_t)s->natms * s->nt * sizeof(double), s->st));
    CU(launch_dmd_calc_g(d, chk, alpha, rows, s->st));
    CU(launch_reduce_partials(d, *rows, 1, s->red_out, s->st));
    return MG_OK;
}
int mg::system_enqueue_calc_g_dev(mg_system* s, const int* chk_dev, const double* alpha_dev, int* rows)
{
    if (!s->dmd) return fail(MG_ERR_UNSUPPORTED, "calc_g needs a DMD force field");
    if (!s->crd_built) return fail(MG_ERR_STATE, "create_2nd_neigh_lst must run before calc_g");
    CHK(ensure_pair_values(s));
    Dev d = s->d;
    d.g_chk = chk_dev;
    d.g_alpha = alpha_dev;
    CU(cudaMemsetAsync(d.E, 0, (size_t)s->natms * s->nt * sizeof(double), s->st));
    CU(launch_dmd_calc_g(d, 0, 0.0, rows, s->st));
    CU(launch_reduce_partials(d, *rows, 1, s->red_out, s->st));
    return MG_OK;
}
int mg::system_set_active_pairs(mg_system* s, bool on)
{
    Dev& d = s->d;
    if (!on) {
        d.act_on = 0;
        return MG_OK;
    }
    if (!s->dmd || s->form != MG_FORM_FP64 || s->natms == 0) return MG_OK;
    if ((size_t)s->natms + 1 > s->nact_cap) {
        CHK(dalloc(&d.nact, (size_t)s->natms + 1));
        CHK(dalloc(&d.act_off, (size_t)s->natms + 1));
        s->nact_cap = (size_t)s->natms + 1;
    }
    d.act_on = 0;
    CHK(ensure_pair_values(s));
    CU(launch_active_count(d, s->st));
    CU(launch_exclusive_scan(d.nact, d.act_off, s->natms + 1, s->scan_tmp, s->scan_tmp_bytes, s->st));
    CU(cudaMemcpyAsync(&s->hp->count, d.act_off + s->natms, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    const int total = s->hp->count;
    const int nvals = s->nt * s->nt + s->nt * (s->nt + 1) / 2;
    if ((size_t)total + 1 > s->act_cap) {
        const size_t cap = (size_t)total + (size_t)total / 8 + 64;
        CHK(dalloc(&d.act_pj, cap));
        CHK(dalloc(&d.act_pv, cap * nvals));
        s->act_cap = cap;
    }
    d.act_cap = (long long)s->act_cap;
    CU(launch_active_fill(d, s->st));
    d.act_on = 1;
    return MG_OK;
}

int mg::system_enqueue_c_d(mg_system* s)
{
    if (!s->dmd) return fail(MG_ERR_UNSUPPORTED, "c_d_calc needs a DMD force field");
    if (!s->crd_built) return fail(MG_ERR_STATE, "create_2nd_neigh_lst must run before c_d_calc");
    CHK(ensure_pair_values(s));
    Dev& d = s->d;
    size_t bytes = (size_t)s->natms * s->nt * sizeof(double);
    CU(cudaMemsetAsync(d.E, 0, bytes, s->st));
    CU(cudaMemsetAsync(d.c_d, 0, bytes, s->st));
    CU(launch_dmd_cdot(d, s->st));
    return MG_OK;
}

// WriteCFG::write_file for the system's current owned state (the arrays
// writer, mg_cfg.cu, does the formatting)
extern "C" int mg_cfg_write(mg_system* s, const char* prefix, int step)
{
    CHK(check_sys(s));
    if (!s->initialized) return fail(MG_ERR_STATE, "ff_init must run before a CFG is written");
    const int n = s->natms, nt = s->nt;
    int name_len = 1;
    for (auto& nm : s->names) name_len = std::max(name_len, (int)nm.size() + 1);
    std::vector<char> names((size_t)nt * name_len, 0);
    for (int t = 0; t < nt; t++) memcpy(&names[(size_t)t * name_len], s->names[t].data(), s->names[t].size());
    std::vector<double> x((size_t)n * s->x_dim + 1), c;
    std::vector<int> type;
    double H[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) H[3 * i + j] = s->H[i][j];
    if (n > 0) {
        CHK(mg_atoms_get_x(s, x.data()));
        if (s->dmd) {
            c.resize((size_t)n * nt);
            CU(cudaMemcpyAsync(c.data(), s->d.c, c.size() * sizeof(double), cudaMemcpyDeviceToHost, s->st));
        } else {
            type.resize(n);
            CU(cudaMemcpyAsync(type.data(), s->d.type, n * sizeof(int), cudaMemcpyDeviceToHost, s->st));
        }
        CU(cudaStreamSynchronize(s->st));
    }
    return mg_cfg_write_arrays(prefix, step, s->dmd, n, nt, names.data(), name_len, s->masses.data(), H, x.data(),
                               s->dmd ? nullptr : type.data(), s->dmd ? c.data() : nullptr);
}
