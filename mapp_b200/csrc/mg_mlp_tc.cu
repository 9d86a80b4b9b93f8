// Learned form (MG_FORM_MLP) inside force_calc, on the 5th-generation tensor
// cores: the network of mg_mlp_common.cuh replaces the Gauss-Hermite smearing
// (ff_dmd_I.cpp:178-259) of every row (site pair, ordered species pair)
// inside its training box.
//
// k_mlp_rows classifies every row: rows beyond the smeared cut store zeros,
// rows inside the training box are appended to the front of the row list
// (and a hashed 1% of them to the audit list), pairs with rows outside it to
// the back.  k_mlp_fallback gives those rows the FP32 quadrature of the
// precision form, every lane on a fallback pair (no divergence against
// network rows).
// k_mlp_tc runs the network on the front rows, one tile of 128 rows per
// warpgroup at a time (persistent):
//   * thread t puts row t of the tile into the BF16 A operand of layer 1 in
//     shared memory (its TMEM lane is t);
//   * one thread issues the layer's tcgen05.mma instructions (M = 128,
//     N = 64, K = 16 each, BF16 operands from shared-memory descriptors, FP32
//     accumulator in TMEM) and commits them to an mbarrier;
//   * every thread reads its row's accumulators back with tcgen05.ld, adds
//     the bias, applies the activation and writes the BF16 row into the next
//     layer's A operand; layer 4 (N = 16, 6 used) gives the corrections, to
//     which the unsmeared spline values at r are added.
// The network runs on x = z / 8 (mg_mlp_common.cuh): inputs and biases of
// the hidden layers are stored divided by 8 and the output layer's scale
// multiplied by 8, all exact, so the activation needs no scaling.
// k_mlp_audit evaluates the audit list by the FP64 quadrature and records
// the largest deviation per output (mg_mlp_audit).
// Per-pair results go to the FP32 pair scratch in the precision form's
// layout; densities (k_mlp_densities), the embedding and pass 2 follow.
//
// Shared-memory operands use the canonical K-major layout without swizzle:
// 8-row x 16-byte core matrices, the two 8-element halves of a K = 16 step
// LBO bytes apart, consecutive 8-row groups SBO = 128 bytes apart.
// Every wait on the tensor core is bounded (200 ms of %globaltimer); a wait
// that runs out sets status[5], frees the CTA's TMEM and ends the CTA.
#include "mg_reduce.cuh"
#include "mg_dmd_common.cuh"
#include "mg_mlp_common.cuh"
#include "mg_split.cuh"

namespace mg {
namespace {

using namespace mlp;

constexpr int kTile = 128;     // rows per tile = M of the MMA = TMEM lanes
constexpr int kPipes = 4;      // independent tile pipelines per CTA, one per warpgroup
constexpr int kTcThreads = 128 * kPipes;
constexpr int kN4 = 16;        // output layer padded to N = 16
constexpr int kTmemCols = 64 * kPipes;  // accumulator columns: 64 (N of layers 1-3) per pipeline
constexpr unsigned long long kTcWaitNs = 200000000ull;

// byte offset of element (row, k) of a K-major operand with `rows` rows
__host__ __device__ constexpr int kmaj_off(int rows, int r, int k)
{
    return (((k >> 3) * (rows >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1);
}

struct TcSmem {
    __nv_bfloat16 w1[H * 16];   // B of layer 1: 64 rows (n) x 16 (k)
    __nv_bfloat16 w2[H * H];
    __nv_bfloat16 w3[H * H];
    __nv_bfloat16 w4[kN4 * H];  // 16 rows (n, 8..15 zero) x 64 (k)
    // per pipeline (warpgroup): layer 1's A operand and the activations (each
    // layer's epilogue overwrites the operand its own MMAs have finished reading)
    __nv_bfloat16 a0[kPipes][kTile * 16];
    __nv_bfloat16 a1[kPipes][kTile * H];
    float b1[H], b2[H], b3[H];  // biases / 8
    float s4[kN4], m4[kN4];     // output q = s4[q] acc + m4[q] (+ the spline base)
    unsigned long long bar[kPipes];  // mbarriers of MMA completion
    unsigned int tmem_base;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t start, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1, no swizzle, base offset 0
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n
__device__ __forceinline__ uint32_t idesc_bf16(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTile >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ unsigned long long gtime()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bounded wait for phase `parity` of the mbarrier; false when it runs out.
// try_wait with a suspend-time hint parks the thread until the phase
// completes (or 100 us pass), so a waiting warp issues almost nothing and
// leaves the issue slots to the other pipelines of the SM.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    const unsigned long long t0 = gtime();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity), "r"(100000u)
            : "memory");
        if (ok) return true;
        if (gtime() - t0 > kTcWaitNs) return false;
    }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 / 64 FP32 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

// one layer's epilogue for this thread's row: bias + activation of 64
// accumulators (x = z / 8), 16 columns per TMEM load, BF16 into the K-major
// A operand `a` of the next layer
template <int ACT>
__device__ __forceinline__ void epilogue64(uint32_t taddr, const float* __restrict__ bias, __nv_bfloat16* a, int row)
{
#pragma unroll
    for (int c = 0; c < 4; c++) {
        float v[16];
        tmem_ld16(taddr + 16 * c, v);
        uint32_t w[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int col = 16 * c + 2 * k;
            w[k] = pack2f(gx<ACT>(col, v[2 * k] + bias[col]), gx<ACT>(col + 1, v[2 * k + 1] + bias[col + 1]));
        }
        *reinterpret_cast<uint4*>(reinterpret_cast<char*>(a) + kmaj_off(kTile, row, 16 * c)) =
            make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4*>(reinterpret_cast<char*>(a) + kmaj_off(kTile, row, 16 * c + 8)) =
            make_uint4(w[4], w[5], w[6], w[7]);
    }
}

// named barrier of one warpgroup (ids 1.. so that __syncthreads's 0 stays free)
__device__ __forceinline__ void wg_sync(int wg) { asm volatile("bar.sync %0, 128;" ::"r"(1 + wg) : "memory"); }
__device__ __forceinline__ bool wg_sync_or(int wg, bool v)
{
    uint32_t out;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, %2, 128, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(out)
        : "r"((uint32_t)v), "r"(1 + wg)
        : "memory");
    return out != 0;
}

// the six outputs of one row into the pair scratch (precision form layout)
template <int NT>
__device__ __forceinline__ void store_row(const Dev& d, long long p, int a, int b, const float (&o)[6])
{
    using SL = Slots<NT>;
    const size_t mp = (size_t)d.maxp;
    float* out = d.prf + p;
    const int rs = b * NT + a, ps = comp_idx(a, b);
    out[(SL::RHO + rs) * mp] = o[1];
    out[(SL::DRR + rs) * mp] = o[3];
    out[(SL::DRA + rs) * mp] = o[5];
    if (a >= b) {
        out[(SL::PHI + ps) * mp] = o[0];
        out[(SL::DPR + ps) * mp] = o[2];
        out[(SL::DPA + ps) * mp] = o[4];
    }
}

// species pair in the ordering the network was trained on for (a, b): the
// cross pair is always (1, 0)
__device__ __forceinline__ void trained_order(int a, int b, int& aa, int& bb)
{
    aa = (a == b) ? a : 1;
    bb = (a == b) ? b : 0;
}

// Row (pair p, species a, b): 0 beyond the smeared cut, 1 inside the training
// box (network; normalised inputs in `in`), 2 outside it (quadrature).
template <int NT>
__device__ __forceinline__ int classify(const Dev& d, const MlpState& S, const F32Consts& kc, long long p, int a,
                                        int b, float4& in, float& r, float& alpha, bool& below_rc)
{
    const int i = d.pair_i[p], j = d.pair_j[p];
    const double4 xi = d.pos[i], xj = d.pos[j];
    const double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
    const double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
    if (!(rsq < d.cut_sq_mod)) return 0;
    const float ai = (float)d.alpha[(size_t)i * NT + a], aj = (float)d.alpha[(size_t)j * NT + b];
    alpha = (ai * aj) / (ai + aj);
    r = sqrtf((float)rsq);
    below_rc = rsq < d.cut_sq;
    const float wi = rsqrtf(ai), wj = rsqrtf(aj);
    const int code = NT == 1 ? 0 : (a == b ? 2 * a : 1);
    const bool inbox = r >= S.box.r_lo && r <= S.box.r_hi && wi >= S.box.w_lo && wi <= S.box.w_hi &&
                       wj >= S.box.w_lo && wj <= S.box.w_hi && alpha > kc.alpha_min && alpha < kc.alpha_max;
    if (!inbox) return 2;
    float v[4];
    net_inputs(S.box, r, wi, wj, code, v);
    in = make_float4(v[0], v[1], v[2], v[3]);
    return 1;
}

// unsmeared spline values at r of the trained ordering (aa, bb), FP32 from
// the split table (the base the network's corrections are added to)
template <int NT>
__device__ __forceinline__ void base_f32(const Dev& d, int aa, int bb, float r, float (&o)[6])
{
    const float dr_inv = d.drS_inv;
    const float pp = fminf(r * dr_inv, (float)(d.nrS - 1));
    const int m = (int)pp;
    const float t = pp - (float)m;
    const float4 cr = __ldg(d.pkS + (size_t)(aa * NT + bb) * d.nrS + m);
    const float4 cp = __ldg(d.pkS + (size_t)(NT * NT + comp_idx(aa, bb)) * d.nrS + m);
    const float z2 = fmaf(fmaf(fmaf(cp.w, t, cp.z), t, cp.y), t, cp.x);
    const float z2p = fmaf(fmaf(3.0f * cp.w, t, 2.0f * cp.z), t, cp.y) * dr_inv;
    const float r_inv = 1.0f / r;
    o[0] = z2 * r_inv;
    o[1] = fmaf(fmaf(fmaf(cr.w, t, cr.z), t, cr.y), t, cr.x);
    o[2] = (z2p - z2 * r_inv) * r_inv;
    o[3] = fmaf(fmaf(3.0f * cr.w, t, 2.0f * cr.z), t, cr.y) * dr_inv;
    o[4] = 0.0f;
    o[5] = 0.0f;
}

// B operand of one layer: element (n, k) = W[k][n] of the row-major [K][N]
// weights (n >= nsrc zero)
__device__ __forceinline__ void load_b(__nv_bfloat16* dst, const __nv_bfloat16* __restrict__ w, int rows, int nsrc,
                                       int K)
{
    for (int e = threadIdx.x; e < rows * K; e += blockDim.x) {
        const int n = e / K, k = e - n * K;
        const __nv_bfloat16 v = n < nsrc ? w[(size_t)k * nsrc + n] : __float2bfloat16(0.0f);
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(dst) + kmaj_off(rows, n, k)) = v;
    }
}

// MMAs of one layer: D[128 x N] (TMEM) = A[128 x K] B^T, K = 16 ksteps
__device__ __forceinline__ void issue_layer(uint32_t tmem, const __nv_bfloat16* a, const __nv_bfloat16* b, int n,
                                            int ksteps)
{
    const uint32_t sa = smem_u32(a), sb = smem_u32(b);
    const uint32_t lbo_a = (kTile / 8) * 128, lbo_b = (uint32_t)(n / 8) * 128;
    const uint32_t id = idesc_bf16(n);
    for (int s = 0; s < ksteps; s++)
        umma(tmem, umma_desc(sa + 2 * s * lbo_a, lbo_a, 128), umma_desc(sb + 2 * s * lbo_b, lbo_b, 128), id,
             s > 0 ? 1u : 0u);
}

// ---- the rows: classification and the row lists ---------------------------
// 1% audit selection of network row (pair p, species pair ab)
__device__ __forceinline__ bool audited(unsigned long long seed, long long p, int ab, int rp)
{
    return (mix64(seed ^ ((unsigned long long)p * rp + (unsigned long long)ab)) >> 40) % 100 == 0;
}

// One thread per listed pair: a pair beyond the smeared cut stores zero
// densities and pair energies; of an in-cut pair's NT^2 rows (ordered species
// pairs), those inside the training box go to the front of the row list (one
// atomic per block and round); a pair with rows outside it goes to the back
// with the mask of those rows (one atomic per warp and round).
template <int NT>
__global__ void __launch_bounds__(kFFBlock) k_mlp_rows(Dev d, MlpState S, unsigned long long audit_seed)
{
    using SL = Slots<NT>;
    constexpr int RP = NT * NT;
    __shared__ int warp_n[kFFWarps];
    __shared__ unsigned blk_base;
    // a warp's network rows of one round, in slot order, so that they leave
    // for the row list with coalesced stores
    __shared__ float4 st_in[kFFWarps][32 * RP];
    __shared__ int2 st_id[kFFWarps][32 * RP];
    __shared__ float st_r[kFFWarps][32 * RP];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const SplitK k = split_consts(d);
    const size_t mp = (size_t)d.maxp;
    for (long long base = (long long)blockIdx.x * kFFBlock; base < d.npairs; base += (long long)gridDim.x * kFFBlock) {
        const long long p = base + threadIdx.x;
        unsigned net = 0, fb = 0;  // bit ab: row (a, b) goes through the network / the quadrature
        float4 in[RP];
        float r = 0.f;
        if (p < d.npairs) {
            const int i = d.pair_i[p], j = d.pair_j[p];
            const double4 xi = d.pos[i], xj = d.pos[j];
            const double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
            const double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
            if (!(rsq < d.cut_sq_mod)) {
                float* out = d.prf + p;
#pragma unroll
                for (int q = 0; q < NT * NT; q++) out[(SL::RHO + q) * mp] = 0.0f;
#pragma unroll
                for (int q = 0; q < SL::NC; q++) out[(SL::PHI + q) * mp] = 0.0f;
            } else {
                const float rsqf = (float)rsq;
                r = rsqf * rsqrtf(rsqf);
                float ai[NT], aj[NT];
#pragma unroll
                for (int a = 0; a < NT; a++) {
                    ai[a] = (float)d.alpha[(size_t)i * NT + a];
                    aj[a] = (float)d.alpha[(size_t)j * NT + a];
                }
#pragma unroll
                for (int a = 0; a < NT; a++)
#pragma unroll
                    for (int b = 0; b < NT; b++) {
                        const int ab = a * NT + b;
                        const float alpha = __fdividef(ai[a] * aj[b], ai[a] + aj[b]);
                        const float wi = rsqrtf(ai[a]), wj = rsqrtf(aj[b]);
                        const bool inbox = r >= S.box.r_lo && r <= S.box.r_hi && wi >= S.box.w_lo &&
                                           wi <= S.box.w_hi && wj >= S.box.w_lo && wj <= S.box.w_hi &&
                                           alpha > k.alpha_min && alpha < k.alpha_max;
                        if (inbox) {
                            float v[4];
                            net_inputs(S.box, r, wi, wj, NT == 1 ? 0 : (a == b ? 2 * a : 1), v);
                            in[ab] = make_float4(v[0] * kSigInvZ, v[1] * kSigInvZ, v[2] * kSigInvZ, v[3] * kSigInvZ);
                            net |= 1u << ab;
                        } else
                            fb |= 1u << ab;
                    }
            }
        }
        // pairs with fallback rows: the back of the list, (pair, row mask), one
        // atomic per warp
        {
            const int cnt = fb ? 1 : 0;
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const int tot = __shfl_sync(0xffffffffu, incl, 31);
            unsigned wbase = 0;
            if (lane == 31 && tot) wbase = atomicAdd(S.row_n + 2, (unsigned)tot);
            wbase = __shfl_sync(0xffffffffu, wbase, 31);
            const long long slot = (long long)wbase + incl - cnt;
            if (cnt) {
                if (slot < S.row_cap) S.row_id[S.row_cap - 1 - slot] = make_int2((int)p, (int)fb);
                else d.status[5] = 2;
            }
        }
        // network rows: block-wide slots at the front, one atomic per block
        const int cnt = __popc(net);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_n[warp] = incl;
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int w = 0; w < kFFWarps; w++) {
                const int c = warp_n[w];
                warp_n[w] = tot;
                tot += c;
            }
            blk_base = tot ? atomicAdd(S.row_n, (unsigned)tot) : 0u;
        }
        __syncthreads();
        int q = incl - cnt;  // this lane's first row in the warp's staging
#pragma unroll
        for (int ab = 0; ab < RP; ab++)
            if (net >> ab & 1u) {
                st_in[warp][q] = in[ab];
                st_id[warp][q] = make_int2((int)p, ab);
                st_r[warp][q] = r;
                q++;
            }
        __syncwarp();
        const int wtot = __shfl_sync(0xffffffffu, incl, 31);
        const long long wbase = (long long)blk_base + warp_n[warp];
        for (int e = lane; e < wtot; e += 32) {
            const long long slot = wbase + e;
            if (slot < S.row_cap) {
                const int2 id = st_id[warp][e];
                S.row_in[slot] = st_in[warp][e];
                S.row_id[slot] = id;
                S.row_r[slot] = st_r[warp][e];
                if (audited(audit_seed, id.x, id.y, RP)) {
                    const unsigned ka = atomicAdd(S.row_n + 1, 1u);
                    if (ka < S.audit_cap) S.audit_rows[ka] = (int)slot;
                }
            } else
                d.status[5] = 2;
        }
        __syncthreads();
    }
}

// The fallback rows (back of the row list: pair, mask of its fallback rows):
// the FP32 quadrature of the precision form (split table), one pair per
// thread.
template <int NT, int NQ>
__global__ void __launch_bounds__(kFFBlock) k_mlp_fallback(Dev d, MlpState S)
{
    // the split table in shared memory, as the precision form's force pass has it
    extern __shared__ float4 tab[];
    load_split_table(d, tab, NT * NT + Slots<NT>::NC);
    const SplitK k = split_consts(d);
    const long long nfb = min((long long)S.row_n[2], S.row_cap);
    unsigned long long nrows = 0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nfb; e += (long long)gridDim.x * blockDim.x) {
        const int2 id = S.row_id[S.row_cap - 1 - e];
        const long long p = id.x;
        const int i = d.pair_i[p], j = d.pair_j[p];
        const double4 xi = d.pos[i], xj = d.pos[j];
        const double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
        const double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
        const float rsqf = (float)rsq;
        const float r_inv = rsqrtf(rsqf);
        const float r = rsqf * r_inv;
        const bool below_rc = rsq < d.cut_sq;
        const Knot k0 = knot_at(r, k);
        float ai[NT], aj[NT];
#pragma unroll
        for (int a = 0; a < NT; a++) {
            ai[a] = (float)d.alpha[(size_t)i * NT + a];
            aj[a] = (float)d.alpha[(size_t)j * NT + a];
        }
#pragma unroll
        for (int a = 0; a < NT; a++)
#pragma unroll
            for (int b = 0; b < NT; b++) {
                const int ab = a * NT + b;
                if (!(id.y >> ab & 1)) continue;
                const float alpha = __fdividef(ai[a] * aj[b], ai[a] + aj[b]);
                const float4* tr = tab + (size_t)ab * d.nrS;
                const float4* tp = tab + (size_t)(NT * NT + comp_idx(a, b)) * d.nrS;
                VDer g, f;
                if (a >= b) smear_full<NQ, true, false>(d, tr, tp, k, r, r_inv, below_rc, alpha, k0, g, f);
                else smear_full<NQ, false, false>(d, tr, tp, k, r, r_inv, below_rc, alpha, k0, g, f);
                const float o[6] = {f.v, g.v, f.dr, g.dr, f.da, g.da};
                store_row<NT>(d, p, a, b, o);
                nrows++;
            }
    }
    for (int off = 16; off > 0; off >>= 1) nrows += __shfl_xor_sync(0xffffffffu, nrows, off);
    if ((threadIdx.x & 31) == 0 && nrows) atomicAdd(reinterpret_cast<unsigned long long*>(S.audit + 8), nrows);
}

// ---- the network on the listed rows, 128 at a time -------------------------
// Two warpgroups per CTA, each an independent tile pipeline (its own A
// operands, mbarrier, TMEM columns and named barrier) over the shared weight
// operands, so one pipeline's MMAs run while the other's epilogue computes.
template <int NT, int ACT>
__global__ void __launch_bounds__(kTcThreads, 2) k_mlp_tc(Dev d, MlpState S)
{
    extern __shared__ __align__(1024) unsigned char smraw[];
    TcSmem& T = *reinterpret_cast<TcSmem*>(smraw);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int wg = tid >> 7, row = tid & (kTile - 1);  // pipeline and tile row (= TMEM lane)

    // ---- set-up: operands of the weights, biases, barriers, TMEM ------------
    load_b(T.w1, S.wbf + OW1, H, H, 16);
    load_b(T.w2, S.wbf + OW2, H, H, H);
    load_b(T.w3, S.wbf + OW3, H, H, H);
    load_b(T.w4, S.wbf + OW4, kN4, 8, H);
    for (int k = tid; k < H; k += kTcThreads) {
        T.b1[k] = S.par[OB1 + k] * kSigInvZ;
        T.b2[k] = S.par[OB2 + k] * kSigInvZ;
        T.b3[k] = S.par[OB3 + k] * kSigInvZ;
    }
    // y = W4 silu(z3) + b4 = 8 W4 g3 + b4; output = y scale + mean
    if (tid < kN4) {
        T.s4[tid] = tid < 6 ? kSigZ * S.out_scale[tid] : 0.0f;
        T.m4[tid] = tid < 6 ? fmaf(S.par[OB4 + tid], S.out_scale[tid], S.out_mean[tid]) : 0.0f;
    }
    // layer 1's K = 16 columns: the 4 inputs, then zeros (the second 8-column
    // half is never rewritten)
    for (int e = tid; e < kPipes * kTile * 16; e += kTcThreads) (&T.a0[0][0])[e] = __float2bfloat16(0.0f);
    if (tid < kPipes) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&T.bar[tid])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&T.tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    async_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = T.tmem_base + 64u * wg;                     // this pipeline's columns
    const uint32_t tlane = tmem + ((uint32_t)((warp & 3) * 32) << 16);  // this warp's lanes
    const uint32_t bar = smem_u32(&T.bar[wg]);
    __nv_bfloat16* a0 = T.a0[wg];
    __nv_bfloat16* a1 = T.a1[wg];

    uint32_t phase = 0;
    bool failed = false;
    const long long nrows = min((long long)*S.row_n, S.row_cap);
    const long long ntiles = (nrows + kTile - 1) / kTile;

    // one tensor-core step of this pipeline: MMAs issued by its first thread,
    // committed, waited for by the warpgroup
    auto mma_step = [&](const __nv_bfloat16* a, const __nv_bfloat16* b, int n, int ksteps) -> bool {
        async_fence();
        tc_fence_before();
        wg_sync(wg);
        if (row == 0) {
            tc_fence_after();
            issue_layer(tmem, a, b, n, ksteps);
            umma_commit(bar);
        }
        const bool ok = mbar_wait(bar, phase & 1u);
        phase++;
        if (wg_sync_or(wg, !ok)) return false;
        tc_fence_after();
        return true;
    };

    long long t = (long long)blockIdx.x * kPipes + wg;
    const long long tstride = (long long)gridDim.x * kPipes;
    // this thread's row of the next tile, loaded one tile ahead
    long long rw = t * kTile + row;
    float4 in = rw < nrows ? __ldg(S.row_in + rw) : make_float4(0.f, 0.f, 0.f, 0.f);
    int2 id = rw < nrows ? __ldg(S.row_id + rw) : make_int2(-1, 0);
    float rr = rw < nrows ? __ldg(S.row_r + rw) : 1.0f;
    for (; t < ntiles; t += tstride) {
        const bool on = rw < nrows;
        const int2 cid = id;
        const float cr = rr;
        *reinterpret_cast<uint4*>(reinterpret_cast<char*>(a0) + kmaj_off(kTile, row, 0)) =
            make_uint4(pack2f(in.x, in.y), pack2f(in.z, in.w), 0u, 0u);
        rw = (t + tstride) * kTile + row;
        if (rw < nrows) {
            in = __ldg(S.row_in + rw);
            id = __ldg(S.row_id + rw);
            rr = __ldg(S.row_r + rw);
        }
        if (!mma_step(a0, T.w1, H, 1)) { failed = true; break; }
        epilogue64<ACT>(tlane, T.b1, a1, row);
        if (!mma_step(a1, T.w2, H, H / 16)) { failed = true; break; }
        epilogue64<ACT>(tlane, T.b2, a1, row);
        if (!mma_step(a1, T.w3, H, H / 16)) { failed = true; break; }
        epilogue64<ACT>(tlane, T.b3, a1, row);
        if (!mma_step(a1, T.w4, kN4, H / 16)) { failed = true; break; }
        float y[16];
        tmem_ld16(tlane, y);
        if (on) {
            const long long p = cid.x;
            const int a = cid.y / NT, b = cid.y - (cid.y / NT) * NT;
            int aa, bb;
            trained_order(a, b, aa, bb);
            float base[6], o[6];
            base_f32<NT>(d, aa, bb, cr, base);
#pragma unroll
            for (int q = 0; q < 6; q++) o[q] = fmaf(y[q], T.s4[q], T.m4[q]) + base[q];
            store_row<NT>(d, p, a, b, o);
        }
    }
    // ---- tear-down: TMEM back ---------------------------------------------------
    if (failed && row == 0) d.status[5] = 1;
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(T.tmem_base), "r"(kTmemCols)
                     : "memory");
}

// ---- the 1% audit: network rows against the FP64 quadrature ----------------
// The audit list (a hashed 1% of the network rows, chosen by k_mlp_rows) is
// evaluated by the FP64 quadrature and compared with what the network
// stored; the largest deviation per output and the number of audited rows go
// to MlpState::audit.
template <int NT, int NQ>
__global__ void __launch_bounds__(kFFBlock) k_mlp_audit(Dev d, MlpState S)
{
    using SL = Slots<NT>;
    const int lane = threadIdx.x & 31;
    const F32Consts kc = f32_consts(d);
    const long long na = min((long long)S.row_n[1], S.audit_cap);
    const size_t mp = (size_t)d.maxp;
    if (blockIdx.x == 0 && threadIdx.x == 0) *reinterpret_cast<unsigned long long*>(S.audit + 6) = (unsigned long long)na;
    float audit_err[6] = {0, 0, 0, 0, 0, 0};
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < na; e += (long long)gridDim.x * blockDim.x) {
        const int2 id = S.row_id[S.audit_rows[e]];
        const long long p = id.x;
        const int a = id.y / NT, b = id.y - (id.y / NT) * NT;
        int aa, bb;
        trained_order(a, b, aa, bb);
        float4 in;
        float r = 0.f, alpha = 0.f;
        bool brc = false;
        classify<NT>(d, S, kc, p, a, b, in, r, alpha, brc);
        double g0 = 0, gdr = 0, gda = 0, f0 = 0, fdr = 0, fda = 0;
        const double r64 = r;
        if (!smear<true, true, NQ>(d, bb * NT + aa, comp_idx(aa, bb), r64, 1.0 / r64, r64 * r64, (double)alpha, g0,
                                   gdr, gda, f0, fdr, fda))
            g0 = gdr = gda = f0 = fdr = fda = 0.0;
        const float* out = d.prf + p;
        const int rs = b * NT + a, ps = comp_idx(a, b);
        const double qv[6] = {f0, g0, fdr, gdr, fda, gda};
        const float o[6] = {out[(SL::PHI + ps) * mp], out[(SL::RHO + rs) * mp], out[(SL::DPR + ps) * mp],
                            out[(SL::DRR + rs) * mp], out[(SL::DPA + ps) * mp], out[(SL::DRA + rs) * mp]};
        // a < b rows store no phi slots of their own (those are the (b, a) row's)
        const int nq = a >= b ? 6 : 0;
#pragma unroll
        for (int q = 0; q < 6; q++)
            if (q & 1 || q < nq) audit_err[q] = fmaxf(audit_err[q], fabsf((float)(qv[q] - o[q])));
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
        float e = audit_err[q];
        for (int off = 16; off > 0; off >>= 1) e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, off));
        if (lane == 0 && e > 0.f) atomicMax(reinterpret_cast<unsigned int*>(S.audit) + q, __float_as_uint(e));
    }
}

// Densities E and pair energy from the pair scratch the learned pass wrote
// (ff_dmd_I.cpp:196-259 sums): one thread per compact pair, i-side sums by
// segmented shuffles, one FP64 atomic per site run and per owned j.
template <int NT>
__global__ void __launch_bounds__(kFFBlock, 4) k_mlp_densities(Dev d, int row0)
{
    using SL = Slots<NT>;
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const size_t mp = (size_t)d.maxp;
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
            const bool own_j = j < d.natms;
            const double w = own_j ? 0.5 : 0.25;
            double ci[NT], cj[NT], Ej[NT];
#pragma unroll
            for (int a = 0; a < NT; a++) {
                ci[a] = d.c[(size_t)i * NT + a];
                cj[a] = d.c[(size_t)j * NT + a];
                Ej[a] = 0.0;
            }
            const float* in = d.prf + p;
#pragma unroll
            for (int a = 0; a < NT; a++)
#pragma unroll
                for (int b = 0; b < NT; b++) {
                    const double g0 = (double)__ldg(in + (SL::RHO + b * NT + a) * mp);
                    Ei[a] += g0 * cj[b];
                    Ej[b] += g0 * ci[a];
                    if (a >= b)
                        acc[0] += w * (cj[b] * ci[a] + cj[a] * ci[b]) * (double)__ldg(in + (SL::PHI + comp_idx(a, b)) * mp);
                }
            if (own_j)
#pragma unroll
                for (int b = 0; b < NT; b++)
                    if (Ej[b] != 0.0) atomicAdd(&d.E[(size_t)j * NT + b], Ej[b]);
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

template <int NT, int ACT>
cudaError_t mlp_force_nt(const Dev& d, const MlpState& S, unsigned long long audit_seed, int st_clc, int* nb,
                         cudaStream_t st, cudaEvent_t* evs)
{
    if (!S.row_in || !S.row_id || !S.row_r || !S.row_n || !S.audit_rows || S.row_cap < d.npairs * NT * NT)
        return cudaErrorInvalidValue;
    const size_t sm = sizeof(TcSmem);
    static int attr_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev != dev) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_tc<NT, ACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_mlp_tc<NT, ACT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
        attr_dev = dev;
    }
    // every resident CTA (the tile count is only known on the device): two
    // per SM when their shared memory and registers fit (TMEM holds two
    // 256-column allocations), from the kernel's own attributes
    static int per_sm = 0;
    if (!per_sm) {
        cudaFuncAttributes fa;
        int smem_sm = 0;
        if (cudaFuncGetAttributes(&fa, k_mlp_tc<NT, ACT>) != cudaSuccess ||
            cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess)
            return cudaErrorInvalidConfiguration;
        const long long per_cta_smem = (long long)sm + fa.sharedSizeBytes + 1024;  // + the driver's reserve
        const int by_smem = (int)(smem_sm / per_cta_smem), by_regs = 65536 / (fa.numRegs * kTcThreads);
        per_sm = std::max(1, std::min(2, std::min(by_smem, by_regs)));
    }
    const int g1 = num_sms() * per_sm;
    const int g0 = (int)std::min<long long>((d.npairs + kFFBlock - 1) / kFFBlock, (long long)num_sms() * 8);
    const bool nq3 = d.nq == 3 && d.xi_f[1] == 0.0f;
    const int gd = persistent_grid(d.npairs, 4);
    cudaError_t e = cudaMemsetAsync(S.row_n, 0, 4 * sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    if (evs) cudaEventRecord(evs[0], st);
    k_mlp_rows<NT><<<std::max(g0, 1), kFFBlock, 0, st>>>(d, S, audit_seed);
    const size_t smF = (size_t)(NT * NT + NT * (NT + 1) / 2) * d.nrS * sizeof(float4);
    if (smF > 48 * 1024) {
        e = cudaFuncSetAttribute(nq3 ? k_mlp_fallback<NT, 3> : k_mlp_fallback<NT, 0>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smF);
        if (e != cudaSuccess) return e;
    }
    if (nq3) k_mlp_fallback<NT, 3><<<num_sms() * 4, kFFBlock, smF, st>>>(d, S);
    else k_mlp_fallback<NT, 0><<<num_sms() * 4, kFFBlock, smF, st>>>(d, S);
    k_mlp_tc<NT, ACT><<<g1, kTcThreads, sm, st>>>(d, S);
    if (d.nq == 3) k_mlp_audit<NT, 3><<<num_sms(), kFFBlock, 0, st>>>(d, S);
    else k_mlp_audit<NT, 0><<<num_sms(), kFFBlock, 0, st>>>(d, S);
    k_mlp_densities<NT><<<gd, kFFBlock, 0, st>>>(d, 0);
    if (evs) cudaEventRecord(evs[1], st);
    int rows = 0;
    e = launch_dmd_force_f32_after_pass1(d, st_clc, gd, &rows, st, evs);
    *nb = gd + rows;
    return e;
}

}  // namespace

cudaError_t launch_dmd_force_mlp(const Dev& d, const MlpState& S, unsigned long long audit_seed, int st_clc, int* nb,
                                 cudaStream_t st, cudaEvent_t* evs)
{
    if (d.npairs > 2147483647LL / 4) return cudaErrorInvalidValue;  // queued rows keep the pair index in an int
    if (d.nt == 1) return S.act == 2   ? mlp_force_nt<1, 2>(d, S, audit_seed, st_clc, nb, st, evs)
                          : S.act == 1 ? mlp_force_nt<1, 1>(d, S, audit_seed, st_clc, nb, st, evs)
                                       : mlp_force_nt<1, 0>(d, S, audit_seed, st_clc, nb, st, evs);
    if (d.nt == 2) return S.act == 2   ? mlp_force_nt<2, 2>(d, S, audit_seed, st_clc, nb, st, evs)
                          : S.act == 1 ? mlp_force_nt<2, 1>(d, S, audit_seed, st_clc, nb, st, evs)
                                       : mlp_force_nt<2, 0>(d, S, audit_seed, st_clc, nb, st, evs);
    return cudaErrorInvalidValue;
}

}  // namespace mg
