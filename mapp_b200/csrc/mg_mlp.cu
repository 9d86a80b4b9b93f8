// Learned form (MG_FORM_MLP), training side: a 4 -> 64 -> 64 -> 64 -> 6
// network (activation silu_p, mg_mlp_common.cuh) learns the correction that
// the DMD Gauss-Hermite smearing (ff_dmd_I.cpp:178-259) adds to the unsmeared
// spline values of phi, rho and their r / alpha derivatives.  Inputs (r, w_i,
// w_j, species pair) with w = alpha^-1/2; outputs (phi, rho, dphi/dr,
// drho/dr, dphi/dalpha, drho/dalpha) of the pair exponent
// alpha = alpha_i alpha_j / (alpha_i + alpha_j), minus their unsmeared values.
//
// Everything runs in this library's own kernels:
//   * k_mlp_labels  -- training samples drawn from a counter-based hash RNG,
//     labelled by the FP64 quadrature of the loaded tables minus the FP64
//     unsmeared spline values;
//   * k_mlp_train   -- one 64-row tile per CTA: forward and backward with
//     BF16 tensor-core MMAs (mma.sync m16n8k16, FP32 accumulation), weight
//     gradients written as per-CTA partials;
//   * k_mlp_adam    -- sums the partials, Adam with a cosine learning rate,
//     refreshes the BF16 weight copy.
// Deployment inside force_calc is mg_mlp_tc.cu (tcgen05 tensor cores, TMEM
// accumulators).
// Species pairs: code 0 = (0,0), 1 = the unordered cross pair, 2 = (1,1); the
// cross code uses one network for (0,1) and (1,0), which needs rho_AB =
// rho_BA (true for the potentials this form is trained on).
#include <cmath>
#include <cstdint>
#include <cuda_bf16.h>

#include "mg_reduce.cuh"
#include "mg_dmd_common.cuh"
#include "mg_mlp_common.cuh"

namespace mg {
namespace {

using namespace mlp;

constexpr int kRows = 64;       // rows per tile
constexpr int kMlpThreads = 128;

__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Warp-tiled product out(m, n) = sum_k A(m, k) B(k, n) over M x N x K (multiples
// of 16, 8, 16).  A and B are accessors returning bf16; out receives FP32.
// The warps of the CTA split the 16x8 output tiles.
template <int M, int N, int K, class FA, class FB, class FO>
__device__ __forceinline__ void cta_gemm(const FA& A, const FB& B, const FO& out)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int nwarps = blockDim.x >> 5;
    constexpr int TN = N / 8, NTILE = (M / 16) * TN;
    for (int tile = warp; tile < NTILE; tile += nwarps) {
        const int m0 = (tile / TN) * 16, n0 = (tile % TN) * 8;
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k0 = 0; k0 < K; k0 += 16) {
            uint32_t a[4], b[2];
            a[0] = pack2(A(m0 + g, k0 + 2 * t), A(m0 + g, k0 + 2 * t + 1));
            a[1] = pack2(A(m0 + g + 8, k0 + 2 * t), A(m0 + g + 8, k0 + 2 * t + 1));
            a[2] = pack2(A(m0 + g, k0 + 2 * t + 8), A(m0 + g, k0 + 2 * t + 9));
            a[3] = pack2(A(m0 + g + 8, k0 + 2 * t + 8), A(m0 + g + 8, k0 + 2 * t + 9));
            b[0] = pack2(B(k0 + 2 * t, n0 + g), B(k0 + 2 * t + 1, n0 + g));
            b[1] = pack2(B(k0 + 2 * t + 8, n0 + g), B(k0 + 2 * t + 9, n0 + g));
            mma16816(c, a, b);
        }
        out(m0 + g, n0 + 2 * t, c[0]);
        out(m0 + g, n0 + 2 * t + 1, c[1]);
        out(m0 + g + 8, n0 + 2 * t, c[2]);
        out(m0 + g + 8, n0 + 2 * t + 1, c[3]);
    }
}


// shared-memory image of one tile's forward state
struct Tile {
    __nv_bfloat16 x[kRows][16];
    __nv_bfloat16 h[3][kRows][H];
    float z[3][kRows][H];
    float y[kRows][8];
    __nv_bfloat16 w1[16][H], w2[H][H], w3[H][H], w4[H][8];
    float b1[H], b2[H], b3[H], b4[8];
};

// the weights, BF16 for the MMAs, biases FP32
__device__ void load_weights(Tile& T, const __nv_bfloat16* __restrict__ wbf, const float* __restrict__ par)
{
    for (int k = threadIdx.x; k < 16 * H; k += blockDim.x) (&T.w1[0][0])[k] = wbf[OW1 + k];
    for (int k = threadIdx.x; k < H * H; k += blockDim.x) {
        (&T.w2[0][0])[k] = wbf[OW2 + k];
        (&T.w3[0][0])[k] = wbf[OW3 + k];
    }
    for (int k = threadIdx.x; k < H * 8; k += blockDim.x) (&T.w4[0][0])[k] = wbf[OW4 + k];
    for (int k = threadIdx.x; k < H; k += blockDim.x) {
        T.b1[k] = par[OB1 + k];
        T.b2[k] = par[OB2 + k];
        T.b3[k] = par[OB3 + k];
    }
    if (threadIdx.x < 8) T.b4[threadIdx.x] = par[OB4 + threadIdx.x];
}

// forward pass of the tile (T.x filled); leaves z, h and y in shared memory
__device__ void forward(Tile& T, int act)
{
    cta_gemm<kRows, H, 16>([&](int m, int k) { return T.x[m][k]; }, [&](int k, int n) { return T.w1[k][n]; },
                           [&](int m, int n, float v) { T.z[0][m][n] = v + T.b1[n]; });
    __syncthreads();
    for (int e = threadIdx.x; e < kRows * H; e += blockDim.x) (&T.h[0][0][0])[e] = __float2bfloat16(act_rt(act, e & (H - 1), (&T.z[0][0][0])[e]));
    __syncthreads();
    cta_gemm<kRows, H, H>([&](int m, int k) { return T.h[0][m][k]; }, [&](int k, int n) { return T.w2[k][n]; },
                          [&](int m, int n, float v) { T.z[1][m][n] = v + T.b2[n]; });
    __syncthreads();
    for (int e = threadIdx.x; e < kRows * H; e += blockDim.x) (&T.h[1][0][0])[e] = __float2bfloat16(act_rt(act, e & (H - 1), (&T.z[1][0][0])[e]));
    __syncthreads();
    cta_gemm<kRows, H, H>([&](int m, int k) { return T.h[1][m][k]; }, [&](int k, int n) { return T.w3[k][n]; },
                          [&](int m, int n, float v) { T.z[2][m][n] = v + T.b3[n]; });
    __syncthreads();
    for (int e = threadIdx.x; e < kRows * H; e += blockDim.x) (&T.h[2][0][0])[e] = __float2bfloat16(act_rt(act, e & (H - 1), (&T.z[2][0][0])[e]));
    __syncthreads();
    cta_gemm<kRows, 8, H>([&](int m, int k) { return T.h[2][m][k]; }, [&](int k, int n) { return T.w4[k][n]; },
                          [&](int m, int n, float v) { T.y[m][n] = v + T.b4[n]; });
    __syncthreads();
}

// ---- training set -----------------------------------------------------------
// Sample k: r ~ U[r_lo, r_hi], w_i, w_j ~ U[w_lo, w_hi], code uniform over the
// species pairs; labels = FP64 quadrature (outputs of smear() for the ordered
// pair (a, b) = (0,0), (1,0), (1,1)) minus the unsmeared spline values at r.
__global__ void k_mlp_labels(Dev d, MlpBox box, unsigned long long seed, int n, float* __restrict__ X,
                             float* __restrict__ Y)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    unsigned long long h = mix64(seed ^ (0x1000000ull * (unsigned long long)k));
    double r = box.r_lo + (box.r_hi - box.r_lo) * u01(h);
    int ncode = d.nt == 1 ? 1 : 3;
    int code = (int)(mix64(h + 3) % (unsigned long long)ncode);
    int a = code == 0 ? 0 : 1, b = code == 2 ? 1 : 0;
    // (w_i, w_j) redrawn (at most 16 times) until the pair exponent lies where
    // the quadrature is defined, alpha_min < alpha < alpha_max; the network is
    // never evaluated outside that range, so zero labels there would only put a
    // step into the fitted function
    double wi = 0, wj = 0, alpha = 0;
    for (int t = 0; t < 16; t++) {
        wi = box.w_lo + (box.w_hi - box.w_lo) * u01(mix64(h + 4 + 2 * t));
        wj = box.w_lo + (box.w_hi - box.w_lo) * u01(mix64(h + 5 + 2 * t));
        double ai = 1.0 / (wi * wi), aj = 1.0 / (wj * wj);
        alpha = (ai * aj) / (ai + aj);
        if (d.alpha_min < alpha && alpha < d.alpha_max) break;
    }
    double r_inv = 1.0 / r, rsq = r * r;
    double g0 = 0, gdr = 0, gda = 0, f0 = 0, fdr = 0, fda = 0;
    if (!smear<true, true, 0>(d, b * d.nt + a, comp_idx(a, b), r, r_inv, rsq, alpha, g0, gdr, gda, f0, fdr, fda))
        g0 = gdr = gda = f0 = fdr = fda = 0.0;
    double base[6];
    base_f64(d, b * d.nt + a, comp_idx(a, b), r, base);
    X[4 * (size_t)k + 0] = (float)r;
    X[4 * (size_t)k + 1] = (float)wi;
    X[4 * (size_t)k + 2] = (float)wj;
    X[4 * (size_t)k + 3] = (float)code;
    // label: the smearing correction (quadrature minus the unsmeared values)
    float* y = Y + 6 * (size_t)k;
    y[0] = (float)(f0 - base[0]);
    y[1] = (float)(g0 - base[1]);
    y[2] = (float)(fdr - base[2]);
    y[3] = (float)(gdr - base[3]);
    y[4] = (float)(fda - base[4]);
    y[5] = (float)(gda - base[5]);
}

// ---- one training step --------------------------------------------------------
// CTA c takes rows idx = hash(seed, step, c*64 + r) % n of the training set,
// or rows [c*64, c*64+64) of the given batch when `fixed` is set (gradient
// checks).  Loss = mean over rows and outputs of the squared error of the
// standardised outputs.
__global__ void __launch_bounds__(kMlpThreads) k_mlp_train(MlpState S, const float* __restrict__ X,
                                                           const float* __restrict__ Y, int n, int batch,
                                                           unsigned long long seed, int step, int fixed)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Tile& T = *reinterpret_cast<Tile*>(smem_raw);
    __shared__ float tgt[kRows][8];
    __shared__ float dsum[H];
    __shared__ __nv_bfloat16 dy[kRows][16];
    __shared__ __nv_bfloat16 dzb[kRows][H];
    __shared__ float loss_sh;
    load_weights(T, S.wbf, S.par);
    if (threadIdx.x == 0) loss_sh = 0.f;
    for (int r = threadIdx.x; r < kRows; r += blockDim.x) {
        long long row = (long long)blockIdx.x * kRows + r;
        long long idx = fixed ? row : (long long)(mix64(seed ^ (0x10000000000ull * (unsigned long long)(step + 1)) ^
                                                        (unsigned long long)row) %
                                                  (unsigned long long)n);
        float in[4];
        net_inputs(S.box, X[4 * idx], X[4 * idx + 1], X[4 * idx + 2], (int)X[4 * idx + 3], in);
        for (int k = 0; k < 16; k++) T.x[r][k] = __float2bfloat16(k < 4 ? in[k] : 0.f);
        for (int q = 0; q < 8; q++) tgt[r][q] = q < 6 ? (Y[6 * idx + q] - S.out_mean[q]) / S.out_scale[q] : 0.f;
    }
    __syncthreads();
    forward(T, S.act);
    float* gp = S.gpart + (size_t)blockIdx.x * NPART;
    const float inv = 2.0f / ((float)batch * 6.0f);
    // dL/dy
    for (int e = threadIdx.x; e < kRows * 16; e += blockDim.x) {
        int r = e / 16, q = e % 16;
        float v = 0.f;
        if (q < 6) {
            float diff = T.y[r][q] - tgt[r][q];
            v = inv * diff;
            atomicAdd(&loss_sh, diff * diff / ((float)batch * 6.0f));
        }
        dy[r][q] = __float2bfloat16(v);
        if (q < 8) T.y[r][q] = q < 6 ? v : 0.f;  // keep FP32 dL/dy for the bias gradient
    }
    __syncthreads();
    // layer 4: dW4 = h3^T dy, db4 = sum dy, dh3 = dy W4^T
    cta_gemm<H, 8, kRows>([&](int m, int k) { return T.h[2][k][m]; }, [&](int k, int n2) { return dy[k][n2]; },
                          [&](int m, int n2, float v) { gp[OW4 + m * 8 + n2] = v; });
    if (threadIdx.x < 8) {
        float s = 0.f;
        for (int r = 0; r < kRows; r++) s += T.y[r][threadIdx.x];
        gp[OB4 + threadIdx.x] = s;
    }
    cta_gemm<kRows, H, 16>([&](int m, int k) { return dy[m][k]; },
                           [&](int k, int n2) { return k < 8 ? T.w4[n2][k] : __float2bfloat16(0.f); },
                           [&](int m, int n2, float v) { T.z[2][m][n2] = v * dact_rt(S.act, n2, T.z[2][m][n2]); });
    __syncthreads();
    // layers 3, 2, 1: z[l] now holds dL/dz_l
    for (int l = 2; l >= 0; l--) {
        for (int e = threadIdx.x; e < kRows * H; e += blockDim.x) (&dzb[0][0])[e] = __float2bfloat16((&T.z[l][0][0])[e]);
        for (int c = threadIdx.x; c < H; c += blockDim.x) {
            float s = 0.f;
            for (int r = 0; r < kRows; r++) s += T.z[l][r][c];
            dsum[c] = s;
        }
        __syncthreads();
        const int ow = l == 2 ? OW3 : (l == 1 ? OW2 : OW1), ob = l == 2 ? OB3 : (l == 1 ? OB2 : OB1);
        for (int c = threadIdx.x; c < H; c += blockDim.x) gp[ob + c] = dsum[c];
        if (l > 0) {
            cta_gemm<H, H, kRows>([&](int m, int k) { return T.h[l - 1][k][m]; }, [&](int k, int n2) { return dzb[k][n2]; },
                                  [&](int m, int n2, float v) { gp[ow + m * H + n2] = v; });
            const __nv_bfloat16(*W)[H] = l == 2 ? T.w3 : T.w2;
            cta_gemm<kRows, H, H>([&](int m, int k) { return dzb[m][k]; }, [&](int k, int n2) { return W[n2][k]; },
                                  [&](int m, int n2, float v) { T.z[l - 1][m][n2] = v * dact_rt(S.act, n2, T.z[l - 1][m][n2]); });
        } else {
            cta_gemm<16, H, kRows>([&](int m, int k) { return T.x[k][m]; }, [&](int k, int n2) { return dzb[k][n2]; },
                                   [&](int m, int n2, float v) { gp[OW1 + m * H + n2] = v; });
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) gp[OLOSS] = loss_sh;
}

// Sum of the per-CTA partial gradients; Adam (Kingma & Ba 2015) with a cosine
// learning rate; BF16 copy of the weights.  With lr == 0 only the summed
// gradient is written (gradient checks).
__global__ void k_mlp_adam(MlpState S, int nblocks, int step, int total_steps, float lr0, float* __restrict__ grad_out,
                           float* __restrict__ loss_hist)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > NPARAM) return;
    float g = 0.f;
    for (int c = 0; c < nblocks; c++) g += S.gpart[(size_t)c * NPART + p];
    if (p == NPARAM) {
        if (loss_hist) loss_hist[step] = g;
        return;
    }
    if (grad_out) grad_out[p] = g;
    if (lr0 <= 0.f) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float lr = 0.5f * lr0 * (1.0f + cospif((float)step / (float)total_steps));
    float m = b1 * S.m[p] + (1.f - b1) * g;
    float v = b2 * S.v[p] + (1.f - b2) * g * g;
    S.m[p] = m;
    S.v[p] = v;
    float mh = m / (1.f - powf(b1, (float)(step + 1)));
    float vh = v / (1.f - powf(b2, (float)(step + 1)));
    float w = S.par[p] - lr * mh / (sqrtf(vh) + eps);
    S.par[p] = w;
    S.wbf[p] = __float2bfloat16(w);
}

// Evaluate the network on n raw inputs (r, w_i, w_j, code); y receives its
// outputs in physical units: the smearing corrections of (phi, rho, dphi/dr,
// drho/dr, dphi/dalpha, drho/dalpha).
__global__ void __launch_bounds__(kMlpThreads) k_mlp_eval(MlpState S, const float* __restrict__ X, int n,
                                                          float* __restrict__ Y)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Tile& T = *reinterpret_cast<Tile*>(smem_raw);
    load_weights(T, S.wbf, S.par);
    for (long long t0 = (long long)blockIdx.x * kRows; t0 < n; t0 += (long long)gridDim.x * kRows) {
        __syncthreads();
        for (int r = threadIdx.x; r < kRows; r += blockDim.x) {
            long long k = t0 + r;
            float in[4] = {0, 0, 0, 0};
            if (k < n) net_inputs(S.box, X[4 * k], X[4 * k + 1], X[4 * k + 2], (int)X[4 * k + 3], in);
            for (int q = 0; q < 16; q++) T.x[r][q] = __float2bfloat16(q < 4 ? in[q] : 0.f);
        }
        __syncthreads();
        forward(T, S.act);
        for (int e = threadIdx.x; e < kRows * 6; e += blockDim.x) {
            int r = e / 6, q = e % 6;
            long long k = t0 + r;
            if (k < n) Y[6 * k + q] = T.y[r][q] * S.out_scale[q] + S.out_mean[q];
        }
    }
}

}  // namespace

size_t mlp_smem_bytes() { return sizeof(Tile); }
int mlp_nparam() { return NPARAM; }
int mlp_npart() { return NPART; }

cudaError_t launch_mlp_labels(const Dev& d, const MlpBox& box, unsigned long long seed, int n, float* X, float* Y,
                              cudaStream_t st)
{
    k_mlp_labels<<<div_up(n, 128), 128, 0, st>>>(d, box, seed, n, X, Y);
    return cudaGetLastError();
}

cudaError_t launch_mlp_train_step(const MlpState& S, const float* X, const float* Y, int n, int batch,
                                  unsigned long long seed, int step, int total, float lr, int fixed, float* grad_out,
                                  float* loss_hist, cudaStream_t st)
{
    static bool attr = false;
    size_t sm = sizeof(Tile);
    if (!attr) {
        cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        cudaFuncSetAttribute(k_mlp_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        attr = true;
    }
    int nb = batch / kRows;
    k_mlp_train<<<nb, kMlpThreads, sm, st>>>(S, X, Y, n, batch, seed, step, fixed);
    k_mlp_adam<<<div_up(NPARAM + 1, 256), 256, 0, st>>>(S, nb, step, total, lr, grad_out, loss_hist);
    return cudaGetLastError();
}

cudaError_t launch_mlp_eval(const MlpState& S, const float* X, int n, float* Y, cudaStream_t st)
{
    size_t sm = sizeof(Tile);
    cudaFuncSetAttribute(k_mlp_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int grid = div_up(n, kRows);
    if (grid > num_sms() * 4) grid = num_sms() * 4;
    k_mlp_eval<<<grid, kMlpThreads, sm, st>>>(S, X, n, Y);
    return cudaGetLastError();
}

}  // namespace mg
