// Learned form (MG_FORM_MLP): a 4 -> 64 -> 64 -> 64 -> 6 SiLU MLP replaces the
// DMD Gauss-Hermite smearing (ff_dmd_I.cpp:178-259) of phi, rho and their r /
// alpha derivatives.  Inputs (r, w_i, w_j, species pair) with w = alpha^-1/2;
// outputs (phi, rho, dphi/dr, drho/dr, dphi/dalpha, drho/dalpha) of the pair
// exponent alpha = alpha_i alpha_j / (alpha_i + alpha_j).
//
// Everything runs in this library's own kernels:
//   * k_mlp_labels  -- training samples drawn from a counter-based hash RNG,
//     labelled by the FP64 quadrature of the loaded tables;
//   * k_mlp_train   -- one 64-row tile per CTA: forward and backward with
//     BF16 tensor-core MMAs (mma.sync m16n8k16, FP32 accumulation), weight
//     gradients written as per-CTA partials;
//   * k_mlp_adam    -- sums the partials, Adam with a cosine learning rate,
//     refreshes the BF16 weight copy;
//   * k_dmd_pass1_mlp -- force pass 1 with the MLP (only on rows inside the
//     training box, gathered per warp), quadrature fallback
//     outside the training box and a 1% audit of MLP pairs against the
//     quadrature.
// Species pairs: code 0 = (0,0), 1 = the unordered cross pair, 2 = (1,1); the
// cross code uses one network for (0,1) and (1,0), which needs rho_AB =
// rho_BA (true for the potentials this form is trained on).
#include <cmath>
#include <cstdint>
#include <cuda_bf16.h>

#include "mg_reduce.cuh"
#include "mg_dmd_common.cuh"

namespace mg {
namespace {

constexpr int kRows = 64;       // rows per tile
constexpr int kMlpThreads = 128;
constexpr int H = 64;           // hidden width
// parameter offsets (FP32 master vector)
constexpr int OW1 = 0, OB1 = OW1 + 16 * H, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + H * H,
              OW4 = OB3 + H, OB4 = OW4 + H * 8, NPARAM = OB4 + 8, OLOSS = NPARAM, NPART = NPARAM + 1;

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

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

// SiLU z * sigmoid(z) with sigmoid(z) = (1 + tanh(z/2)) / 2 from the hardware
// tanh (tanh.approx.f32, absolute error about 2^-11, below the BF16 rounding of
// the activations); training, evaluation and the force pass share it.
__device__ __forceinline__ float tanh_hw(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigm(float z) { return fmaf(0.5f, tanh_hw(0.5f * z), 0.5f); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z)
{
    float s = sigm(z);
    return s * (1.0f + z * (1.0f - s));
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
__device__ void forward(Tile& T)
{
    cta_gemm<kRows, H, 16>([&](int m, int k) { return T.x[m][k]; }, [&](int k, int n) { return T.w1[k][n]; },
                           [&](int m, int n, float v) { T.z[0][m][n] = v + T.b1[n]; });
    __syncthreads();
    for (int e = threadIdx.x; e < kRows * H; e += blockDim.x) (&T.h[0][0][0])[e] = __float2bfloat16(silu((&T.z[0][0][0])[e]));
    __syncthreads();
    cta_gemm<kRows, H, H>([&](int m, int k) { return T.h[0][m][k]; }, [&](int k, int n) { return T.w2[k][n]; },
                          [&](int m, int n, float v) { T.z[1][m][n] = v + T.b2[n]; });
    __syncthreads();
    for (int e = threadIdx.x; e < kRows * H; e += blockDim.x) (&T.h[1][0][0])[e] = __float2bfloat16(silu((&T.z[1][0][0])[e]));
    __syncthreads();
    cta_gemm<kRows, H, H>([&](int m, int k) { return T.h[1][m][k]; }, [&](int k, int n) { return T.w3[k][n]; },
                          [&](int m, int n, float v) { T.z[2][m][n] = v + T.b3[n]; });
    __syncthreads();
    for (int e = threadIdx.x; e < kRows * H; e += blockDim.x) (&T.h[2][0][0])[e] = __float2bfloat16(silu((&T.z[2][0][0])[e]));
    __syncthreads();
    cta_gemm<kRows, 8, H>([&](int m, int k) { return T.h[2][m][k]; }, [&](int k, int n) { return T.w4[k][n]; },
                          [&](int m, int n, float v) { T.y[m][n] = v + T.b4[n]; });
    __syncthreads();
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    // splitmix64 finaliser (Steele, Lea & Flood 2014)
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double u01(unsigned long long h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

// normalised network inputs of (r, w_i, w_j, code)
__device__ __forceinline__ void net_inputs(const MlpBox& b, float r, float wi, float wj, int code, float (&in)[4])
{
    in[0] = (r - 0.5f * (b.r_lo + b.r_hi)) / (0.5f * (b.r_hi - b.r_lo));
    in[1] = (wi - 0.5f * (b.w_lo + b.w_hi)) / (0.5f * (b.w_hi - b.w_lo));
    in[2] = (wj - 0.5f * (b.w_lo + b.w_hi)) / (0.5f * (b.w_hi - b.w_lo));
    in[3] = (float)code - 1.0f;
}

// ---- training set -----------------------------------------------------------
// Sample k: r ~ U[r_lo, r_hi], w_i, w_j ~ U[w_lo, w_hi], code uniform over the
// species pairs; labels = FP64 quadrature (outputs of smear() for the ordered
// pair (a, b) = (0,0), (1,0), (1,1)).
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
    X[4 * (size_t)k + 0] = (float)r;
    X[4 * (size_t)k + 1] = (float)wi;
    X[4 * (size_t)k + 2] = (float)wj;
    X[4 * (size_t)k + 3] = (float)code;
    float* y = Y + 6 * (size_t)k;
    y[0] = (float)f0;
    y[1] = (float)g0;
    y[2] = (float)fdr;
    y[3] = (float)gdr;
    y[4] = (float)fda;
    y[5] = (float)gda;
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
    forward(T);
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
                           [&](int m, int n2, float v) { T.z[2][m][n2] = v * dsilu(T.z[2][m][n2]); });
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
                                  [&](int m, int n2, float v) { T.z[l - 1][m][n2] = v * dsilu(T.z[l - 1][m][n2]); });
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

// Evaluate the network on n raw inputs (r, w_i, w_j, code); y receives the
// physical outputs (phi, rho, dphi/dr, drho/dr, dphi/dalpha, drho/dalpha).
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
        forward(T);
        for (int e = threadIdx.x; e < kRows * 6; e += blockDim.x) {
            int r = e / 6, q = e % 6;
            long long k = t0 + r;
            if (k < n) Y[6 * k + q] = T.y[r][q] * S.out_scale[q] + S.out_mean[q];
        }
    }
}

// ---- force pass 1 with the network (one or two species) ------------------
// One warp takes 32 rows at a time: 32 / NT^2 consecutive compact pairs, row
// (pair, a, b).  The network runs on two 16-row m-tiles with the activations
// kept in registers: the FP32 accumulator fragment of one layer, after SiLU
// and BF16 packing, is exactly the A fragment of the next layer's
// m16n8k16 MMA, so only the inputs and the 8 outputs of a row touch shared
// memory.  The weights sit in shared memory in fragment order (one 8-byte load
// per lane per MMA, conflict-free).
//
// Rows inside the training box take the network's outputs; other rows inside
// the smeared cut take the FP32 quadrature of the precision form; a hashed 1%
// of network rows is also evaluated by the FP64 quadrature and the largest
// deviation per output is recorded.  Per-pair results go to the FP32 pair
// scratch in the precision form's layout, so embedding and pass 2 are that
// form's kernels.
constexpr int kInfWarps = 8;
constexpr int kInfThreads = kInfWarps * 32;

struct MlpFrag {
    uint2 w1[8][32];     // [n-tile][lane]            (K = 16: one k-chunk)
    uint2 w2[4][8][32];  // [k-chunk][n-tile][lane]
    uint2 w3[4][8][32];
    uint2 w4[4][32];     // [k-chunk][lane]           (N = 8: one n-tile)
    float b1[H], b2[H], b3[H], b4[8];
};

// per-warp queue of rows that go through the network
constexpr int kQueue = 64;
struct MlpWarpBuf {
    float xin[kQueue][4];  // normalised inputs of the queued rows
    float y[32][8];        // network outputs (standardised) of the first 32
    int pair[kQueue];      // compact pair index of each queued row
    unsigned char ab[kQueue];  // a * 2 + b
};

// B fragment of W (row-major [K][N] BF16 at w) for k-chunk kc, n-tile nt, lane
__device__ __forceinline__ uint2 bfrag(const __nv_bfloat16* __restrict__ w, int N, int kc, int nt, int lane)
{
    const int g = lane >> 2, t = lane & 3, n = nt * 8 + g, k = kc * 16 + 2 * t;
    uint2 f;
    f.x = pack2(w[(size_t)k * N + n], w[(size_t)(k + 1) * N + n]);
    f.y = pack2(w[(size_t)(k + 8) * N + n], w[(size_t)(k + 9) * N + n]);
    return f;
}

__device__ void build_frags(MlpFrag& F, const __nv_bfloat16* __restrict__ wbf, const float* __restrict__ par)
{
    for (int e = threadIdx.x; e < 8 * 32; e += blockDim.x) F.w1[e >> 5][e & 31] = bfrag(wbf + OW1, H, 0, e >> 5, e & 31);
    for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
        int kc = e >> 8, nt = (e >> 5) & 7, ln = e & 31;
        F.w2[kc][nt][ln] = bfrag(wbf + OW2, H, kc, nt, ln);
        F.w3[kc][nt][ln] = bfrag(wbf + OW3, H, kc, nt, ln);
    }
    for (int e = threadIdx.x; e < 4 * 32; e += blockDim.x) F.w4[e >> 5][e & 31] = bfrag(wbf + OW4, 8, e >> 5, 0, e & 31);
    for (int k = threadIdx.x; k < H; k += blockDim.x) {
        F.b1[k] = par[OB1 + k];
        F.b2[k] = par[OB2 + k];
        F.b3[k] = par[OB3 + k];
    }
    if (threadIdx.x < 8) F.b4[threadIdx.x] = par[OB4 + threadIdx.x];
}

__device__ __forceinline__ uint32_t pack2f(float lo, float hi)
{
    return pack2(__float2bfloat16(lo), __float2bfloat16(hi));
}

__device__ __forceinline__ void mma_b(float (&c)[4], const uint32_t (&a)[4], uint2 b)
{
    const uint32_t bb[2] = {b.x, b.y};
    mma16816(c, a, bb);
}

// bias into the accumulators of a 64-wide layer
__device__ __forceinline__ void bias64(float (&c)[8][4], const float* __restrict__ bias, int t)
{
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        float b0 = bias[nt * 8 + 2 * t], b1 = bias[nt * 8 + 2 * t + 1];
        c[nt][0] = b0;
        c[nt][1] = b1;
        c[nt][2] = b0;
        c[nt][3] = b1;
    }
}

// SiLU of a 64-wide accumulator set, packed as the next layer's A fragments
__device__ __forceinline__ void act64(const float (&c)[8][4], uint32_t (&a)[4][4])
{
#pragma unroll
    for (int kc = 0; kc < 4; kc++) {
        a[kc][0] = pack2f(silu(c[2 * kc][0]), silu(c[2 * kc][1]));
        a[kc][1] = pack2f(silu(c[2 * kc][2]), silu(c[2 * kc][3]));
        a[kc][2] = pack2f(silu(c[2 * kc + 1][0]), silu(c[2 * kc + 1][1]));
        a[kc][3] = pack2f(silu(c[2 * kc + 1][2]), silu(c[2 * kc + 1][3]));
    }
}

// the network on rows 0..31 of the queue (B.xin -> B.y), one 16-row m-tile
// at a time (one unrolled tile keeps the body inside the instruction cache)
__device__ __forceinline__ void warp_mlp(const MlpFrag& F, MlpWarpBuf& B, int lane)
{
    const int g = lane >> 2, t = lane & 3;
#pragma unroll 1
    for (int mt = 0; mt < 2; mt++) {
        const int r0 = mt * 16 + g, r1 = r0 + 8;
        uint32_t ax[4] = {0u, 0u, 0u, 0u};
        if (t < 2) {
            ax[0] = pack2f(B.xin[r0][2 * t], B.xin[r0][2 * t + 1]);
            ax[1] = pack2f(B.xin[r1][2 * t], B.xin[r1][2 * t + 1]);
        }
        float c[8][4];
        uint32_t ah[4][4];
        bias64(c, F.b1, t);
#pragma unroll
        for (int nt = 0; nt < 8; nt++) mma_b(c[nt], ax, F.w1[nt][lane]);
        act64(c, ah);
        bias64(c, F.b2, t);
#pragma unroll
        for (int kc = 0; kc < 4; kc++)
#pragma unroll
            for (int nt = 0; nt < 8; nt++) mma_b(c[nt], ah[kc], F.w2[kc][nt][lane]);
        act64(c, ah);
        bias64(c, F.b3, t);
#pragma unroll
        for (int kc = 0; kc < 4; kc++)
#pragma unroll
            for (int nt = 0; nt < 8; nt++) mma_b(c[nt], ah[kc], F.w3[kc][nt][lane]);
        act64(c, ah);
        float y[4] = {F.b4[2 * t], F.b4[2 * t + 1], F.b4[2 * t], F.b4[2 * t + 1]};
#pragma unroll
        for (int kc = 0; kc < 4; kc++) mma_b(y, ah[kc], F.w4[kc][lane]);
        B.y[r0][2 * t] = y[0];
        B.y[r0][2 * t + 1] = y[1];
        B.y[r1][2 * t] = y[2];
        B.y[r1][2 * t + 1] = y[3];
    }
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

// Geometry of row (pair p, species a, b): in-cut test, r, pair exponent.
struct RowGeo {
    int mode;  // 0 beyond the smeared cut, 1 network, 2 quadrature
    float r, alpha;
    bool below_rc;
};

template <int NT>
__device__ __forceinline__ RowGeo row_geo(const Dev& d, const MlpState& S, const F32Consts& kc, long long p, int a,
                                          int b, float (&in)[4])
{
    RowGeo g{0, 1.f, 0.f, false};
    const int i = d.pair_i[p], j = d.pair_j[p];
    const double4 xi = d.pos[i], xj = d.pos[j];
    const double dx0 = xi.x - xj.x, dx1 = xi.y - xj.y, dx2 = xi.z - xj.z;
    const double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
    if (!(rsq < d.cut_sq_mod)) return g;
    const float ai = (float)d.alpha[(size_t)i * NT + a], aj = (float)d.alpha[(size_t)j * NT + b];
    g.alpha = (ai * aj) / (ai + aj);
    g.r = sqrtf((float)rsq);
    g.below_rc = rsq < d.cut_sq;
    const float wi = rsqrtf(ai), wj = rsqrtf(aj);
    const int code = NT == 1 ? 0 : (a == b ? 2 * a : 1);
    const bool inbox = g.r >= S.box.r_lo && g.r <= S.box.r_hi && wi >= S.box.w_lo && wi <= S.box.w_hi &&
                       wj >= S.box.w_lo && wj <= S.box.w_hi && g.alpha > kc.alpha_min && g.alpha < kc.alpha_max;
    g.mode = inbox ? 1 : 2;
    if (inbox) net_inputs(S.box, g.r, wi, wj, code, in);
    return g;
}

// Force pass 1 of the learned form: the six smeared quantities of every row
// into the pair scratch.  A warp walks its rows 32 at a time (32 / NT^2 pairs);
// rows beyond the smeared cut write zeros, rows outside the training box take
// the FP32 quadrature at once, and rows inside it join the warp's queue, which
// runs through the network whenever it holds 32 rows, so the network never
// evaluates a row it does not use.  A hashed 1% of network rows is re-evaluated
// by the FP64 quadrature (audit).  Densities and pair energy follow in
// k_mlp_densities.
template <int NT>
__global__ void __launch_bounds__(kInfThreads, 2) k_dmd_pass1_mlp(Dev d, MlpState S, unsigned long long audit_seed)
{
    constexpr int RP = NT * NT;   // rows per pair
    constexpr int PPW = 32 / RP;  // pairs per warp step
    __shared__ MlpFrag F;
    __shared__ MlpWarpBuf WB[kInfWarps];
    build_frags(F, S.wbf, S.par);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    MlpWarpBuf& B = WB[warp];
    const F32Consts kc = f32_consts(d);
    unsigned long long n_audit = 0, n_fallback = 0;
    float audit_err[6] = {0, 0, 0, 0, 0, 0};
    int qn = 0;  // queued rows (warp-uniform)

    // the network on queue rows 0..31; rows >= nvalid are stale and ignored
    auto drain = [&](int nvalid) {
        __syncwarp();
        warp_mlp(F, B, lane);
        __syncwarp();
        if (lane < nvalid) {
            const long long p = B.pair[lane];
            const int a = B.ab[lane] >> 1, b = B.ab[lane] & 1;
            float o[6];
#pragma unroll
            for (int q = 0; q < 6; q++) o[q] = B.y[lane][q] * S.out_scale[q] + S.out_mean[q];
            store_row<NT>(d, p, a, b, o);
            const unsigned long long h = mix64(audit_seed ^ ((unsigned long long)p * RP + a * NT + b));
            if ((h >> 40) % 100 == 0) {
                float in[4];
                const RowGeo g = row_geo<NT>(d, S, kc, p, a, b, in);
                double g0, gdr, gda, f0 = 0, fdr = 0, fda = 0;
                const int aa = (a == b) ? a : 1, bb = (a == b) ? b : 0;  // the ordering the network was trained on
                const double rr = g.r;
                bool hit = smear<true, true, 0>(d, bb * NT + aa, comp_idx(aa, bb), rr, 1.0 / rr, rr * rr,
                                                (double)g.alpha, g0, gdr, gda, f0, fdr, fda);
                if (!hit) g0 = gdr = gda = f0 = fdr = fda = 0.0;
                const double qv[6] = {f0, g0, fdr, gdr, fda, gda};
#pragma unroll
                for (int q = 0; q < 6; q++) audit_err[q] = fmaxf(audit_err[q], fabsf((float)(qv[q] - o[q])));
                n_audit++;
            }
        }
        __syncwarp();
    };

    const long long ngroups = (d.npairs + PPW - 1) / PPW;
    for (long long grp = (long long)blockIdx.x * kInfWarps + warp; grp < ngroups;
         grp += (long long)gridDim.x * kInfWarps) {
        const long long p = grp * PPW + lane / RP;
        const int a = (lane % RP) / NT, b = lane % NT;
        float in[4] = {0.f, 0.f, 0.f, 0.f};
        RowGeo g{0, 1.f, 0.f, false};
        if (p < d.npairs) g = row_geo<NT>(d, S, kc, p, a, b, in);
        // network rows join the queue
        const unsigned net = __ballot_sync(0xffffffffu, p < d.npairs && g.mode == 1);
        if (p < d.npairs && g.mode == 1) {
            const int slot = qn + __popc(net & ((1u << lane) - 1u));
            B.xin[slot][0] = in[0];
            B.xin[slot][1] = in[1];
            B.xin[slot][2] = in[2];
            B.xin[slot][3] = in[3];
            B.pair[slot] = (int)p;
            B.ab[slot] = (unsigned char)(a * 2 + b);
        }
        qn += __popc(net);
        // the others now: zeros beyond the cut, FP32 quadrature outside the box
        if (p < d.npairs && g.mode != 1) {
            float o[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (g.mode == 2) {
                const float4* pk = d.pkT + (size_t)(a * NT + b) * d.nr * 2;
                const float r_inv = 1.0f / g.r;
                float g0 = 0, gdr = 0, gda = 0, f0 = 0, fdr = 0, fda = 0;
                const bool hit =
                    (a >= b) ? smear_f<true, 0>(d, kc, pk, g.r, r_inv, g.below_rc, g.alpha, g0, gdr, gda, f0, fdr, fda)
                             : smear_f<false, 0>(d, kc, pk, g.r, r_inv, g.below_rc, g.alpha, g0, gdr, gda, f0, fdr, fda);
                if (hit) {
                    o[0] = f0;
                    o[1] = g0;
                    o[2] = fdr;
                    o[3] = gdr;
                    o[4] = fda;
                    o[5] = gda;
                }
                n_fallback++;
            }
            store_row<NT>(d, p, a, b, o);
        }
        if (qn >= 32) {
            drain(32);
            // move the rows queued after the first 32 to the front
            const int rest = qn - 32;
            float x0 = 0.f, x1 = 0.f, x2 = 0.f, x3 = 0.f;
            int pr = 0;
            unsigned char ab = 0;
            if (lane < rest) {
                x0 = B.xin[32 + lane][0];
                x1 = B.xin[32 + lane][1];
                x2 = B.xin[32 + lane][2];
                x3 = B.xin[32 + lane][3];
                pr = B.pair[32 + lane];
                ab = B.ab[32 + lane];
            }
            __syncwarp();
            if (lane < rest) {
                B.xin[lane][0] = x0;
                B.xin[lane][1] = x1;
                B.xin[lane][2] = x2;
                B.xin[lane][3] = x3;
                B.pair[lane] = pr;
                B.ab[lane] = ab;
            }
            __syncwarp();
            qn = rest;
        }
    }
    if (qn > 0) drain(qn);
    // audit and fallback counters: one atomic per warp
#pragma unroll
    for (int q = 0; q < 6; q++) {
        float e = audit_err[q];
        for (int off = 16; off > 0; off >>= 1) e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, off));
        if (lane == 0 && e > 0.f) atomicMax(reinterpret_cast<unsigned int*>(S.audit) + q, __float_as_uint(e));
    }
    for (int off = 16; off > 0; off >>= 1) {
        n_audit += __shfl_xor_sync(0xffffffffu, n_audit, off);
        n_fallback += __shfl_xor_sync(0xffffffffu, n_fallback, off);
    }
    if (lane == 0) {
        if (n_audit) atomicAdd(reinterpret_cast<unsigned long long*>(S.audit + 6), n_audit);
        if (n_fallback) atomicAdd(reinterpret_cast<unsigned long long*>(S.audit + 8), n_fallback);
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
                    if (a >= b) acc[0] += w * (cj[b] * ci[a] + cj[a] * ci[b]) * (double)__ldg(in + (SL::PHI + comp_idx(a, b)) * mp);
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

cudaError_t launch_dmd_force_mlp(const Dev& d, const MlpState& S, unsigned long long audit_seed, int st_clc, int* nb,
                                 cudaStream_t st, cudaEvent_t* evs)
{
    if (d.npairs > 2147483647LL) return cudaErrorInvalidValue;  // queued rows keep the pair index in an int
    const int ppw = 32 / (d.nt * d.nt);
    long long groups = (d.npairs + ppw - 1) / ppw;
    long long need = (groups + kInfWarps - 1) / kInfWarps;
    long long cap = (long long)num_sms() * 2;
    int g1 = (int)(need < cap ? (need > 0 ? need : 1) : cap);
    int gd = persistent_grid(d.npairs, 4);
    if (evs) cudaEventRecord(evs[0], st);
    if (d.nt == 1) {
        k_dmd_pass1_mlp<1><<<g1, kInfThreads, 0, st>>>(d, S, audit_seed);
        k_mlp_densities<1><<<gd, kFFBlock, 0, st>>>(d, 0);
    } else {
        k_dmd_pass1_mlp<2><<<g1, kInfThreads, 0, st>>>(d, S, audit_seed);
        k_mlp_densities<2><<<gd, kFFBlock, 0, st>>>(d, 0);
    }
    if (evs) cudaEventRecord(evs[1], st);
    int rows = 0;
    cudaError_t e = launch_dmd_force_f32_after_pass1(d, st_clc, gd, &rows, st, evs);
    *nb = gd + rows;
    return e;
}

}  // namespace mg
