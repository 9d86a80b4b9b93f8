// Allocation-free Finnis-Sinclair energy: the variant of the FS energy_calc
// kernels (mg_eam.cu, k_fs_pass1 / k_fs_embed) for callers that cannot call
// cudaMalloc -- code running where another allocator owns all device memory
// (a framework's caching allocator or a preallocated pool), where dynamic
// allocation after start-up is not allowed, or that must not trigger the
// implicit device synchronisation an allocation can cause.
//
// The caller passes every input and the output as its own device buffers; the
// kernels' scratch (per-atom densities and per-block partial sums) lives in
// one file-scope __device__ array of fixed size, which every GPU that loads
// the library holds until the process exits.  No cudaMalloc / cudaFree or
// allocating library routine is called on this path.
//
// The scratch is shared by every call: the densities are cleared at the start
// of each call, and calls that overlap on the GPU (on different streams, or
// from different threads) race on it.  Callers serialise them.
//
// The first call on a device resolves the array's device address there
// (cudaGetSymbolAddress).  With the runtime's lazy module loading that lookup
// can be what loads this library's device code onto the device, which may
// allocate and synchronise once; callers make that first call during set-up.
// The cached address belongs to the device's current context: after a
// cudaDeviceReset the cache is stale and this entry point must not be used.
#include <mutex>

#include "../../include/mapp_b200.h"
#include "mg_internal.h"
#include "mg_reduce.cuh"

namespace mg {
namespace {

constexpr int kNaBlock = 256;
constexpr int kNaMaxBlocks = 1024;              // grid cap of each kernel (grid-stride loops)
constexpr int kNaRows = 2 * kNaMaxBlocks;       // partial rows: pair kernel + embedding kernel
constexpr size_t kNaPartialBytes = (size_t)kNaRows * 8 * sizeof(double);

__device__ __align__(256) unsigned char g_noalloc_scratch[MG_NOALLOC_SCRATCH_BYTES];

// per-device address of g_noalloc_scratch (host code may not use the symbol itself)
std::mutex g_na_mutex;
void* g_na_ptr[64] = {nullptr};

__device__ __forceinline__ double na_warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void na_block_partial(double v, double* partial, int row)
{
    __shared__ double sh[kNaBlock / 32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = na_warp_sum(v);
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < kNaBlock / 32; k++) s += sh[k];
        partial[(size_t)row * 8] = s;
    }
}

// Pair sums of ForceField_fs::energy_calc (ff_fs.cpp:633-678): density of i
// and of owned j, pair energy with weight 1/2 for ghost j.  One warp per owned
// atom, grid-stride.
__global__ void __launch_bounds__(kNaBlock) k_na_fs_pairs(mg_fs_coeffs cf, int natms, const double* __restrict__ x,
                                                          const int* __restrict__ type, const int* __restrict__ off,
                                                          const int* __restrict__ nbr, double* __restrict__ rho,
                                                          double* __restrict__ partial)
{
    int lane = threadIdx.x & 31;
    int nwarps = gridDim.x * (blockDim.x >> 5);
    double en = 0.0;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < natms; i += nwarps) {
        int ti = type[i];
        double xi0 = x[3 * (size_t)i], xi1 = x[3 * (size_t)i + 1], xi2 = x[3 * (size_t)i + 2];
        double rho_i = 0.0;
        for (int k = off[i] + lane; k < off[i + 1]; k += 32) {
            int j = nbr[k];
            int tj = type[j];
            int cs = comp_idx(ti, tj);
            if (!cf.chk[cs]) continue;
            double dx0 = xi0 - x[3 * (size_t)j], dx1 = xi1 - x[3 * (size_t)j + 1], dx2 = xi2 - x[3 * (size_t)j + 2];
            double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx0, dx0), __dmul_rn(dx1, dx1)), __dmul_rn(dx2, dx2));
            double crho = cf.cut_rho[cs], cphi = cf.cut_phi[cs];
            double csq = crho * crho > cphi * cphi ? crho * crho : cphi * cphi;
            if (!(rsq < csq)) continue;
            double r = sqrt(rsq);
            bool own_j = j < natms;
            if (r < crho) {
                double d = r - crho;
                rho_i += d * d * (cf.t1[tj][ti] + cf.t2[tj][ti] * d);
                if (own_j) atomicAdd(&rho[j], d * d * (cf.t1[ti][tj] + cf.t2[ti][tj] * d));
            }
            if (r < cphi) {
                double d = r - cphi;
                en += (own_j ? 1.0 : 0.5) * (d * d * (cf.k1[cs] + cf.k2[cs] * r + cf.k3[cs] * rsq));
            }
        }
        rho_i = na_warp_sum(rho_i);
        if (lane == 0) atomicAdd(&rho[i], rho_i);
    }
    na_block_partial(en, partial, blockIdx.x);
}

// Embedding energy -A sqrt(rho) per owned atom (ff_fs.cpp:679).
__global__ void __launch_bounds__(kNaBlock) k_na_fs_embed(mg_fs_coeffs cf, int natms, const int* __restrict__ type,
                                                          const double* __restrict__ rho, double* __restrict__ partial,
                                                          int row0)
{
    double en = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < natms; i += gridDim.x * blockDim.x)
        en -= cf.A[type[i]] * sqrt(rho[i]);
    na_block_partial(en, partial, row0 + blockIdx.x);
}

// Sum of the partial rows into out[0] (one block).
__global__ void __launch_bounds__(kNaBlock) k_na_sum(const double* __restrict__ partial, int rows, double* __restrict__ out)
{
    double s = 0.0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) s += partial[(size_t)r * 8];
    __shared__ double sh[kNaBlock / 32];
    s = na_warp_sum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < kNaBlock / 32; k++) t += sh[k];
        out[0] = t;
    }
}

bool on_device(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace
}  // namespace mg

extern "C" int mg_fs_energy_noalloc(const mg_fs_coeffs* coeffs, int natms, int nall, const double* x, const int* type,
                                    const int* nbr_off, const int* nbr, double* energy, void* stream)
{
    using namespace mg;
    if (!coeffs || !x || !type || !nbr_off || !nbr || !energy)
        return internal_fail(MG_ERR_ARG, "mg_fs_energy_noalloc: null argument");
    if (coeffs->ntypes < 1 || coeffs->ntypes > kMaxTypes)
        return internal_fail(MG_ERR_ARG, "mg_fs_energy_noalloc: ntypes must be 1..4");
    if (natms < 0 || nall < natms) return internal_fail(MG_ERR_ARG, "mg_fs_energy_noalloc: need 0 <= natms <= nall");
    if (natms > MG_NOALLOC_MAX_ATOMS)
        return internal_fail(MG_ERR_CAPACITY,
                                "mg_fs_energy_noalloc: natms exceeds MG_NOALLOC_MAX_ATOMS (the fixed scratch holds "
                                "densities for at most 1000000 atoms)");
    if (!on_device(x) || !on_device(type) || !on_device(nbr_off) || !on_device(nbr))
        return internal_fail(MG_ERR_ARG, "mg_fs_energy_noalloc: x, type, nbr_off and nbr must be device memory");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return internal_fail(MG_ERR_CUDA, "mg_fs_energy_noalloc: no current CUDA device");
    void* base = nullptr;
    {
        // set-up, once per device, with that device current: the device
        // address of the scratch array
        std::lock_guard<std::mutex> lk(g_na_mutex);
        if (!g_na_ptr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return internal_fail(MG_ERR_CUDA, "mg_fs_energy_noalloc: cudaGetSymbolAddress of the scratch failed");
            g_na_ptr[dev] = p;
        }
        base = g_na_ptr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    double* partial = (double*)base;
    double* rho = (double*)((char*)base + kNaPartialBytes);
    double* total = partial + (size_t)(kNaRows - 1) * 8 + 1;  // spare column of the last row
    if (cudaMemsetAsync(rho, 0, (size_t)natms * sizeof(double), st) != cudaSuccess)
        return internal_fail(MG_ERR_CUDA, "mg_fs_energy_noalloc: clearing the scratch failed");
    int g1 = natms ? div_up((long long)natms * 32, kNaBlock) : 1;
    if (g1 > kNaMaxBlocks) g1 = kNaMaxBlocks;
    int g2 = natms ? div_up(natms, kNaBlock) : 1;
    if (g2 > kNaMaxBlocks) g2 = kNaMaxBlocks;
    k_na_fs_pairs<<<g1, kNaBlock, 0, st>>>(*coeffs, natms, x, type, nbr_off, nbr, rho, partial);
    k_na_fs_embed<<<g2, kNaBlock, 0, st>>>(*coeffs, natms, type, rho, partial, g1);
    k_na_sum<<<1, kNaBlock, 0, st>>>(partial, g1 + g2, total);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return internal_fail(MG_ERR_CUDA, cudaGetErrorString(e));
    e = cudaMemcpyAsync(energy, total, sizeof(double), on_device(energy) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && !on_device(energy)) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return internal_fail(MG_ERR_CUDA, cudaGetErrorString(e));
    return MG_OK;
}
