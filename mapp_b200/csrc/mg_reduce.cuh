// Warp / block reduction helpers shared by the force-field kernels.
#pragma once

#include "mg_internal.h"

namespace mg {

constexpr int kFFBlock = 256;           // threads per force-field block (8 warps)
constexpr int kFFWarps = kFFBlock / 32;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_sumf(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over an aligned group of G lanes (G = 8, 16 or 32) of one warp; every
// lane of the group must call it (other groups of the warp may be elsewhere).
template <int G>
__device__ __forceinline__ double group_sum(double v)
{
    const unsigned mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}

// Lanes of a warp that hold the same key: pairs are sorted by their first
// site, so equal keys are contiguous lanes [first, last].
struct Seg {
    int first, last;
};

__device__ __forceinline__ Seg seg_of(int key)
{
    unsigned m = __match_any_sync(0xffffffffu, key);
    Seg s;
    s.first = __ffs(m) - 1;
    s.last = 31 - __clz(m);
    return s;
}

// Sum of v over the lanes of the caller's segment, returned in the segment's
// first lane (every lane of the warp must call it).
__device__ __forceinline__ double seg_sum(double v, const Seg& s)
{
    int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double t = __shfl_down_sync(0xffffffffu, v, o);
        if (lane + o <= s.last) v += t;
    }
    return v;
}

// Batched form: is the cell of owned site i still being evaluated?
__device__ __forceinline__ bool site_active(const Dev& d, int i)
{
    return d.cell_active == nullptr || d.cell_active[d.site_cell[i]] != 0;
}

// Batched form: adds e (this lane's energy term of owned site i; i < 0 for a
// lane without one) to the energy of i's cell, one atomic per run of equal
// cells in the warp (sites and pairs are numbered cell by cell).  Every lane
// of the warp must call it.
__device__ __forceinline__ void cell_energy_add(const Dev& d, int i, double e)
{
    const int cell = i >= 0 ? d.site_cell[i] : -1;
    const Seg s = seg_of(cell);
    const double t = seg_sum(e, s);
    if (cell >= 0 && (int)(threadIdx.x & 31) == s.first && t != 0.0) atomicAdd(&d.cell_E[cell], t);
}

// Persistent grid size for a force kernel: enough blocks to fill every SM at
// the kernel's resident-block count, never more than the work needs.
inline int persistent_grid(long long threads_needed, int blocks_per_sm)
{
    long long need = (threads_needed + kFFBlock - 1) / kFFBlock;
    long long cap = (long long)num_sms() * blocks_per_sm;
    return (int)(need < cap ? (need > 0 ? need : 1) : cap);
}

// Sums NV per-thread values over the block (up to 1024 threads) and writes them to
// partial[(row) * 8 + v] (row = blockIdx.x + row_offset).  Every thread of the
// block must call it.
template <int NV>
__device__ __forceinline__ void block_partials(const double (&vals)[NV], double* partial, int row)
{
    __shared__ double sh[32][8];  // up to 1024 threads
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < NV; v++) {
        double s = warp_sum(vals[v]);
        if (lane == 0) sh[w][v] = s;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += sh[k][threadIdx.x];
        partial[(size_t)row * 8 + threadIdx.x] = s;
    }
}

}  // namespace mg
