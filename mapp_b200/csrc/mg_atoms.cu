// Atoms / Neighbor kernels: x<->s conversion, ghost (phantom) build and
// refresh, binning, half neighbour list, skin check.
//
// Every floating-point step that decides list membership uses explicit
// round-to-nearest intrinsics (no fused multiply-add) in the reference's
// operation order, so positions, bins and the (i, j) pair set are bit-identical
// to the reference's: x2s atoms.cpp:1869-1897, s2x atoms.cpp:1924-1941,
// s2bin neighbor.cpp:507-525, rsq neighbor.cpp:212-215, ghost s shift
// atoms.cpp:489-495, ghost x refresh atoms.cpp:1340-1348, skin check
// atoms.cpp:1804-1819.
#include <cub/device/device_scan.cuh>

#include "mg_internal.h"

namespace mg {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ double comp3(const double4& p, int k) { return k == 0 ? p.x : (k == 1 ? p.y : p.z); }

__device__ __forceinline__ void set3(double4& p, int k, double v)
{
    if (k == 0) p.x = v;
    else if (k == 1) p.y = v;
    else p.z = v;
}

__global__ void k_split_x(Dev d, const double* __restrict__ x, int frac)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.natms) return;
    const double* p = x + (size_t)i * d.x_dim;
    double4 v = make_double4(p[0], p[1], p[2], 0.0);
    if (frac) d.sfr[i] = v;
    else d.pos[i] = v;
    for (int a = 0; a < d.x_dim - 3; a++) d.alpha[(size_t)i * d.nt + a] = p[3 + a];
}

// Atoms::x2s for owned atoms, including the wrap loops into [0, 1).
__global__ void k_x2s(Dev d)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.natms) return;
    double4 p = d.pos[i];
    for (int j = 0; j < 3; j++) {
        double v = dmul(comp3(p, j), d.B[j][j]);
        for (int k = j + 1; k < 3; k++) v = dadd(v, dmul(d.B[k][j], comp3(p, k)));
        set3(p, j, v);
    }
    for (int j = 0; j < 3; j++) {
        double v = comp3(p, j);
        // the reference steps by one until inside; bounded here by a generous
        // iteration limit so an absurd coordinate cannot spin a thread forever
        for (int it = 0; v < 0.0 && it < (1 << 20); it++) v = dadd(v, 1.0);
        for (int it = 0; v >= 1.0 && it < (1 << 20); it++) v = dsub(v, 1.0);
        set3(p, j, v);
    }
    p.w = 0.0;
    d.sfr[i] = p;
    d.root[i] = i;
    d.gchain[i] = 0ull;
}

// One swap pass of Atoms::ph_setup (atoms.cpp:317-372): the atoms of
// [lo, hi) whose s in `dim` lies in the low (dir 0) or high (dir 1) phantom
// shell are appended, in order, as new ghosts: s[dim] shifted by +1 (dir 0)
// or -1 (dir 1), the phantom vectors copied, (dim, dir) appended to the image
// chain. The pass's bounds and the ghost count live in a GhostCtl on the
// device, written by the previous pass, so the passes run back to back
// without the host.
//
// One launch per pass: a stable compaction by decoupled look-back. Each
// block takes the next tile of kGhostTile atoms (a ticket, so every earlier
// tile belongs to a block that already runs), counts its flagged atoms,
// publishes the count, and walks back over the earlier tiles' published
// counts until it meets an inclusive prefix; then it publishes its own
// inclusive prefix and scatters. Status words: value in the low 30 bits,
// bit 30 "count of this tile", bit 31 "prefix through this tile". The block
// of the last tile writes the next pass's control: next_mode 0 = another
// pass of this direction (over the ghosts just made), 1 = the other
// direction of this dimension (over [0, hi_dim)), 2 = the next dimension
// (over every atom so far). Ghosts beyond `cap` are counted in `over` and not
// written; the host then grows the arrays and builds again. The tile words
// and the ticket of the next pass (the other half of the ping-pong) are
// zeroed here. A look-back wait is bounded; if it runs out, status[6] is set
// and the host reports the build as failed.
constexpr int kGhostTile = 2 * kBlock;
constexpr unsigned kTileAgg = 1u << 30, kTilePrefix = 1u << 31, kTileVal = (1u << 30) - 1;

__global__ void __launch_bounds__(kBlock) k_ghost_pass(Dev d, const GhostCtl* __restrict__ c, GhostCtl* __restrict__ nx,
                                                       unsigned* __restrict__ tiles, unsigned* __restrict__ tiles_next,
                                                       int* __restrict__ ticket, int* __restrict__ ticket_next, int cap,
                                                       int dim, int dir, int next_mode)
{
    __shared__ int s_tile, s_excl;
    __shared__ int s_warp[kBlock / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // the other half of the ping-pong, for the next pass
    tiles_next[blockIdx.x] = 0u;
    if (blockIdx.x == 0 && tid == 0) *ticket_next = 0;
    const int lo = c->lo, n = min(c->hi, cap) - lo, nph = c->nph;
    const int base = d.natms + nph;
    const int ntiles = n > 0 ? (n + kGhostTile - 1) / kGhostTile : 0;
    if (tid == 0) s_tile = atomicAdd(ticket, 1);
    __syncthreads();
    const int tile = s_tile;
    if (ntiles == 0 && tile == 0 && tid == 0) {
        // nothing to scan: the next pass's control with no new ghosts
        GhostCtl o;
        o.nph = nph;
        o.over = c->over;
        o.lo = next_mode == 0 ? base : 0;
        o.hi = next_mode == 1 ? c->hi_dim : d.natms + nph;
        o.hi_dim = next_mode == 2 ? d.natms + nph : c->hi_dim;
        *nx = o;
    }
    if (tile >= ntiles) return;
    // flags of this thread's two atoms
    const int k0 = tile * kGhostTile + 2 * tid;
    int f[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int k = k0 + q;
        f[q] = 0;
        if (k < n) {
            const double sv = comp3(d.sfr[lo + k], dim);
            f[q] = dir == 0 ? (sv <= d.s_ph_lo[dim]) : (d.s_ph_hi[dim] <= sv);
        }
    }
    // block-wide exclusive scan of the counts
    const int mine = f[0] + f[1];
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kBlock / 32 ? s_warp[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kBlock / 32) s_warp[lane] = wi - w;  // exclusive offset of each warp
        if (lane == kBlock / 32 - 1) {
            // lane holding the block total: publish, look back, publish the prefix
            const unsigned total = (unsigned)wi;
            unsigned excl = 0;
            bool ok = true;
            if (tile == 0) {
                atomicExch(&tiles[0], kTilePrefix | total);
            } else {
                atomicExch(&tiles[tile], kTileAgg | total);
                for (int j = tile - 1; j >= 0;) {
                    unsigned v = 0;
                    for (int it = 0; it < (1 << 22); it++) {
                        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(tiles + j) : "memory");
                        if (v) break;
                        __nanosleep(64);
                    }
                    if (!v) {
                        ok = false;
                        break;
                    }
                    excl += v & kTileVal;
                    if (v & kTilePrefix) break;
                    j--;
                }
                atomicExch(&tiles[tile], kTilePrefix | (excl + total));
            }
            if (!ok) atomicExch(&d.status[6], 1);
            s_excl = (int)excl;
            if (tile == ntiles - 1) {
                GhostCtl o;
                o.nph = nph + (int)(excl + total);
                o.over = max(c->over, d.natms + o.nph - cap);
                if (next_mode == 0) {
                    o.lo = base;
                    o.hi = d.natms + o.nph;
                    o.hi_dim = c->hi_dim;
                } else if (next_mode == 1) {
                    o.lo = 0;
                    o.hi = c->hi_dim;
                    o.hi_dim = c->hi_dim;
                } else {
                    o.lo = 0;
                    o.hi = d.natms + o.nph;
                    o.hi_dim = o.hi;
                }
                *nx = o;
            }
        }
    }
    __syncthreads();
    int slot = s_excl + s_warp[warp] + incl - mine;
#pragma unroll
    for (int q = 0; q < 2; q++) {
        if (!f[q]) continue;
        const int src = lo + k0 + q, g = base + slot++;
        if (g >= cap) continue;
        double4 s = d.sfr[src];
        double v = comp3(s, dim);
        set3(s, dim, dir == 0 ? dadd(v, 1.0) : dsub(v, 1.0));
        d.sfr[g] = s;
        for (int a = 0; a < d.x_dim - 3; a++) d.alpha[(size_t)g * d.nt + a] = d.alpha[(size_t)src * d.nt + a];
        if (d.c)
            for (int a = 0; a < d.nt; a++) d.c[(size_t)g * d.nt + a] = d.c[(size_t)src * d.nt + a];
        if (d.type) d.type[g] = d.type[src];
        d.root[g] = d.root[src];
        unsigned long long ch = d.gchain[src];
        int used = __popcll(ch & 0x8888888888888888ull);
        if (used < kMaxChain) ch |= (unsigned long long)(8 | (dim << 1) | dir) << (4 * used);
        else atomicExch(&d.status[4], 1);  // chain too deep: reported as a capacity error
        d.gchain[g] = ch;
    }
}

__global__ void k_ghost_ctl_init(Dev d, GhostCtl* c)
{
    GhostCtl o;
    o.lo = 0;
    o.hi = d.natms;
    o.nph = 0;
    o.hi_dim = d.natms;
    o.over = 0;
    *c = o;
}

// owned + ghost atoms: from the ghost build's control on the device (at
// most cap) when given, else d.nall
__device__ __forceinline__ int nall_of(const Dev& d, const GhostCtl* gc, int cap)
{
    return gc ? min(d.natms + gc->nph, cap) : d.nall;
}

// Neighbor::s2bin for every atom, then Atoms::s2x (owned + ghost), counting
// atoms per bin.
__global__ void k_bin_s2x(Dev d, const GhostCtl* __restrict__ gc, int cap)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nall_of(d, gc, cap)) return;
    double4 s = d.sfr[i];
    int no = 0;
    for (int k = 0; k < 3; k++) {
        double q = __ddiv_rn(dsub(dadd(comp3(s, k), d.cut_ph_s[k]), 0.0), d.cut_ph_s[k]);
        no += (int)q * d.denom[k];
    }
    d.bin[i] = no;
    atomicAdd(&d.cell_count[no], 1);
    double4 x = s;
    for (int j = 0; j < 3; j++) {
        double v = dmul(comp3(s, j), d.H[j][j]);
        for (int k = j + 1; k < 3; k++) v = dadd(v, dmul(d.H[k][j], comp3(s, k)));
        set3(x, j, v);
    }
    x.w = 0.0;
    d.pos[i] = x;
}

__device__ __forceinline__ double pack_idx(int idx, int type)
{
    return __longlong_as_double(((long long)type << 32) | (unsigned int)idx);
}
__device__ __forceinline__ int unpack_idx(double w) { return (int)(__double_as_longlong(w) & 0xffffffffll); }
__device__ __forceinline__ int unpack_type(double w) { return (int)(__double_as_longlong(w) >> 32); }

__global__ void k_cell_fill(Dev d, int* __restrict__ cursor, const GhostCtl* __restrict__ gc, int cap)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nall_of(d, gc, cap)) return;
    int b = d.bin[i];
    int slot = d.cell_start[b] + atomicAdd(&cursor[b], 1);
    double4 p = d.pos[i];
    p.w = pack_idx(i, d.type ? d.type[i] : 0);
    d.cell_pos[slot] = p;
}

// Neighbor::create_list, one warp per owned atom: the 27-bin stencil is nine
// contiguous rows of the bin-sorted atom array; each lane tests one candidate,
// and a ballot compacts the accepted j (> i, rsq < cut_sk_sq) into the list.
__global__ void __launch_bounds__(kBlock) k_neigh(Dev d)
{
    int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (i >= d.natms) return;
    double4 xi = d.pos[i];
    int ti = d.type ? d.type[i] : 0;
    int b = d.bin[i];
    int b2 = b / d.denom[2];
    int rem = b - b2 * d.denom[2];
    int b1 = rem / d.denom[1];
    int b0 = rem - b1 * d.denom[1];
    int x_lo = max(b0 - 1, 0), x_hi = min(b0 + 1, d.grid[0] - 1);
    unsigned lt = (1u << lane) - 1u;
    int cnt = 0;
    int* out = d.nbr + (size_t)i * d.maxnb;
    const bool md = d.style <= STYLE_FS;
    for (int dz = -1; dz <= 1; dz++) {
        int z = b2 + dz;
        if (z < 0 || z >= d.grid[2]) continue;
        for (int dy = -1; dy <= 1; dy++) {
            int y = b1 + dy;
            if (y < 0 || y >= d.grid[1]) continue;
            int row = y * d.denom[1] + z * d.denom[2];
            int start = d.cell_start[row + x_lo], end = d.cell_start[row + x_hi + 1];
            for (int k0 = start; k0 < end; k0 += 32) {
                int k = k0 + lane;
                bool ok = false;
                int j = 0;
                if (k < end) {
                    double4 e = d.cell_pos[k];
                    j = unpack_idx(e.w);
                    if (j > i) {
                        double d0 = dsub(xi.x, e.x), d1 = dsub(xi.y, e.y), d2 = dsub(xi.z, e.z);
                        double rsq = dadd(dadd(dmul(d0, d0), dmul(d1, d1)), dmul(d2, d2));
                        double cut = md ? d.cut_sk_sq[comp_idx(ti, unpack_type(e.w))] : d.cut_sk_sq[0];
                        ok = rsq < cut;
                    }
                }
                unsigned m = __ballot_sync(0xffffffffu, ok);
                if (ok) {
                    int slot = cnt + __popc(m & lt);
                    if (slot < d.maxnb) out[slot] = j;
                }
                cnt += __popc(m);
            }
        }
    }
    if (lane == 0) {
        d.nnb[i] = min(cnt, d.maxnb);
        if (i == 0) d.nnb[d.natms] = 0;  // the scan's extra element (pair count at poff[natms])
        if (cnt > d.maxnb) {
            d.status[0] = 1;
            atomicMax(&d.status[1], cnt);
        }
    }
}

// Compact CSR copy of the half list: pair p = poff[i] + k is (i, nbr[i][k]).
__global__ void __launch_bounds__(kBlock) k_pairs_compact(Dev d)
{
    int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (i >= d.natms) return;
    int nn = d.nnb[i], o = d.poff[i];
    for (int k = lane; k < nn; k += 32) {
        d.pair_i[o + k] = i;
        d.pair_j[o + k] = d.nbr[(size_t)i * d.maxnb + k];
    }
}

__global__ void k_store_x0(Dev d)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.natms) d.pos0[i] = d.pos[i];
}

// Atoms::update for x (update_0) in one launch.  Owned sites take the new x
// (position and alpha) and test their displacement since the last build
// against the skin (Neighbor's rebuild test); each ghost is its root's new x
// with the chain of +-H[dim][0..dim] additions applied in creation order, read
// straight from the caller's x (roots are owned sites), so no second launch has
// to wait for the owned copy.  A site past the skin writes `gen`, which the
// caller makes new for every call, to *flag, so the word needs no reset.
__global__ void k_update_x(Dev d, const double* __restrict__ x, double sq_skin, int* __restrict__ flag, int gen)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < d.natms) {
        const double* p = x + (size_t)k * d.x_dim;
        const double4 v = make_double4(p[0], p[1], p[2], 0.0);
        d.pos[k] = v;
        for (int a = 0; a < d.x_dim - 3; a++) d.alpha[(size_t)k * d.nt + a] = p[3 + a];
        const double4 q = d.pos0[k];
        const double dx0 = dsub(v.x, q.x), dx1 = dsub(v.y, q.y), dx2 = dsub(v.z, q.z);
        const double sq = dadd(dadd(dmul(dx0, dx0), dmul(dx1, dx1)), dmul(dx2, dx2));
        if (sq > sq_skin) *flag = gen;  // (every writer stores the same value)
    } else if (k < d.natms + d.nph) {
        const int r = d.root[k];
        const double* p = x + (size_t)r * d.x_dim;
        d.pos[k] = ghost_image(d, d.gchain[k], make_double4(p[0], p[1], p[2], 0.0));
        for (int a = 0; a < d.x_dim - 3; a++) d.alpha[(size_t)k * d.nt + a] = p[3 + a];
    }
}

__global__ void k_refresh_c(Dev d)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.nph) return;
    int g = d.natms + k, r = d.root[g];
    for (int a = 0; a < d.nt; a++) d.c[(size_t)g * d.nt + a] = d.c[(size_t)r * d.nt + a];
}

__global__ void k_merge_x(Dev d, double* __restrict__ x, int first, int count)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    int i = first + k;
    double* p = x + (size_t)k * d.x_dim;
    double4 v = d.pos[i];
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
    for (int a = 0; a < d.x_dim - 3; a++) p[3 + a] = d.alpha[(size_t)i * d.nt + a];
}

// Deterministic final reduction of per-block partial sums: one block of 1024
// threads; each thread sums its strided rows for all columns at once (rows are
// 64-byte records), then a warp-shuffle and shared-memory tree per column.
__global__ void __launch_bounds__(1024) k_reduce_partials(const double* __restrict__ partial, int nblocks, int nvals,
                                                         double* __restrict__ out)
{
    __shared__ double sh[32][8];
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        const double2* row = reinterpret_cast<const double2*>(partial + (size_t)b * 8);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            double2 v = row[q];
            acc[2 * q] += v.x;
            acc[2 * q + 1] += v.y;
        }
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < 8; v++) {
        double s = acc[v];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) sh[w][v] = s;
    }
    __syncthreads();
    if (threadIdx.x < nvals) {
        double s = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += sh[k][threadIdx.x];
        out[threadIdx.x] = s;
    }
}

}  // namespace

int num_sms()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

cudaError_t launch_split_x(const Dev& d, const double* x_aos, int frac, cudaStream_t st)
{
    if (d.natms) k_split_x<<<div_up(d.natms, kBlock), kBlock, 0, st>>>(d, x_aos, frac);
    return cudaGetLastError();
}

cudaError_t launch_x2s(const Dev& d, cudaStream_t st)
{
    if (d.natms) k_x2s<<<div_up(d.natms, kBlock), kBlock, 0, st>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_ghost_init(const Dev& d, GhostCtl* ctl, cudaStream_t st)
{
    k_ghost_ctl_init<<<1, 1, 0, st>>>(d, ctl);
    return cudaGetLastError();
}

int ghost_tiles(int cap) { return (cap + kGhostTile - 1) / kGhostTile; }

cudaError_t launch_ghost_pass(const Dev& d, const GhostCtl* ctl, GhostCtl* next, unsigned* tiles, unsigned* tiles_next,
                              int* ticket, int* ticket_next, int cap, int dim, int dir, int next_mode, cudaStream_t st)
{
    k_ghost_pass<<<std::max(ghost_tiles(cap), 1), kBlock, 0, st>>>(d, ctl, next, tiles, tiles_next, ticket,
                                                                   ticket_next, cap, dim, dir, next_mode);
    return cudaGetLastError();
}

cudaError_t launch_bin_and_s2x(const Dev& d, const GhostCtl* gc, int cap, cudaStream_t st)
{
    const int n = gc ? cap : d.nall;
    if (n) k_bin_s2x<<<div_up(n, kBlock), kBlock, 0, st>>>(d, gc, cap);
    return cudaGetLastError();
}

cudaError_t launch_cell_fill(const Dev& d, int* cursor, const GhostCtl* gc, int cap, cudaStream_t st)
{
    const int n = gc ? cap : d.nall;
    if (n) k_cell_fill<<<div_up(n, kBlock), kBlock, 0, st>>>(d, cursor, gc, cap);
    return cudaGetLastError();
}

cudaError_t launch_neigh(const Dev& d, cudaStream_t st)
{
    if (d.natms) k_neigh<<<div_up((long long)d.natms * 32, kBlock), kBlock, 0, st>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_pairs_compact(const Dev& d, cudaStream_t st)
{
    if (d.natms) k_pairs_compact<<<div_up((long long)d.natms * 32, kBlock), kBlock, 0, st>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_store_x0(const Dev& d, cudaStream_t st)
{
    if (d.natms) k_store_x0<<<div_up(d.natms, kBlock), kBlock, 0, st>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_update_x(const Dev& d, const double* x_aos, double sq_skin, int* flag, int gen, cudaStream_t st)
{
    const int n = d.natms + d.nph;
    if (n) k_update_x<<<div_up(n, kBlock), kBlock, 0, st>>>(d, x_aos, sq_skin, flag, gen);
    return cudaGetLastError();
}

cudaError_t launch_refresh_c(const Dev& d, cudaStream_t st)
{
    if (d.nph && d.c) k_refresh_c<<<div_up(d.nph, kBlock), kBlock, 0, st>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_merge_x(const Dev& d, double* x_aos, int first, int count, cudaStream_t st)
{
    if (count) k_merge_x<<<div_up(count, kBlock), kBlock, 0, st>>>(d, x_aos, first, count);
    return cudaGetLastError();
}

cudaError_t launch_reduce_partials(const Dev& d, int nblocks, int nvals, double* out, cudaStream_t st)
{
    k_reduce_partials<<<1, 1024, 0, st>>>(d.partial, nblocks, nvals, out);
    return cudaGetLastError();
}

size_t scan_temp_bytes(int n)
{
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const int*)nullptr, (int*)nullptr, n);
    return bytes;
}

cudaError_t launch_exclusive_scan(const int* in, int* out, int n, void* temp, size_t temp_bytes, cudaStream_t st)
{
    return cub::DeviceScan::ExclusiveSum(temp, temp_bytes, in, out, n, st);
}

}  // namespace mg
