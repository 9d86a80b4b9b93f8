// Internal state and kernel launchers of the mapp_b200 library.
//
// Device data layout (reference index space: owned atoms [0, natms) first,
// then ghosts [natms, natms+nph) in the exact order Atoms::ph_setup creates
// them, atoms.cpp:317-372):
//   pos[i]    double4  Cartesian x, y, z (w = 0)              owned + ghost
//   sfr[i]    double4  fractional s during a rebuild          owned + ghost
//   alpha[i*nt+a], c[i*nt+a]   DMD per-site vectors           owned + ghost
//   type[i]   int      species (EAM / FS)                     owned + ghost
//   root[g]   int      owned atom a ghost images (owned: itself)
//   gchain[g] uint64   the ordered (dim, dir) image shifts that made ghost g
//                      from root[g]: 4 bits each, low bits first, bit 3 set
//                      marks a used slot; ghosts refresh as
//                      x_g = ((x_root (+-) H[d1]) (+-) H[d2]) ... in that order,
//                      the same sequence of additions as Atoms::update
//                      (atoms.cpp:1320-1352) performs along the swap chain.
//   nbr[i*maxnb+k] int half neighbour list (j > i), nnb[i] its length
//   pair slots (DMD)  SoA over pair index i*maxnb+k, 21 double per pair for
//                      two species: rho[nt*nt], drho_dr, drho_dalpha,
//                      phi[nt(nt+1)/2], dphi_dr, dphi_dalpha
// A ghost refresh of a plain vector v is never materialised: kernels read
// v[root[j]] for j >= natms.
#pragma once

#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <nvtx3/nvToolsExt.h>

struct mg_system;

namespace mg {

enum Style { STYLE_EAM = 0, STYLE_FS = 1, STYLE_DMD_I = 2, STYLE_DMD_II = 3, STYLE_DMD = 4 };

constexpr int kMaxTypes = 4;
constexpr int kMaxQuad = 14;
// 256 knots: the force error against the FP64 form stays at 2.4-2.6e-6 eV/A
// (the FP32 arithmetic, not the table, sets it), and the force pass's table
// (28 KB for two species) leaves room for four blocks per SM
#ifndef MG_SPLIT_KNOTS
#define MG_SPLIT_KNOTS 256
#endif
constexpr int kSplitKnots = MG_SPLIT_KNOTS;  // knots per slot of the precision form's shared-memory table
constexpr int kMaxPassBlocksPerSM = 8;    // resident 256-thread blocks per SM at most
constexpr int kSiteRec = 2;               // float4 per site of the precision form's site record (nt <= 4)
constexpr int kMaxChain = 15;

// Everything a kernel needs, passed by value.
struct Dev {
    // sizes
    int natms, nph, nall, nt, x_dim, maxnb, maxcrd, style, form;
    // box
    double H[3][3], B[3][3];
    double cut_ph_s[3], s_ph_lo[3], s_ph_hi[3];
    int grid[3], denom[3], tot_bin;
    // atoms
    double4* pos;
    double4* sfr;
    double4* pos0;
    double* alpha;
    double* c;
    int* type;
    int* root;
    unsigned long long* gchain;
    // bins / list
    int* bin;
    int* cell_start;
    int* cell_count;
    double4* cell_pos;  // sorted copy: x,y,z and (index | type<<24) in .w bits
    int* nbr;
    int* nnb;      // natms + 1 (last entry 0, so its exclusive scan ends in the pair count)
    int* poff;     // natms + 1: first compact pair of each owned atom
    int* pair_i;   // compact pair list sorted by i (DMD pair scratch is indexed by it)
    int* pair_j;
    long long npairs;
    int* crdl;
    int* ncrd;
    int* crd;
    // per-atom FF vectors
    double* f;     // natms * x_dim
    double* rho;   // EAM/FS rho then F'(rho), nall
    double* E;     // nall * nt
    double* dE;
    double* ddE;
    double* n;
    double* s;
    double* t;
    double* v;
    double* c_d;
    double* a_in;
    double* g;
    // per-pair scratch
    double* pr;    // EAM/FS: drhoi[maxp], drhoj[maxp]; DMD: 21 SoA blocks of maxp
    long long maxp;
    // while act_on: the listed pairs whose stored densities and pair
    // energies are not all zero, as CSR over the owned sites (act_off[i],
    // nact[i] entries): the partner act_pj and the pair's NT^2 densities and
    // NC pair energies copied contiguously (value q of entry k at
    // act_pv[q * act_cap + k], densities first); c_d_calc and calc_g then
    // stream these instead of the list and its per-pair buffers
    int* act_pj;
    double* act_pv;
    int* act_off;
    int* nact;
    long long act_cap;
    int act_on;
    // calc_g's chk and alpha read from device memory (a device-steered solve
    // changes them between graph iterations) when set, else the launch's
    // arguments; with g_chk set the g passes are always enqueued and return
    // at once when *g_chk is non-zero
    const int* g_chk;
    const double* g_alpha;
    // reductions
    double* partial;   // [nblocks][8]
    int* status;       // [0] overflow of nbr, [1] needed maxnb, [2] overflow crd, [3] needed maxcrd,
                       // [4] overflow of the precision form's in-cut list (in a rebuild: ghost
                       // chain too deep), [5] a learned-form tensor-core wait ran out, [6] a
                       // ghost pass's look-back wait ran out
    // tables (device)
    int nr, nrho;
    double dr, drho, dr_inv, drho_inv, rho_max, cut_sq, cut_sq_mod, rc;
    const double* rhoT;  // [nt*nt][nr][8]
    const double* phiT;  // [ncomp][nr][8]
    const double* FT;    // [nt][nrho+1][Fw]
    int Fw;
    // precision form: per ordered species pair (a,b) and knot, one 32-byte
    // sector {rho c0..c3 of slot b*nt+a, phi c0..c3 of slot COMP(a,b) (zero when a < b)}
    const float4* pkT;
    // the plain form's copy of the same pairing in FP64: per ordered species
    // pair (a,b) and knot one 64-byte record {rho c0..c3, phi c0..c3}, so the
    // two knots a quadrature node needs share one cache line
    const double* pk64;
    // the precision form's table: the same splines resampled onto nrS =
    // kSplitKnots knots over [0, rc] (FP32 cubic Hermite pieces, float4
    // {c0..c3} per knot), rho slots of the ordered species pairs (a*nt+b holds
    // density slot b*nt+a) then phi slots in COMP order, nrS rows each; row
    // nrS-1 of a slot is the constant f(rc)
    const float4* pkS;
    int nrS;
    float drS_inv;
    // in-cut pair list of the precision form, written by its density pass in
    // batches of 32 padded with i = -1, two int4 per pair: {i, j, owner of j,
    // 0} and the bits of {dx, dy, dz, rsq} (FP32); warp w of that pass fills
    // region w and writes its batch count to icut_n[w]; capacity icut_cap pairs
    int4* icut;
    unsigned* icut_n;
    long long icut_cap;
    float* prf;          // FP32 pair scratch, same SoA layout as pr
    // precision form per-site FP32 records: srec[i*kSiteRec..] = {alpha_0..,
    // c_0..} of site i (owned + ghost), dE32[i*nt+a] = F'(E) of owned site i,
    // facc[i*8..] the j-side force sums of owned site i (x, y, z, alpha_0..)
    float4* srec;
    float* dE32;
    float* facc;
    double cut_sk_sq[16];
    // FS analytic
    double fsA[kMaxTypes], fst1[kMaxTypes][kMaxTypes], fst2[kMaxTypes][kMaxTypes];
    double fs_cut_rho[16], fs_cut_phi[16], fsk1[16], fsk2[16], fsk3[16], fs_cut_sq[16];
    int fs_chk[16];
    // DMD
    double rsq_crd, alpha_min, alpha_max, kbT, beta, c0[kMaxTypes];
    int nq;
    double xi[kMaxQuad], w0[kMaxQuad], w1[kMaxQuad], w2[kMaxQuad];
    float xi_f[kMaxQuad], w0_f[kMaxQuad], w1_f[kMaxQuad], w2_f[kMaxQuad];  // FP32 copies (precision form)
    // batched form (many independent cells in one site / pair numbering);
    // all null for a single system
    const int* site_cell;              // owned site -> cell
    const unsigned char* cell_active;  // cells whose pairs / sites are evaluated
    double* cell_E;                    // per-cell energy accumulators
    int tune_bps, tune_bps2;           // blocks per SM of pair pass 1 / pass 2 (0: built-in)
};

__host__ __device__ inline int comp_idx(int i, int j)
{
    return i < j ? (j + 1) * j / 2 + i : (i + 1) * i / 2 + j;
}

#ifdef __CUDACC__
// A ghost's position from its root's: the shifts +-H[dim][0..dim] of its chain
// applied in creation order with round-to-nearest adds, as Atoms::update
// refreshes x along the swap chain (atoms.cpp:1320-1352).
__device__ __forceinline__ double4 ghost_image(const Dev& d, unsigned long long ch, double4 p)
{
    for (int s = 0; s < kMaxChain; s++) {
        unsigned code = (unsigned)(ch >> (4 * s)) & 15u;
        if (!(code & 8u)) break;
        int dim = (code >> 1) & 3, dir = code & 1;
        p.x = dir == 0 ? __dadd_rn(p.x, d.H[dim][0]) : __dsub_rn(p.x, d.H[dim][0]);
        if (dim >= 1) p.y = dir == 0 ? __dadd_rn(p.y, d.H[dim][1]) : __dsub_rn(p.y, d.H[dim][1]);
        if (dim >= 2) p.z = dir == 0 ? __dadd_rn(p.z, d.H[dim][2]) : __dsub_rn(p.z, d.H[dim][2]);
    }
    p.w = 0.0;
    return p;
}
#endif

// training box of the learned form (inputs outside it fall back to quadrature)
struct MlpBox {
    float r_lo, r_hi, w_lo, w_hi;
};

// network parameters, optimiser state and deployment bookkeeping
struct MlpState {
    float* par;             // FP32 master parameters
    __nv_bfloat16* wbf;     // BF16 copy used by the tensor-core kernels
    float* m;               // Adam moments
    float* v;
    float* gpart;           // per-CTA partial gradients
    float* audit;           // [0..5] max |network - quadrature| per output, [6..7] audited rows (u64), [8..9] fallback rows (u64)
    MlpBox box;
    float out_mean[6], out_scale[6];
    int act;                // activation kind (MG_MLP_ACT_*): 0 silu_p, 1 silu_t, 2 split
    // deployment: the rows (site pair, species pair) listed by k_mlp_rows.
    // Network rows fill the list from the front (normalised inputs / 8,
    // (pair, a*nt+b), r), quadrature-fallback rows from the back (row_id
    // only); row_cap entries.  row_n: [0] network rows, [1] audited rows
    // (indices into the list, in audit_rows, capacity audit_cap), [2] fallback
    // rows.
    float4* row_in;
    int2* row_id;
    float* row_r;
    unsigned* row_n;
    long long row_cap;
    int* audit_rows;
    long long audit_cap;
};

// ---- launchers (defined in the .cu files) ---------------------------------
// atoms / neighbour
cudaError_t launch_x2s(const Dev& d, cudaStream_t st);
cudaError_t launch_split_x(const Dev& d, const double* x_aos, int frac, cudaStream_t st);
// bounds of one ghost pass ([lo, hi) scanned), the ghost count so far, the
// end of the range the current dimension's passes start from, and the number
// of ghosts that did not fit
struct GhostCtl {
    int lo, hi, nph, hi_dim, over;
};
cudaError_t launch_ghost_init(const Dev& d, GhostCtl* ctl, cudaStream_t st);
// one ghost pass: tile words and tickets of this pass and of the next
// (ping-pong halves, ghost_tiles(cap) words each)
int ghost_tiles(int cap);
cudaError_t launch_ghost_pass(const Dev& d, const GhostCtl* ctl, GhostCtl* next, unsigned* tiles, unsigned* tiles_next,
                              int* ticket, int* ticket_next, int cap, int dim, int dir, int next_mode, cudaStream_t st);
// over owned + ghost atoms, their count from gc (the ghost build's control,
// clamped to cap) when gc is given, else d.nall
cudaError_t launch_bin_and_s2x(const Dev& d, const GhostCtl* gc, int cap, cudaStream_t st);
cudaError_t launch_cell_fill(const Dev& d, int* cursor, const GhostCtl* gc, int cap, cudaStream_t st);
cudaError_t launch_neigh(const Dev& d, cudaStream_t st);
cudaError_t launch_pairs_compact(const Dev& d, cudaStream_t st);
cudaError_t launch_store_x0(const Dev& d, cudaStream_t st);
cudaError_t launch_update_x(const Dev& d, const double* x_aos, double sq_skin, int* flag, int gen, cudaStream_t st);
cudaError_t launch_refresh_c(const Dev& d, cudaStream_t st);
cudaError_t launch_merge_x(const Dev& d, double* x_aos, int first, int count, cudaStream_t st);
cudaError_t launch_reduce_partials(const Dev& d, int nblocks, int nvals, double* out, cudaStream_t st);
size_t scan_temp_bytes(int n);
cudaError_t launch_exclusive_scan(const int* in, int* out, int n, void* temp, size_t temp_bytes, cudaStream_t st);
// EAM / FS
cudaError_t launch_eam_force(const Dev& d, int st_clc, int* nblocks_out, cudaStream_t st);
cudaError_t launch_eam_energy(const Dev& d, int* nblocks_out, cudaStream_t st);
cudaError_t launch_fs_force(const Dev& d, int st_clc, int* nblocks_out, cudaStream_t st);
cudaError_t launch_fs_energy(const Dev& d, int* nblocks_out, cudaStream_t st);
// DMD
// evs (may be null): 4 events recorded before pass 1, before the embedding
// kernel, before pass 2 and after pass 2, for per-kernel device times
cudaError_t launch_dmd_force(const Dev& d, int st_clc, int* nblocks_out, cudaStream_t st, cudaEvent_t* evs);
cudaError_t launch_dmd_energy(const Dev& d, int* nblocks_out, cudaStream_t st);
// precision form (MG_FORM_FP32) force_calc; evs as for launch_dmd_force
cudaError_t launch_dmd_force_f32(const Dev& d, int st_clc, int* nblocks_out, cudaStream_t st, cudaEvent_t* evs);
// the precision form's embedding and pass 2 after a pass 1 that filled the FP32 pair scratch
// the precision form's per-pair densities and pair energies (rho and phi blocks
// of prf) at the current positions, for c_d_calc / calc_g after its force call
cudaError_t launch_dmd32_pair_values(const Dev& d, cudaStream_t st);
// entries the in-cut list needs for maxp listed pairs, and the number of
// per-warp batch counts (icut_n) it needs
long long dmd32_icut_capacity(long long maxp);
int dmd32_icut_warps();
cudaError_t launch_dmd_force_f32_after_pass1(const Dev& d, int st_clc, int row0, int* nblocks_out, cudaStream_t st,
                                             cudaEvent_t* evs);
// learned form
size_t mlp_smem_bytes();
int mlp_nparam();
int mlp_npart();
cudaError_t launch_mlp_labels(const Dev& d, const MlpBox& box, unsigned long long seed, int n, float* X, float* Y,
                              cudaStream_t st);
cudaError_t launch_mlp_train_step(const MlpState& S, const float* X, const float* Y, int n, int batch,
                                  unsigned long long seed, int step, int total, float lr, int fixed, float* grad_out,
                                  float* loss_hist, cudaStream_t st);
cudaError_t launch_mlp_eval(const MlpState& S, const float* X, int n, float* Y, cudaStream_t st);
cudaError_t launch_dmd_force_mlp(const Dev& d, const MlpState& S, unsigned long long audit_seed, int st_clc, int* nb,
                                 cudaStream_t st, cudaEvent_t* evs);
cudaError_t launch_dmd_crd(const Dev& d, cudaStream_t st);
cudaError_t launch_dmd_cdot(const Dev& d, cudaStream_t st);
cudaError_t launch_dmd_calc_g(const Dev& d, int chk, double alpha, int* nblocks_out, cudaStream_t st);
// the active sublist: per-site counts (nact, nact[natms] = 0), then, after the
// caller's scan into act_off and with act_cap set, the CSR copy
cudaError_t launch_active_count(const Dev& d, cudaStream_t st);
cudaError_t launch_active_fill(const Dev& d, cudaStream_t st);

// One NVTX range per hot-path entry point, named after it, so a profiler's
// timeline shows force_calc, calc_g, list builds and solver runs the way the
// reference's per-phase timers report them (thermo_dynamics.cpp:188-206).
// Without an attached tool a range costs one pointer test.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
#define MG_NVTX(name) ::mg::NvtxRange mg_nvtx_range_(name)

// records msg as the calling thread's last error and returns code
int internal_fail(int code, const char* msg);
const char* internal_last_error();

// grid sizing helpers
int num_sms();
inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// accessors of a single system for the batched form and the MD loop (mg_api.cu)
Dev& system_dev(mg_system* s);
cudaStream_t system_stream(mg_system* s);
int system_device(mg_system* s);
void system_shape(mg_system* s, int* style, int* nt, int* x_dim, int* form, double* B_out);
double system_skin(mg_system* s);
void system_box(mg_system* s, double* H_out);
int system_natms(mg_system* s);
// MG_OK when ff_init has run (else records the error and returns its code)
int system_check_ready(mg_system* s);
void system_masses(mg_system* s, double* out);
// x2s of the owned atoms, then the ghost / bin / list rebuild (Atoms::update_0's rebuild branch)
int system_rebuild(mg_system* s);
// enqueue force_calc's device work only (zero f and rho unless the caller has,
// the EAM / FS passes); capturable
int system_enqueue_force(mg_system* s, int st_clc, int zero, int* rows);
double* system_red_out(mg_system* s);
// enqueue calc_g's device work on the system's a_in (cost * 4 left in red_out[0],
// g in the system's g unless chk) and c_d_calc's (c_d in the system's c_d); capturable
int system_enqueue_calc_g(mg_system* s, int chk, double alpha, int* rows);
// the same with chk and alpha read from device memory at run time (for a
// captured loop whose iterations change them)
int system_enqueue_calc_g_dev(mg_system* s, const int* chk_dev, const double* alpha_dev, int* rows);
int system_enqueue_c_d(mg_system* s);
// builds the active-pair sublist from the last force_calc's pair values and
// makes c_d_calc / calc_g walk it (on), or walk the full list again (off);
// valid while the positions and the list stay as they are
int system_set_active_pairs(mg_system* s, bool on);

}  // namespace mg
