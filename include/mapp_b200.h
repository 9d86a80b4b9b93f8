/*
 * mapp_b200 -- B200-native force-field hot path of MAPP, behind a C ABI.
 *
 * One mg_system is one MAPP single-rank system (Atoms + Neighbor + ForceField)
 * resident on one GPU.  Entry points mirror the reference's own boundary:
 *
 *   ForceField  (ff.h:12-29)          coef / init / force_calc / energy_calc /
 *                                     create_2nd_neigh_lst / c_d_calc / calc_g / fin
 *   Neighbor    (neighbor.h:46-58)    create_list, neighbor_list, no_pairs
 *   Atoms       (atoms.h:255-287)     H / skin / per-atom vectors, update_0, update(c)
 *
 * so a MAPP ForceField subclass can forward its virtuals one-to-one.
 * Conventions:
 *   - every function returns MG_OK (0) or an MG_ERR_* code; mg_last_error()
 *     returns the message of the last failure on the calling thread (the
 *     reference prints the same text and exits, error.cpp:29-43);
 *   - array arguments may be host or device memory (detected per call);
 *     host arrays are copied through the system's stream, except that
 *     force_calc and calc_g copy their finished per-site result (f, g) into
 *     page-locked host memory on a second stream of the library's own,
 *     beside the reduction of the totals, and join it before returning;
 *     page-locked host buffers give the fastest calls from host memory;
 *   - per-atom arrays use the reference's layouts: x is natms * x_dim with
 *     x_dim = 3 (EAM, FS) or 3 + ntypes (DMD: x y z alpha_1..alpha_n),
 *     c is natms * ntypes, type is natms ints, f has the layout of x;
 *   - en_st receives 7 doubles if st_clc != 0 (energy, then the virial
 *     xx yy zz yz zx xy as in ff_eam.cpp:150-155), else 1.
 */
#ifndef MAPP_B200_H
#define MAPP_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mg_system mg_system;

#define MG_OK 0
#define MG_ERR_ARG 1          /* bad argument (style name, sizes, null pointer)   */
#define MG_ERR_FILE 2         /* potential file cannot be opened                  */
#define MG_ERR_FORMAT 3       /* potential file malformed / ended prematurely     */
#define MG_ERR_STATE 4        /* call out of order (e.g. force before init)       */
#define MG_ERR_CUDA 5         /* CUDA runtime error                               */
#define MG_ERR_CAPACITY 6     /* a device buffer limit could not be met          */
#define MG_ERR_UNSUPPORTED 7  /* feature not available for this style / form      */
#define MG_ERR_TIMEOUT 8      /* a bounded device-side wait ran out               */
#define MG_ERR_DOMAIN 9       /* an integration left its domain (reference aborts) */

#define MG_FORM_FP64 0        /* plain form: FP64 arithmetic throughout            */
#define MG_FORM_FP32 1        /* precision form: FP32 pair/quadrature/spline,
                                 Kahan-compensated per-site sums, FP64 totals      */
#define MG_FORM_MLP 2         /* learned form: BF16 MLP replaces DMD quadrature    */

#define MG_LAUNCH_WHOLE_GPU -1 /* lbfgs_cluster: a one-cell batch's step on every SM */

#define MG_MIN_LBFGS 0        /* Min_LBFGS's two-loop direction (min_l-bfgs.cpp)    */
#define MG_MIN_CG 1           /* Min_CG's Polak-Ribiere direction (min_cg.cpp)      */

/* ---- library ---------------------------------------------------------- */
const char* mg_last_error(void);
int mg_version(void);

/* ---- lifecycle -------------------------------------------------------- */
/* style: a ForceField style name of ff_styles.h: "EAM", "FS", "DMD_I",
   "DMD_II" or "DMD" (MAPP::ff_style, MAPP.cpp:243-264). */
int mg_create(const char* style, int device, mg_system** out);
int mg_destroy(mg_system* s);
int mg_set_stream(mg_system* s, void* cuda_stream);
int mg_set_form(mg_system* s, int form);

/* ---- Atoms ------------------------------------------------------------ */
/* AtomTypes::add_type (atom_types.cpp): names and masses in type order. */
int mg_atoms_set_types(mg_system* s, int ntypes, const char* const* names, const double* masses);
/* Atoms::H (atoms.h:266), 3x3 row-major, lower triangular as ReadCFG::set_box
   leaves it (read_cfg.cpp:365-460); B = H^-1 is formed as M3INV (init.h:72). */
int mg_atoms_set_box(mg_system* s, const double* H);
/* Atoms::skin (atoms.cpp:19, 2908-2915); default 0.5. */
int mg_atoms_set_skin(mg_system* s, double skin);
/* Owned atoms in the state ReadCFG leaves them: vector 0 holds FRACTIONAL
   coordinates s in [0,1) (plus alpha for DMD), then type (MD) or c (DMD). */
int mg_atoms_set(mg_system* s, int natms, const double* x_frac, const int* type, const double* c);
/* Atoms::update_0(0,1,...) (atoms.cpp:1780-1865) after the caller wrote the
   owned Cartesian x (natms * x_dim): skin check against the positions at the
   last rebuild, then either a ghost refresh or x2s + ghost build + list
   rebuild.  *rebuilt reports which, and the call waits for the test.  With
   rebuilt NULL the call does not wait: the test is read by the next entry
   point that needs the positions, ghosts or list (mg_ff_force_calc reads it
   with its results and, when the skin was exceeded, rebuilds and evaluates
   again), with the same outcome as the waiting call. */
int mg_atoms_update_x(mg_system* s, const double* x, int* rebuilt);
/* Owned c written, then Atoms::update(c_n) ghost refresh. */
int mg_atoms_update_c(mg_system* s, const double* c);
/* Owned x (natms * x_dim, Cartesian; a rebuild wraps it into the box). */
int mg_atoms_get_x(mg_system* s, double* x);
/* Ghost ("phantom") atoms: x (natms_ph * x_dim) and the owned atom each one
   images (natms_ph ints); either pointer may be NULL. */
int mg_atoms_get_ghosts(mg_system* s, double* x, int* owner);

/* ---- ForceField ------------------------------------------------------- */
/* ForceField::coef(narg, arg) with the reference's arguments, arg[0] being
   "ff_coef":  EAM  ff_coef {SetFL|FS|FuncFL} file...     (ff_eam.cpp:400-429)
               FS   ff_coef file                          (ff_fs.cpp:113-335)
               DMD* ff_coef r_crd n alpha_min alpha_max T {FS|SetFL|FuncFL} file...
                                                          (ff_dmd_I.cpp:735-796) */
int mg_ff_coef(mg_system* s, int narg, const char* const* arg);
/* ForceField::init, then Atoms::ph_setup(1), Neighbor::init,
   Neighbor::create_list(0,1), Atoms::store_0 -- the order every reference
   caller uses (min_l-bfgs.cpp:178-182, md_nh.cpp:486-503, clock_bdf.cpp:223-236). */
int mg_ff_init(mg_system* s);
/* ForceField::force_calc (ff_eam.cpp:44, ff_fs.cpp:379, ff_dmd_I.cpp:88).
   f receives the owned forces (natms * x_dim; DMD includes the alpha
   components). f may be NULL to keep them on the device. */
int mg_ff_force_calc(mg_system* s, int st_clc, double* f, double* en_st);
/* ForceField::energy_calc (ff_eam.cpp:268, ff_fs.cpp:609, ff_dmd_I.cpp:454). */
int mg_ff_energy_calc(mg_system* s, double* energy);
/* ForceField::create_2nd_neigh_lst (ff_dmd_I.cpp:2138-2217). */
int mg_ff_create_2nd_neigh_lst(mg_system* s);
/* ForceField::c_d_calc (ff_dmd_I.cpp:2241-2398); c_d receives natms * ntypes
   (may be NULL). Uses the per-pair densities of the last force_calc. */
int mg_ff_c_d_calc(mg_system* s, double* c_d);
/* ForceField::calc_g (ff_dmd_I.cpp:2402-2674): a and g are natms * ntypes;
   *cost receives the return value; chk != 0 computes the cost only and
   leaves g zeroed, as the reference does. */
int mg_ff_calc_g(mg_system* s, int chk, double alpha, const double* a, double* g, double* cost);
/* ForceField::fin (releases the per-pair scratch and FF vectors). */
int mg_ff_fin(mg_system* s);

/* ---- Neighbor --------------------------------------------------------- */
/* Neighbor::create_list(0,1) preceded by x2s and a ghost rebuild, as the
   rebuild branch of Atoms::update_0 runs it. */
int mg_neighbor_create_list(mg_system* s);
/* natms, natms_ph and Neighbor::no_pairs (any pointer may be NULL). */
int mg_neighbor_counts(mg_system* s, int* natms, int* natms_ph, long long* no_pairs);
/* Neighbor::neighbor_list_size (natms) and the concatenated per-atom half
   lists (no_pairs ints, j > i, indices in the reference's owned+ghost index
   space); the order inside one atom's list is unspecified. */
int mg_neighbor_get_list(mg_system* s, int* sizes, int* pairs);

/* ---- diagnostics ------------------------------------------------------ */
/* Per-atom double vectors of the force field, owned entries (natms * nt, or
   natms for "rho"): "E", "dE", "ddE", "n", "c_d", "c" (DMD), "rho" (EAM/FS:
   F'(rho)). */
int mg_get_vector(mg_system* s, const char* name, double* out);
/* Per-atom int vectors: "crd" (owned + ghost). */
int mg_get_int_vector(mg_system* s, const char* name, int* out);
/* Device time in ms of the last call of each phase, measured with CUDA events
   on the system's stream: "list" (always), "force", "energy", "c_d", "calc_g"
   (timing level 1 or 2), and for DMD styles the three force kernels
   "force.pass1", "force.embed", "force.pass2" (level 2); MG_ERR_STATE when the
   last call of that phase was not timed. */
int mg_last_time(mg_system* s, const char* phase, double* ms);
/* Device timing level: 0 no events, 1 (default) one event pair around the
   whole call of force_calc, energy_calc, c_d_calc and calc_g, 2 also an event
   between the kernels of the DMD force call. Each event costs a call a few
   microseconds, so a production caller that does not read the times sets 0.
   A profiling switch with no counterpart in the reference (whose force timer,
   thermo_dynamics.cpp:188-206, times the whole call on the host). */
int mg_set_timing(mg_system* s, int level);

/* ---- learned form (MG_FORM_MLP) ------------------------------------------ */
/* A 4 -> 64 -> 64 -> 64 -> 6 SiLU network replaces the Gauss-Hermite smearing
   of phi, rho and their r and alpha derivatives (ff_dmd_I.cpp:178-259) for
   pairs inside its training box; other pairs keep the quadrature, and a
   hashed 1% of network pairs is re-evaluated by the quadrature every
   force_calc (mg_mlp_audit).  Inputs (r, w_i, w_j, species pair) with
   w = alpha^-1/2 per site; outputs (phi, rho, dphi/dr, drho/dr, dphi/dalpha,
   drho/dalpha).  DMD styles with one or two species. */
int mg_mlp_nparam(void);
/* allocate the network for the training box r in [r_lo, r_hi] A and
   w_i, w_j in [w_lo, w_hi] A; random initial weights from `seed` */
/* activation of the learned form's network (before mg_mlp_train: training and
   deployment use the same one): MG_MLP_ACT_POLY is z times a
   degree-15 polynomial stand-in for the logistic function on the FP32 FMA
   pipe (|sigma_p - sigma| <= 9.2e-4); MG_MLP_ACT_TANH is SiLU with the
   logistic from the transcendental unit (tanh.approx); MG_MLP_ACT_SPLIT uses
   the second on the first 48 units of each hidden layer and the first on the
   other 16, so that both pipes evaluate activations at once (default). */
#define MG_MLP_ACT_POLY 0
#define MG_MLP_ACT_TANH 1
#define MG_MLP_ACT_SPLIT 2
int mg_mlp_set_activation(mg_system* s, int act);
int mg_mlp_init(mg_system* s, double r_lo, double r_hi, double w_lo, double w_hi, unsigned long long seed);
/* label nsamples seeded samples with the FP64 quadrature of the loaded tables
   and train `steps` Adam steps of `batch` rows (multiple of 64), cosine
   learning rate from lr; *final_loss = last batch loss (standardised MSE) */
int mg_mlp_train(mg_system* s, long long nsamples, int steps, int batch, double lr, unsigned long long seed,
                 double* final_loss);
int mg_mlp_loss_history(mg_system* s, int n, float* loss);
/* read and/or write the FP32 parameters (mg_mlp_nparam floats) and the output
   standardisation (6 means then 6 scales); any pointer may be NULL */
int mg_mlp_state(mg_system* s, float* params_out, const float* params_in, float* scaling_out,
                 const float* scaling_in);
/* physical outputs y (n * 6) of raw inputs x (n * 4: r, w_i, w_j, code) */
int mg_mlp_eval(mg_system* s, int n, const float* x, float* y);
/* gradient (mg_mlp_nparam floats) of the standardised MSE over n rows
   (multiple of 64) and the loss, without updating the weights */
int mg_mlp_grad(mg_system* s, int n, const float* x, const float* y, float* grad, double* loss);
/* audit of the last learned-form force_calc: max |network - quadrature| per
   output (6 doubles); counts[0] audited rows, counts[1] rows that fell back */
int mg_mlp_audit(mg_system* s, double* max_err, long long* counts);

/* ---- allocation-free entry point ---------------------------------------- */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc:
   code where another allocator owns all device memory (a framework's caching
   allocator, a preallocated pool), code that may not allocate once started,
   or code that must not trigger the implicit synchronisation an allocation
   can cause.  It computes the Finnis-Sinclair energy of ForceField_fs::
   energy_calc (ff_fs.cpp:609-684) from caller-owned device buffers and
   allocates nothing: its scratch (per-atom densities, per-block partial sums)
   is one fixed array of MG_NOALLOC_SCRATCH_BYTES in the library's device
   memory, held by every GPU that loads the library until the process exits.
     x        nall * 3 Cartesian positions, owned atoms first, then ghosts
     type     nall species indices
     nbr_off  natms + 1 offsets into nbr (CSR)
     nbr      half neighbour list: for owned i, the j > i (indices < nall)
     energy   one double, host or device
   x, type, nbr_off and nbr must be device memory; natms may not exceed
   MG_NOALLOC_MAX_ATOMS (MG_ERR_CAPACITY otherwise).  The first call on a
   device looks up the scratch's device address with that device current, so
   make it before any stream capture; under the CUDA runtime's lazy module
   loading that first lookup may also load the library's device code on that
   device, which can allocate and synchronise once, so make the first call
   during set-up.  Later calls allocate nothing.  Every call shares the
   scratch and clears the densities it uses: calls that overlap on the GPU
   race. */
#define MG_NOALLOC_SCRATCH_BYTES (8u << 20)
#define MG_NOALLOC_MAX_ATOMS 1000000

typedef struct mg_fs_coeffs {
    int ntypes;          /* 1..4 */
    int chk[10];         /* 1 where the pair is defined, COMP order (i <= j: j(j+1)/2 + i) */
    double A[4];         /* F = -A sqrt(rho) per type */
    double t1[4][4];     /* rho coefficients [i][j], as in the coefficient file */
    double t2[4][4];
    double cut_rho[10];  /* COMP order */
    double cut_phi[10];
    double k1[10];
    double k2[10];
    double k3[10];
} mg_fs_coeffs;

int mg_fs_energy_noalloc(const mg_fs_coeffs* coeffs, int natms, int nall, const double* x, const int* type,
                         const int* nbr_off, const int* nbr, double* energy, void* cuda_stream);

/* ---- batched form: many independent DMD cells relaxed together ----------- */
/* No counterpart in the reference, which relaxes one system per process with
   Min_LBFGS::run (min_l-bfgs.cpp:616-773) and LineSearch_BackTrack::line_min
   (line_search.cpp:223-342).  Every cell of a batch runs that algorithm on the
   GPU -- m-entry two-loop recursion, Armijo backtracking with c = 0.4,
   rho = 0.5 and first step min(1, max|h|) after |h| = 1, the reference's
   stopping codes -- with all cells advancing together: one force evaluation
   per active cell per iteration, inside one CUDA-graph launch whose
   device-side while loop runs until every cell has stopped.  Cells may
   differ in size and box.  Line-search energies are those of the force pass
   (see the oracle's orc_lbfgs), the L-BFGS dot products, Armijo tests and
   energies are FP64, and the force passes are FP64 or the FP32 precision
   form (mg_batch_set_form).

   The batch builds each cell's ghosts and neighbour list with `builder`, a
   DMD system with types, skin and ff_coef set: its own atoms are replaced. */
typedef struct mg_batch mg_batch;

typedef struct mg_batch_stats {
    double relax_ms;        /* device-loop wall time, list rebuilds included */
    double build_ms;        /* ghosts + lists of every cell, gathered into the batch */
    double tune_ms;         /* autotuning (0 when the choice came from the cache) */
    long long iterations;   /* while-loop iterations (force evaluations of the longest cell) */
    long long evaluations;  /* force evaluations summed over cells */
    int rebuild_rounds;     /* list rebuilds triggered by the skin rule */
    int converged;          /* cells stopped by max|f| < fmax_tol */
    int bps1, bps2;         /* blocks per SM of force pass 1 and pass 2 */
    int lbfgs_threads;      /* threads per CTA of the L-BFGS step */
    int from_cache;         /* launch shapes read from the tuning cache */
    int lbfgs_cluster;      /* CTAs per cell of the L-BFGS step (a thread-block cluster),
                               or MG_LAUNCH_WHOLE_GPU */
} mg_batch_stats;

typedef struct mg_cell_result {
    double energy;          /* free energy at the final point */
    double max_f;           /* max |f| over the cell's degrees of freedom at the last accepted point */
    double t_ms;            /* time from the start of the relaxation to this cell's stop */
    int code;               /* line_search.h codes: 0 running, 1 not downhill, 2 zero gradient,
                               3 minimum step, 4 max iterations, 5 tolerance (energy or max|f|) */
    int iterations;         /* line searches */
    int evaluations;        /* force evaluations */
    int natms;
} mg_cell_result;

int mg_batch_create(mg_system* builder, mg_batch** out);
int mg_batch_destroy(mg_batch* b);
/* one periodic cell: box H (3x3, lower triangular as Atoms::H), natms sites
   with x_frac = natms * (3 + nt) (fractional position, then alpha per
   species) and c = natms * nt */
int mg_batch_add_cell(mg_batch* b, int natms, const double* H, const double* x_frac, const double* c, int* index);
/* history m (1..8), iteration limit, stop when max|f| < fmax_tol (0: off),
   reference energy tolerance, backtracking limit (halvings per line search) */
int mg_batch_set_params(mg_batch* b, int m, int max_iter, double fmax_tol, double energy_tol, int max_halvings);
/* MG_FORM_FP64 or MG_FORM_FP32 force passes */
int mg_batch_set_form(mg_batch* b, int form);
/* MG_MIN_LBFGS (default) or MG_MIN_CG: Min_CG::run's fixed-box branch
   (min_cg.cpp:449-562) with the same line search; m is unused for CG */
int mg_batch_set_method(mg_batch* b, int method);
/* autotune = 1: time candidate launch shapes on the batch (or read them from
   cache_path, a text file of earlier choices, which is then extended);
   0: built-in shapes.  The search covers the blocks per SM of the two pair
   passes and the threads and cluster size of the L-BFGS step.  cache_path
   may be NULL. */
int mg_batch_set_tuning(mg_batch* b, int autotune, const char* cache_path);
/* fixed launch shapes instead of autotuning: blocks per SM of force pass 1
   and pass 2 (0: built-in), threads per CTA (32..1024) and CTAs per cell
   (1, 2, 4, 8 or 16: a thread-block cluster whose CTAs share the cell's
   vectors; MG_LAUNCH_WHOLE_GPU for a batch of one cell: one CTA per SM) of
   the L-BFGS step */
int mg_batch_set_launch(mg_batch* b, int bps1, int bps2, int lbfgs_threads, int lbfgs_cluster);
/* failure limits of a relaxation: at most iteration_budget loop iterations in
   one launch (0: every cell's max_iter times its halvings, the default), and
   a grid-barrier wait of the whole-GPU step that gives up after
   barrier_wait_s seconds (default 2; 0 gives up at the first wait, to test
   the failure path).  Either running out ends the relaxation with
   MG_ERR_TIMEOUT and leaves the GPU usable.  The reference has no such
   limits: its loops end or abort (error.cpp:29-43). */
int mg_batch_set_limits(mg_batch* b, long long iteration_budget, double barrier_wait_s);
int mg_batch_relax(mg_batch* b, mg_batch_stats* stats);
/* final state of one cell: x = natms * (3 + nt) Cartesian positions and
   alpha, f the same shape; either may be NULL */
int mg_batch_cell_result(mg_batch* b, int cell, double* x, double* f, mg_cell_result* r);

/* ---- configuration files ------------------------------------------------ */
/* ReadCFG (read_cfg.cpp:225-700): standard or extended CFG files as the
   reference reads them -- header keys, H0 x Transform x basic length turned
   into the lower-triangular H of Atoms::H, fractional positions wrapped into
   [0, 1), species in the order of their mass / name lines, MD velocities (each
   times R twice and in the frame of the file's box, as the reference converts
   them), DMD rows (s, alpha per species, c per species; dmd != 0, extended
   format only).  eta(i,j) strains are rejected (MG_ERR_UNSUPPORTED).  Host
   code; pass the results to mg_atoms_set_types / _set_box / _set. */
typedef struct mg_cfg mg_cfg;
int mg_cfg_read(const char* path, int dmd, mg_cfg** out);
int mg_cfg_info(const mg_cfg* c, int* natms, int* ntypes, double* H, int* has_velocity);
/* names: ntypes slots of name_len chars each; masses: ntypes doubles */
int mg_cfg_types(const mg_cfg* c, char* names, int name_len, double* masses);
/* x_frac natms * 3 (MD) or natms * (3 + nt) (DMD), type natms (MD), conc
   natms * nt (DMD), velocity natms * 3 (MD); any may be NULL */
int mg_cfg_atoms(const mg_cfg* c, double* x_frac, int* type, double* conc, double* velocity);
int mg_cfg_free(mg_cfg* c);
/* WriteCFG::write_file (write_cfg.cpp:119-433) for the default vector set
   ("write cfg n prefix x" in MD mode, "... x c" in DMD mode; no auxiliary
   vectors, no id sorting): writes <prefix>.<step as %08d>.cfg, and in DMD
   mode the companion .usr file, byte for byte as the reference formats them
   (six decimals, positions as unwrapped fractional coordinates).
   mg_cfg_write_arrays takes host arrays: names ntypes slots of name_len
   chars, masses ntypes, H the 3x3 lower-triangular box, x natms * x_dim
   Cartesian (x_dim 3, or 3 + ntypes in DMD mode with the alphas), type
   natms (MD) or c natms * ntypes (DMD).  mg_cfg_write writes an initialised
   system's current owned state. */
int mg_cfg_write_arrays(const char* prefix, int step, int dmd, int natms, int ntypes, const char* names,
                        int name_len, const double* masses, const double* H, const double* x, const int* type,
                        const double* c);
int mg_cfg_write(mg_system* s, const char* prefix, int step);

/* ---- device-resident minimiser for one system ---------------------------- */
/* Min_LBFGS::run with LineSearch_BackTrack::line_min (min_l-bfgs.cpp:616-773,
   line_search.cpp:223-342) for the system itself, on the GPU: the same
   algorithm, stop codes and line-search energies as the batched form (one
   cell), with the L-BFGS vector work of each step spread over a
   thread-block cluster of lbfgs_cluster CTAs (1, 2, 4, 8 or 16), or on every SM
   (MG_LAUNCH_WHOLE_GPU: one CTA per SM, launched cooperatively, reductions
   through a global array after grid barriers whose waits give up after 2 s
   with MG_ERR_TIMEOUT); 0 = autotune among all of them.
   It replaces the reference's host loop, which copies x and f through the
   boundary on every force evaluation.  The system (DMD style, initialised,
   FP64 or FP32 form) starts from its current state and holds the final state
   on return, ghosts and lists rebuilt; r receives the energy, max|f|, stop code
   and counts, stats the launch statistics (either may be NULL). */
int mg_min_lbfgs(mg_system* s, int m, int max_iter, double fmax_tol, double energy_tol, int max_halvings,
                 int lbfgs_cluster, mg_cell_result* r, mg_batch_stats* stats);
/* Min_CG::run (min_cg.cpp:449-562, fixed box) with LineSearch_BackTrack
   for the system itself on the device, as mg_min_lbfgs does for Min_LBFGS:
   the conjugate direction h = ratio h + f (ratio = (f.f - f.f0) / f0.f0,
   h = f when h.f < 0) instead of the two-loop recursion. */
int mg_min_cg(mg_system* s, int max_iter, double fmax_tol, double energy_tol, int max_halvings, int cluster,
              mg_cell_result* r, mg_batch_stats* stats);

/* ---- concentration clock -------------------------------------------------- */
/* Clock_Adams "clock adams order nsteps delta_t" then run (clock_adams.cpp:
   13-124 constructor, init :128-167, run :187-240, solve :246-365) for an
   initialised DMD system in the plain form: fixed-step Adams-Moulton steps of
   the concentrations, each solved by the reference's box-constrained
   nonlinear conjugate gradient on calc_g.  The vectors stay on the device;
   only the scalars that steer the solve cross to the host.  On return the
   system holds the final c (read with mg_get_vector "c"); err (nsteps
   doubles, may be NULL) receives each step's final calc_g cost and n_calc_g
   (may be NULL) the number of calc_g evaluations. */
int mg_clock_adams(mg_system* s, int order, int nsteps, double delta_t, double* err, long long* n_calc_g);

/* The options of "clock bdf nsteps [key value ...]" (clock_bdf.cpp:14-111);
   mg_bdf_defaults fills the constructor's defaults (clock_bdf.cpp:14-24).
   initial_del_t < 0 means "not given": the first step is then
   a_tol / rms(c_d) clamped to [min_del_t, max_del_t] (clock_bdf.cpp:257-269). */
typedef struct mg_bdf_opts {
    int max_order;        /* 6 (at most 12 here)  */
    int max_iter;         /* 50                   */
    double min_gamma;     /* 1e-10                */
    double gamma_red;     /* 0.8 ("red_gamma")    */
    double slope;         /* 0.4                  */
    double m_tol;         /* 1e-10                */
    double a_tol;         /* 1e-6                 */
    double e_tol;         /* 0: no early stop     */
    double min_del_t;     /* 1e-12                */
    double max_del_t;     /* 1e4                  */
    double initial_del_t; /* -1: from rms(c_d)    */
} mg_bdf_opts;
void mg_bdf_defaults(mg_bdf_opts* o);
/* Clock_BDF init + run (clock_bdf.cpp:201-275, 479-884) for an initialised
   DMD system in the plain form: variable-order (1..max_order),
   variable-step BDF steps of the concentrations, each solved by the
   reference's box-constrained nonlinear conjugate gradient on calc_g, with
   the reference's error estimates and step/order control.  opts may be NULL
   (the defaults).  The run ends after nsteps steps or when
   rms(c_d) / e_tol < 1.  The vectors stay on the device; only the scalars
   that steer the solve and the step control cross to the host.  On return
   the system holds the final c; hist (3 * nsteps doubles, may be NULL)
   receives per step its size, the order it ran at and the time after it;
   steps_taken and n_calc_g (may be NULL) the steps run and the calc_g
   evaluations.  Where the reference aborts (c outside [0, 1] after a solve)
   this returns MG_ERR_DOMAIN, as it does where the reference's unbounded
   step-size retry loops would not end: a predictor outside [0, 1] at
   min_del_t, a retry at the size just tried (at min_del_t), or 100000
   retries.  The error estimate
   reads a local time the reference never sets (clock_bdf.cpp:838-854); the
   reference built with gcc -O2 evaluates it as 0.0 and so does this. */
int mg_clock_bdf(mg_system* s, int nsteps, const mg_bdf_opts* opts, double* hist, int* steps_taken,
                 long long* n_calc_g);

/* ---- Nose-Hoover molecular dynamics ------------------------------------- */
/* MD_NH "md nh nvt temp t_tar t_period eta_iteration .. eta_chains .." with
   time_step dt and boltzmann boltz, then "run nsteps" (md_nh.cpp:23-330
   constructor options, init :385-567, run :636-677), without a barostat and
   without a dof vector, for an initialised EAM / FS system whose species
   masses were given to mg_atoms_set_types.  Velocities: seed > 0 draws them as
   create_vel does (Park-Miller Gaussian, md_nh.cpp:1211-1280); otherwise
   xd_in (natms * 3, host or device) is rescaled to t_tar as init_vel does
   (zero velocities are an MG_ERR_ARG, where the reference aborts).  As in the
   reference, x_0 is not stored at init, so the first step rebuilds the ghosts
   and the list.  On return the system holds the final positions (read them
   with mg_atoms_get_x) and forces; xd_out (natms * 3, may be NULL) receives
   the velocities; thermo (9 + eta_chains doubles, may be NULL) the energy and
   six virial terms of force_calc(1) at the final positions, ke_cur, t_cur and
   the chain velocities eta_d; rebuilds (may be NULL) the number of list
   rebuilds during the run. */
int mg_md_nh(mg_system* s, double t_tar, double t_period, int eta_iteration, int eta_chains, double dt,
             double boltz, int seed, const double* xd_in, int nsteps, double* xd_out, double* thermo,
             int* rebuilds);

#ifdef __cplusplus
}
#endif

#endif /* MAPP_B200_H */
