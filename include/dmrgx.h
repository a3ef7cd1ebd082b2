/* dmrgx: B200-native effective-Hamiltonian path for symmetry-blocked DMRG.
 *
 * C ABI of libdmrgx.so.  Plain pointers and sizes only.  Every function returns
 * 0 on success and a negative DMRGX_E* code on failure; dmrgx_last_error()
 * gives the message of the last failure on the calling thread.
 *
 * Terms follow the reference code (clover199/DMRG):
 *  - a block-sparse tensor ("qtensor", include/qtensor.h:20-31) has, per leg, a
 *    list of sector sizes, per block one sector label per leg, per leg a
 *    fermion direction, and its blocks stored dense row-major (last index
 *    fastest), packed one after another in block order;
 *  - the wavefunction psi is the packed concatenation of its blocks in the order
 *    generate_dim_sym produces (src/useful.cpp:151-194);
 *  - a matvec plan is the pair of task lists ("maps") that get_map builds
 *    (src/qtensor.cpp:997-1119), seven ints per row:
 *    [env block, in offset, out offset, rows, cols, beta, alpha].
 *
 * Qtensor metadata ("meta") is an int array:
 *   nleg, nblk, nsec[0..nleg), dims (all legs' sector sizes, leg by leg),
 *   dir[0..nleg), sym[blk][leg] (nblk*nleg ints).
 *
 * Element types: DMRGX_F64 (double) or DMRGX_C128 (interleaved re,im doubles).
 * A context owns one GPU stream, the device copies of the environments, the
 * plan and its scratch; it is not shared between host threads.
 */
#ifndef DMRGX_H
#define DMRGX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  DMRGX_OK = 0,
  DMRGX_E_ARG = -1,      /* bad argument / inconsistent metadata */
  DMRGX_E_CUDA = -2,     /* CUDA runtime or kernel error */
  DMRGX_E_STATE = -3,    /* call not valid in this state (e.g. no plan) */
  DMRGX_E_NOCONV = -4,   /* eigensolver did not converge */
  DMRGX_E_TIMEOUT = -5,  /* a bounded device wait gave up */
};

enum { DMRGX_F64 = 0, DMRGX_C128 = 1 };

/* matvec arithmetic of a context */
enum {
  DMRGX_PREC_FP64 = 0,   /* FP64 tensor-core (DMMA) grouped GEMM */
  DMRGX_PREC_BF16X3 = 1, /* split precision: hi*hi + hi*lo + lo*hi in BF16, FP32 accumulate */
  DMRGX_PREC_TF32X3 = 2, /* split precision in TF32, FP32 accumulate */
};

/* how the block GEMMs of one matvec are launched */
enum {
  DMRGX_SCHED_GROUPED = 0,   /* one grouped persistent kernel per stage (default) */
  DMRGX_SCHED_PER_BLOCK = 1, /* one cuBLAS GEMM per task row: the reference's own av()
                                loop (src/qtensor.cpp:986-994 -> src/tensor.cpp:698-718)
                                moved to the GPU as-is; FP64 only */
};

enum { DMRGX_MEM_HOST = 0, DMRGX_MEM_DEVICE = 1 };

/* group_n value selecting the Z2 x Z2 x Z2 fusion rule (S4E, src/useful.cpp:4-27) */
enum { DMRGX_GROUP_Z2CUBED = -8 };

/* chain boundary of dmrgx_dmrg (the reference's PBC switch, global.h:14) */
enum { DMRGX_BOUNDARY_OPEN = 0, DMRGX_BOUNDARY_PERIODIC = 1 };

typedef struct dmrgx_ctx dmrgx_ctx;

const char* dmrgx_last_error(void);
const char* dmrgx_version(void);

/* Create a context on CUDA device `device` for element type `dtype`. */
int dmrgx_ctx_create(dmrgx_ctx** ctx, int dtype, int device);
void dmrgx_ctx_destroy(dmrgx_ctx* ctx);

/* Select the matvec arithmetic (DMRGX_PREC_*).  Default FP64. */
int dmrgx_set_precision(dmrgx_ctx* ctx, int prec);

/* Kernel launches of one dmrgx_av with the current plan and settings: FP64
 * grouped 2 (one per stage), split precision 3 (operand split, two stages) plus
 * one per stage that reduces K-split partials, per-block one library GEMM per
 * task row.  Memsets are not counted. */
int dmrgx_matvec_launches(dmrgx_ctx* ctx, int* out);

/* The tiling the autotuner chose for the current split-precision plan.  The
 * split stages run one of four kernel configurations: 0 tiles up to 256 columns
 * with a 4-deep shared-memory ring, 1 up to 128 with a 7-deep ring (one CTA per
 * SM), 2 up to 128 with a 3-deep ring and 3 up to 64 with a 4-deep ring (two
 * CTAs per SM); when a
 * plan's block-shape histogram (rows, columns and K-tiles of every output block,
 * rounded) is new and no plan of its coarse class (half-octave buckets of its
 * tile count, total and longest K, and its widest block) has been tuned, every
 * candidate tiling is timed once on the device and the fastest is cached for
 * later plans of that histogram and class (DMRGX_TUNE=0 in the environment
 * turns the tuner off).  out[0..3] stage 1, out[4..7] stage 2: configuration, halving of
 * one-tile blocks, K-split threshold scale x100 (-100: no K-split), 1 if
 * measured for this plan (0: from the cache).  cap >= 8. */
int dmrgx_split_tuning(dmrgx_ctx* ctx, int* out, int cap);

/* The work units the FP64 grouped kernel runs for one stage (host only: no
 * context, no device work).  The stage is n_outs output blocks; block i is
 * out_desc[3i..3i+2] = (rows, real columns, segment count), and seg_k lists the
 * real K extent of every segment, block by block.  grid: CTAs; mode: 0 whole
 * 64 x 64 tiles longest first onto the least-loaded CTA, 1 equal per-CTA shares
 * of all k-tiles (stream-K) where they shorten the longest CTA by a tenth, 2
 * always shares, -1 tiles in order (the matvec stages use DMRGX_F64_SPLIT, default
 * 1).  Writes min(cap, count) units of 8 ints (out, tm, tn, kt0, kt1, slot, part,
 * nparts; k-tiles 16 wide; out = -1 marks a padding entry; unit j runs on CTA
 * j % grid unless mode is -1 or there are at most grid units), the count to
 * *n_units and the K-split workspace slots to *n_slots. */
int dmrgx_f64_units(int n_outs, const int* out_desc, const int* seg_k, int grid, int mode,
                    int* units, int64_t cap, int64_t* n_units, int64_t* n_slots);

/* Select the launch schedule of the matvec (DMRGX_SCHED_*).  Default grouped.
 * The per-block schedule is the plain FP64 GPU path: same plan, same
 * eigensolver, one library GEMM per task row with the row's sign as alpha. */
int dmrgx_set_schedule(dmrgx_ctx* ctx, int schedule);

/* Build a matvec plan from two block-sparse environments, the way the
 * reference step functions do before calling the eigensolver
 * (src/core.cpp:201-202, :236-247): psi layout from
 * generate_dim_sym(lenv, l_num-1, renv, r_num, sector) (src/useful.cpp:151-194),
 * rmap = renv.get_map(..., 'N','T', r_num, 0) and
 * lmap = lenv.get_map(..., 'N','T', l_num, 0, back=true) (src/qtensor.cpp:997-1119).
 * group_n: N >= 1 for the Z_N fusion rule (src/useful.cpp:30), or
 * DMRGX_GROUP_Z2CUBED for the Z2 x Z2 x Z2 rule of the reference's S4E build
 * (src/useful.cpp:4-27: labels 0..7 fuse by XOR, parity odd for labels 2..5);
 * fermion: apply the direction signs (src/qtensor.cpp:1078-1085); 0 for
 * bosonic models.
 * Environment values (host pointers) are copied to the device. */
int dmrgx_plan_build(dmrgx_ctx* ctx, const int* lenv_meta, const void* lenv_vals,
                     const int* renv_meta, const void* renv_vals, int l_num, int r_num,
                     int sector, int group_n, int fermion);

/* Build a plan from the reference's own task lists: the drop-in for a caller
 * that already holds lanczos<T>::rmap/lmap (include/val_for_lanczos.h:7-24).
 * n: psi length; d_store: length of the intermediate (get_dimension of the
 * store layout, src/core.cpp:239).  env_vals: blocks packed in block order;
 * env_sizes: element count of each block. */
int dmrgx_plan_from_maps(dmrgx_ctx* ctx, int64_t n, int64_t d_store,
                         const int* rmap, int n_rmap, const void* renv_vals,
                         const int64_t* renv_sizes, int n_renv_blocks,
                         const int* lmap, int n_lmap, const void* lenv_vals,
                         const int64_t* lenv_sizes, int n_lenv_blocks);

/* The sector bookkeeping of dmrgx_plan_build alone, on the host (no context, no
 * GPU): psi layout and both task lists in the reference's row format.
 * info[0]=n, info[1]=d_store, info[2]=rows of rmap, info[3]=rows of lmap.
 * rmap/lmap may be NULL (or too small: caps are in rows) to query the sizes;
 * returns DMRGX_E_ARG with the sizes in info when a buffer is too small. */
int dmrgx_build_maps(const int* lenv_meta, const int* renv_meta, int l_num, int r_num,
                     int sector, int group_n, int fermion, int64_t* info, int* rmap,
                     int64_t rmap_cap, int* lmap, int64_t lmap_cap);

/* Periodic chains: the edge pair of av() (src/core.cpp:27-30, PBC build).  The
 * matvec becomes
 *   out = lenv (x) (renv (x) in) + ledge (x) (redge (x) in)
 * with the edge pair's task lists built as the step functions build them
 * (src/core.cpp:241-247): remap = redge.get_map(psi layout, 'N','T', r_num, 0)
 * with its own intermediate (e_store elements), lemap = ledge.get_map(...,
 * l_num, beta = 1, back = true).  The reference shares one store of
 * max(d_store, e_store) between the pairs and runs them one after the other;
 * here each pair has its own intermediate and both run in the same two
 * launches (the edge rows are further tasks of each stage).  Arguments as for
 * the open-chain calls; ledge/redge have the legs of lenv/renv. */
int dmrgx_plan_build_pbc(dmrgx_ctx* ctx, const int* lenv_meta, const void* lenv_vals,
                         const int* renv_meta, const void* renv_vals, const int* ledge_meta,
                         const void* ledge_vals, const int* redge_meta, const void* redge_vals,
                         int l_num, int r_num, int sector, int group_n, int fermion);

/* dmrgx_build_maps with the edge pair: info (7 slots) adds info[4]=e_store,
 * info[5]=rows of remap, info[6]=rows of lemap. */
int dmrgx_build_maps_pbc(const int* lenv_meta, const int* renv_meta, const int* ledge_meta,
                         const int* redge_meta, int l_num, int r_num, int sector, int group_n,
                         int fermion, int64_t* info, int* rmap, int64_t rmap_cap, int* lmap,
                         int64_t lmap_cap, int* remap, int64_t remap_cap, int* lemap,
                         int64_t lemap_cap);

/* dmrgx_plan_from_maps with the edge pair: the drop-in for a PBC build's
 * lanczos<T> (include/val_for_lanczos.h:18-23: ledge, redge, lemap, remap). */
int dmrgx_plan_from_maps_pbc(dmrgx_ctx* ctx, int64_t n, int64_t d_store, const int* rmap,
                             int n_rmap, const void* renv_vals, const int64_t* renv_sizes,
                             int n_renv_blocks, const int* lmap, int n_lmap,
                             const void* lenv_vals, const int64_t* lenv_sizes, int n_lenv_blocks,
                             int64_t e_store, const int* remap, int n_remap,
                             const void* redge_vals, const int64_t* redge_sizes,
                             int n_redge_blocks, const int* lemap, int n_lemap,
                             const void* ledge_vals, const int64_t* ledge_sizes,
                             int n_ledge_blocks);

/* Plan facts: out[0]=n, out[1]=d_store, out[2]=rows of rmap, out[3]=rows of lmap
 * (the main pair), out[4]=useful real flops of one matvec (2*M*N*K per task, x4
 * for complex, both pairs), out[5]=psi blocks, out[6]=store blocks. */
int dmrgx_plan_info(dmrgx_ctx* ctx, int64_t* out);

/* Edge pair of the current plan: out[0]=e_store, out[1]=rows of remap,
 * out[2]=rows of lemap (all 0 on an open chain). */
int dmrgx_plan_edge_info(dmrgx_ctx* ctx, int64_t* out);

/* Copy out the task lists of the current plan, reference row format. */
int dmrgx_plan_maps(dmrgx_ctx* ctx, int* rmap, int* lmap);

/* Copy out the edge pair's task lists (remap, lemap), reference row format. */
int dmrgx_plan_edge_maps(dmrgx_ctx* ctx, int* remap, int* lemap);

/* Copy out the psi layout: nleg, nblk, nsec[], dims..., sym[blk][leg]. */
int dmrgx_plan_psi_layout(dmrgx_ctx* ctx, int* out, int64_t cap);

/* out = H_eff in, exactly av() of the reference (src/core.cpp:22-31):
 * store = renv (x)_{r_num} in, out = lenv (x)_{l_num} store.
 * mem = DMRGX_MEM_HOST: in/out are host arrays (copied straight from and to
 * them); DMRGX_MEM_DEVICE: device arrays on this context's
 * device, ordered on the context's stream.  Psi sectors no task writes are set
 * to zero (the reference leaves them untouched). */
int dmrgx_av(dmrgx_ctx* ctx, const void* in, void* out, int mem);

/* H_eff matvec that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc/cudaFree while they apply H_eff: an
 * eigensolver loop inside a host framework whose own allocator has reserved the
 * device memory, or a loop that cannot afford the device-wide synchronisation
 * that allocation may cause.  Same arithmetic as dmrgx_plan_from_maps followed
 * by dmrgx_av, without a context:
 *   renv/lenv  device arrays: each environment's blocks packed one after
 *              another in block order, every block dense row-major;
 *   rmap/lmap  host arrays: the task rows of stage 1 (renv applied to `in`)
 *              and stage 2 (lenv applied to the intermediate), 7 ints per row:
 *              [block, in offset, out offset, rows, cols, beta, sign];
 *   *_sizes    host arrays, element count of every environment block;
 *   in/out     device arrays of n elements; stream: a cudaStream_t (NULL = legacy
 *              default stream).  The work is queued on `stream`; the call returns
 *              without waiting for it.
 * The intermediate (d_store elements) and the task descriptors live in one
 * static device array of the library (32 MiB for the intermediate, 4 MiB for
 * descriptors), held by every GPU that loads the library until exit.  Larger
 * problems (d_store * element size > 32 MiB, more than 16384 task rows per
 * stage or 65536 blocks per environment) return DMRGX_E_ARG.  The first call on a
 * device looks the array up on that device.  Every call uploads its descriptors
 * from host buffers that the next call reuses, so a call made while `stream`
 * is being captured into a CUDA graph returns DMRGX_E_STATE.  All calls share
 * the array: calls whose GPU work overlaps race. */
int dmrgx_av_noalloc(int dtype, int64_t n, int64_t d_store, const int* rmap, int n_rmap,
                     const void* renv, const int64_t* renv_sizes, int n_renv_blocks,
                     const int* lmap, int n_lmap, const void* lenv, const int64_t* lenv_sizes,
                     int n_lenv_blocks, const void* in, void* out, void* stream);

/* The nev lowest eigenvalues of H_eff and the eigenvector of the lowest: the
 * replacement of the reference's ARPACK wrapper znaupd(n, nev, Evals, Evecs,
 * pass_val) (src/dsaupd.cpp:65-155, src/znaupd.cpp:78-197), run on the device.
 * Thick-restart Lanczos with FP64 basis, inner products and reorthogonalisation;
 * with a split-precision context the lowest Ritz pair is finished by defect
 * correction against the FP64 matvec (residual measured in FP64).
 *   ncv      basis size (<= 0: 4*nev real, 6*nev complex, as the reference)
 *   tol      convergence |H v - theta v| <= tol |theta| (<= 0: 1e-10)
 *   maxiter  restart cycles (<= 0: 3n)
 *   v0       host start vector of n elements, or NULL for a fixed default
 *   evals    host, nev values ascending; evec: host, n elements, unit norm
 *   info     NULL or 6 slots: matvecs, FP64 matvecs, cycles, defect corrections,
 *            converged Ritz values, final residual norm (a double's bits). */
int dmrgx_eigsolve(dmrgx_ctx* ctx, int nev, int ncv, double tol, int maxiter, const void* v0,
                   double* evals, void* evec, int64_t* info);

/* The reference's dmrg() schedule (src/functions.cpp:157-227) with every site
 * step on the GPU: env (x) MPO fusion, the device eigensolver (with this
 * context's matvec precision), block SVD truncation and environment update.
 * model: 0 Kitaev(t, p, u) on an F64 context, 1 XYZ(jx, jy, jz) and 2 Potts3
 * (f, j, p, t) on C128 contexts, built as the reference's drivers build them
 * (kitaev.cpp, xyz.cpp, potts.cpp; src/operators.cpp); 3 the same XYZ chain with
 * a real MPO (sigma_y sigma_y = -(i sigma_y)(i sigma_y)) on an F64 context.  m: bond dimension, sweeps:
 * the reference's n.  Per step (up to cap steps): energies[6*i..] the six lowest
 * values, trunc[i] the truncation error, steps_lr[2*i..] the (l, r) sites,
 * matvecs[i] the matvec count; nsteps: steps done.  seconds (5 slots, may be
 * NULL): total, eigensolver, SVD, environment update, env (x) MPO fusion. */
int dmrgx_dmrg(dmrgx_ctx* ctx, int model, int L, int m, int sweeps, int sector,
               const double* params, int nparams, double* energies, double* trunc, int* steps_lr,
               int64_t* matvecs, int64_t cap, int64_t* nsteps, double* seconds);

/* Boundary condition of the next dmrgx_dmrg: DMRGX_BOUNDARY_OPEN (default) or
 * DMRGX_BOUNDARY_PERIODIC, the reference's PBC build (global.h:14): the MPS
 * carries edge environments seeded with the edge operators the drivers give
 * (kitaev.cpp:42-45 H_Kitaev(t, -p, 0), xyz.cpp:39-42 H_XYZ(jx, jy, jz),
 * potts.cpp:44-47 H_Potts3(0, j, p, t); left() / right()), carried across the
 * chain by the identity operator id(W) (src/qtensor.cpp:157-184) and updated
 * with the bulk environments (src/core.cpp:93-97, :193-199, :272-282, ...);
 * every step's matvec adds the edge pair.  dmrgx_adjoint and dmrgx_expect
 * refuse a periodic run. */
int dmrgx_set_boundary(dmrgx_ctx* ctx, int boundary);

/* Eigensolver of the next dmrgx_dmrg's site steps.  New options; the defaults
 * (6, 0, 0) are the reference's settings.
 *   nev      1..6 eigenvalues converged per step (the reference's NEV = 6,
 *            global.h:21); energies past nev are reported as 0
 *   ncv      Krylov basis size (0: the reference's 4 nev real / 6 nev complex,
 *            src/dsaupd.cpp:76, src/znaupd.cpp:94)
 *   predict  1: start every sweep step from White's prediction of the new
 *            centre (the last step's state carried one site on through the
 *            site tensors, or the same state at a turn), where the reference
 *            starts from a random vector (src/dsaupd.cpp:97).  Needs nev = 1: a
 *            start this close to the lowest eigenvector spans the excited ones
 *            too weakly for their values to be trusted. */
int dmrgx_set_solver(dmrgx_ctx* ctx, int nev, int ncv, int predict);
/* XYZ (models 1 and 3) accept a fourth parameter h: a field h sum_i sigma^z_i,
 * absent from the reference (nparams = 3, or h = 0, is the reference's MPO).
 * The final state of dmrgx_dmrg (MPS site tensors, environments and the one-site
 * centre of the last step) stays in the context for the two calls below. */

/* The block SVD with truncation of the reference's qtensor<T>::svd(U, S, V,
 * num, cutoff) (src/qtensor.cpp:1122-1262), on the device: the tensor (meta,
 * host vals) is reshaped with its first num legs as rows and the rest as
 * columns, every symmetry sector is decomposed, the singular values of all
 * sectors are merged in descending order (ties to the lower sector), the
 * cutoff largest are kept (0: all) and U / V are padded with complement
 * columns to min(dim, cutoff) per sector, as the reference does.  group_n and
 * fermion as for dmrgx_plan_build.  The results stay in the context;
 * sizes[0..5) = U meta ints, U elements, V meta ints, V elements, number of
 * singular values (the whole spectrum, descending).  dmrgx_svd_result copies
 * them out (any pointer may be NULL): U as [legs 0..num), k], V as [k, legs
 * num..), metadata in the layout of dmrgx_plan_psi_layout. */
int dmrgx_svd(dmrgx_ctx* ctx, const int* meta, const void* vals, int num, int cutoff,
              int group_n, int fermion, int64_t* sizes);
int dmrgx_svd_result(dmrgx_ctx* ctx, int* u_meta, void* u_vals, int* v_meta, void* v_vals,
                     double* s);

/* The rest of the reference's singular-value rows (print_singular,
 * src/useful.cpp:75-102) for every step of the last dmrgx_dmrg, in schedule
 * order (the truncation error is dmrgx_dmrg's trunc):
 *   entropy  cap values, S = -sum_i s_i^2 log(s_i^2 + 1e-10) over the whole
 *            spectrum of the step's block SVD (the reference's TOL)
 *   s20      cap * 20 values, the 20 largest singular values (the reference's
 *            NSI), descending, 0 past the spectrum's length
 *   nsv      cap values, the spectrum's length
 * Each output may be NULL; nsteps gets the step count. */
int dmrgx_singular(dmrgx_ctx* ctx, double* entropy, double* s20, int* nsv, int64_t cap,
                   int64_t* nsteps);

/* Solve groups: one batched launch for several chains.  New work (BASELINE
 * config 5): the reference solves chains one after another, each site step's
 * matvec as one serial BLAS call per task row (src/core.cpp:22-31).
 *
 * Contexts that join one group (dmrgx_set_group) and run dmrgx_dmrg from their
 * own host threads meet at every site step's eigensolve: the last to arrive
 * runs one lock-step Lanczos over all members, in which each Krylov round
 * applies every member's H_eff in one grouped FP64 launch per stage (the task
 * lists of all members merged).  The members must run the same schedule (same
 * L, m, sweeps and solver settings, so that their site steps pair up), in FP64
 * on the grouped schedule.  A member that waits 5 minutes for the others gives
 * up with DMRGX_E_TIMEOUT.  members: the number of contexts that will join.
 * dmrgx_set_group(ctx, NULL) leaves the group. */
typedef struct dmrgx_group dmrgx_group;
int dmrgx_group_create(dmrgx_group** group, int members);
void dmrgx_group_destroy(dmrgx_group* group);
int dmrgx_set_group(dmrgx_ctx* ctx, dmrgx_group* group);
/* Work of the group so far: out[0] Krylov rounds, out[1] grouped matvec
 * launches (one per stage per round), out[2] member matvecs they served. */
int dmrgx_group_stats(dmrgx_group* group, int64_t* out);

/* Wall seconds of every site step of the last dmrgx_dmrg (eigensolver, SVD,
 * environment update and fusion of the step), in schedule order; nsteps gets the
 * count, out (cap values, may be NULL) the times. */
int dmrgx_step_seconds(dmrgx_ctx* ctx, double* out, int64_t cap, int64_t* nsteps);

/* Per-step time split of the last dmrgx_dmrg (wall seconds), schedule order:
 * out[5*i..5*i+5) = eigensolver, block SVD, environment update, env (x) MPO
 * fusion, plan building of step i (cap steps at most; out may be NULL). */
int dmrgx_step_split(dmrgx_ctx* ctx, double* out, int64_t cap, int64_t* nsteps);

/* Time split of the last dmrgx_dmrg (wall seconds): out[0] all site steps,
 * [1] eigensolver, [2] block SVD, [3] environment update, [4] env (x) MPO fusion,
 * [5] plan building (sector bookkeeping, task lists, device images, split-precision
 * images and tuning).  cap >= 6.  With cap >= 10 the plan building is also
 * split: [6] sector bookkeeping and task lists, [7] FP64 images and
 * descriptors, [8] split-precision images and descriptors, [9] autotuning. */
int dmrgx_run_seconds(dmrgx_ctx* ctx, double* out, int cap);

/* Gradient of the ground-state energy of the last dmrgx_dmrg with respect to the
 * MPO tensors and the model parameters, by adjoint contractions of the
 * effective Hamiltonian.  New work: the reference has no derivatives; it
 * replaces the finite differences a reference user would take over whole runs
 * (src/functions.cpp:157-227 per parameter value).  The centre walks to the left
 * edge and across the chain without changing the state; at each site k
 *   dE/dW_k = adjoint of <psi| Lop (x) (Rop (x) psi)> w.r.t. the operator that
 *             holds W_k, pulled back through the env (x) MPO fusion
 *             (src/core.cpp:188-192) with the reference's fermion signs.
 * FP64 throughout.  recompute=1 drops the stored environments and rebuilds them
 * from the MPS site tensors first.
 *   dE_dparams  nparams values (model parameter order of dmrgx_dmrg, nparams <=
 *               3 Kitaev, 4 XYZ (jx, jy, jz, h) and Potts)
 *   dE_dW       NULL or L * w_len doubles: per site, dE/dW_k in the bulk MPO's
 *               block layout (edge sites land in row D-1 / column 0)
 *   w_len       NULL or: doubles per site (MPO elements x 1 real / 2 complex)
 *   checks      NULL or 4 slots: E0 of the last step, max |<psi|H|psi> - E0| over
 *               the centres visited, max_k |<dE/dW_k, W_k> - E0| (E is linear in
 *               each W_k), max weight dropped by the centre moves
 *   seconds     NULL or 1 slot: wall time of the adjoint sweep */
int dmrgx_adjoint(dmrgx_ctx* ctx, int recompute, double* dE_dparams, int nparams,
                  double* dE_dW, int64_t w_cap, int64_t* w_len, double* checks,
                  double* seconds);

/* Checkpoint of the state after dmrgx_dmrg (new work; the reference has no MPS
 * file format, only tensor::write_file / read_file for one dense tensor,
 * src/tensor.cpp:249-296).  Text file: a header (model, L, sector, m, centre
 * site, element type, final energy, model parameters), then every site tensor
 * left and right of the one-site centre and the centre tensor, each as its
 * block metadata followed by one line per block in tensor::write_file's format
 * (index count, extents, values at 32 significant digits; complex "(re,im)").
 * dmrgx_load_state reads such a file into a context of the same element type,
 * builds the model's MPO and the environments from the site tensors, and
 * leaves the state for dmrgx_adjoint / dmrgx_expect / dmrgx_save_state.  Open
 * chains only. */
int dmrgx_save_state(dmrgx_ctx* ctx, const char* path);
int dmrgx_load_state(dmrgx_ctx* ctx, const char* path);

/* <Psi|H(params)|Psi> of the current state of the last dmrgx_dmrg for the same
 * model with other parameters (the reference's calc(mps, mpo),
 * src/functions.cpp:469-511, on the device): environments rebuilt from the MPS
 * site tensors with the new MPO, closed at the centre.  For a Hamiltonian linear
 * in its couplings, params = e_p gives the Hellmann-Feynman value dE/dp. */
int dmrgx_expect(dmrgx_ctx* ctx, const double* params, int nparams, double* value);

/* Per-launch device timing of the matvec, for roofline measurements: CUDA
 * events recorded on the context's stream around each launch of every matvec
 * while enabled (enable=1 clears the totals and starts, 0 stops).
 * dmrgx_profile_read synchronises the stream and fills out[0] = matvecs timed,
 * out[1..3] = summed milliseconds of the launch slots [operand split (split
 * precision only), stage 1, stage 2].  cap >= 4. */
int dmrgx_profile(dmrgx_ctx* ctx, int enable);
int dmrgx_profile_read(dmrgx_ctx* ctx, double* out, int cap);

/* The context's CUDA stream (a cudaStream_t), for callers that order their own
 * device work with dmrgx_av(..., DMRGX_MEM_DEVICE). */
void* dmrgx_stream(dmrgx_ctx* ctx);

/* Block until all work queued on the context's stream is done. */
int dmrgx_sync(dmrgx_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* DMRGX_H */
