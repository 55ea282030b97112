/*
 * ccq_b200 — C ABI of the B200 coupled-cluster amplitude-update engine.
 *
 * Drop-in boundary for ccq (piecuch-group/ccq).  Every entry point is
 * extern "C", takes plain pointers, 64-bit integers (ccq is built with
 * -fdefault-integer-8 / ILP64 BLAS) and FP64 data in the reference's
 * Fortran (column-major) layout, and returns 0 on success or a negative
 * CCQ_B200_E* code; ccq_b200_last_error() gives the message.  A Fortran
 * caller binds them with ISO_C_BINDING interfaces and calls stop_all() on a
 * non-zero status, which keeps ccq's exit-code behaviour (errors.f90:11-27).
 *
 * Two levels:
 *  1. The dgemm.f90 call surface (egemm / egemm1 / egemm2) on host arrays.
 *  2. A resident solver context: integrals and T1..T4 stay in HBM across
 *     iterations; the host driver keeps ccq's loop (solve_cc.f90:175-269)
 *     and calls update + energy through the procedure-pointer slots
 *     update_ptr / calculate_energy_ptr (proc_pointers.f90:7-31).
 */
#ifndef CCQ_B200_H
#define CCQ_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CCQ_B200_OK 0
#define CCQ_B200_EINVAL (-1)     /* bad argument / size                  */
#define CCQ_B200_ECUDA (-2)      /* CUDA runtime error                   */
#define CCQ_B200_ENOMEM (-3)     /* device allocation failed             */
#define CCQ_B200_EPLAN (-4)      /* plan text could not be parsed        */
#define CCQ_B200_ESINGULAR (-5)  /* DIIS system singular (diis.F90:64)   */
#define CCQ_B200_ENODEV (-6)     /* no CUDA device                       */
#define CCQ_B200_ERANGE (-7)     /* size beyond a fixed maximum          */

typedef struct ccq_b200_ctx ccq_b200_ctx;

/* Problem sizes (sys_t, system.f90:60-98).  froz/occ_a/occ_b/orbs are the
 * reference's spatial-orbital counts: occupied alpha = occ_a - froz, etc. */
typedef struct {
    int64_t froz;
    int64_t occ_a;
    int64_t occ_b;
    int64_t orbs;
} ccq_b200_dims;

/* Precision of the bulk contractions (GETT operations on T3/T4 blocks). */
#define CCQ_B200_PREC_FP64 0     /* FP64 DMMA tensor cores                */
#define CCQ_B200_PREC_SPLIT 1    /* Ozaki int8 slices, tcgen05, INT32 acc */

/* ---- level 1: dgemm.f90 call surface (host arrays) ---------------------- */

/* Replaces egemm (src/dgemm.f90:1-29): C(k2,k1) = B(k3,k2)^T A(k3,k1),
 * i.e. dgemm('t','n',k2,k1,k3,1,B,k3,A,k3,0,C,k2).  Column-major host
 * arrays; copies in and out of device memory on every call. */
int ccq_b200_egemm(int64_t k1, int64_t k2, int64_t k3,
                   const double *A, const double *B, double *C);
/* Replaces egemm1 (src/dgemm.f90:31-57): C(k1) = A(k3,k1)^T B(k3). */
int ccq_b200_egemm1(int64_t k1, int64_t k3, const double *A, const double *B, double *C);
/* Replaces egemm2 (src/dgemm.f90:59-73): C(k2) = B(k3,k2)^T A(k3). */
int ccq_b200_egemm2(int64_t k2, int64_t k3, const double *A, const double *B, double *C);

/* egemm in split precision: FP64 operands cut into nslices (2..4) int8
 * slices with a power-of-two scale per row, slice products on the tcgen05
 * tensor pipe with INT32 accumulation, recombined in FP64.  Absolute error
 * about nslices * 2^(-7 nslices - 5) * k3 * max|A col| * max|B col|. */
int ccq_b200_egemm_split(int64_t k1, int64_t k2, int64_t k3,
                         const double *A, const double *B, double *C, int64_t nslices);
/* The same with the kernel chosen: persistent = 0 one CTA per output tile,
 * 1 one CTA per SM walking the tiles with the epilogue overlapped. */
int ccq_b200_egemm_split_kernel(int64_t k1, int64_t k2, int64_t k3, const double *A, const double *B, double *C,
                                int64_t nslices, int64_t persistent);

/* Fortran link-level drop-ins with gfortran's names and by-reference
 * arguments (ILP64 integers): link libccq_b200 in place of dgemm.o. */
void egemm_(const int64_t *k1, const int64_t *k2, const int64_t *k3,
            const double *A, const double *B, double *C);
void egemm1_(const int64_t *k1, const int64_t *k3, const double *A, const double *B, double *C);
void egemm2_(const int64_t *k2, const int64_t *k3, const double *A, const double *B, double *C);

/* egemm on device buffers for callers that cannot allocate device memory.
 * No counterpart in the reference.  Some hosts own all of the GPU's memory
 * through their own pool allocator, or run a time-critical loop in which a
 * cudaMalloc/cudaFree would synchronise the device; this entry point makes no
 * allocation of any kind.  A, B, C are device pointers in the column-major
 * layout of ccq_b200_egemm (C(k2,k1) = B(k3,k2)^T A(k3,k1)); stream is a
 * cudaStream_t (NULL: legacy default stream) and the call only enqueues work
 * on it.  Its scratch (GETT offset tables) is a fixed 1.5 MiB array that each
 * GPU holds from library load until process exit, so k1, k2 and k3 must each
 * be at most 65536 (else CCQ_B200_ERANGE, nothing enqueued).  The first call on
 * a device looks up that array's address; make that first call before any
 * stream capture.  All calls share the one array: calls that overlap on the
 * GPU (different streams, no ordering between them) race on it.  The return
 * code reports argument and launch errors only (a launch error left pending by
 * earlier, unrelated work is cleared on entry and not blamed on this call);
 * errors during execution surface on the stream, like any kernel's. */
int ccq_b200_egemm_dev_noalloc(int64_t k1, int64_t k2, int64_t k3,
                               const double *A, const double *B, double *C, void *stream);

/* ---- level 2: resident solver ------------------------------------------- */

/* Builds a context for calc_type "CCSD", "CCSDT" or "CCSDTQ"
 * (parser.f90:316-432).  f_a, f_b: Fock matrices (orbs x orbs, Fortran
 * order, sys%ints%f_a / f_b); v_aa, v_ab, v_bb: antisymmetrised two-body
 * blocks over the active range ((orbs-froz)^4, Fortran order,
 * sys%ints%v_aa/v_ab/v_bb, integrals.f90:264-276).  rhf != 0 selects the
 * closed-shell copies of update_cc.F90:125-317.  diis_space as in
 * run%diis_space.  The arrays are copied; the caller keeps ownership. */
int ccq_b200_init(const ccq_b200_dims *dims, const char *calc_type,
                  const double *f_a, const double *f_b,
                  const double *v_aa, const double *v_ab, const double *v_bb,
                  int64_t rhf, double shift, int64_t diis_space,
                  ccq_b200_ctx **out);

/* ccq_b200_init for hosts that hold the integrals row-major (C order:
 * f[p][q] over orbs x orbs, v[p][q][r][s] over the active range), such as
 * numpy or C++ arrays.  No counterpart in the reference, whose arrays are
 * Fortran-ordered; it spares such a host two transposed copies of every
 * (orbs-froz)^4 block (one on the host to reach Fortran order, one on the
 * device back to the engine's row-major layout).  Same semantics, sizes and
 * error codes as ccq_b200_init otherwise. */
int ccq_b200_init_rowmajor(const ccq_b200_dims *dims, const char *calc_type,
                           const double *f_a, const double *f_b,
                           const double *v_aa, const double *v_ab, const double *v_bb,
                           int64_t rhf, double shift, int64_t diis_space,
                           ccq_b200_ctx **out);

/* Options of ccq_b200_init_ex. */
typedef struct {
    int64_t rowmajor;     /* 0: f and v Fortran-ordered (as ccq_b200_init), 1: row-major (as ccq_b200_init_rowmajor) */
    int64_t act_occ_b;    /* calc_type "CCSDt": ccq's sys%act_occ_b; -1 otherwise */
    int64_t act_unocc_a;  /* calc_type "CCSDt": ccq's sys%act_unocc_a; -1 otherwise */
} ccq_b200_init_opts;

/* ccq_b200_init with options; the one way to build calc_type "CCSDt"
 * (parser.f90:380-388, update_clusters_t3_opt update_cc.F90:325-2191):
 * triples with at least one active occupied orbital (above act_occ_b) and one
 * active virtual (up to act_unocc_a) are iterated, the others stay zero, and
 * every T3 residual contraction runs only over the active triples' index
 * ranges.  The T vector keeps the full-block layout of get_t_sizes here;
 * ccq_b200_t3_compress / _expand convert to and from ccq's compressed
 * CCSDt layout (get_t_sizes_act). */
int ccq_b200_init_ex(const ccq_b200_dims *dims, const char *calc_type, const ccq_b200_init_opts *opts,
                     const double *f_a, const double *f_b,
                     const double *v_aa, const double *v_ab, const double *v_bb,
                     int64_t rhf, double shift, int64_t diis_space,
                     ccq_b200_ctx **out);

/* ccq's compressed CCSDt T vector (get_t_sizes_act, cc_utils.f90:560-630;
 * the sub-blocks t3A, t3B1..t3B4, t3C1..t3C4, t3D of
 * cc_opt_ccsdt/t2B0000_update_opt.f:48-57) and the full-block T vector of a
 * CCSDt context (get_t_sizes).  Host functions, no context or device needed.
 * ccq_b200_t_size_act returns the compressed length (pos(16) - 1) or a
 * negative error code.  compress copies the active slices out of a full
 * vector; expand writes them back with every antisymmetric copy and zeros
 * elsewhere.  n_full / n_act must equal the two lengths (else
 * CCQ_B200_EINVAL). */
int64_t ccq_b200_t_size_act(const ccq_b200_dims *dims, int64_t act_occ_b, int64_t act_unocc_a);
int ccq_b200_t_compress(const ccq_b200_dims *dims, int64_t act_occ_b, int64_t act_unocc_a,
                        const double *t_full, int64_t n_full, double *t_act, int64_t n_act);
int ccq_b200_t_expand(const ccq_b200_dims *dims, int64_t act_occ_b, int64_t act_unocc_a,
                      const double *t_act, int64_t n_act, double *t_full, int64_t n_full);

/* ---- many independent solves at once --------------------------------------
 * No counterpart in the reference (it solves one system per run).  A batch
 * groups contexts of one calc_type, rhf and diis_space on one device (ccq's
 * CCSD, CCSDT or CCSDTQ plans; not CCSDt or CR-CC(2,3) contexts).  Each
 * batch iteration runs operation k of every active context as one launch (one
 * GETT launch over all their output tiles, one assemble launch over all their
 * canonical elements), then each context's own ring write, residuum and DIIS
 * step (jacobi_iter, solve_cc.f90:175-269, per context).  active[j] != 0 runs
 * context j; e_cor, res and did_diis (arrays of n, may be NULL) receive what
 * ccq_b200_iterate returns for each active context.  The contexts must not be
 * iterated otherwise while in a batch; freeing the batch leaves them intact. */
typedef struct ccq_b200_batch ccq_b200_batch;
int ccq_b200_batch_create(ccq_b200_ctx *const *ctxs, int64_t n, ccq_b200_batch **out);
int ccq_b200_batch_iterate(ccq_b200_batch *batch, int64_t iter, const int64_t *active,
                           double *e_cor, double *res, int64_t *did_diis);
/* launches and device ms of the last batch iteration's sweep */
int ccq_b200_batch_stats(const ccq_b200_batch *batch, int64_t *launches, double *sweep_ms);
int ccq_b200_batch_free(ccq_b200_batch *batch);

/* Length of t_vec (get_t_sizes, cc_utils.f90:479-559) and of the DIIS
 * vector (solve_cc.f90:66-77). */
int ccq_b200_sizes(const ccq_b200_ctx *ctx, int64_t *t_size, int64_t *vec_size);

/* Copy the whole T vector (cc%t_vec layout) to / from the device. */
int ccq_b200_set_t(ccq_b200_ctx *ctx, const double *t_vec, int64_t n);
int ccq_b200_get_t(const ccq_b200_ctx *ctx, double *t_vec, int64_t n);

/* Copy one amplitude block ("T1A".."T3D" inside t_vec, or the T4 blocks
 * "T4A".."T4E" that the reference keeps in its T4 scratch files,
 * cc_utils.f90:89-168) to the device (to_device=1) or back (0).  n must equal
 * the block's element count; layout as the reference's Fortran array. */
int ccq_b200_block(ccq_b200_ctx *ctx, const char *name, double *host, int64_t n, int64_t to_device);

/* One sweep of update_clusters_t4 (update_cc.F90:12-323): the update_ptr
 * slot.  Blocks are updated in place in the reference's order. */
int ccq_b200_update(ccq_b200_ctx *ctx);

/* calculate_unsorted_energy (energy.f90:138-270): calculate_energy_ptr. */
int ccq_b200_energy(ccq_b200_ctx *ctx, double *e_cor);

/* One jacobi_iter step (solve_cc.f90:215-245): update, energy, ring write,
 * residuum, and DIIS when iter % (diis_space+1) == 0.  *did_diis is set to
 * 1 when an extrapolation was applied. */
int ccq_b200_iterate(ccq_b200_ctx *ctx, int64_t iter, double *e_cor,
                     double *residuum, int64_t *did_diis);

/* One iteration from a host t_vec to a host t_vec (the reference's loop when
 * it keeps cc%t_vec on the host): t_in is copied to the device, the sweep
 * runs, and every T1..T3 block is copied to t_out as soon as the sweep has
 * written it for the last time, overlapping the rest of the sweep (in a DIIS
 * iteration the extrapolated vector is copied out whole after the sweep instead).  t_in may equal t_out.  With
 * pageable t_out the copy-out follows the sweep instead of overlapping it.
 * With pinned t_in and t_out and the dependency-graph sweep (use_graph 1),
 * the input is read inside the sweep, block by block, each operation waiting
 * only for the blocks it reads; when t_in is mapped into the device's address
 * space (pinned by cudaHostAlloc, or registered as mapped) the T3 blocks are
 * read there at their canonical elements only (sorted indices within each
 * same-spin run of occupied and of virtual labels), every other element being
 * the antisymmetric image that the reference's t*_update fill writes.
 * Returns what ccq_b200_iterate does. */
int ccq_b200_iterate_host(ccq_b200_ctx *ctx, int64_t iter, const double *t_in, double *t_out, int64_t n,
                          double *e_cor, double *residuum, int64_t *did_diis);

/* Bytes the last ccq_b200_iterate_host moved from host to device and back.
 * No counterpart in the reference. */
int ccq_b200_io_bytes(ccq_b200_ctx *ctx, int64_t *h2d, int64_t *d2h);

/* ccq_b200_iterate in two halves, for many independent solves at once (one
 * context per Hamiltonian, each on its own stream): _async enqueues the
 * iteration and returns; _wait blocks until it is done and returns its
 * outputs.  A context takes one pending iteration at a time. */
int ccq_b200_iterate_async(ccq_b200_ctx *ctx, int64_t iter);
int ccq_b200_iterate_wait(ccq_b200_ctx *ctx, double *e_cor, double *residuum, int64_t *did_diis);

/* Autotuner (no counterpart in the reference): one eager sweep that times every
 * contraction in each candidate configuration (64 x 64 DMMA tiles, skinny DMMA
 * tiles, the small-K FMA kernel; split-K chunk; in split mode int8 slices or
 * DMMA) on scratch output, keeps the
 * fastest per contraction for the later sweeps and restores the amplitudes, so
 * tuning does not count as an iteration.  reps timed runs per candidate;
 * *ms_default / *ms_tuned = summed per-contraction times before / after.
 * Re-run after ccq_b200_set_precision to tune the other mode. */
int ccq_b200_autotune(ccq_b200_ctx *ctx, int64_t reps, double *ms_default, double *ms_tuned);
/* Externally corrected CC (calc_type=CADFCIQMC, src/ext_cor/ext_cor.f90:12-149,
 * src/update_cc.F90:104-109): on a CCSDT or CCSDTQ context, the T3 (and T4)
 * amplitudes stay at the values given by ccq_b200_set_t / ccq_b200_block and
 * only T1 and T2 iterate, with their full T3 / T4 contributions (T1-dressed);
 * DIIS covers T1 + T2 as in the reference's ext_cor runs.  on = 0 restores
 * the full method. */
int ccq_b200_set_external(ccq_b200_ctx *ctx, int64_t on);

/* Active-space CCSDt (calc_type=CCSDt, src/parser.f90:380-388 with
 * act_ind_t = 1): on a CCSDT context, keeps only the triples with at least
 * one active occupied and at least one active virtual index and holds the
 * others at zero.  Active: spatial orbitals act_occ_b < p <= occ (occupied)
 * and occ < p <= act_unocc_a (virtual), both spins, with ccq's
 * act_occ_b = max(occ_b - act_occ, froz), act_unocc_a = min(occ_a + act_unocc,
 * orbs) (src/parser.f90:495-499; 1-based).
 * On a CR-CC(2,3) context (CC(t;3), src/parser.f90:400-411): ccq_b200_crcc23
 * sums only the triples outside that active space, the skip of crcc23
 * (src/mm_correct.f90:61-62,131,190,244,300), for amplitudes set from a
 * CCSDt solve. */
int ccq_b200_set_active(ccq_b200_ctx *ctx, int64_t act_occ_b, int64_t act_unocc_a);

/* Pins every contraction to one GETT kernel family: 0 = by shape, 1 = 64 x 64
 * DMMA tiles, 2 = skinny DMMA tiles (where one side is <= 32), 3 = small-K
 * FMA kernel, 4 = 64 x 64 DMMA tiles with a 3-stage operand pipeline, 5 = skinny
 * DMMA tiles with a 2-stage ring, 6 = register-direct small-K DMMA kernel (the
 * whole K range in one pass).  A family that does not fit a shape falls back to the shape's
 * default.  For tests and experiments; ccq_b200_autotune picks per contraction. */
int ccq_b200_force_tile(ccq_b200_ctx *ctx, int64_t tile);

/* ---- checkpoint / restart ------------------------------------------------
 * The reference's restart (src/solve_cc.f90:56-60, src/utils/cc_utils.f90:89-168)
 * keeps only the T4 files and restarts T1-T3 from zero.  Here a checkpoint
 * holds the resident t_vec, the amplitude blocks kept outside it (T4) and,
 * with with_ring, the DIIS ring, so that a solve continued from it follows
 * the uninterrupted trajectory.  iteration and state[8] are the caller's
 * solver state (iteration number, energy, convergence history), stored
 * as given.  checkpoint_load refuses a file of another system, method or
 * diis_space, and a truncated file, before touching device state.
 * checkpoint_info reads the header: dims = froz, oa, ob, va, vb, rhf,
 * diis_space, t_dev, vec_size. */
int ccq_b200_checkpoint_save(ccq_b200_ctx *ctx, const char *path, int64_t with_ring, int64_t iteration,
                             const double *state);
int ccq_b200_checkpoint_load(ccq_b200_ctx *ctx, const char *path, int64_t *iteration, double *state,
                             int64_t *with_ring);
int ccq_b200_checkpoint_info(const char *path, int64_t *dims, int64_t *iteration, int64_t *with_ring,
                             double *state, char *calc_type, int64_t len);

/* ---- FCIDUMP integrals ---------------------------------------------------
 * Replaces get_fcidump (src/parser.f90:260-313) and load_fcidump
 * (src/integrals.f90:93-210).  fcidump_header: NORB and NELEC of the header
 * (-1 when absent; the reference then sets nel = NELEC, nvirt = 2 NORB - NELEC).
 * fcidump_read: e1int(norb,norb) and e2int(norb,norb,norb,norb), Fortran order,
 * e2int(i,j,a,b) = <ij|ab> = (ia|jb), from the unique integrals of the file
 * (8-fold permutational expansion, orbitals renumbered by ascending orbital
 * energy, later records overwrite earlier ones), *enuc = nuclear repulsion.
 * fcidump_read_device: the same with e2int in device memory, expanded on the
 * GPU (e1int stays a host array). */
int ccq_b200_fcidump_header(const char *path, int64_t *norb, int64_t *nelec);
int ccq_b200_fcidump_read(const char *path, int64_t norb, double *e1, double *e2, double *enuc);
int ccq_b200_fcidump_read_device(const char *path, int64_t norb, double *e1, double *e2_dev, double *enuc,
                                 void *stream);

/* ---- FCIQMC walker files (calc_type=CADFCIQMC) ------------------------------
 * Replaces parse_fciqmc_c3 (src/ext_cor/ext_cor.f90:146-283), the C4 pass of
 * process_fciqmc_c4 (src/ext_cor/contract_t4.f90:12-125) and the cluster
 * analysis (cluster_analysis_up_t3, src/ext_cor/cluster_analysis.f90:10-258;
 * the C4 / T1..T3 products of drive_t4_contraction, contract_t4.f90:241-479).
 * Reads records "c_id coef occ_1 .. occ_m" (m = nel - 2 froz spin orbitals,
 * numbered from the first unfrozen one, odd alpha, even beta), divides every
 * CI coefficient by the Hartree-Fock one and writes T = ln(1 + C) rank by
 * rank: t_vec (t_size = the T1..T3 size, ccq's t_vec layout) holds T1 and T2
 * (zero unless with_sd, the ext_cor_sd key) and T3 on every triple; t4 (may be
 * NULL; t4_size = the five T4 blocks in the layout of ccq_b200_block, T4A..T4E
 * one after the other) holds T4 on every quadruple, C4 entering where the file
 * has one.  info[0..3] = the Hartree-Fock coefficient, records read,
 * distinct quadruples, records above quadruples (skipped).  Host only. */
int ccq_b200_walkers_read(const char *path, const ccq_b200_dims *dims, int64_t nel, int64_t with_sd,
                          double *t_vec, int64_t t_size, double *t4, int64_t t4_size, double *info);

/* ---- learned warm start ---------------------------------------------------------
 * A per-amplitude multilayer perceptron (no counterpart in the reference, which
 * starts every solve from T = 0): y = w3 . tanh(W2 tanh(W1 x + b1) + b2) + b3 with
 * x in R^nfeat (nfeat <= CCQ_B200_MLP_MAXF) and CCQ_B200_MLP_HIDDEN hidden units, FP32.
 * Parameters are one array: W1[H][F] | b1[H] | W2[H][H] | b2[H] | w3[H] | b3.
 * All pointers are device pointers; stream may be NULL (the legacy stream).
 * _params returns the number of parameters for nfeat (or a negative error). */
#define CCQ_B200_MLP_HIDDEN 32
#define CCQ_B200_MLP_MAXF 8
int ccq_b200_mlp_params(int64_t nfeat);
/* y[n] = network(x[n][nfeat]) */
int ccq_b200_mlp_forward(const float *params, int64_t nfeat, const float *x, int64_t n, float *y, void *stream);
/* grad[nparams] = d/dparams of (1/n) sum (y - target)^2, *loss = that mean (both overwritten) */
int ccq_b200_mlp_grad(const float *params, int64_t nfeat, const float *x, const float *target, int64_t n,
                      float *grad, float *loss, void *stream);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected; step counts from 1) */
int ccq_b200_mlp_adam(float *params, const float *grad, float *m, float *v, int64_t nparams, double lr,
                      int64_t step, void *stream);

/* ---- CR-CC(2,3) (calc_type "CR-CC(2,3)") -------------------------------------
 * After the CCSD solve of a context created with calc_type "CR-CC(2,3)", the
 * reference runs hbar2, solve_lcc and crcc23 (src/calc_driver.f90:55-73).
 *
 * ccq_b200_lambda_init replaces hbar2 (src/hbar.f90:10-720) and the setup of
 * solve_lcc (src/solve_cc.f90:101-173): it dresses the Hamiltonian with the
 * current T1, builds the Hbar(CCSD) diagonals used by the left Jacobi step and
 * by crcc23, stores e_cor (the converged CCSD correlation energy, cc%en_cor) and
 * zeroes lambda and its DIIS ring.  Lambda has the T1 + T2 layout of t_vec. */
int ccq_b200_lambda_init(ccq_b200_ctx *ctx, double e_cor);

/* One left-CCSD iteration: update_l2 (every LH from the old lambda, then the
 * Jacobi step with h(a,a) - h(i,i) - E_cor + shift, src/update_lcc.f90:10-280),
 * calculate_left_energy (sqrt(sum LH^2) + E_cor, src/energy.f90:103-136), the
 * ring write, residuum and DIIS of jacobi_iter on l_vec (src/solve_cc.f90:175-269).
 * Outputs as ccq_b200_iterate, with *e_left the left energy. */
int ccq_b200_lambda_iterate(ccq_b200_ctx *ctx, int64_t iter, double *e_left,
                            double *res, int64_t *did_diis);

/* crcc23 (src/mm_correct.f90:11-344): e[0..3] = the triples corrections with
 * denominators A (Fock), B (Hbar one-body), C (+ two-body), D (+ three-body),
 * summed over the unique triples of the four spin blocks.  The reference adds
 * e[3] to the correlation energy (src/mm_correct.f90:342). */
int ccq_b200_crcc23(ccq_b200_ctx *ctx, double e[4]);

/* Copies lambda (T1 + T2 layout, n = T1 + T2 size) to the host. */
int ccq_b200_get_l(ccq_b200_ctx *ctx, double *l_vec, int64_t n);

/* Precision of the bulk contractions; nslices = int8 slices per operand
 * (2..7) for CCQ_B200_PREC_SPLIT. */
int ccq_b200_set_precision(ccq_b200_ctx *ctx, int64_t mode, int64_t nslices);

/* Capture one update+energy sweep in a CUDA graph and replay it: 1 = a graph
 * whose independent contractions run concurrently (side streams, dependencies
 * from the buffers each operation reads and writes), 2 = a single-stream graph
 * (for many contexts running at once), 0 = launch the kernels one by one. */
int ccq_b200_use_graph(ccq_b200_ctx *ctx, int64_t enable);

/* Counters: kernels launched by the last iterate, algorithmic FP64 FLOPs of
 * one update+energy sweep, and the device time of the last sweep in ms. */
int ccq_b200_stats(const ccq_b200_ctx *ctx, int64_t *launches, double *flops, double *sweep_ms);

/* Device time of the last iterate: the update+energy sweep and the whole
 * step including ring write, residuum and DIIS (CUDA events, ms). */
int ccq_b200_timing(const ccq_b200_ctx *ctx, double *sweep_ms, double *iter_ms);

/* Per-kernel profiling of eager sweeps (CUDA events around every launch;
 * disables graph replay while on).  kind: 0 FP64 GETT, 1 split GETT,
 * 2 assemble (gather + Jacobi + fill), 3 other.  Enabling resets the sums. */
int ccq_b200_profile(ccq_b200_ctx *ctx, int64_t enable);
int ccq_b200_profile_get(const ccq_b200_ctx *ctx, int64_t kind, double *ms, double *flops, int64_t *launches);

int ccq_b200_free(ccq_b200_ctx *ctx);

/* Last error message of this thread (NUL-terminated, truncated to len). */
int ccq_b200_last_error(char *buf, int64_t len);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif
