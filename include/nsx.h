/*
 * nsx.h -- C ABI of the B200 (sm_100a) Lanczos hot path for pn-factorised
 * J-scheme shell-model Hamiltonians (the NuLnz / NuTRL solver of NuShellX).
 *
 * The reference has no library API: its hot path is a set of Fortran module
 * subroutines working on module globals.  Each entry point below replaces one
 * of them (cited file:line relative to the NuShellX source tree):
 *
 *   nsx_create / nsx_load_files  <- Lnz_TRD setup          src/NuLnz/NuCoreX.f90:807-1367
 *                                   (+ drdbh pn table        src/NuLnz/NuCoreX.f90:1428-1577)
 *   nsx_matvec                   <- multiplyx(); multiplya(); multiplyb()
 *                                                           src/NuLnz/NuCoreX.f90:76-226
 *   nsx_solve                    <- Lnz_OP + lnzort (standard and thick restart)
 *                                                           src/NuLnz/NuCoreX.f90:240-791
 *   nsx_destroy                  <- (module deallocation at program end)
 *
 * Conventions: every function returns 0 on success or a negative NSX_E* code;
 * nsx_last_error() gives the message of the last failure on the calling
 * thread.  No exceptions or aborts cross this boundary.  A handle is used by
 * one host thread at a time; all device work goes to the stream passed in
 * (NULL = the legacy default stream).  Vectors are FP64 in the reference's
 * layout: blocks (2Ja,2Jb) in ascending order, each a column-major
 * d_a(Ja) x d_b(Jb) matrix with proton partitions along the rows.
 */
#ifndef NSX_H
#define NSX_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NSX_OK 0
#define NSX_E_ARG (-1)      /* invalid argument / inconsistent problem data */
#define NSX_E_IO (-2)       /* file missing, short or malformed record      */
#define NSX_E_CUDA (-3)     /* CUDA runtime failure                          */
#define NSX_E_NOMEM (-4)    /* device or host allocation failed              */
#define NSX_E_NUMERIC (-5)  /* NaN/Inf in the recurrence, eigensolver failure */
#define NSX_E_NOCONV (-6)   /* iteration limit reached before convergence    */

#define NSX_FP64 0          /* matvec contractions in FP64                   */
#define NSX_FP32 1          /* matvec contractions in FP32, FP64 in/out      */

/* One nucleon species, in the content and order of its .tri/.trd/.mat files
 * (src/NuOpd/NuOpd.f90:484-494, 678-680; src/NuOrth/NuOrth.f90:218-223). */
typedef struct nsx_species {
  int32_t nspart;            /* number of partitions                            */
  int32_t minJ2, maxJ2;      /* 2J range of the species (step 2)                */
  const int32_t *njt;        /* [nJ][nspart]: nJT(partition, J), nJ=(maxJ2-minJ2)/2+1 */
  const int32_t *parity;     /* [nspart]: +1 / -1                               */
  int32_t shell_first;       /* global number (1-based) of the species' first shell */
  int32_t nshell;            /* number of shells of the species                 */
  /* one-body reduced densities, one entry per .trd key */
  int32_t nkeys;
  const uint8_t *keys;       /* [nkeys][8]: 2Jl, 2Jr, shell_l, shell_r, 2lam, 0,0,0 */
  const int64_t *val_off;    /* [nkeys+1]: offsets into vals                    */
  const double *vals;        /* values in .trd order (per right partition r, left l
                                with bit l of mask r: nJT(l,Jl) x nJT(r,Jr) col-major) */
  int32_t words;             /* 32-bit mask words per partition                 */
  const uint32_t *masks;     /* [nkeys][nspart][words]                          */
  /* like-particle Hamiltonian segments (.mat), npr >= np */
  int32_t nseg;
  const int32_t *seg_J2;     /* [nseg]                                          */
  const int32_t *seg_np;     /* [nseg] left partition (1-based, as in .mat)     */
  const int32_t *seg_npr;    /* [nseg] right partition (1-based), >= seg_np      */
  const int64_t *seg_off;    /* [nseg+1] offsets into seg_vals                  */
  const double *seg_vals;    /* matrix(dimptr, dimpt) column-major per segment  */
  /* occupation of each of the species' nshell shells per partition (the .tri partition record,
   * [nspart][nshell]); may be null.  With it the result files include NuVec's .xva / .lp. */
  const int16_t *occ;
} nsx_species;

typedef struct nsx_problem {
  int32_t J2;                /* total 2J                                        */
  int32_t parity;            /* +1, -1, or 0 for both (the reference's Tparity) */
  nsx_species a;             /* species "a" (protons)                           */
  nsx_species b;             /* species "b" (neutrons)                          */
  int32_t nop;               /* pn multipole matrix elements (.oph)             */
  const uint8_t *op_keys;    /* [nop][8]: shell_al, shell_ar, shell_bl, shell_br, 2lam, 0,0,0 */
  const double *op_vals;     /* [nop] V_lam in MeV (before renorm)              */
  double renorm;             /* .spe line 2 (src/NuLnz/NuCoreX.f90:1664-1670)   */
} nsx_problem;

typedef struct nsx_params {
  int32_t nev;               /* eigenpairs wanted (reference: no_level)         */
  int32_t max_iter;          /* total Lanczos steps allowed                     */
  int32_t window;            /* thick-restart window (basis vectors kept in HBM)*/
  int32_t keep;              /* Ritz vectors kept at a restart (0 = automatic)  */
  double tol;                /* residual tolerance ||H y - theta y|| (MeV)      */
  int32_t precision;         /* NSX_FP64 or NSX_FP32                            */
  int32_t pre_iter;          /* power pre-iterations on the start vector (ref: 2) */
  uint64_t seed;             /* start-vector seed                               */
  const double *start;       /* optional host start vector [no_state] or NULL   */
  int32_t refine;            /* 1: FP64 Rayleigh-Ritz refinement of the result  */
} nsx_params;

typedef struct nsx_report {
  int32_t iterations;        /* Lanczos steps (matvecs after the pre-iterations) */
  int32_t matvecs;           /* all H.v products, including pre-iterations       */
  int32_t restarts;
  int32_t converged;         /* number of eigenpairs with residual <= tol       */
  double seconds;            /* wall time of nsx_solve                          */
  double matvec_seconds;     /* device time in H.v                              */
  double residual[64];       /* residual norms of the first min(nev,64) pairs    */
} nsx_report;

typedef struct nsx_handle nsx_handle;

/* Build a solver handle from host arrays.  The library copies what it needs
 * to the device; the caller keeps ownership of the host buffers.  With device < 0
 * the handle is plan only: no device memory and no CUDA call, for inspecting a
 * problem (nsx_dim, nsx_blocks, nsx_lcoef, nsx_matvec_flops), loading new
 * interactions and writing result files on a host without a GPU; H.v and solves
 * on it fail with NSX_E_ARG (NSX_E_CUDA from nsx_matvec_noalloc). */
int nsx_create(const nsx_problem *prob, int device, nsx_handle **out);

/* The reference's input file set (src/NuLnz/NuCoreX.f90:1659-1670, 1216-1319).
 * Files read: <a>.tri <a>.trd <b>.tri <b>.trd <inter>.oph <inter>.spe and, for every
 * 2J of each species, <like>file_code(J, T2/2, nmp/2+36)<xtra>.sgt / .mat
 * (src/NuCommon/NuModules.F90:553-597). */
typedef struct nsx_files {
  const char *a, *b, *inter;      /* base names (paths without extension)        */
  const char *like_a, *like_b;    /* nucleus prefix of the .sgt/.mat files        */
  int32_t T2_a, nmp_a;            /* file-code arguments of species a            */
  int32_t T2_b, nmp_b;            /* file-code arguments of species b            */
  char xtra;                      /* character between file code and extension   */
  int32_t J2, parity;             /* target 2J and parity (0 = both)             */
  int32_t nshells;                /* shells of the model space (protons first)   */
  int32_t nshells_p;              /* how many of them are proton shells          */
  const int32_t *shell_parity;    /* [nshells] +1/-1 (the .nus file's sp(i))      */
} nsx_files;

int nsx_load_files(const nsx_files *files, int device, nsx_handle **out);

/* The compressed pn interaction of NuTRLZ (src/NuTRLZ/NuCoreXZ.f90:1613-1887, read from the
 * .dop file that src/NuDiop/NuDiop.f90 writes): for each (2lam, parity) the kept eigenpairs
 * (e, u_e) of the multipole matrix V_lam(proton pair; neutron pair), one term per kept
 * component of an eigenvector.  The handle's proton densities are folded into the combined
 * operators sum_a e u_e(a) rho_a, the neutron densities into sum_b u_e(b) rho_b, and the pn
 * product pairs the combined operators of the same e with the Racah weight alone (the
 * problem's own op_keys / op_vals are not used; renorm is).  Without truncation this is the
 * exact product; with it, the approximation NuTRLZ makes. */
typedef struct nsx_dop {
  int32_t nterms;            /* kept eigenvector components                          */
  const int32_t *lam2;       /* [nterms] 2lam                                         */
  const int32_t *parity;     /* [nterms] +1 / -1: parity of the orbit pairs           */
  const int32_t *eig;        /* [nterms] eigenvector number within its (2lam, parity), 1.. */
  const double *e;           /* [nterms] its eigenvalue (MeV)                          */
  const uint8_t *shells;     /* [nterms][4]: proton shells s1 s3, neutron shells s2 s4 */
  const double *u;           /* [nterms] the component u_e(s1 s3) = u_e(s2 s4)         */
} nsx_dop;
int nsx_create_z(const nsx_problem *prob, const nsx_dop *dop, int device, nsx_handle **out);
/* The same from the file set of nsx_load_files plus the .dop file at dop_path. */
int nsx_load_files_z(const nsx_files *files, const char *dop_path, int device, nsx_handle **out);

/* Replace the interaction of a handle without re-planning: new pn multipole values
 * (op_vals, same count and order as nsx_problem.op_keys at creation, renorm applied as
 * then) and new like-particle segment values (same segments and order as the
 * nsx_species seg_vals at creation, a_nvals / b_nvals values).  The densities, the
 * block structure and every buffer stay as they are; the call copies the new operands
 * to the device synchronously and allocates nothing.  The reference re-runs NuOp and
 * reloads its files for a new interaction (src/NuLnz/NuCoreX.f90:1133-1142 reads the
 * .oph values, 1216-1319 the .mat segments); this is that reload for a handle already
 * in memory, used by interaction sweeps. */
int nsx_set_interaction(nsx_handle *h, const double *op_vals, int32_t nop, const double *a_seg_vals,
                        int64_t a_nvals, const double *b_seg_vals, int64_t b_nvals);

/* The 3-character NuShellX file code (src/NuCommon/NuModules.F90:22-35). */
int nsx_file_code(int32_t i, int32_t j, int32_t k, char out[4]);

int64_t nsx_dim(const nsx_handle *h);          /* no_state (both parities)   */
int32_t nsx_nblocks(const nsx_handle *h);
/* Block list: [nblocks][4] = 2Ja, 2Jb, d_a, d_b, and offsets [nblocks+1]. */
int nsx_blocks(const nsx_handle *h, int32_t *blocks4, int64_t *offsets);
/* Parity mask (the reference's lcoef): [no_state] bytes 0/1. */
int nsx_lcoef(const nsx_handle *h, uint8_t *mask);
/* Algorithmic flop count of one H.v (partition-sparse, reuse-aware). */
double nsx_matvec_flops(const nsx_handle *h);

/* y = H x.  x and y are DEVICE pointers of no_state doubles (stream-ordered).  The first
 * product of a handle creates its auxiliary streams and events (the like-particle stage and the
 * tensor-core classes run beside the main stream, forked from and joined back into it with
 * events): make it outside a stream capture. */
int nsx_matvec(nsx_handle *h, const double *x, double *y, int32_t precision, void *stream);
/* y = H x in FP64 without allocating device memory (no counterpart in the
 * reference).  For callers that cannot have device memory allocated during
 * the call: cudaMalloc synchronises the whole device, and some hosts give all
 * device memory to their own pool.  The intermediates (Y and the stacked
 * Zbar) go to a fixed file-scope device array of 8 Mi FP64 elements (64 MiB, held by every GPU
 * that loads the library until exit); larger problems are rejected with
 * NSX_E_ARG.  The first call on a device looks up the array's address: make it
 * before any stream capture.  All calls share the array; calls that overlap on
 * the GPU race.  x and y are DEVICE pointers; the operator data is the handle's.  It never
 * calls a shard's exchange: on a shard handle it writes the rank's rows only. */
int nsx_matvec_noalloc(nsx_handle *h, const double *x, double *y, void *stream);

/* The same with HOST pointers: copies in, multiplies, copies out, synchronises. */
int nsx_matvec_host(nsx_handle *h, const double *x, double *y, int32_t precision);

/* <psi_i|H|psi_j> between nvec host vectors (vecs: [nvec][no_state], at most 64): the
 * matrix NuXpct forms between stored eigenvectors (src/NuXpct/NuCoreXE.f90:1417-1471),
 * matrixc(i, j) = (H psi_i) . psi_j, returned column-major in out[nvec][nvec]
 * (out[i + nvec*j]).  For eigenvectors it is diagonal with the eigenvalues on it. */
int nsx_expectation_matrix(nsx_handle *h, const double *vecs, int32_t nvec, int32_t precision, double *out);
/* The same on files, as NuXpct runs: the levels of the .xvc file at xvc_path (NuVec's
 * eigenvector file) in, <out_prefix>.ovl (text, 8f10.4 per column) and <out_prefix>.ovx
 * (unformatted: no_levels, then each column in FP32) out. */
int nsx_xpct_files(nsx_handle *h, const char *xvc_path, const char *out_prefix, int32_t precision);

/* Lowest nev eigenpairs.  evals: host [nev]; evecs: host [nev][no_state] or NULL. */
int nsx_solve(nsx_handle *h, const nsx_params *params, double *evals, double *evecs,
              nsx_report *report);

/* The thick-restart state of a solve (the reference's TRL records: .abz matrix and counters,
 * .trl basis vectors, src/NuLnz/NuCoreX.f90:266-292, 455-533): an orthonormal basis V, its
 * projection T = V^T H V (tridiagonal with an arrowhead row after restarts) and the next
 * Lanczos vector, with H V = V T + beta next e_m^T.  As output of nsx_solve_ex, m is the
 * room of V and T in vectors on entry (window + 1 is always enough) and the vectors written
 * on return; the state is the one at convergence. */
typedef struct nsx_state {
  int32_t m;                 /* basis vectors                                         */
  double *V;                 /* [m][no_state] host                                    */
  double *T;                 /* [m][m] column-major host                              */
  double *next;              /* [no_state] host, unit norm                            */
  double beta;               /* coupling of next to the last basis vector             */
  int32_t iterations;        /* Lanczos steps made so far                             */
  int32_t restarts;          /* thick restarts so far                                 */
} nsx_state;
/* nsx_solve, optionally resuming from a saved state (resume: the lowest params->keep Ritz
 * vectors of its basis are kept, its next vector continues the recurrence; the start-vector
 * fields of params are ignored) and optionally returning the final state (state_out). */
int nsx_solve_ex(nsx_handle *h, const nsx_params *params, const nsx_state *resume, nsx_state *state_out,
                 double *evals, double *evecs, nsx_report *report);

/* Many independent solves at once (different J^pi, interaction variants or problems
 * of uneven size): problem i is nsx_solve(handles[i], &params[i], evals[i],
 * evecs ? evecs[i] : NULL, reports ? &reports[i] : NULL).  Every handle solves on its
 * own non-blocking stream from a pool of host threads, so the small problems' kernels
 * and host round trips overlap on the GPU.  The handles must be distinct.  Returns the
 * first failing problem's code, with "problem i: ..." in nsx_last_error().  The
 * reference runs one NuLnz process per J^pi (src/NuShellx/NuShellx.f90:1060-1061). */
int nsx_batch_solve(nsx_handle *const *handles, int32_t n, const nsx_params *params, double *const *evals,
                    double *const *evecs, nsx_report *reports);

/* Write eigenpairs (evals[nev], evecs[nev][no_state], e.g. from nsx_solve) in the
 * reference's output files, as NuTRL leaves them for NuVec (src/NuLnz/NuCoreX.f90:526-533,
 * 280-281; src/NuVec/NuVec.f90:120-131, 182, 281, 285-286, 298-321):
 *   <prefix>.abz  thick-restart form, 4 records: isave = nev, alpha = E, betat = 0,
 *                 matrix = diag(E); imax = iterations, no_level = nev, tt, no_state, basd,
 *                 count = 2, no_keep = no_conv = nev, first_iter, second_iter, noiter;
 *                 bas; alpha_copy, betat(isave+1), indx
 *   <prefix>.trl  one FP32 direct-access record of no_state values per eigenvector
 *   <prefix>.lev  header (intfile, 2J and 2T = T2) and the levels as 5(f10.3,a1)
 *   <prefix>.xvc  NuVec's eigenvector file: (no_state, nev), then (E_i, vector_i) in FP32
 * NuVec's reconstruction from these files returns exactly the given eigenpairs.
 * The reference names prefix Nucleus // file_code(J2/2, no_cA, no_cB). */
int nsx_write_results(const nsx_handle *h, const char *prefix, const double *evals, const double *evecs,
                      int32_t nev, int32_t iterations, const char *intfile, int32_t T2);

/* The thick-restart state in the reference's TRL files, as NuTRL leaves them at convergence
 * (src/NuLnz/NuCoreX.f90:526-533, 280-281): <prefix>.abz with isave = state->m, alpha = diag T,
 * betat = the subdiagonal, matrix = T, the counters, betat(isave+1) = beta; <prefix>.trl with the
 * basis vectors and then the next vector (FP32 records); and, for the given eigenpairs, .lev
 * and (evecs not NULL) .xvc.  NuVec's reconstruction from .abz/.trl gives the Ritz vectors. */
int nsx_write_state(const nsx_handle *h, const char *prefix, const nsx_state *state, const double *evals,
                    const double *evecs, int32_t nev, const char *intfile, int32_t T2);
/* Reads <prefix>.abz / .trl written by nsx_write_state into a state for nsx_solve_ex's resume
 * (the reference's TRL resume reads them at NuCoreX.f90:266-292); state->m is the room of
 * state->V / state->T in vectors on entry. */
int nsx_read_state(const nsx_handle *h, const char *prefix, nsx_state *state);

/* Device-side statistics of a handle (for benchmarking and profiling).
 * Stages of one H.v: 0 = like-particle products (k_like), 1 = neutron-side Y
 * products (k_y), 2 = mixing into the stacked operands (k_z), 3 = proton-side
 * products (k_a), 4 = FP64 <-> FP32 conversions.  With timing enabled every
 * stage launch is bracketed by CUDA events on its stream; nsx_get_stats
 * synchronises and sums them. */
#define NSX_STAGES 5
typedef struct nsx_stats {
  int64_t launches;           /* kernels launched by the library since the reset   */
  int64_t matvecs;            /* H.v products since the reset                        */
  int64_t stage_launches[NSX_STAGES];
  double stage_ms[NSX_STAGES];     /* summed device time per stage (timing enabled only) */
  double stage_bytes[NSX_STAGES];  /* algorithmic HBM bytes of one launch of each stage  */
  double stage_flops[NSX_STAGES];  /* algorithmic flops of one launch of each stage      */
} nsx_stats;

/* Shape of a handle's H.v plan (no counterpart in the reference): which kernel paths its
 * products take and the sizes that select them.  For tests and profiling; works on plan-only
 * handles. */
typedef struct nsx_plan_info {
  int64_t y_elems;            /* Y intermediate elements (k_y path)                           */
  int64_t zbar_elems;         /* stacked operand elements, FP64 row-major layout              */
  int64_t zbar_tc_elems;      /* stacked operand elements, FP32 tensor-core tile layout       */
  int32_t y_row_tiles_max;    /* most 256-row tiles of one Y matrix (k_y)                     */
  int32_t group_sources_max;  /* most sources (h, b) of one mixing group                      */
  int32_t fused_fp32;         /* 1: the fused FP32 variant (Y formed inside the mixing stage)
                               *    is available (every mixing group has at most 16 sources)  */
  int32_t slab_rows_max;      /* longest stacked operand of an output slab                    */
  int32_t slab_splits_max;    /* most K pieces of one FP64 k_a slab tile (atomic partial sums) */
  int32_t slab_nl_max;        /* most rows of a proton partition (an output slab)             */
  int64_t tc_tiles[4];        /* k_a_tc tiles with N = 16, 32, 48, 64                         */
  int64_t tc_chunks_max;      /* most 32-row groups of stacked rows in one k_a_tc tile (piece) */
  int32_t fp32_path;          /* FP32 variant in use (NSX_FP32_*; 0 before the first FP32 H.v) */
  int32_t tc_pieces;          /* k_a_tc tiles that are K pieces of a longer slab (atomic sums)  */
} nsx_plan_info;
int nsx_get_plan_info(const nsx_handle *h, nsx_plan_info *out);

/* Variants of the FP32 product (no counterpart in the reference); all give the FP32 form's
 * accuracy and differ in speed by problem:
 *   NSX_FP32_FUSED  the neutron-side products formed inside the mixing stage (no Y in HBM,
 *                   k_yz), the proton side on the tensor cores (k_a_tc, tcgen05);
 *   NSX_FP32_TC     Y in HBM (k_y), mixing into the tensor-core operand layout (k_z), k_a_tc;
 *   NSX_FP32_SIMT   k_y, k_z and the SIMT proton side (k_a).
 * NSX_FP32_AUTO (the default) times the available variants on the handle's first FP32 product
 * and keeps the fastest; that product synchronises its stream, so make it outside a stream
 * capture (or choose a variant).  The buffers of the variants not kept are freed.  The fused
 * variant needs every mixing group to have at most 16 sources (nsx_plan_info.fused_fp32). */
#define NSX_FP32_AUTO 0
#define NSX_FP32_FUSED 1
#define NSX_FP32_TC 2
#define NSX_FP32_SIMT 3
int nsx_set_fp32_path(nsx_handle *h, int32_t path);

/* Output-block sharding of H.v over `world` GPUs, one process per GPU (the reference splits
 * the same work over OpenMP threads by output block and J_ar, src/NuLnz/NuCoreX.f90:142-220).
 * The blocks are cut into `world` contiguous ranges that minimise the largest range's flops;
 * the handle of rank `rank` plans and computes the output rows of its range only, reading the
 * whole input vector.  Without an exchange, its H.v writes rows [row_begin[rank],
 * row_begin[rank+1]) of y and leaves the others as they were.  With an exchange (below),
 * every product of the handle (nsx_matvec, nsx_solve, nsx_expectation_matrix, ...) ends with
 * fn(user, y, no_state, stream): fn gets y with this rank's rows fresh and must fill the other
 * ranks' rows (an all-gather, e.g. ncclAllGather over the ranks' communicator) before the work
 * it enqueues on `stream` completes, and return 0.  Every rank then runs the same Lanczos
 * recurrence on the whole vector.  Solves and expectation values on a handle with world > 1
 * need an exchange.  world = 1 is the ordinary handle. */
typedef int (*nsx_exchange_fn)(void *user, double *y, int64_t n, void *stream);
int nsx_create_shard(const nsx_problem *prob, int device, int32_t rank, int32_t world, nsx_handle **out);
int nsx_load_files_shard(const nsx_files *files, int device, int32_t rank, int32_t world, nsx_handle **out);
/* rank, world, the rows of every rank (row_begin: world + 1 entries, may be null) and the
 * flops of every rank's product as the split estimated them (world entries, may be null) */
int nsx_shard_info(const nsx_handle *h, int32_t *rank, int32_t *world, int64_t *row_begin, double *est_flops);
int nsx_set_exchange(nsx_handle *h, nsx_exchange_fn fn, void *user);
/* The flops of every output block's rows (nsx_nblocks entries), the costs the split balances;
 * a Y matrix read by several blocks counts for each of them. */
int nsx_block_flops(const nsx_handle *h, double *out);

/* Reset the counters; enable (1) or disable (0) per-stage event timing.  With timing enabled
 * the stages of a product run one after another (no overlap), so each stage's time is its
 * own; a product's whole time is then the stages' sum. */
int nsx_stats_reset(nsx_handle *h, int32_t timing);
int nsx_get_stats(nsx_handle *h, nsx_stats *out);

void nsx_destroy(nsx_handle *h);
const char *nsx_last_error(void);

/* ---- Learned start vector: the network --------------------------------------
 * No counterpart in the reference, whose start vector is always the seeded random
 * one (src/NuLnz/NuCoreX.f90:625-654).  A 3-layer MLP n_in -> width -> width -> n_out
 * with SiLU, FP32 weights and BF16 hidden activations, trained (full-batch Adam on a
 * mean-squared error) and evaluated by the library's own CUDA kernels.  It maps the
 * coefficients of an interaction variant to the compressed ground state (weights on
 * the dominant proton x neutron sub-blocks) from which the host builds the start
 * vector passed to nsx_solve.  Parameters are one flat FP32 array:
 * W1[width][n_in], b1[width], W2[width][width], b2[width], W3[n_out][width], b3[n_out].
 * Inputs x are [batch][n_in], targets and outputs [batch][n_out], all FP32 host
 * arrays.  Errors: negative NSX_E_* codes with nsx_mlp_last_error(). */
typedef struct nsx_mlp nsx_mlp;
int nsx_mlp_create(int32_t n_in, int32_t width, int32_t n_out, uint64_t seed, int device, nsx_mlp **out);
int64_t nsx_mlp_param_count(const nsx_mlp *net);
int nsx_mlp_set_params(nsx_mlp *net, const float *params, int64_t n);  /* also resets Adam */
int nsx_mlp_get_params(const nsx_mlp *net, float *params, int64_t n);
/* y = net(x) */
int nsx_mlp_forward(nsx_mlp *net, const float *x, int32_t batch, float *y);
/* loss = mean (net(x) - t)^2 over batch x n_out, and its gradient w.r.t. the
 * parameters (grad may be NULL; the gradient stays on the device for nsx_mlp_train) */
int nsx_mlp_gradients(nsx_mlp *net, const float *x, const float *t, int32_t batch, float *loss, float *grad);
/* steps of full-batch Adam (beta 0.9 / 0.999, eps 1e-8) at learning rate lr on the
 * batch (uploaded once); loss = the loss after the last step */
int nsx_mlp_train(nsx_mlp *net, const float *x, const float *t, int32_t batch, int32_t steps, float lr, float *loss);
void nsx_mlp_destroy(nsx_mlp *net);
const char *nsx_mlp_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
