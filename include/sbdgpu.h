/*
 * sbdgpu.h -- C ABI of the B200 (sm_100a) tensor-product-basis Davidson path.
 *
 * This is the boundary the header-only C++ host library (sbd::tpb::diag, the
 * drop-in for the reference entry point chemistry/tpb/sbdiag.h:102-113) calls.
 * Plain C types only: pointers, sizes, status codes.  Nothing throws across it.
 *
 * Conventions (all shared with the reference):
 *  - norb <= 64; a string is a uint64 with orbital i at bit i (the reference
 *    packs bit_length bits per size_t word, framework/bit_manipulation.h:158-172;
 *    the host side re-packs).  alpha/beta strings are given in the order the
 *    reference holds them (sorted ascending unless shuffled, main.cc:122-132).
 *  - Wavefunction and sigma vectors are row-major [na][nb]: index ia*nb + ib
 *    (chemistry/tpb/qcham.h:359, mult.h:503), in the reference's interleaved
 *    spin-orbital sign convention (chemistry/basic/determinants.h:98-119).
 *  - One-body integrals h1[p*norb+q] (spatial); two-body integrals in the
 *    reference's 8-fold packed store (chemistry/basic/integrals.h:34-43):
 *    ij = max(i,j)(max(i,j)+1)/2 + min(i,j), element at a(a+1)/2+b with
 *    a = max(ij,kl), b = min(ij,kl); length P(P+1)/2, P = norb(norb+1)/2.
 *  - Status: 0 = success; nonzero = error, text from sbdgpu_last_error().
 *  - Host pointers are synchronous in/out and stay owned by the caller.  Device
 *    memory, the stream and kernels belong to the context.  A context is not
 *    thread-safe: use one per host thread.
 */
#ifndef SBDGPU_H
#define SBDGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sbdgpu_ctx sbdgpu_ctx;

#define SBDGPU_OK 0
#define SBDGPU_ERR_ARG 1
#define SBDGPU_ERR_CUDA 2
#define SBDGPU_ERR_ALLOC 3
#define SBDGPU_ERR_LIMIT 4
#define SBDGPU_ERR_STATE 5

/* Arithmetic of a sigma build. */
#define SBDGPU_FP64 0  /* plain path: every product and sum in FP64 */
#define SBDGPU_MIXED 1 /* FP32 vectors and FP32 sigma; FP64 dot products, Ritz
                          step, residual norms and a final FP64 refinement sigma */
#define SBDGPU_MIXED_TC 2 /* as SBDGPU_MIXED, with the alpha-beta term of sigma on the
                             tensor cores (BF16 operands, FP32 accumulation); the
                             Davidson switches to FP32 sigma once the residual norm
                             is below 1e-2, then refines in FP64 */

/* Davidson options: the reference SBD fields that steer the solver
 * (chemistry/tpb/sbdiag.h:12-30). */
typedef struct sbdgpu_opts {
  int max_it;       /* SBD::max_it (--iteration), restarts */
  int max_nb;       /* SBD::max_nb (--block), Krylov block <= 32 */
  double eps;       /* SBD::eps (--tolerance), residual-norm target */
  double max_time;  /* SBD::max_time, wall-time budget in seconds */
  int precision;    /* SBDGPU_FP64, SBDGPU_MIXED or SBDGPU_MIXED_TC */
  int verbose;      /* 1: print the reference's "Davidson iteration" lines */
  int restart_keep; /* mixed precisions only: Ritz vectors kept at a restart; 0 or 1 =
                       the reference's collapse to the lowest Ritz vector
                       (davidson.h:911-915), k > 1 = thick restart with the k lowest,
                       whose sigma vectors are carried over instead of recomputed */
  int restart_prev; /* mixed precisions only: 1 = also keep the previous step's Ritz
                       vector at a restart (the "+1" of a GD+k restart), with its
                       sigma vector; 0 = not (the reference's behaviour) */
  int precond;      /* mixed precisions only: SBDGPU_PRECOND_DIAGONAL (the reference's
                       correction), SBDGPU_PRECOND_LEARNED or SBDGPU_PRECOND_OLSEN */
} sbdgpu_opts;

/* Davidson correction (sbdgpu_opts.precond). */
#define SBDGPU_PRECOND_DIAGONAL 0 /* t_i = r_i / (E0 - H_ii), davidson.h:853-862 */
#define SBDGPU_PRECOND_LEARNED 1  /* t_i = r_i / (E0 - H_ii - s_i), s_i from the context's
                                     trained network (sbdgpu_precond_train or
                                     sbdgpu_precond_set); falls back to the diagonal
                                     correction when the context has no network, or
                                     for the rest of the run after a restart cycle in
                                     which the residual norm fell by less than 10 % */
#define SBDGPU_PRECOND_OLSEN 2    /* t = P r - eps P w, P = (E0 - H_ii)^-1 regularised as
                                     the diagonal correction, w the Ritz vector and
                                     eps = <w|P r> / <w|P w> (Olsen's correction; no
                                     counterpart in the reference) */

/* Training of the learned preconditioner (no counterpart in the reference). */
typedef struct sbdgpu_learn_opts {
  int pairs;      /* (Ritz vector, residual, correction) triples to harvest: one at the
                     end of each Davidson cycle (FP64, the reference's algorithm) */
  int cycle;      /* Davidson steps per cycle, 1..32 */
  int cg_iters;   /* MINRES steps of each correction solve
                     (I - uu^T)(H - E0)(I - uu^T) t = -r, t orthogonal to u */
  int samples;    /* determinants sampled per triple: half with the largest
                     |t_i|^2 + |r_i|^2, half uniform (weighted), >= 64 */
  int steps;      /* Adam steps, one whole triple's sample per step */
  float lr;       /* Adam learning rate */
  unsigned seed;  /* initial weights and uniform samples */
} sbdgpu_learn_opts;

/* Create a context on CUDA device `device` for one alpha x beta product basis
 * and Hamiltonian.  Replaces the set-up half of sbd::tpb::diag
 * (chemistry/tpb/sbdiag.h:143-166: SetupIntegrals, TaskCommunicator,
 * MakeHelpers/RemakeHelpers).  Copies all inputs. */
int sbdgpu_create(sbdgpu_ctx** out, int norb, size_t na, size_t nb, const uint64_t* astr,
                  const uint64_t* bstr, double ecore, const double* h1, const double* eri_packed,
                  int device);

/* Build the excitation tables on the GPU.  Replaces GenerateExcitation /
 * MakeSmartHelper (chemistry/tpb/helper.h:132-182, 352-422).  Called
 * implicitly by every routine that needs the tables. */
int sbdgpu_build_tables(sbdgpu_ctx* ctx);

/* Table sizes for spin (0 alpha, 1 beta): total singles and doubles entries. */
int sbdgpu_table_sizes(sbdgpu_ctx* ctx, int spin, uint64_t* n_singles, uint64_t* n_doubles);

/* Copy one spin's tables to the host in the reference helper layout: for bra
 * string i, kets single_idx[single_off[i] .. single_off[i+1]) ascending
 * (SinglesFromAlphaSM / SinglesFromAlphaLen, helper.h:352-422); same for
 * doubles.  Offsets have n+1 entries. */
int sbdgpu_get_tables(sbdgpu_ctx* ctx, int spin, uint64_t* single_off, uint64_t* single_idx,
                      uint64_t* double_off, uint64_t* double_idx);

/* Diagonal H_ii for every determinant (row-major).  Replaces
 * makeQChamDiagTerms (chemistry/tpb/qcham.h:314-366). */
int sbdgpu_diag(sbdgpu_ctx* ctx, double* hii);

/* sigma = H*C with host vectors (na*nb doubles each).  Replaces the direct
 * mult (chemistry/tpb/mult.h:387-648); unlike mult, sigma is overwritten
 * rather than accumulated into. */
int sbdgpu_sigma(sbdgpu_ctx* ctx, const double* C, double* sigma, int precision);

/* sigma = H*C with device vectors (na*nb doubles each, on this context's
 * device).  The work is issued on the context's stream; the call returns
 * after it completes. */
int sbdgpu_sigma_device(sbdgpu_ctx* ctx, const double* dC, double* dsigma, int precision);

/* Rows [r0, r1) of sigma = H*C, FP64, for the full vector C (device, na*nb
 * doubles) into sigma_rows (device, (r1-r0)*nb doubles): one rank's share when
 * W and sigma are split into blocks of alpha rows over several GPUs, the
 * reference's adet_comm split (chemistry/tpb/helper.h:505-540, ranges from
 * get_mpi_range, framework/mpi_utility.h:14-36).  The rank gathers C from the
 * others first (one all-gather per sigma, the counterpart of the reference's
 * Mpi2dSlide ring, mult.h:440-443, 612-621); every term of its rows is then
 * summed locally, so no reduction of sigma follows (mult.h:630-631). */
int sbdgpu_sigma_rows_device(sbdgpu_ctx* ctx, const double* dC, double* dsigma_rows, size_t r0, size_t r1);

/* sigma = H*C with device vectors, for callers that cannot allocate device
 * memory during the call (a pre-reserved memory pool or arena owns the
 * device, or the call sits on a path that must not synchronise the device as
 * cudaMalloc/cudaFree can).  No counterpart in the reference.  It allocates
 * nothing: its scratch is one 12 MiB file-scope device array (3 x 524,288
 * doubles) that every GPU with a context holds until exit.  Limits:
 * na*nb <= 524,288 (SBDGPU_ERR_LIMIT otherwise); the context's set-up must be
 * done first (sbdgpu_build_tables and sbdgpu_diag, else SBDGPU_ERR_STATE).
 * sbdgpu_create resolves the array's address on its device and loads the
 * sigma kernels there, so the call itself loads no module (CUDA's lazy
 * loading would otherwise allocate inside it).  All calls share the array, so
 * calls that overlap on the GPU race.  Same result as sbdgpu_sigma_device,
 * FP64 only. */
int sbdgpu_sigma_device_noalloc(sbdgpu_ctx* ctx, const double* dC, double* dsigma);

/* Block Davidson for the nroots lowest roots, FP64 (an extension: the
 * reference's Davidson, chemistry/tpb/davidson.h:661-923, follows the lowest
 * root only).  Each cycle adds one diagonally preconditioned correction per
 * unconverged root; when the basis would pass opts->max_nb vectors
 * (2*nroots <= max_nb <= 32) it collapses to the Ritz vectors.  Stops when
 * every residual norm is below opts->eps, after opts->max_it cycles, or at
 * opts->max_time seconds.
 *   W         [nroots][na*nb], reference convention.  In: initial vectors, or
 *             all zeros for determinant 0 and the lowest-H_ii determinants.  Out: the
 *             normalised Ritz vectors.
 *   energies  out [nroots]: Ritz values, ascending
 *   resid     out [nroots] (may be NULL): residual norms
 *   n_iter, n_sigma  out (may be NULL): cycles, sigma builds */
int sbdgpu_davidson_roots(sbdgpu_ctx* ctx, const sbdgpu_opts* opts, int nroots, double* W, double* energies,
                          double* resid, int* n_iter, int* n_sigma);

/* Lowest-root Davidson (as sbdgpu_davidson, same opts) for nprob independent
 * problems at once (an extension; the reference has none).  FP64 contexts on
 * one device run a device-resident Davidson: every step of a problem (its
 * correction, Gram-Schmidt, sigma, projected row, small eigenproblem, Ritz
 * update and norms) is one replayed CUDA graph on the context's stream, one
 * host thread launches a step for every unconverged problem and waits once
 * per round, and all vectors come from one device allocation made before the
 * first round.  Other precisions, stored Hamiltonians or several devices run
 * each problem's sbdgpu_davidson in turn.  W[i]: problem i's initial vector
 * in, Ritz vector out (reference convention); energies[i], n_steps[i] (may be
 * NULL) and status[i] (may be NULL) per problem.  Returns SBDGPU_OK or the
 * first error status.  The contexts must be distinct and not used by other
 * threads meanwhile.  max_threads is not used (kept for the signature). */
int sbdgpu_davidson_batch(int nprob, sbdgpu_ctx* const* ctxs, const sbdgpu_opts* opts, double* const* W,
                          double* energies, int* n_steps, int* status, int max_threads);

/* Method 1 (--method 1): build the Hamiltonian's off-diagonal elements once
 * and keep them in device memory, CSR by bra determinant (4-byte ket index and
 * FP64 value per element, 12 bytes); every later FP64 sigma of this context,
 * the ones inside sbdgpu_davidson included, is then a sparse product with it.
 * Replaces makeQCham (chemistry/tpb/qcham.h:10-312), which stores the same
 * elements as (bra, ket, Hij) triplets, and the stored mult
 * (chemistry/tpb/mult.h:13-123).  FP32 and the no-allocation sigma keep the
 * on-the-fly build.  nnz (out, may be NULL): elements stored.
 * SBDGPU_ERR_LIMIT when the elements do not fit in free device memory (with
 * 1 GiB to spare) or na*nb >= 2^32. */
int sbdgpu_store_hamiltonian(sbdgpu_ctx* ctx, uint64_t* nnz);

/* Frees the stored Hamiltonian; later sigma builds are on the fly again. */
int sbdgpu_release_hamiltonian(sbdgpu_ctx* ctx);

/* Restarted Davidson for the lowest root, the reference algorithm of
 * chemistry/tpb/davidson.h:661-923 (block <= max_nb, collapse restart,
 * diagonal preconditioner with eps_reg = 1e-12, modified Gram-Schmidt,
 * wall-time budget), followed by E = <W|HW> from one more sigma
 * (sbdiag.h:239-262).
 *   W         in: initial vector (na*nb, normalised or not); out: Ritz vector
 *   energy    out: <W|HW>
 *   trace_e / trace_tol  optional (may be NULL): lowest Ritz value and residual
 *             norm per step, up to max_trace entries
 *   n_steps   out: steps taken (sigma builds inside the loop) */
int sbdgpu_davidson(sbdgpu_ctx* ctx, const sbdgpu_opts* opts, double* W, double* energy,
                    double* trace_e, double* trace_tol, int max_trace, int* n_steps);

/* One- and two-particle RDMs of W in the reference layout
 * one[s*L*L + i + L*j], two[(s + 2t)*L^4 + i + L*j + L^2*k + L^3*l]
 * (chemistry/tpb/correlation.h:194-443, docs/user-guide.md:138-139). */
int sbdgpu_rdm(sbdgpu_ctx* ctx, const double* W, double* one, double* two);

/* Orbital occupations density[2p] (alpha), density[2p+1] (beta).  Replaces
 * OccupationDensity (chemistry/tpb/occupation.h:10-95). */
int sbdgpu_occupation(sbdgpu_ctx* ctx, const double* W, double* density);

/* Per-alpha-string weights D[ia] = sum_ib W[ia,ib]^2, the input of the
 * carry-over selection (DiagonalReducedDensityMatrix, chemistry/tpb/rdmat.h:11-58). */
int sbdgpu_alpha_weights(sbdgpu_ctx* ctx, const double* W, double* D);

/* CUDA-event times in milliseconds of the last sigma build, on the context's
 * stream: ms5[0] diagonal + alpha same-spin kernel, [1] beta same-spin
 * (transposes included), [2] alpha-beta kernel, [3] the whole build on device
 * vectors (sign phases included), [4] for sbdgpu_sigma only: end to end from
 * the start of the host-to-device copy to the end of the device-to-host copy
 * (0 after a device-vector call).  No counterpart in the reference, which
 * prints wall-clock timers (chemistry/tpb/mult.h:435-446, 619-646). */
int sbdgpu_last_sigma_ms(sbdgpu_ctx* ctx, float* ms5);

/* Diagnostic of the bounded wait that the tensor-core kernel uses on its
 * MMA-completion barrier (no reference counterpart).  Launches one warp that
 * waits on a barrier nobody arrives on, polling at most spin_limit times, and
 * one that arrives first.  status[0] = 1 when the first wait gave up (the
 * expected outcome), status[1] = 0 when the second completed.  The context
 * stays usable either way.  spin_limit in [1, 2^26] (the kernel's own limit),
 * else SBDGPU_ERR_ARG; each wait also gives up after 2 s of GPU time. */
int sbdgpu_wait_selftest(sbdgpu_ctx* ctx, long long spin_limit, int* status);

/* Learned preconditioner (no counterpart in the reference; it replaces the
 * diagonal correction of chemistry/tpb/davidson.h:853-862 when
 * opts->precond = SBDGPU_PRECOND_LEARNED).  A network of 3 layers (48 features
 * -> 128 -> 128 -> 1, BF16 weights) maps per-determinant features (H_ii - E0,
 * |r_i|, holes and particles within 8 orbitals of each spin's Fermi level,
 * excitation ranks) to a shift s_i of the diagonal denominator.
 * sbdgpu_precond_train harvests triples on this context's system (on the GPU,
 * with this library's sigma) and trains the network on them with the
 * library's own forward and backward kernels.  loss_trace [steps] and
 * seconds [2] (harvest, training) may be NULL. */
int sbdgpu_precond_train(sbdgpu_ctx* ctx, const sbdgpu_learn_opts* opts, double* loss_trace, double* seconds);

/* The context's network weights (FP32 master copy): with w == NULL only *n is
 * set.  A network trained on one system may be loaded into the context of
 * another with sbdgpu_precond_set (the features do not depend on norb). */
int sbdgpu_precond_get(sbdgpu_ctx* ctx, float* w, int* n);
int sbdgpu_precond_set(sbdgpu_ctx* ctx, const float* w, int n);

/* The learned correction of one residual: out_i = R_i / (e0 - H_ii - s_i),
 * host vectors of na*nb doubles (either sign convention: the network sees
 * |R_i|).  Runs the tensor-core inference kernel. */
int sbdgpu_precond_apply(sbdgpu_ctx* ctx, const double* R, double e0, double* out);

/* Loss and gradient of the network's training kernels for master weights w
 * and B samples with features X [B][48] (FP32), residuals r, denominators
 * den = E0 - H_ii, Ritz-vector components u, target corrections t and
 * weights wt, on CUDA device `device` (for checking the kernels' gradients;
 * S = the shift scale, 0.5 in training). */
int sbdgpu_mlp_loss_grad(int device, const float* w, int B, const float* X, const double* r, const double* den,
                         const double* u, const double* t, const double* wt, double S, double eps_reg,
                         double* loss, float* grad);

/* Launch shape of the FP64 alpha-beta kernel (an extension): ab_group alpha
 * singles per CTA (16, 8, 4, 2 or 1, where the integral block fits in shared
 * memory beside a row of C) and ab_threads threads per CTA (128, 256, 512 or
 * 1024); (0, 0) restores the default (the largest group that fits; 512
 * threads while two CTAs fit an SM, else 1024, halved down to 128 while the
 * warps outnumber the 32-string slices of beta strings).  A shape that does not fit the
 * basis is refused. */
int sbdgpu_set_tuning(sbdgpu_ctx* ctx, int ab_group, int ab_threads);

/* Time every alpha-beta shape that fits (reps FP64 sigma builds each, after
 * one warm-up) and keep the fastest on the context; its shape and sigma time
 * in *ab_group, *ab_threads, *best_ms (each may be NULL). */
int sbdgpu_autotune(sbdgpu_ctx* ctx, int reps, int* ab_group, int* ab_threads, float* best_ms);

/* How the FP64 sigma forms its same-spin terms (an extension): method 0 (the
 * default) = as exact INT8 tensor-core products of the dense string-only
 * operator (residues modulo 15 primes, CRT reconstruction; FP64-accurate: the
 * scaled operands are rounded to 49-bit integers) where both spins have at
 * least 1,024 strings (multiples of 4) and the residues fit in device memory,
 * else the rows kernels; method 1 = the rows kernels always (and the device
 * memory of the integer products is released). */
int sbdgpu_set_fp64_same_spin(sbdgpu_ctx* ctx, int method);

const char* sbdgpu_last_error(sbdgpu_ctx* ctx);
void sbdgpu_destroy(sbdgpu_ctx* ctx);

/* ---- The generic path: a second-quantised operator on a basis of bit strings
 * (basic/generalop.h GeneralOp, basic/basis.h Basis,
 * basic/out_of_place_func/mult.h, lanczos.h, davidson.h). ---- */

typedef struct sbdgpu_genop sbdgpu_genop;

/* Maximum field operators in one term, and words (64 sites each) per state. */
#define SBDGPU_GENOP_MAX_OPS 16
#define SBDGPU_GENOP_MAX_WORDS 4

/* A basis of nstates bit strings on CUDA device `device`: state i is
 * states[i*nwords .. i*nwords+nwords), site q at bit q%64 of word q/64
 * (1 <= nwords <= 4).  Any order; vectors follow it.  A repeated state is
 * refused (SBDGPU_ERR_ARG).  sign = 1: fermionic signs (each operator counts
 * the occupied sites below its own, basic/out_of_place_func/mult.h:213-240 with
 * framework/bit_manipulation.h:943-962); 0: none.  Replaces Basis::Init
 * (basis.h:208-256) at one rank.  Copies all inputs. */
int sbdgpu_genop_create(sbdgpu_genop** out, int device, int nwords, size_t nstates, const uint64_t* states,
                        int sign);

/* The operator, as GeneralOp keeps it (generalop.h:17-826): n_diag terms of
 * the diagonal list (d_, e_) and n_off of the off-diagonal list (o_, c_).
 * Term k of a list has the field operators ops[off[k] .. off[k+1]) in the
 * order written, each site | dag << 16, n_dag[k] of them creation operators
 * (ProductOp::n_dag), coefficient coef[k].  As in mult.h:118-144 a diagonal
 * term adds coef * C_i where the sites of its first n_dag operators are all
 * occupied; as in mult.h:207-256 an off-diagonal term annihilates the sites of
 * its first n_dag operators from the bra state in turn and creates those of
 * the rest, and adds coef * sign * C_j when the result is basis state j.
 * Replaces any earlier operator.  At most SBDGPU_GENOP_MAX_OPS operators per
 * term, sites below 64 * nwords. */
int sbdgpu_genop_set_terms(sbdgpu_genop* g, size_t n_diag, const int64_t* diag_off, const int32_t* diag_ops,
                           const int32_t* diag_ndag, const double* diag_coef, size_t n_off, const int64_t* off_off,
                           const int32_t* off_ops, const int32_t* off_ndag, const double* off_coef);

/* The quantum-chemistry Hamiltonian of an FCIDUMP file as the operator
 * (GeneralOp_From_FCIDump, basic/out_of_place_func/stdmodel.h:13-98: alpha
 * orbital p at site p, beta at site p + norb), in place of
 * sbdgpu_genop_set_terms; *norb and *nelec from the file's header.  The
 * integrals are used at full precision (the reference's MpiBcast of the
 * FCIDUMP re-reads them at six significant digits). */
int sbdgpu_genop_set_fcidump(sbdgpu_genop* g, const char* path, int* norb, int* nelec);

/* W += H C (mult.h:268-291 at one rank: the diagonal list, then the
 * off-diagonal one).  Host vectors of nstates doubles; the _device form takes
 * device pointers, runs on the object's stream and returns when it is done. */
int sbdgpu_genop_mult(sbdgpu_genop* g, const double* C, double* W);
int sbdgpu_genop_mult_device(sbdgpu_genop* g, const double* dC, double* dW);

/* <i|H|i> for every basis state (the diagonal terms plus the off-diagonal ones
 * that map a state onto itself). */
int sbdgpu_genop_diagonal(sbdgpu_genop* g, double* hii);

/* Lanczos for the lowest eigenvalue (lanczos.h:176-310): W (normalised) is the
 * start vector and receives the Ritz vector, rebuilt by a second pass of the
 * recurrence; stops when the lowest Ritz value moves by less than eps, when a
 * new Lanczos coefficient is below eps, or after max_it steps.  *energy = the
 * lowest Ritz value; *n_iter = Lanczos steps taken.  No reorthogonalisation,
 * as in the reference. */
int sbdgpu_genop_lanczos(sbdgpu_genop* g, double* W, int max_it, double eps, double* energy, int* n_iter);

/* Davidson for the lowest eigenvalue with on-the-fly sigma (the algorithm of
 * basic/out_of_place_func/davidson.h:19-196 and chemistry/tpb/davidson.h:
 * collapse restart, diagonal correction r_i / (E0 - H_ii)); opts->max_it,
 * max_nb, eps, verbose are used.  Traces as sbdgpu_davidson. */
int sbdgpu_genop_davidson(sbdgpu_genop* g, const sbdgpu_opts* opts, double* W, double* energy, double* trace_e,
                          double* trace_tol, int max_trace, int* n_steps);

/* <W|H^2|W> as MeasHamSquare computes it (expand.h:10-215): every basis
 * state weighted by the diagonal list, every configuration an off-diagonal
 * term reaches from basis state i weighted coef * sign * W_i (inside the basis
 * or not), equal configurations summed, then the sum of squares.  W: host
 * vector of nstates doubles. */
int sbdgpu_genop_ham_square(sbdgpu_genop* g, const double* W, double* res);

/* The expanded basis of ExpandBasis (expand.h:217-366): the basis states and
 * every configuration an off-diagonal term reaches from basis state i with
 * |coef * sign * W_i| > eps_hb, distinct, ascending as nwords-word integers
 * (word nwords-1 most significant).  *n_out receives their number; with out
 * == NULL nothing else is written, else out must hold capacity >= *n_out
 * states of nwords words (SBDGPU_ERR_LIMIT otherwise). */
int sbdgpu_genop_expand(sbdgpu_genop* g, const double* W, double eps_hb, uint64_t* out, size_t capacity,
                        size_t* n_out);

const char* sbdgpu_genop_last_error(sbdgpu_genop* g);
void sbdgpu_genop_destroy(sbdgpu_genop* g);

#ifdef __cplusplus
}
#endif

#endif /* SBDGPU_H */
