/*
 * sbdx.h: C-ABI of the B200 (sm_100a) implementation of the sbd
 * tensor-product-basis selected-CI hot path (walkup/sbd-ykt, namespace
 * sbd::tpb). Plain pointers and sizes only; every call returns an int status
 * (SBDX_OK = 0) and sbdx_last_error() describes the last failure. No C++
 * exception crosses this boundary. A context is affine to one host thread and
 * one CUDA device; it owns every device buffer it allocates, the caller owns
 * every host buffer it passes.
 *
 * Layout conventions (shared by all entry points):
 *   - a spin string is one uint64, bit p = spatial orbital p, L <= 64. The
 *     reference packs bit_length bits per size_t word
 *     (framework/bit_manipulation.h:158-172); numeric uint64 order equals the
 *     reference's word-reversed lexicographic order (bit_manipulation.h:26-43);
 *   - determinant (ia, ib) has vector index ia*nb + ib (alpha-major), as the
 *     reference's braIdx (chemistry/tpb/mult.h:487-488);
 *   - h is the L*L one-electron matrix (row-major, symmetric); eri is the
 *     8-fold packed two-electron array of twoInt::store
 *     (chemistry/basic/integrals.h:51-59): index canon(pq, rs) with
 *     pq = max(p,q)*(max(p,q)+1)/2 + min(p,q) and
 *     canon(x, y) = max(x,y)*(max(x,y)+1)/2 + min(x,y);
 *   - 1-RDM: 2 blocks of L*L, element [s][p + L*q]; 2-RDM: 4 blocks of L^4,
 *     element [s + 2t][i + L*j + L^2*k + L^3*l], the reference's
 *     one_p_rdm / two_p_rdm (chemistry/tpb/correlation.h:211-218).
 */
#ifndef SBDX_H
#define SBDX_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SBDX_OK 0
#define SBDX_ERR_ARG 1      /* invalid argument (size, pointer, range)         */
#define SBDX_ERR_CUDA 2     /* CUDA runtime error                               */
#define SBDX_ERR_STATE 3    /* call out of order (e.g. sigma before strings)    */
#define SBDX_ERR_NOMEM 4    /* device allocation failed                         */
#define SBDX_ERR_NUMERIC 5  /* non-finite input or breakdown                    */

#define SBDX_FP64 0
#define SBDX_FP32 1

typedef struct sbdx_ctx sbdx_ctx;

/* Context lifetime. Replaces the MPI communicator set-up of tpb::diag at
 * world size 1 (chemistry/tpb/helper.h:199-233, TaskCommunicator). */
int sbdx_ctx_create(sbdx_ctx** ctx, int device);
int sbdx_ctx_destroy(sbdx_ctx* ctx);
const char* sbdx_last_error(const sbdx_ctx* ctx);
/* Stream used by all subsequent work (a cudaStream_t; NULL = legacy stream). */
int sbdx_set_stream(sbdx_ctx* ctx, void* cuda_stream);
/* Kernels launched by this context since creation (instrumentation). */
unsigned long long sbdx_launch_count(const sbdx_ctx* ctx);
/* Instrumentation with no reference counterpart (the reference prints wall
 * timers, sbdiag.h:171-262): when on, every sigma records CUDA events between
 * its five phases (alpha same-spin, transpose, beta same-spin, alpha-beta,
 * combine) and accumulates their durations; this adds one host sync per sigma.
 * sbdx_phase_times copies up to n accumulated milliseconds and returns the
 * number of sigma calls timed; on == 0 also resets the accumulators. */
int sbdx_set_profiling(sbdx_ctx* ctx, int on);
long long sbdx_phase_times(sbdx_ctx* ctx, double* ms, int n);
/* Launch shapes of the sigma kernels (no reference counterpart), applied to
 * both precisions; 0 selects the built-in default (alpha-first kernels; the
 * blocked same-spin kernel from 2 M determinants in FP64 and 1 M with FP32
 * storage, the one-string-per-CTA kernel below).
 * Alpha-first kernels (the sigma evaluated in the alpha-before-beta
 * determinant ordering, conjugated by the +-1 basis phase):
 *   same_code: 21/22/24/28 = 1/2/4/8 columns per thread, one bra string per
 *              CTA; 31/32/34/38 = the same widths for blocks of 4 bra strings
 *              that walk the union of their double-excitation lists once;
 *   ab_code:   61-64 = 1-4 staged ket rows of the balanced alpha-beta kernel,
 *              71 = the same with the rows packed in 16-byte elements (2 FP64
 *              or 4 FP32 rows per group; falls back to 62/64 when nb is too
 *              large for the packs to fit in shared memory).
 * Interleaved-ordering kernels (kept for comparison; both codes must then
 * come from this family):
 *   same_code: 1/2/4/8 = columns per thread of the prefix-parity-table
 *              same-spin kernel, 11/12/14 = 1/2/4 columns of the popcount one;
 *   ab_code:   10*variant + staged ket rows (1-4) of the alpha-beta kernel,
 *              variant 0 = L1 gathers, 1 = shared-memory staging, 2 =
 *              double-buffered TMA staging, 3 = staging with two 512-thread
 *              CTAs per SM, 4 = staging with SELL-32 beta records.
 * Shapes that do not fit the problem (alignment, shared memory) are narrowed. */
int sbdx_set_tuning(sbdx_ctx* ctx, int same_code, int ab_code);
/* Autotuner: times the candidate codes on the current problem (a few sigma
 * products on scratch vectors, for FP64 and for FP32 separately) and keeps the
 * fastest; writes the FP64 choice. */
int sbdx_autotune(sbdx_ctx* ctx, int* same_code, int* ab_code);

/* Integrals. Replaces SetupIntegrals (chemistry/basic/makeintegrals.h:81-126)
 * with exact doubles (the struct path of tpb::diag, sbdiag.h:157). eri_len
 * must equal P*(P+1)/2 with P = L*(L+1)/2. Non-finite values -> SBDX_ERR_NUMERIC. */
int sbdx_set_integrals(sbdx_ctx* ctx, int norb, double I0, const double* h, const double* eri,
                       size_t eri_len);

/* Sampled alpha and beta strings (the adet/bdet arguments of tpb::diag,
 * chemistry/tpb/sbdiag.h:116-117). Strings must be unique; sorted ascending for
 * index 0 to be the Aufbau start vector, as LoadAlphaDets leaves them
 * (chemistry/basic/makedeterminants.h:184). All alpha strings must have the
 * same popcount, and all beta strings likewise. At most 16,777,215 strings
 * per spin (the excitation records hold 24-bit string indices). */
int sbdx_set_strings(sbdx_ctx* ctx, const uint64_t* alpha, size_t na, const uint64_t* beta, size_t nb);

/* Excitation connectivity. Replaces MakeHelpers/RemakeHelpers + GenerateExcitation
 * (chemistry/tpb/helper.h:132-197, 447-968) at world size 1. */
int sbdx_build_connectivity(sbdx_ctx* ctx);
/* Total entries (singles + doubles) of spin 0 (alpha) or 1 (beta). */
int sbdx_connectivity_size(sbdx_ctx* ctx, int spin, uint64_t* n_entries);
/* The helper lists in MakeSmartHelper's flattened layout
 * (chemistry/tpb/helper.h:367-437): per bra string, its singles then its
 * doubles, ascending ket index; slen/dlen: per-bra list lengths. */
int sbdx_get_connectivity(sbdx_ctx* ctx, int spin, uint64_t* slen, uint64_t* dlen, uint64_t* idx);

/* Stored Hamiltonian, the reference's method 1 (chemistry/tpb/sbdiag.h:275-330:
 * makeQCham, chemistry/tpb/qcham.h:10-312, then the stored-element mult,
 * chemistry/tpb/mult.h:13-123). Builds every off-diagonal H_IJ on the device
 * (CSR over determinant rows, FP64 values with the determinant phases, 32-bit
 * columns: 12 bytes per element) after the connectivity and the diagonal;
 * from then on every FP64 sigma of this context (sbdx_sigma, sbdx_sigma_device
 * with SBDX_FP64, the Davidson solvers' FP64 products) is its sparse product,
 * and FP32 sigmas stay on the fly. *nnz (may be NULL) receives the number of
 * stored elements. SBDX_ERR_NOMEM, with the size in the message, when the
 * matrix does not fit. New strings, integrals or connectivity drop it. */
int sbdx_build_hamiltonian(sbdx_ctx* ctx, uint64_t* nnz);
/* Frees the stored matrix; FP64 sigmas go back to the on-the-fly kernels. */
int sbdx_release_hamiltonian(sbdx_ctx* ctx);

/* Diagonal H_II for all determinants. Replaces makeQChamDiagTerms
 * (chemistry/tpb/qcham.h:314-366). hii: host buffer of na*nb doubles (may be
 * NULL to only compute the device copy). */
int sbdx_diag_terms(sbdx_ctx* ctx, double* hii);

/* Diagonal H_II computed without any device allocation. This entry point has no
 * counterpart in the reference; it returns the same values as sbdx_diag_terms.
 *
 * For callers that must not have a library allocate or free device memory:
 * code whose device memory all comes from its own pre-sized pool or framework
 * allocator, and code that records its stream into a replayable sequence where
 * a cudaMalloc/cudaFree would either be refused or synchronise the device.
 * No context is used: every input is a device pointer the caller owns.
 *   d_h     L*L FP64, row-major;  d_eri  8-fold packed (pq|rs) FP64
 *   d_alpha na uint64 strings;    d_beta nb uint64 strings (bits >= norb ignored)
 *   d_hii   na*nb FP64 output, alpha-major (index ia*nb + ib)
 *   stream  cudaStream_t to launch on (NULL = legacy default stream)
 * The intermediate per-string energies and beta Coulomb rows live in one
 * fixed file-scope device array of 524288 doubles (4 MiB) per GPU; a call needs
 * na + nb + nb*norb <= 524288 and na <= 65535, else it returns SBDX_ERR_ARG
 * with a message in errbuf and launches nothing. Nothing has to start at zero:
 * each call writes every scratch word before reading it.
 * The first call on each device (with that device current) looks up the
 * array's device address with cudaGetSymbolAddress, which may initialise the
 * CUDA context; make that first call before any stream capture begins. The
 * address is cached per device ordinal, so the entry point assumes the
 * device's primary context (the one the CUDA runtime uses); a caller that
 * switches between its own driver contexts on one device must not use it.
 * All calls on one device share the array: calls that can overlap (on
 * different streams, or from several host threads) race and give wrong
 * results; serialise them on one stream. Asynchronous: synchronise the stream
 * before reading d_hii. errbuf (may be NULL) receives a NUL-terminated
 * message of at most errlen bytes when the status is not SBDX_OK. */
int sbdx_diag_terms_noalloc(int norb, double I0, const double* d_h, const double* d_eri,
                            const uint64_t* d_alpha, size_t na, const uint64_t* d_beta, size_t nb,
                            double* d_hii, void* stream, char* errbuf, size_t errlen);

/* One H*C product. Replaces mult (chemistry/tpb/mult.h:376-632). C and S are
 * host buffers of na*nb doubles (S is overwritten, not accumulated). On large
 * problems the copies run in chunks of alpha rows on a second stream,
 * overlapped with the product's kernels (page-locked host buffers let them
 * overlap; pageable ones give the same result, serialised). */
int sbdx_sigma(sbdx_ctx* ctx, const double* C, double* S);
/* Chunks of that pipeline: 0 = automatic (about 8 M determinants per chunk,
 * at most 8; none below about 12.6 M determinants), 1 = no pipeline (one copy in, the
 * product, one copy out), K >= 2 = K chunks of equal alpha-row counts. The
 * pipeline runs with the default alpha-first launch codes and no stored
 * Hamiltonian; otherwise sbdx_sigma copies around one whole product. */
int sbdx_set_io_chunks(sbdx_ctx* ctx, int chunks);
/* Same on device buffers of na*nb elements of the given precision
 * (SBDX_FP64: double; SBDX_FP32: float storage with FP64 row accumulation),
 * on the context stream. */
int sbdx_sigma_device(sbdx_ctx* ctx, int precision, const void* dC, void* dS);

/* One shard of the product for a distributed solve: output rows [a0, a1) of
 * S = H C, i.e. the determinants of alpha strings a0 .. a1-1. dC is the whole
 * vector (na*nb elements of the given precision, the ket side); dS receives
 * (a1-a0)*nb elements (its element 0 is determinant (a0, 0)). a0 must be a
 * multiple of 8 (or a0 == a1). The reference distributes the vector in 2-D
 * blocks, rotates ket blocks between ranks (Mpi2dSlide,
 * framework/mpi_utility.h:441-515; chemistry/tpb/mult.h:429-432, 599-607) and
 * sums partial products (MpiAllreduce, mult.h:614-615); here each GPU owns a
 * block of alpha rows, gathers the whole C into its HBM (one all-gather per
 * product) and evaluates its own rows completely, so no partial products are
 * summed. Evaluated on the fly (SBDX_ERR_STATE while a stored Hamiltonian is
 * held). The rows' work items are built on first use of a range. */
int sbdx_sigma_rows_device(sbdx_ctx* ctx, int precision, const void* dC, void* dS, size_t a0, size_t a1);

/* The subspace projection of every Davidson step: dP[i*nx + r] = <V_i, X_r>
 * for m device vectors V_i (element stride ldv) and 1 <= nx <= 8 device
 * vectors X_r (stride ldx), D elements each, of the given precision; dP holds
 * m*nx doubles on the device. The reference forms these dots one pair at a
 * time (InnerProduct, framework/dm_vector.h:179-243, called from
 * chemistry/tpb/davidson.h:756-797 and 865-873); here one pass over the
 * vectors evaluates all of them as (m x D)(D x nx) tiles on the FP64 tensor
 * pipe (FP32 vectors widened exactly), with a fixed-order reduction, on the
 * context stream; returns after the result is written. */
int sbdx_project_device(sbdx_ctx* ctx, int precision, const void* dV, size_t ldv, int m, const void* dX, size_t ldx,
                        int nx, size_t D, double* dP);

typedef struct {
  int max_it;          /* outer restarts (SBD::max_it, sbdiag.h:19)            */
  int max_nb;          /* subspace size (SBD::max_nb, sbdiag.h:20)            */
  double eps;          /* residual-norm tolerance (SBD::eps, sbdiag.h:21)     */
  double max_time;     /* seconds (SBD::max_time, sbdiag.h:22)                */
  int precision;       /* SBDX_FP64: the reference algorithm; SBDX_FP32:
                          FP32-stored subspace with FP64 defect correction    */
  int defect_every;    /* FP32 mode: 0 = exact FP64 refresh when the estimated
                          residual fell 1e4-fold (default); k > 0 = every k steps */
  int verbose;         /* print one line per step, as davidson.h:834-846      */
} sbdx_davidson_params;

typedef struct {
  double energy;       /* <W|H|W> after one extra FP64 sigma (sbdiag.h:250-273) */
  double residual;     /* last residual norm                                    */
  int n_sigma;         /* sigma products of the working precision              */
  int n_sigma64;       /* FP64 sigma products (defect corrections + final)     */
  int converged;       /* residual < eps                                        */
  double seconds;      /* wall time of the solve                                */
} sbdx_davidson_info;

/* Davidson eigensolve + final energy. Replaces Davidson (max_time overload,
 * chemistry/tpb/davidson.h:661-924), BasisInitVector (:101-140) and the energy
 * evaluation of tpb::diag (sbdiag.h:246-273). W: host buffer of na*nb doubles;
 * on input the start vector if init_from_W != 0, else W[0] = 1 (Hartree-Fock);
 * on output the normalised ground-state vector. W may be NULL when
 * init_from_W == 0: the vector then stays on the device only. Either way the
 * result stays resident in the context (sbdx_wavefunction_device) until the
 * next solve or new strings. */
int sbdx_davidson(sbdx_ctx* ctx, const sbdx_davidson_params* params, int init_from_W, double* W,
                  sbdx_davidson_info* info);

/* Several lowest roots; no counterpart in the reference, whose Davidson is
 * single-root. W: host buffer of nroots*na*nb doubles (root r at offset
 * r*na*nb); on input the start vectors if init_from_W != 0, else unit vectors
 * on the nroots lowest diagonal elements; on output the orthonormal Ritz
 * vectors (W may be NULL when init_from_W == 0; the vectors stay resident as
 * for sbdx_davidson). energies and residuals (may be NULL): nroots doubles each, the
 * Rayleigh quotients and exact residual norms |H W_r - E_r W_r|. 1 <= nroots
 * <= 4. SBDX_FP64: block Davidson whose subspace holds the nroots Ritz
 * vectors plus max_nb FP64 corrections; SBDX_FP32: the mixed-precision solver
 * with one FP64 anchor per root and 2*max_nb FP32 corrections. Both add one
 * Olsen-corrected preconditioned residual per unconverged root per step.
 * Converged when every exact residual is below eps. */
int sbdx_davidson_roots(sbdx_ctx* ctx, const sbdx_davidson_params* params, int nroots, int init_from_W,
                        double* W, double* energies, double* residuals, sbdx_davidson_info* info);

/* ---- the converged vector on the device (no device-host round trip) -------
 * The reference reduces its distributed vector where it lies: the density
 * (OccupationDensity, chemistry/tpb/occupation.h:10-95), the alpha weights of
 * the carry-over (DiagonalReducedDensityMatrix, chemistry/tpb/rdmat.h:10-58)
 * and the RDMs (Correlation, chemistry/tpb/correlation.h:194-444) run on the
 * W that Davidson left in memory. These entry points do the same with device
 * vectors: dW is any device buffer of na*nb doubles on the context's device,
 * usually the resident result of the last solve. */
/* Device address of root `root` of the last sbdx_davidson /
 * sbdx_davidson_roots solve of this context (SBDX_ERR_STATE before any solve;
 * invalidated by the next solve or new strings). */
int sbdx_wavefunction_device(sbdx_ctx* ctx, int root, const double** dW);
/* Copies that root to the host buffer W (na*nb doubles), e.g. to save it
 * (SaveWavefunction, chemistry/tpb/restart.h:20-67). */
int sbdx_get_wavefunction(sbdx_ctx* ctx, int root, double* W);
/* As sbdx_rdm, sbdx_occupation, sbdx_alpha_weights and sbdx_energy_backward
 * (below) on a device vector; outputs are host buffers of the same sizes. */
int sbdx_rdm_device(sbdx_ctx* ctx, const double* dW, double* one, double* two);
int sbdx_occupation_device(sbdx_ctx* ctx, const double* dW, double* density);
int sbdx_alpha_weights_device(sbdx_ctx* ctx, const double* dW, double* weights);
int sbdx_energy_backward_device(sbdx_ctx* ctx, const double* dW, double* dE_dh, double* dE_deri);

/* Solver of sbdx_davidson_roots (no counterpart in the reference, whose
 * Davidson steps are host loops over distributed vectors, davidson.h:661-924):
 * on != 0 runs the device-driven form, in which an iteration (expansion of
 * every root, its products, the projections, the generalised Rayleigh-Ritz
 * problem solved on the device, the anchor update) is one CUDA graph launched
 * without a host round trip; the host reads each iteration's residual
 * estimates one iteration later and launches the exact FP64 refreshes from
 * them. Same algorithm and results as the host-driven form (every root is
 * expanded in every iteration, Gram-Schmidt always makes two passes). Needs a
 * non-default stream for the graphs (else the same kernels run unrecorded). */
int sbdx_set_graph_steps(sbdx_ctx* ctx, int on);

/* 1-/2-RDM of a vector W (host, na*nb doubles). Replaces Correlation
 * (chemistry/tpb/correlation.h:194-444). one: 2*L*L doubles; two: 4*L^4
 * doubles (may be NULL to skip the 2-RDM). */
int sbdx_rdm(sbdx_ctx* ctx, const double* W, double* one, double* two);

/* Occupation density[2p+s] of W. Replaces OccupationDensity
 * (chemistry/tpb/occupation.h:10-95) over all orbitals. */
int sbdx_occupation(sbdx_ctx* ctx, const double* W, double* density);

/* Alpha-string weights sum_b |W[a,b]|^2 (DiagonalReducedDensityMatrix,
 * chemistry/tpb/rdmat.h:10-57), the input of CarryOverAlphaDet. */
int sbdx_alpha_weights(sbdx_ctx* ctx, const double* W, double* weights);

/* Adjoint of the energy with respect to the integrals (Hellmann-Feynman):
 * dE/dh (L*L, one entry per unordered pair, set on both triangles) and
 * dE/d(pq|rs) for every 8-fold packed class (eri_len doubles), computed from
 * the RDMs of W, which the call recomputes together with the connectivity.
 * It has no single counterpart in the reference; it contracts the reference's
 * RDM outputs (correlation.h:194-444) the way the sample's energy check uses
 * them (samples/selected_basis_diagonalization/main.cc:166-216). */
int sbdx_energy_backward(sbdx_ctx* ctx, const double* W, double* dE_dh, double* dE_deri);

/* ---- batches of subspaces -------------------------------------------------
 * No counterpart in the reference, which solves one basis per tpb::diag call
 * (sbdiag.h:113-124). A batch holds many independent alpha x beta string sets
 * that share one Hamiltonian and solves them concurrently on one GPU: each
 * subspace has its own context on its own stream, its sigmas are replayed
 * from captured CUDA graphs, and a pool of host threads drives the Davidson
 * solves (sbdx_davidson_roots for every subspace), largest first. */
typedef struct sbdx_batch sbdx_batch;
/* Integrals as in sbdx_set_integrals (exact doubles, copied). */
int sbdx_batch_create(sbdx_batch** batch, int device, int norb, double I0, const double* h, const double* eri,
                      size_t eri_len);
int sbdx_batch_destroy(sbdx_batch* batch);
const char* sbdx_batch_last_error(const sbdx_batch* batch);
/* Adds one subspace (strings as in sbdx_set_strings); builds its
 * connectivity and diagonal. *index receives its position. */
int sbdx_batch_add(sbdx_batch* batch, const uint64_t* alpha, size_t na, const uint64_t* beta, size_t nb,
                   int* index);
int sbdx_batch_size(const sbdx_batch* batch);
int sbdx_batch_dims(const sbdx_batch* batch, int index, size_t* na, size_t* nb);
/* sbdx_set_graph_steps for every subspace of the batch (and those added later). */
int sbdx_batch_set_graph_steps(sbdx_batch* batch, int on);
/* Tunes the sigma launch shapes on the largest subspace (sbdx_autotune) and
 * applies them to the subspaces with at least a quarter of its determinants;
 * smaller ones keep the size-dependent defaults. */
int sbdx_batch_tune(sbdx_batch* batch, int* same_code, int* ab_code);
/* Lowest nroots (1-4) of every subspace, start vectors on the lowest diagonal
 * elements, nthreads host threads (0 = 8). energies, residuals: size*nroots
 * doubles (subspace-major; residuals may be NULL); infos: size entries (may be
 * NULL), each with that subspace's own solve time; *seconds (may be NULL):
 * wall time of the whole batch. */
int sbdx_batch_solve(sbdx_batch* batch, const sbdx_davidson_params* params, int nroots, int nthreads,
                     double* energies, double* residuals, sbdx_davidson_info* infos, double* seconds);
/* Ritz vector `root` of subspace `index` of the last solve (host, na*nb). */
int sbdx_batch_vector(sbdx_batch* batch, int index, int root, double* W);

#ifdef __cplusplus
}
#endif
#endif
