/* sbd_tpb.h -- C ABI of the B200 tensor-product-basis (TPB) selected-basis diagonalization.
 *
 * One process, one GPU.  Inputs are an FCIDUMP-style Hamiltonian (core energy, one-electron
 * integrals, 8-fold packed two-electron integrals) and sorted, duplicate-free alpha and beta
 * occupation strings (uint64, bit p = spatial orbital p, L <= 64).  Outputs are the lowest
 * eigenvalue, the CI vector in the reference's sign convention and determinant order
 * (index Ia*nb + Ib), the orbital occupations and the spin-resolved 1- and 2-RDMs in the
 * reference's layouts.  Every entry point returns an int status (SBD_TPB_OK = 0 or a negative
 * SBD_TPB_ERR_* code); sbd_tpb_last_error() gives the message of the calling thread's last
 * failure.  No entry point throws or exits the process.
 *
 * The reference interfaces each entry point replaces are cited as file:line inside ncsa/sbd-pub.
 */
#ifndef SBD_TPB_H
#define SBD_TPB_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SBD_TPB_API __attribute__((visibility("default")))
#else
#define SBD_TPB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SBD_TPB_OK 0
#define SBD_TPB_ERR_INVALID (-1)       /* bad argument or inconsistent input */
#define SBD_TPB_ERR_CUDA (-2)          /* CUDA runtime error (message says which call) */
#define SBD_TPB_ERR_OOM (-3)           /* device allocation refused */
#define SBD_TPB_ERR_NOT_CONVERGED (-4) /* Davidson stopped at max_it / max_time; result filled */
#define SBD_TPB_ERR_STATE (-5)         /* call order: e.g. sigma before strings/Hamiltonian */
#define SBD_TPB_ERR_IO (-6)            /* file could not be read or parsed */
#define SBD_TPB_ERR_NO_DEVICE (-7)     /* no usable sm_100 device */
#define SBD_TPB_ERR_CAPACITY (-8)      /* caller buffer missing or too small; sizes were returned */

/* Memory location of caller buffers passed to the vector entry points. */
#define SBD_TPB_HOST 0
#define SBD_TPB_DEVICE 1

/* Table kinds for sbd_tpb_table_size / sbd_tpb_get_table. */
#define SBD_TPB_SINGLES_ALPHA 0
#define SBD_TPB_DOUBLES_ALPHA 1
#define SBD_TPB_SINGLES_BETA 2
#define SBD_TPB_DOUBLES_BETA 3

/* Arithmetic of the solver. */
#define SBD_TPB_FP64 0  /* FP64 vectors and sigma throughout (the plain path) */
#define SBD_TPB_MIXED 1 /* FP32 CI/search vectors, FP32 sigma with split-BF16 tensor-core
                           alpha-beta contraction, FP64 dots / Rayleigh-Ritz and a final FP64
                           sigma for the reported energy and residual */

/* Eigensolver (--method of the reference app; the matrix-free ones). */
#define SBD_TPB_METHOD_DAVIDSON 0 /* block Davidson (tpb/davidson.h:667-930) */
#define SBD_TPB_METHOD_LANCZOS 2  /* Lanczos without reorthogonalisation (tpb/lanczos.h:167-320), FP64 */

/* Davidson correction. */
#define SBD_TPB_PRECOND_DIAGONAL 0 /* t = r / (E0 - H_ii)  (tpb/davidson.h:858-868) */
#define SBD_TPB_PRECOND_LEARNED 1  /* MLP correction, diagonal fallback when a step fails */

typedef struct sbd_tpb_handle sbd_tpb_handle;

/* Run parameters: the fields of sbd::tpb::SBD that matter on one rank (tpb/sbdiag.h:22-50). */
typedef struct sbd_tpb_params {
  int max_it;        /* --iteration: restarts of the Davidson subspace (default 1) */
  int max_nb;        /* --block: subspace size (default 10) */
  double eps;        /* --tolerance: residual norm (default 1e-4) */
  double max_time;   /* --max_time in seconds (default 86400) */
  int init;          /* --init: 0 = start from determinant 0 (the reference's HF start);
                        1 = the reference's seeded random start (BasisInitVector with init 1,
                        tpb/davidson.h:138-141: Randomize, framework/dm_vector.h:101-178, the same
                        values for the same seed, normalised) */
  int do_rdm;        /* --rdm: 0 = orbital occupations only, 1 = full 1/2-RDMs */
  int precision;     /* SBD_TPB_FP64 or SBD_TPB_MIXED */
  int preconditioner;/* SBD_TPB_PRECOND_* */
  int verbose;       /* print the reference's " Davidson iteration" lines to stdout */
  int device;        /* CUDA device ordinal used by sbd_tpb_diag */
  int symmetry;      /* 1 (default): when the alpha and beta string lists are identical and the
                        start is the HF determinant, every correction vector is projected onto
                        the alpha<->beta exchange-symmetric sector the start vector lies in
                        (C = C^T in the separated convention), so rounding cannot steer the
                        iteration to a lower state of the other sector; 2: the same, and a
                        random start (init 1) is projected onto that sector too (the reference
                        does not project; its random start reaches the lowest state of either
                        sector); 0: off.  Davidson only. */
  int method;        /* --method: SBD_TPB_METHOD_DAVIDSON (default) or SBD_TPB_METHOD_LANCZOS */
  unsigned long long seed; /* --seed of the random start (default 1729, tpb/sbdiag.h:34) */
} sbd_tpb_params;

/* Fills p with the reference defaults (tpb/sbdiag.h:22-50) and SBD_TPB_FP64 / diagonal. */
SBD_TPB_API void sbd_tpb_default_params(sbd_tpb_params *p);

/* Hamiltonian in FCIDUMP terms.  h1 is L*L row-major and symmetric; eri_packed is the 8-fold
 * store of twoInt (basic/integrals.h:64-107): index a*(a+1)/2+b with a >= b over the pair
 * indices ij = max(i,j)*(max(i,j)+1)/2 + min(i,j); length B*(B+1)/2, B = L*(L+1)/2. */
typedef struct sbd_tpb_hamiltonian {
  int norb;
  int nelec;
  double core_energy;
  const double *h1;
  const double *eri_packed;
  size_t n_eri_packed;
} sbd_tpb_hamiltonian;

/* Carry-over strings: the step after the solver in the sample-based loop (tpb/sbdiag.h:690-736;
 * app flags --carryover_type / --carryover_ratio / --carryover_threshold). */
#define SBD_TPB_CARRYOVER_NONE 0
#define SBD_TPB_CARRYOVER_DOMINANT 1         /* CarryOverAdet/Bdet (tpb/rdmat.h:63-262) */
#define SBD_TPB_CARRYOVER_DOMINANT_SINGLES 2 /* the dominant strings and all their single
                                                excitations, sorted and unique
                                                (SinglesExtendHalfdets, tpb/extend.h:186-320) */
#define SBD_TPB_CARRYOVER_CUTOFF_SINGLES 3   /* the strings of determinants with W^2 > threshold and
                                                their singles, sorted and unique
                                                (SinglesExtendHalfdets, tpb/extend.h:13-177) */

typedef struct sbd_tpb_carryover {
  int type;           /* SBD_TPB_CARRYOVER_* */
  double ratio;       /* types 1, 2: > 0 keeps the first (size_t)(ratio * n) strings of each spin by
                         descending weight; 0 keeps them up to and including the first whose running
                         weight exceeds 1 - threshold (all of them if none does) */
  double threshold;   /* the reference's default is 0.01 */
  uint64_t *astr;     /* out: caller buffer (host) for the alpha strings, or NULL to query */
  size_t acap;        /* its capacity in strings */
  size_t na;          /* out: number of alpha strings (also when the buffer was too small) */
  uint64_t *bstr;     /* out: the same for beta */
  size_t bcap;
  size_t nb;
  double truncated_a; /* out, ratio mode: 1 - weight of the kept alpha strings */
  double truncated_b; /* out, ratio mode: the same for beta */
  double total_weight;/* out, type 3: weight of the determinants above the threshold */
} sbd_tpb_carryover;

/* Results; pointer fields are caller-allocated (host) and may be NULL to skip that output. */
typedef struct sbd_tpb_result {
  double energy;      /* <W|H|W> with an FP64 sigma (tpb/sbdiag.h:431-469) */
  double residual;    /* last Davidson residual norm */
  int iterations;     /* Davidson steps (sigma applications inside the loop) */
  int converged;      /* residual < eps */
  double *ci_vector;  /* [na*nb] reference sign convention, index Ia*nb+Ib */
  double *density;    /* [2L]: alpha/beta occupation per orbital, density[2p+s] */
  double *one_rdm;    /* [2*L*L]  onebody[s][i + L*j] (tpb/correlation.h:378-664) */
  double *two_rdm;    /* [4*L^4]  twobody[s+2t][...] in the reference layout */
  double seconds_tables, seconds_davidson, seconds_rdm, seconds_total;
  int learned_steps;  /* Davidson corrections taken from the learned preconditioner */
  int fallback_steps; /* steps that fell back to the diagonal after a learned step failed */
  sbd_tpb_carryover *carryover; /* optional: with type != 0, carry-over strings of the final
                                   vector (as sbd_tpb_carryover_strings); a buffer that is too small makes
                                   the call return SBD_TPB_ERR_CAPACITY after everything else */
} sbd_tpb_result;

/* ---- one-shot driver: replaces sbd::tpb::diag (tpb/sbdiag.h:139-151, one rank, --method 0) */
SBD_TPB_API int sbd_tpb_diag(const sbd_tpb_params *params, const sbd_tpb_hamiltonian *ham,
                 const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                 sbd_tpb_result *result);

/* Same, starting Davidson from W0 (host, [na*nb], reference convention and order; NULL = the HF
 * start) -- the reference's --loadname restart (tpb/sbdiag.h:280-291). */
SBD_TPB_API int sbd_tpb_diag_from(const sbd_tpb_params *params, const sbd_tpb_hamiltonian *ham,
                                  const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                                  const double *W0, sbd_tpb_result *result);

/* ---- handle API: the stages of the same path, for callers that drive them ---------------- */
SBD_TPB_API const char *sbd_tpb_last_error(void);
SBD_TPB_API int sbd_tpb_create(int device, sbd_tpb_handle **out);
SBD_TPB_API int sbd_tpb_destroy(sbd_tpb_handle *h);

/* Replaces SetupIntegrals (basic/makeintegrals.h:123-174) feeding MultTPBThrust::Init
 * (tpb/mult_thrust.h:98-277). */
SBD_TPB_API int sbd_tpb_set_hamiltonian(sbd_tpb_handle *h, const sbd_tpb_hamiltonian *ham);

/* Strings as LoadAlphaDets + sort_bitarray leave them (basic/makedeterminants.h:160-186):
 * ascending and unique, or in the order --shuffle leaves them (ShuffleDet,
 * basic/determinants.h:622-628); the order fixes the determinant index.  Rejected when
 * duplicated, wider than norb, or when their electron counts differ within a spin. */
SBD_TPB_API int sbd_tpb_set_strings(sbd_tpb_handle *h, const uint64_t *astr, size_t na, const uint64_t *bstr,
                        size_t nb);

/* String files parsed, sorted and de-duplicated on the GPU, as LoadAlphaDets leaves them
 * (basic/makedeterminants.h:160-186): text, one string per line with orbital 0 the last of the first
 * norb characters (from_string, framework/bit_manipulation.h:215-230; trailing '\r'/spaces and
 * empty lines are skipped, a short line or a character other than 0/1 is SBD_TPB_ERR_IO with the
 * line number), or binary, ceil(norb/8)-byte big-endian records holding the string in their low
 * norb bits (DecodeAlphaDets, makedeterminants.h:63-108).  The result is ascending and unique
 * (sort_bitarray), ready for sbd_tpb_set_strings.  Strings go to out (host) when it holds them
 * all; otherwise *count is set and SBD_TPB_ERR_CAPACITY returned (a text file has at most
 * nbytes/(norb+1)+1 strings, a binary one nbytes/ceil(norb/8)). */
#define SBD_TPB_STRINGS_TEXT 0
#define SBD_TPB_STRINGS_BINARY 1
SBD_TPB_API int sbd_tpb_parse_strings(sbd_tpb_handle *h, const void *bytes, size_t nbytes, int format, int norb,
                                      uint64_t *out, size_t cap, size_t *count);
/* The same from a file; the format follows the extension (".bin" binary, anything else text),
 * as LoadAlphaDets decides it. */
SBD_TPB_API int sbd_tpb_read_strings(sbd_tpb_handle *h, const char *path, int norb, uint64_t *out, size_t cap,
                                     size_t *count);
/* Device time (ms) of the last string parse on the handle: host-to-device copy, parse, sort and
 * de-duplication (CUDA events on the handle's stream). */
SBD_TPB_API double sbd_tpb_last_parse_ms(sbd_tpb_handle *h);

/* Excitation tables on the GPU; replaces MakeHelpers/RemakeHelpers with GenerateExcitation
 * (tpb/helper.h:185-323, 710-854, 916-1226) for one rank. */
SBD_TPB_API int sbd_tpb_build_tables(sbd_tpb_handle *h);
SBD_TPB_API int sbd_tpb_table_size(sbd_tpb_handle *h, int kind, size_t *nrows, size_t *nnz);
/* Copies one table to host buffers in the reference's flattened layout: off[nrows+1] CSR
 * offsets, ket[nnz] ket string indices (ascending per bra, TaskHelpers::*FromAlpha),
 * cran[2*nnz] or [4*nnz] CrAn labels (TaskHelpers::*CrAn). */
SBD_TPB_API int sbd_tpb_get_table(sbd_tpb_handle *h, int kind, uint64_t *off, uint64_t *ket, int32_t *cran);

/* H_ii for every determinant; replaces makeQChamDiagTerms (tpb/qcham.h:290-340,
 * tpb/mult_thrust.h:1585-1664). */
SBD_TPB_API int sbd_tpb_diagonal(sbd_tpb_handle *h, double *hii, int mem);

/* sigma (+)= H*C; replaces MultBase<double>::run(hii, Wk, Wb) (basic/mult.h:94-102) as
 * implemented by MultTPBThrust::run (tpb/mult_thrust.h:1172-1582) and sbd::mult
 * (tpb/mult.h:625-881).  accumulate = 1 adds into sigma like the reference (Wb accumulates);
 * accumulate = 0 overwrites.  C and sigma use the reference sign convention. */
SBD_TPB_API int sbd_tpb_sigma(sbd_tpb_handle *h, const double *C, double *sigma, int accumulate, int mem);
/* FP32 vectors (mixed-precision path), same semantics. */
SBD_TPB_API int sbd_tpb_sigma_f32(sbd_tpb_handle *h, const float *C, float *sigma, int accumulate, int mem);

/* Device-vector sigma with an explicit sign convention, for callers that keep their vectors in
 * HBM (their own eigensolver, benchmarks).  dtype 0 = double, 1 = float; convention 0 = the
 * reference's (interleaved determinant, as sbd_tpb_sigma), 1 = the library's internal separated
 * convention (alpha creators before beta creators: x_sep = D x_ref with
 * D = (-1)^#{(p in Ia, q in Ib) : q < p}), which skips the two sign passes.  Same accumulate rule;
 * in convention 1, C and sigma must be distinct buffers (SBD_TPB_ERR_INVALID otherwise).
 * Convention 2 = convention 1 for an exchange-symmetric C (C[Ia, Ib] = C[Ib, Ia] over identical
 * alpha and beta string lists, the sector of an HF-started singlet solve): the beta part of sigma
 * is then the transpose of the alpha part, so it runs one gathering pass and a transpose-add
 * (accumulate must be 0; SBD_TPB_ERR_STATE when the string lists differ).  The answer equals
 * convention 1 up to rounding only for a symmetric C. */
SBD_TPB_API int sbd_tpb_sigma_device(sbd_tpb_handle *h, const void *C, void *sigma, int dtype,
                                     int accumulate, int convention);

/* Size of the fixed device scratch of sbd_tpb_sigma_noalloc (16 MiB). */
#define SBD_TPB_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)

/* sigma (+)= H*C on device vectors in the separated convention (as sbd_tpb_sigma_device with
 * convention 1) that allocates no device memory.  No counterpart in the reference: it serves
 * callers that cannot have a library call cudaMalloc under them -- a code that has already
 * reserved the card's memory through its own pool, or one whose memory policy forbids
 * allocations after set-up.  The C^T staging lives in a static device array of
 * SBD_TPB_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until exit;
 * ndet * element size beyond it is rejected with SBD_TPB_ERR_INVALID, as are C == sigma and
 * tables that sbd_tpb_build_tables did not finish.  All calls on a device share that array
 * (nothing in it must start at zero), so calls whose kernels overlap on the GPU race: serialise
 * them.  The first call on a device looks up the array's address (cudaGetSymbolAddress) and
 * keeps it for the process: make that first call before any stream capture, and do not call it
 * on a device after cudaDeviceReset.  The alpha-beta terms always use the direct loop. */
SBD_TPB_API int sbd_tpb_sigma_noalloc(sbd_tpb_handle *h, const void *C, void *sigma, int dtype,
                                      int accumulate);

/* Davidson (tpb/davidson.h:667-930; basic/davidson_thrust.h:85-373) on the handle's problem,
 * from W (host, [na*nb], reference convention; NULL = HF start).  Writes the energy etc. into
 * result (ci_vector/density/RDM fields as in sbd_tpb_diag). */
SBD_TPB_API int sbd_tpb_davidson(sbd_tpb_handle *h, const sbd_tpb_params *params, const double *W0,
                     sbd_tpb_result *result);

/* Lanczos (tpb/lanczos.h:167-320; --method 2) on the handle's problem from W0 (as
 * sbd_tpb_davidson): params->max_it outer iterations of at most params->max_nb steps, stopping
 * when the lowest eigenvalue of the tridiagonal matrix moves by less than params->eps (result
 * converged = 1) or an off-diagonal falls below it; params->verbose prints the reference's
 * " Lanczos iteration" lines.  FP64 only.  result->residual is |HW - E W| of the final vector. */
SBD_TPB_API int sbd_tpb_lanczos(sbd_tpb_handle *h, const sbd_tpb_params *params, const double *W0,
                                sbd_tpb_result *result);

/* 1/2-RDMs of W; replaces Correlation (tpb/correlation.h:378-664) and
 * MultTPBThrust::correlation (tpb/correlation_thrust.h:504-731).  one: [2*L*L], two: [4*L^4]
 * (two may be NULL for the 1-RDM only).  W in the reference convention. */
SBD_TPB_API int sbd_tpb_rdm(sbd_tpb_handle *h, const double *W, double *one, double *two, int mem);

/* Carry-over strings of W ([na*nb], either sign convention: only W^2 enters), as sbd::tpb::diag
 * selects them after the solve (tpb/sbdiag.h:690-736).  Strings are written to co->astr/bstr when
 * both buffers hold them; otherwise the counts are returned in co->na/nb with
 * SBD_TPB_ERR_CAPACITY (pass NULL buffers to query, or size them with
 * sbd_tpb_carryover_capacity).  Strings of types 1 and 2 come out by descending weight (type 1;
 * equal weights by ascending string index) or ascending as integers (types 2 and 3). */
SBD_TPB_API int sbd_tpb_carryover_strings(sbd_tpb_handle *h, const double *W, int mem, sbd_tpb_carryover *co);
/* Upper bound of the strings one spin (0 alpha, 1 beta) can produce for a carry-over type. */
SBD_TPB_API size_t sbd_tpb_carryover_capacity(sbd_tpb_handle *h, int type, int spin);
/* Times of the last carry-over on the handle, milliseconds: [0] the pass over W that forms the
 * per-string weights or counts (CUDA events on the handle's stream), [1] the whole call (host
 * clock, including sorting, extension and copies). */
SBD_TPB_API int sbd_tpb_last_carryover_ms(sbd_tpb_handle *h, double *ms);

/* Device stream of the handle (cudaStream_t as void*), for callers that order their own work. */
SBD_TPB_API void *sbd_tpb_stream(sbd_tpb_handle *h);

/* Timing of the last sigma call on the handle's stream (CUDA events), milliseconds. */
SBD_TPB_API double sbd_tpb_last_sigma_ms(sbd_tpb_handle *h);

/* Per-stage device times (ms) of the last sigma call, in launch order: [0] alpha pass (diagonal,
 * alpha singles/doubles, C^T), [1] beta pass, [2] alpha-beta term (sparse kernel or dense
 * gather/contract/scatter).  Returns how many were written (<= max_n) or a negative status. */
SBD_TPB_API int sbd_tpb_last_sigma_kernels(sbd_tpb_handle *h, double *ms, int max_n);

/* Number of kernel launches the library has issued on this handle (for accounting). */
SBD_TPB_API uint64_t sbd_tpb_kernel_launches(sbd_tpb_handle *h);

/* Release the handle's cached work memory: the Davidson N-vectors kept between solves, the
 * sigma C^T staging and the sign-conversion vectors.  Tables, diagonal and the problem stay;
 * the next call that needs the work memory allocates it again.  No counterpart in the
 * reference, whose solver frees its vectors at the end of each call. */
SBD_TPB_API int sbd_tpb_release_work(sbd_tpb_handle *h);

/* ---- learned Davidson preconditioner ------------------------------------------------------
 * No counterpart in the reference, whose only correction is the diagonal one
 * t = r / (E0 - H_ii) (tpb/davidson.h:858-868).  A small MLP predicts a per-determinant factor:
 *   t_i = d_i * (1 + 0.5 tanh(y_i)),  d_i = r_i / (E0 - H_ii),
 *   y = w3 . gelu(W2 gelu(W1 x + b1) + b2) + b3   (hidden width 256, tanh-form GELU, BF16
 *   weights and activations on tensor cores, FP32 accumulation),
 * with x = [asinh(E_J - E0)/4, 0, which of the 24 orbitals n-12 .. n+11 around the Fermi level
 * are doubly occupied, which singly, 14 zeros] (orbitals below 0 read as occupied; n = electrons
 * per spin); E_J is the spin-free diagonal, H_ii plus the same-spin exchange integrals of both
 * strings.  The inputs depend only on the spatial occupation, so every determinant of a
 * spin-coupled set gets the same factor and the learned correction keeps the spin symmetry the
 * diagonal one keeps (the residual entry r_i, which differs within such a set, is left out: its
 * input slot is zero).  It is trained by the library's own forward/backward kernels on pairs
 * (d_k, exact correction) recorded from FP64 Davidson runs; w3 = b3 = 0 at creation, so an
 * untrained network is exactly the diagonal preconditioner.  The parameter vector is FP32 in
 * the order W1[256][64], b1[256], W2[256][256], b2[256], w3[256], b3. */
typedef struct sbd_tpb_precond sbd_tpb_precond;
#define SBD_TPB_MLP_HIDDEN 256
#define SBD_TPB_MLP_FEATURES 64
#define SBD_TPB_MLP_PARAMS 82689

SBD_TPB_API int sbd_tpb_precond_create(int device, uint64_t seed, sbd_tpb_precond **out);
SBD_TPB_API int sbd_tpb_precond_destroy(sbd_tpb_precond *p);
/* Runs the plain FP64 diagonal Davidson of params on the handle's problem, recording every
 * correction step, and turns each step into training pairs (importance-sampled, about
 * samples_per_step determinants each) appended to set `role` (0 = training, 1 = held out).
 * energy (may be NULL) receives the converged energy. */
SBD_TPB_API int sbd_tpb_precond_collect(sbd_tpb_precond *p, sbd_tpb_handle *h, const sbd_tpb_params *params,
                                        size_t samples_per_step, int role, double *energy);
SBD_TPB_API int sbd_tpb_precond_num_samples(sbd_tpb_precond *p, int role, size_t *n);
/* Adam on the training set, minibatches of `batch` (multiple of 128); loss is the weighted mean
 * of (a (1 + 0.5 tanh(y)) - b)^2 / 2 with a = d/|d| and b the scaled exact correction. */
SBD_TPB_API int sbd_tpb_precond_train(sbd_tpb_precond *p, int epochs, int batch, double lr, double *last_loss);
/* Weighted squared error of the learned correction and of the diagonal one (y = 0) on a set. */
SBD_TPB_API int sbd_tpb_precond_evaluate(sbd_tpb_precond *p, int role, double *loss_learned,
                                         double *loss_diagonal);
SBD_TPB_API int sbd_tpb_precond_get_params(sbd_tpb_precond *p, float *params, size_t n);
SBD_TPB_API int sbd_tpb_precond_set_params(sbd_tpb_precond *p, const float *params, size_t n);
/* One forward/backward pass of the training kernels on n host samples (x: n x 64 features,
 * a, b, w per sample): grad (SBD_TPB_MLP_PARAMS floats) of 0.5/n sum w (a (1 + 0.5 tanh(y)) - b)^2,
 * its loss and the bounded outputs 0.5 tanh(y).  For gradient checks. */
SBD_TPB_API int sbd_tpb_precond_gradients(sbd_tpb_precond *p, size_t n, const float *x, const float *a,
                                          const float *b, const float *w, float *grad, double *loss,
                                          float *y);
/* The fused inference kernel on the handle's determinants: t = d (1 + 0.5 tanh(y)) from d (host, FP64,
 * separated convention, [na*nb]), E0 and |r|.  Beyond 2^22 determinants only the entries with
 * |d_i| >= |d| / 2^11 are corrected (at most 2^22 of them), as inside the Davidson loop; the
 * others keep t_i = d_i.  For parity tests. */
SBD_TPB_API int sbd_tpb_precond_apply(sbd_tpb_handle *h, sbd_tpb_precond *p, const double *d, double e0,
                                      double rnorm, double *t);
/* Attaches p (or NULL) to the handle: Davidson with preconditioner SBD_TPB_PRECOND_LEARNED uses
 * it.  The handle does not own p. */
SBD_TPB_API int sbd_tpb_set_preconditioner(sbd_tpb_handle *h, sbd_tpb_precond *p);

#ifdef __cplusplus
}
#endif
#endif /* SBD_TPB_H */
