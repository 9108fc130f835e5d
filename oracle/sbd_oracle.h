/* CPU restatement of the reference TPB path: TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker for the GPU path of this repository.  It restates, in plain C,
 * the algorithms of the reference (ncsa/sbd-pub, include/sbd/...) for the one-rank TPB
 * selected-basis diagonalization: FCIDUMP parsing and integral setup, string parsing and sorting,
 * the excitation tables, the Slater-Condon elements on the interleaved determinant, the
 * diagonal, sigma = H*C, the Davidson loop and the 1/2-RDMs.  Each function cites the reference
 * lines it follows.  It is pinned against the reference itself (oracle/_ref, golden fixtures in
 * tests/golden/).  Only tests, the smoke check and the CPU-baseline leg of bench.py may load it.
 *
 * Conventions (as in the reference): strings are uint64 with bit p = spatial orbital p (L <= 64);
 * determinant (Ia, Ib) has index Ia*nb + Ib; spin-orbital 2p is alpha p and 2p+1 is beta p;
 * the one-electron array I1 is 2L x 2L row-major (i*2L + j); the two-electron array is the
 * 8-fold packed store (integrals.h:64-107). */
#ifndef SBD_ORACLE_H
#define SBD_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ham {
  int L;         /* spatial orbitals */
  int nelec;     /* NELEC from the header */
  double I0;     /* core energy */
  double *I1;    /* 2L*2L spin-orbital one-electron integrals */
  double *I2;    /* packed store, (B*(B+1))/2 entries, B = L(L+1)/2 */
  size_t n_I2;
  double *direct;   /* 2L*2L, DirectMat[i + 2L*j] */
  double *exchange; /* 2L*2L, ExchangeMat[i + 2L*j] */
} orc_ham;

/* FCIDUMP text -> integrals (framework/fcidump.h:29-141, basic/makeintegrals.h:123-174).
 * Returns 0 on success, -1 when the file cannot be opened, -2 on a malformed header. */
int orc_load_fcidump(const char *path, orc_ham *out);
/* Same setup from arrays: h1 is L*L (symmetric), eri_packed the packed store. */
int orc_ham_from_arrays(int L, int nelec, double I0, const double *h1, const double *eri_packed,
                        orc_ham *out);
void orc_free_ham(orc_ham *h);

/* Text strings (one per line, orbital 0 is the LAST character) -> sorted uint64
 * (basic/makedeterminants.h:160-186, framework/bit_manipulation.h:149, 215-230, 381-392).
 * With out == NULL only the count is returned in *n.  Returns 0, or -1 on open failure,
 * -2 on a line longer than 64 orbitals or with characters other than 0/1. */
int orc_load_strings(const char *path, int L, uint64_t *out, size_t cap, size_t *n);
/* Binary string file (DecodeAlphaDets, basic/makedeterminants.h:63-108): records of
 * ceil(L/8) bytes read while whole, bits taken from the most significant end of each byte, the
 * first 8*ceil(L/8) - L skipped, the remaining L reversed so the last bit read is orbital 0; then
 * sorted and made unique as the text reader does.  With out == NULL only the count is returned.
 * Returns 0 or -1 on open failure. */
int orc_load_strings_bin(const char *path, int L, uint64_t *out, size_t cap, size_t *n);
/* Ascending sort as an unsigned integer (sort_bitarray / less_from_back). */
void orc_sort_strings(uint64_t *s, size_t n);

/* Excitation table of one spin (tpb/helper.h:185-323): for each bra string, the ket strings
 * whose XOR popcount equals ndiff (2 = single, 4 = double), ket index ascending, with labels
 * CrAn = (2*cr + spin, 2*an + spin) for singles and (2cr0, 2cr1, 2an0, 2an1) (+spin) for
 * doubles; cr are the bra's orbitals missing from the ket, an the ket's missing from the bra,
 * ascending (determinants.h:386-432).  Pass ket_idx == NULL to fill only off[nbra+1].
 * Returns the number of entries. */
size_t orc_excitations(const uint64_t *bra, size_t nbra, const uint64_t *ket, size_t nket,
                       int L, int ndiff, int spin, uint64_t *off, uint64_t *ket_idx,
                       int32_t *cran);

/* Interleaved-determinant Slater-Condon elements (basic/determinants.h:434-501). */
double orc_zero_excite(uint64_t a, uint64_t b, const orc_ham *h);
double orc_one_excite(uint64_t a, uint64_t b, int cr, int an, const orc_ham *h);
double orc_two_excite(uint64_t a, uint64_t b, int i, int j, int ca, int cb, const orc_ham *h);
/* <(a,b)|H|(a2,b2)> by orbital difference (determinants.h:503-568). */
double orc_hij(uint64_t a, uint64_t b, uint64_t a2, uint64_t b2, const orc_ham *h);

/* Diagonal H_ii for all na*nb determinants (tpb/qcham.h:290-340). */
void orc_diagonal(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                  const orc_ham *h, double *hii);

/* Tables for the three one-rank tasks (tpb/helper.h:710-854). */
typedef struct orc_tables {
  size_t na, nb;
  uint64_t *sa_off, *sa_ket;
  int32_t *sa_cran;
  uint64_t *da_off, *da_ket;
  int32_t *da_cran;
  uint64_t *sb_off, *sb_ket;
  int32_t *sb_cran;
  uint64_t *db_off, *db_ket;
  int32_t *db_cran;
} orc_tables;
int orc_build_tables(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb, int L,
                     orc_tables *t);
void orc_free_tables(orc_tables *t);

/* sigma += H*C in the reference's sign convention (tpb/mult.h:625-881): diagonal, task type 2
 * (alpha singles and doubles), type 1 (beta), type 0 (alpha single x beta single). */
void orc_sigma(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
               const orc_tables *t, const orc_ham *h, const double *hii, const double *C,
               double *sigma);

/* The closed-form test vector ((i * 0x9E3779B97F4A7C15 mod 2^64) >> 11) / 2^53 - 1/2. */
double orc_hash_vector(size_t i);
/* sigma = H*C at the determinants rows[0..nrows) (index Ia*nb + Ib), reference sign convention,
 * the terms added in orc_sigma's order; C = NULL takes the closed-form vector. */
void orc_sigma_rows(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                    const orc_tables *t, const orc_ham *h, const double *C, const size_t *rows,
                    size_t nrows, double *out);

/* Block Davidson for the lowest root (tpb/davidson.h:667-930) from W (in/out); the subspace
 * eigenproblem uses a cyclic Jacobi solver with eigenvalues sorted ascending.  Returns the
 * number of sigma applications; *energy is <W|H|W> after the loop as in tpb/sbdiag.h:431-469,
 * *resid the last residual norm.  verbose != 0 prints the reference's iteration lines. */
int orc_davidson(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                 const orc_tables *t, const orc_ham *h, const double *hii, double *W,
                 int max_it, int max_nb, double eps, int verbose, double *energy, double *resid);

/* Lanczos for the lowest root without reorthogonalisation (tpb/lanczos.h:167-320), from W
 * (in/out, not renormalised), with the dense subspace eigenproblem solved by the same sorted
 * Jacobi method as orc_davidson.  Returns the number of sigma applications; *energy is <W|H|W>
 * after the loop (tpb/sbdiag.h:431-469), *steps_printed the number of " Lanczos iteration"
 * lines the reference prints, *converged whether the eigenvalue change fell below eps. */
int orc_lanczos(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                const orc_tables *t, const orc_ham *h, const double *hii, double *W,
                int max_it, int num_block, double eps, int verbose, double *energy, int *steps_printed,
                int *converged);

/* Spin-resolved RDMs of W (tpb/correlation.h:378-664, basic/correlation.h:16-231):
 * one[s*L*L + i + L*j], two[(s+2t)*L^4 + ...] in the reference layout. */
void orc_rdm(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
             const orc_tables *t, int L, const double *W, double *one, double *two);

/* Energy decomposition from spin-summed RDMs as the reference app prints it
 * (apps/chemistry_tpb_selected_basis_diagonalization/main.cc:264-317): out[0..2] =
 * zero-, one- and two-body energies. */
void orc_rdm_energy(const orc_ham *h, const double *one, const double *two, double *out);

/* Sign of the interleaved -> separated (all alpha, then all beta) reordering of
 * determinant (a, b): +1 or -1.  Used by tests to relate the two conventions. */
int orc_reorder_sign(uint64_t a, uint64_t b);

/* Carry-over strings of a CI vector (tpb/sbdiag.h:690-736).
 * orc_string_weights: wa[ia] = sum over ib of W^2 and wb[ib] = sum over ia of W^2, each summed
 * in the reference's loop order (tpb/rdmat.h:47-54, 174-181); ca/cb (may be NULL) count the
 * entries with W^2 > cutoff per row/column and *total (may be NULL) sums those entries in
 * row-major order (tpb/extend.h:45-58). */
void orc_string_weights(const double *W, size_t na, size_t nb, double cutoff, double *wa, double *wb,
                        uint64_t *ca, uint64_t *cb, double *total);
/* Dominant strings (CarryOverAdet/Bdet, tpb/rdmat.h:63-135, 190-262): order[] receives the
 * string indices by descending weight (equal weights by ascending index: the reference leaves
 * their order to std::sort).  ratio > 0 keeps floor(ratio * n) strings and sets *truncated to
 * 1 - their weight; otherwise the strings up to and including the first whose running weight
 * exceeds 1 - threshold are kept (all n when none does: the reference then reads past its
 * arrays).  Returns the number kept. */
size_t orc_carryover_select(const double *w, size_t n, double ratio, double threshold, size_t *order,
                            double *truncated);
/* Each string of s followed by its single excitations (closed orbital j ascending, then open
 * orbital k ascending: basic/excitation.h:9-29), then sorted ascending and made unique
 * (SinglesExtendHalfdets, tpb/extend.h:186-320; sort_bitarray).  out needs n*(1 + e*(L-e))
 * entries (e = electrons of the string); returns the number written. */
size_t orc_singles_extend(const uint64_t *s, size_t n, int L, uint64_t *out);

/* Tiny MLP reference for the learned preconditioner checks (see the product's mlp kernels):
 * y = W3 gelu(W2 gelu(W1 x + b1) + b2) + b3 with fp32 math; weights row-major [out][in]. */
void orc_mlp_forward(int n, int din, int dh, const float *x, const float *W1, const float *b1,
                     const float *W2, const float *b2, const float *W3, const float *b3,
                     float *h1_out, float *h2_out, float *y);
/* Gradients, with respect to all weights (fp64 accumulation), of the learned preconditioner's
 * loss 0.5/n * sum_r w_r (a_r (1 + c tanh(y_r)) - b_r)^2 (a = diagonal correction, b = exact
 * correction, w = sampling weight, c = ORC_MLP_BOUND, y = orc_mlp_forward's output); returns the
 * loss. */
#define ORC_MLP_BOUND 0.5
double orc_mlp_backward(int n, int din, int dh, const float *x, const float *a, const float *b,
                        const float *w, const float *W1, const float *b1, const float *W2,
                        const float *b2, const float *W3, const float *b3, double *gW1, double *gb1,
                        double *gW2, double *gb2, double *gW3, double *gb3);

#ifdef __cplusplus
}
#endif
#endif
