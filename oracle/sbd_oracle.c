/* CPU restatement of the reference TPB path: TEST INFRASTRUCTURE ONLY.
 * See sbd_oracle.h for the contract.  Reference paths are relative to ncsa/sbd-pub. */
#define _GNU_SOURCE
#include "sbd_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------ */
/* Integrals (basic/integrals.h:64-107, basic/makeintegrals.h:123-174)                         */
/* ------------------------------------------------------------------------------------------ */

static inline size_t packed_index(int I, int J, int K, int L_) {
  /* twoInt::Value index for spatial orbitals (integrals.h:86-95) */
  int mij = I > J ? I : J, nij = I > J ? J : I;
  int mkl = K > L_ ? K : L_, nkl = K > L_ ? L_ : K;
  size_t ij = (size_t)mij * (mij + 1) / 2 + nij;
  size_t kl = (size_t)mkl * (mkl + 1) / 2 + nkl;
  size_t a = ij > kl ? ij : kl, b = ij > kl ? kl : ij;
  return a * (a + 1) / 2 + b;
}

/* twoInt::Value(i,j,k,l) on spin-orbitals: zero unless i,j and k,l share a spin. */
static inline double I2v(const orc_ham *h, int i, int j, int k, int l) {
  if (!((i % 2 == j % 2) && (k % 2 == l % 2))) return 0.0;
  return h->I2[packed_index(i / 2, j / 2, k / 2, l / 2)];
}

static inline double I1v(const orc_ham *h, int i, int j) { return h->I1[(size_t)i * 2 * h->L + j]; }

static void finish_ham(orc_ham *h) {
  /* DirectMat / ExchangeMat (makeintegrals.h:160-173) */
  int L = h->L, n2 = 2 * L;
  h->direct = calloc((size_t)n2 * n2, sizeof(double));
  h->exchange = calloc((size_t)n2 * n2, sizeof(double));
  for (int i = 0; i < L; i++) {
    for (int j = 0; j < L; j++) {
      for (int si = 0; si < 2; si++) {
        for (int sj = 0; sj < 2; sj++) {
          int a = 2 * i + si, b = 2 * j + sj;
          h->direct[a + n2 * b] = I2v(h, a, a, b, b);
          h->exchange[a + n2 * b] = I2v(h, a, b, b, a);
        }
      }
    }
  }
}

static void alloc_ham(orc_ham *h, int L) {
  memset(h, 0, sizeof(*h));
  h->L = L;
  h->I1 = calloc((size_t)4 * L * L, sizeof(double));
  size_t B = (size_t)L * (L + 1) / 2;
  h->n_I2 = B * (B + 1) / 2;
  h->I2 = calloc(h->n_I2, sizeof(double));
}

static void set_one(orc_ham *h, int i, int j, double v) {
  /* I1 entries for both spins and both orders (makeintegrals.h:148-152) */
  int n2 = 2 * h->L;
  h->I1[(size_t)(2 * i) * n2 + 2 * j] = v;
  h->I1[(size_t)(2 * i + 1) * n2 + 2 * j + 1] = v;
  h->I1[(size_t)(2 * j) * n2 + 2 * i] = v;
  h->I1[(size_t)(2 * j + 1) * n2 + 2 * i + 1] = v;
}

int orc_load_fcidump(const char *path, orc_ham *out) {
  /* framework/fcidump.h:29-141: header lines until "&END" with "&FCI" removed are joined and
   * split on ','; then "value i j k l" lines.  Lines that are empty or start with '!' skip. */
  FILE *f = fopen(path, "r");
  if (!f) return -1;
  char *line = NULL;
  size_t cap = 0;
  ssize_t len;
  int in_header = 1;
  size_t hcap = 4096, hlen = 0;
  char *header = malloc(hcap);
  header[0] = 0;
  size_t ncap = 1 << 16, nint = 0;
  double *vals = malloc(ncap * sizeof(double));
  int *idx = malloc(ncap * 4 * sizeof(int));
  while ((len = getline(&line, &cap, f)) >= 0) {
    while (len > 0 && (line[len - 1] == '\n' || line[len - 1] == '\r')) line[--len] = 0;
    if (len == 0 || line[0] == '!') continue;
    if (in_header) {
      if (strstr(line, "&END")) {
        in_header = 0;
        continue;
      }
      char *p = strstr(line, "&FCI");
      if (p) memmove(p, p + 4, strlen(p + 4) + 1);
      size_t l = strlen(line);
      if (hlen + l + 1 > hcap) {
        hcap = 2 * (hlen + l + 1);
        header = realloc(header, hcap);
      }
      memcpy(header + hlen, line, l + 1);
      hlen += l;
    } else {
      double v;
      int i, j, k, l;
      if (sscanf(line, "%lf %d %d %d %d", &v, &i, &j, &k, &l) != 5) continue;
      if (nint == ncap) {
        ncap *= 2;
        vals = realloc(vals, ncap * sizeof(double));
        idx = realloc(idx, ncap * 4 * sizeof(int));
      }
      vals[nint] = v;
      idx[4 * nint] = i;
      idx[4 * nint + 1] = j;
      idx[4 * nint + 2] = k;
      idx[4 * nint + 3] = l;
      nint++;
    }
  }
  free(line);
  fclose(f);
  int L = -1, N = -1;
  for (char *tok = strtok(header, ","); tok; tok = strtok(NULL, ",")) {
    char *eq = strchr(tok, '=');
    if (!eq) continue;
    *eq = 0;
    char *key = tok;
    while (*key == ' ' || *key == '\t') key++;
    char *end = key + strlen(key);
    while (end > key && (end[-1] == ' ' || end[-1] == '\t')) *--end = 0;
    if (strcmp(key, "NORB") == 0) L = atoi(eq + 1);
    if (strcmp(key, "NELEC") == 0) N = atoi(eq + 1);
  }
  free(header);
  if (L <= 0 || L > 64) {
    free(vals);
    free(idx);
    return -2;
  }
  alloc_ham(out, L);
  out->nelec = N;
  for (size_t n = 0; n < nint; n++) {
    int i = idx[4 * n], j = idx[4 * n + 1], k = idx[4 * n + 2], l = idx[4 * n + 3];
    if (i == 0 && j == 0 && k == 0 && l == 0) {
      out->I0 = vals[n];
    } else if (k == 0 && l == 0) {
      set_one(out, i - 1, j - 1, vals[n]);
    } else {
      out->I2[packed_index(i - 1, j - 1, k - 1, l - 1)] = vals[n];
    }
  }
  free(vals);
  free(idx);
  finish_ham(out);
  return 0;
}

int orc_ham_from_arrays(int L, int nelec, double I0, const double *h1, const double *eri_packed,
                        orc_ham *out) {
  alloc_ham(out, L);
  out->nelec = nelec;
  out->I0 = I0;
  for (int i = 0; i < L; i++)
    for (int j = 0; j <= i; j++) set_one(out, i, j, h1[(size_t)i * L + j]);
  memcpy(out->I2, eri_packed, out->n_I2 * sizeof(double));
  finish_ham(out);
  return 0;
}

void orc_free_ham(orc_ham *h) {
  free(h->I1);
  free(h->I2);
  free(h->direct);
  free(h->exchange);
  memset(h, 0, sizeof(*h));
}

/* ------------------------------------------------------------------------------------------ */
/* Strings (basic/makedeterminants.h:160-186, framework/bit_manipulation.h:149, 215-230, 381)  */
/* ------------------------------------------------------------------------------------------ */

static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

void orc_sort_strings(uint64_t *s, size_t n) { qsort(s, n, sizeof(uint64_t), cmp_u64); }

int orc_load_strings_bin(const char *path, int L, uint64_t *out, size_t cap, size_t *n) {
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  const int rb = (L + 7) / 8;
  unsigned char rec[8];
  uint64_t *tmp = NULL;
  size_t cnt = 0, tcap = 0;
  int seq[64];
  while (fread(rec, 1, (size_t)rb, f) == (size_t)rb) {
    /* bits of the record from the high end of each byte; the first 8*rb - L are skipped */
    int nb = 0, bit_index = 0;
    for (int b = 0; b < rb; b++)
      for (int i = 7; i >= 0; i--) {
        if (8 * rb - L <= bit_index) seq[nb++] = (rec[b] >> i) & 1;
        bit_index++;
      }
    /* reversed: orbital p is seq[L-1-p] */
    uint64_t v = 0;
    for (int p = 0; p < L; p++)
      if (seq[L - 1 - p]) v |= (uint64_t)1 << p;
    if (cnt == tcap) {
      tcap = tcap ? 2 * tcap : 1024;
      tmp = realloc(tmp, tcap * sizeof(uint64_t));
    }
    tmp[cnt++] = v;
  }
  fclose(f);
  orc_sort_strings(tmp, cnt);
  size_t u = 0;
  for (size_t i = 0; i < cnt; i++)
    if (u == 0 || tmp[i] != tmp[u - 1]) tmp[u++] = tmp[i];
  *n = u;
  if (out) memcpy(out, tmp, (u < cap ? u : cap) * sizeof(uint64_t));
  free(tmp);
  return 0;
}

int orc_load_strings(const char *path, int L, uint64_t *out, size_t cap, size_t *n) {
  FILE *f = fopen(path, "r");
  if (!f) return -1;
  char *line = NULL;
  size_t lcap = 0;
  ssize_t len;
  size_t cnt = 0;
  int rc = 0;
  uint64_t *tmp = NULL;
  size_t tcap = 0;
  while ((len = getline(&line, &lcap, f)) >= 0) {
    while (len > 0 && (line[len - 1] == '\n' || line[len - 1] == '\r' || line[len - 1] == ' '))
      line[--len] = 0;
    if (len == 0) continue;
    if (len < L || L > 64) {
      rc = -2;
      break;
    }
    /* from_string: character s[L-1-i] is orbital i (bit_manipulation.h:215-230) */
    uint64_t v = 0;
    for (int i = 0; i < L; i++) {
      char c = line[L - 1 - i];
      if (c == '1') v |= (uint64_t)1 << i;
      else if (c != '0') rc = -2;
    }
    if (rc) break;
    if (cnt == tcap) {
      tcap = tcap ? 2 * tcap : 1024;
      tmp = realloc(tmp, tcap * sizeof(uint64_t));
    }
    tmp[cnt++] = v;
  }
  free(line);
  fclose(f);
  if (rc) {
    free(tmp);
    return rc;
  }
  /* sort_bitarray: ascending, then duplicates removed (bit_manipulation.h:381-392) */
  orc_sort_strings(tmp, cnt);
  size_t u = 0;
  for (size_t i = 0; i < cnt; i++)
    if (u == 0 || tmp[u - 1] != tmp[i]) tmp[u++] = tmp[i];
  *n = u;
  if (out) memcpy(out, tmp, (u < cap ? u : cap) * sizeof(uint64_t));
  free(tmp);
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Excitation tables (tpb/helper.h:185-323, basic/determinants.h:365-432)                      */
/* ------------------------------------------------------------------------------------------ */

static inline uint64_t lmask(int L) { return L >= 64 ? ~(uint64_t)0 : (((uint64_t)1 << L) - 1); }

size_t orc_excitations(const uint64_t *bra, size_t nbra, const uint64_t *ket, size_t nket,
                       int L, int ndiff, int spin, uint64_t *off, uint64_t *ket_idx,
                       int32_t *cran) {
  const uint64_t m = lmask(L);
  off[0] = 0;
  /* counting pass (helper.h:209-214), then an exclusive scan into CSR offsets */
#pragma omp parallel for schedule(dynamic, 64)
  for (size_t i = 0; i < nbra; i++) {
    uint64_t c = 0;
    for (size_t j = 0; j < nket; j++)
      if (__builtin_popcountll((bra[i] ^ ket[j]) & m) == ndiff) c++;
    off[i + 1] = c;
  }
  for (size_t i = 0; i < nbra; i++) off[i + 1] += off[i];
  if (!ket_idx) return off[nbra];
  const int per = ndiff == 2 ? 2 : 4;
#pragma omp parallel for schedule(dynamic, 64)
  for (size_t i = 0; i < nbra; i++) {
    uint64_t w = off[i];
    for (size_t j = 0; j < nket; j++) {
      uint64_t x = (bra[i] ^ ket[j]) & m;
      if (__builtin_popcountll(x) != ndiff) continue;
      ket_idx[w] = j;
      /* OrbitalDifference(bra, ket): cr = bra \ ket, an = ket \ bra, ascending */
      uint64_t cr = bra[i] & ~ket[j] & m, an = ket[j] & ~bra[i] & m;
      int32_t c[2] = {0, 0}, a[2] = {0, 0};
      int nc = 0, na = 0;
      for (int p = 0; p < L; p++) {
        if ((cr >> p) & 1) c[nc++ & 1] = p;
        if ((an >> p) & 1) a[na++ & 1] = p;
      }
      if (per == 2) {
        cran[2 * w] = 2 * c[0] + spin;
        cran[2 * w + 1] = 2 * a[0] + spin;
      } else {
        cran[4 * w] = 2 * c[0] + spin;
        cran[4 * w + 1] = 2 * c[1] + spin;
        cran[4 * w + 2] = 2 * a[0] + spin;
        cran[4 * w + 3] = 2 * a[1] + spin;
      }
      w++;
    }
  }
  return off[nbra];
}

static void build_one(const uint64_t *bra, size_t nbra, int L, int ndiff, int spin, uint64_t **off,
                      uint64_t **ket, int32_t **cran) {
  *off = malloc((nbra + 1) * sizeof(uint64_t));
  size_t n = orc_excitations(bra, nbra, bra, nbra, L, ndiff, spin, *off, NULL, NULL);
  *ket = malloc((n ? n : 1) * sizeof(uint64_t));
  *cran = malloc((n ? n : 1) * (ndiff == 2 ? 2 : 4) * sizeof(int32_t));
  orc_excitations(bra, nbra, bra, nbra, L, ndiff, spin, *off, *ket, *cran);
}

int orc_build_tables(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb, int L,
                     orc_tables *t) {
  /* One rank: task type 2 (alpha singles + doubles), type 1 (beta singles + doubles) and
   * type 0 (alpha singles x beta singles) all span the full string ranges (helper.h:726-777). */
  memset(t, 0, sizeof(*t));
  t->na = na;
  t->nb = nb;
  build_one(astr, na, L, 2, 0, &t->sa_off, &t->sa_ket, &t->sa_cran);
  build_one(astr, na, L, 4, 0, &t->da_off, &t->da_ket, &t->da_cran);
  build_one(bstr, nb, L, 2, 1, &t->sb_off, &t->sb_ket, &t->sb_cran);
  build_one(bstr, nb, L, 4, 1, &t->db_off, &t->db_ket, &t->db_cran);
  return 0;
}

void orc_free_tables(orc_tables *t) {
  free(t->sa_off); free(t->sa_ket); free(t->sa_cran);
  free(t->da_off); free(t->da_ket); free(t->da_cran);
  free(t->sb_off); free(t->sb_ket); free(t->sb_cran);
  free(t->db_off); free(t->db_ket); free(t->db_cran);
  memset(t, 0, sizeof(*t));
}

/* ------------------------------------------------------------------------------------------ */
/* Interleaved determinant and Slater-Condon elements (basic/determinants.h:97-142, 230-501)   */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
  uint64_t w[2]; /* spin-orbitals 0..63 and 64..127 */
} det128;

static inline det128 interleave(uint64_t a, uint64_t b) {
  /* DetFromAlphaBeta: alpha orbital p -> bit 2p, beta orbital p -> bit 2p+1 */
  det128 d = {{0, 0}};
  for (int p = 0; p < 64; p++) {
    if ((a >> p) & 1) d.w[(2 * p) >> 6] |= (uint64_t)1 << ((2 * p) & 63);
    if ((b >> p) & 1) d.w[(2 * p + 1) >> 6] |= (uint64_t)1 << ((2 * p + 1) & 63);
  }
  return d;
}

static inline int getocc(const det128 *d, int x) { return (int)((d->w[x >> 6] >> (x & 63)) & 1); }

/* number of set bits in the half-open spin-orbital range [s, e) */
static inline int count_range(const det128 *d, int s, int e) {
  int c = 0;
  for (int x = s; x < e; x++) c += getocc(d, x);
  return c;
}

/* parity(det, start, end, sgn): bits counted in [start, end), then the sign flipped once more
 * when bit `start` is set -- i.e. the sign of the open interval (determinants.h:230-281). */
static inline double parity(const det128 *d, int start, int end, double sgn) {
  int nz = count_range(d, start, end);
  sgn *= (-2. * (nz % 2) + 1);
  if (getocc(d, start)) sgn *= -1.;
  return sgn;
}

double orc_zero_excite(uint64_t a, uint64_t b, const orc_ham *h) {
  /* ZeroExcite (determinants.h:434-457) */
  det128 d = interleave(a, b);
  int n2 = 2 * h->L;
  double e = 0.0;
  for (int i = 0; i < n2; i++) {
    if (!getocc(&d, i)) continue;
    e += I1v(h, i, i);
    for (int j = i + 1; j < n2; j++) {
      if (!getocc(&d, j)) continue;
      e += h->direct[i + n2 * j];
      if ((i % 2) == (j % 2)) e -= h->exchange[i + n2 * j];
    }
  }
  return e + h->I0;
}

static double one_excite_det(const det128 *d, int i, int a, const orc_ham *h) {
  /* OneExcite(det, i, a) (determinants.h:459-481): sign from the open interval, value
   * I1(a,i) + sum over occupied j of [(ai|jj) - (aj|ji)], j ascending. */
  double sgn = parity(d, i < a ? i : a, i < a ? a : i, 1.0);
  double e = I1v(h, a, i);
  for (int x = 0; x < 2; x++) {
    uint64_t bits = d->w[x];
    for (int pos = 0; pos < 64; pos++) {
      if (bits & 1ULL) {
        int j = x * 64 + pos;
        e += (I2v(h, a, i, j, j) - I2v(h, a, j, j, i));
      }
      bits >>= 1;
    }
  }
  return e * sgn;
}

static double two_excite_det(const det128 *d, int i, int j, int a, int b, const orc_ham *h) {
  /* TwoExcite(det, i, j, a, b) (determinants.h:483-501) */
  double sgn = 1.0;
  int I = i < j ? i : j, J = i < j ? j : i, A = a < b ? a : b, B = a < b ? b : a;
  sgn = parity(d, I < A ? I : A, I < A ? A : I, sgn);
  sgn = parity(d, J < B ? J : B, J < B ? B : J, sgn);
  if (A > J || B < I) sgn *= -1.0;
  return sgn * (I2v(h, A, I, B, J) - I2v(h, A, J, B, I));
}

double orc_one_excite(uint64_t a, uint64_t b, int cr, int an, const orc_ham *h) {
  det128 d = interleave(a, b);
  return one_excite_det(&d, cr, an, h);
}

double orc_two_excite(uint64_t a, uint64_t b, int i, int j, int ca, int cb, const orc_ham *h) {
  det128 d = interleave(a, b);
  return two_excite_det(&d, i, j, ca, cb, h);
}

double orc_hij(uint64_t a, uint64_t b, uint64_t a2, uint64_t b2, const orc_ham *h) {
  /* Hij(DetA, DetB) (determinants.h:503-568): c = DetA \ DetB, d = DetB \ DetA; the element
   * is evaluated on DetB. */
  det128 A = interleave(a, b), B = interleave(a2, b2);
  int c[4], dd[4], nc = 0, nd = 0;
  for (int x = 0; x < 128; x++) {
    int ia = getocc(&A, x), ib = getocc(&B, x);
    if (ia && !ib) {
      if (nc < 4) c[nc] = x;
      nc++;
    }
    if (ib && !ia) {
      if (nd < 4) dd[nd] = x;
      nd++;
    }
  }
  if (nc == 0) return orc_zero_excite(a2, b2, h);
  if (nc == 1) return one_excite_det(&B, dd[0], c[0], h);
  if (nc == 2) return two_excite_det(&B, dd[0], dd[1], c[0], c[1], h);
  return 0.0;
}

int orc_reorder_sign(uint64_t a, uint64_t b) {
  /* moving every alpha electron (at spin-orbital 2p) in front of all beta electrons passes
   * the beta electrons at orbitals q < p */
  int n = 0;
  for (int p = 0; p < 64; p++)
    if ((a >> p) & 1) n += __builtin_popcountll(b & (((uint64_t)1 << p) - 1));
  return (n & 1) ? -1 : 1;
}

/* ------------------------------------------------------------------------------------------ */
/* Diagonal and sigma (tpb/qcham.h:290-340, tpb/mult.h:625-881)                               */
/* ------------------------------------------------------------------------------------------ */

void orc_diagonal(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                  const orc_ham *h, double *hii) {
#pragma omp parallel for schedule(static)
  for (size_t ia = 0; ia < na; ia++)
    for (size_t ib = 0; ib < nb; ib++) hii[ia * nb + ib] = orc_zero_excite(astr[ia], bstr[ib], h);
}

void orc_sigma(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
               const orc_tables *t, const orc_ham *h, const double *hii, const double *C,
               double *sigma) {
  /* Per bra element the additions happen in the reference's order: the diagonal, task type 2
   * (alpha singles then doubles, ket ascending), type 1 (beta singles then doubles), type 0
   * (alpha single outer, beta single inner). */
#pragma omp parallel for schedule(dynamic, 4)
  for (size_t ia = 0; ia < na; ia++) {
    for (size_t ib = 0; ib < nb; ib++) {
      const size_t bra = ia * nb + ib;
      det128 d = interleave(astr[ia], bstr[ib]);
      double acc = sigma[bra];
      acc += hii[bra] * C[bra];
      for (uint64_t j = t->sa_off[ia]; j < t->sa_off[ia + 1]; j++) {
        size_t ket = t->sa_ket[j] * nb + ib;
        acc += one_excite_det(&d, t->sa_cran[2 * j], t->sa_cran[2 * j + 1], h) * C[ket];
      }
      for (uint64_t j = t->da_off[ia]; j < t->da_off[ia + 1]; j++) {
        size_t ket = t->da_ket[j] * nb + ib;
        const int32_t *c = t->da_cran + 4 * j;
        acc += two_excite_det(&d, c[0], c[1], c[2], c[3], h) * C[ket];
      }
      for (uint64_t j = t->sb_off[ib]; j < t->sb_off[ib + 1]; j++) {
        size_t ket = ia * nb + t->sb_ket[j];
        acc += one_excite_det(&d, t->sb_cran[2 * j], t->sb_cran[2 * j + 1], h) * C[ket];
      }
      for (uint64_t j = t->db_off[ib]; j < t->db_off[ib + 1]; j++) {
        size_t ket = ia * nb + t->db_ket[j];
        const int32_t *c = t->db_cran + 4 * j;
        acc += two_excite_det(&d, c[0], c[1], c[2], c[3], h) * C[ket];
      }
      for (uint64_t j = t->sa_off[ia]; j < t->sa_off[ia + 1]; j++) {
        size_t ja = t->sa_ket[j];
        for (uint64_t k = t->sb_off[ib]; k < t->sb_off[ib + 1]; k++) {
          size_t ket = ja * nb + t->sb_ket[k];
          acc += two_excite_det(&d, t->sa_cran[2 * j], t->sb_cran[2 * k], t->sa_cran[2 * j + 1],
                                t->sb_cran[2 * k + 1], h) *
                 C[ket];
        }
      }
      sigma[bra] = acc;
    }
  }
}

/* The closed-form test vector x_i = ((i * 0x9E3779B97F4A7C15 mod 2^64) >> 11) / 2^53 - 1/2 (the
 * input of the reference dumps made with --sigma_hash). */
double orc_hash_vector(size_t i) {
  return (double)(((uint64_t)i * 0x9E3779B97F4A7C15ull) >> 11) * 0x1p-53 - 0.5;
}

void orc_sigma_rows(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                    const orc_tables *t, const orc_ham *h, const double *C, const size_t *rows,
                    size_t nrows, double *out) {
  /* orc_sigma for the determinants rows[0..nrows) only, each added in the same order; H_ii from
   * orc_zero_excite, C[k] from the array or, when C is NULL, orc_hash_vector(k) */
#define CV(k) (C ? C[(k)] : orc_hash_vector((k)))
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t r = 0; r < nrows; r++) {
    const size_t bra = rows[r], ia = bra / nb, ib = bra % nb;
    det128 d = interleave(astr[ia], bstr[ib]);
    double acc = 0.0;
    acc += orc_zero_excite(astr[ia], bstr[ib], h) * CV(bra);
    for (uint64_t j = t->sa_off[ia]; j < t->sa_off[ia + 1]; j++)
      acc += one_excite_det(&d, t->sa_cran[2 * j], t->sa_cran[2 * j + 1], h) * CV(t->sa_ket[j] * nb + ib);
    for (uint64_t j = t->da_off[ia]; j < t->da_off[ia + 1]; j++) {
      const int32_t *c = t->da_cran + 4 * j;
      acc += two_excite_det(&d, c[0], c[1], c[2], c[3], h) * CV(t->da_ket[j] * nb + ib);
    }
    for (uint64_t j = t->sb_off[ib]; j < t->sb_off[ib + 1]; j++)
      acc += one_excite_det(&d, t->sb_cran[2 * j], t->sb_cran[2 * j + 1], h) * CV(ia * nb + t->sb_ket[j]);
    for (uint64_t j = t->db_off[ib]; j < t->db_off[ib + 1]; j++) {
      const int32_t *c = t->db_cran + 4 * j;
      acc += two_excite_det(&d, c[0], c[1], c[2], c[3], h) * CV(ia * nb + t->db_ket[j]);
    }
    for (uint64_t j = t->sa_off[ia]; j < t->sa_off[ia + 1]; j++) {
      const size_t ja = t->sa_ket[j];
      for (uint64_t k = t->sb_off[ib]; k < t->sb_off[ib + 1]; k++)
        acc += two_excite_det(&d, t->sa_cran[2 * j], t->sb_cran[2 * k], t->sa_cran[2 * j + 1],
                              t->sb_cran[2 * k + 1], h) *
               CV(ja * nb + t->sb_ket[k]);
    }
    out[r] = acc;
  }
#undef CV
}

/* ------------------------------------------------------------------------------------------ */
/* Davidson (tpb/davidson.h:667-930, framework/dm_vector.h:23-87)                              */
/* ------------------------------------------------------------------------------------------ */

static double kahan_dot(const double *x, const double *y, size_t n) {
  /* InnerProduct: Kahan summation per thread, thread sums added in order (dm_vector.h:23-51) */
  int nth = omp_get_max_threads();
  double *part = calloc((size_t)nth, sizeof(double));
#pragma omp parallel
  {
    int tid = omp_get_thread_num();
    double s = 0.0, eps = 0.0, val, tmp;
#pragma omp for schedule(static)
    for (size_t i = 0; i < n; i++) {
      val = x[i] * y[i] - eps;
      tmp = s + val;
      eps = (tmp - s) - val;
      s = tmp;
    }
    part[tid] = s;
  }
  double sum = 0.0;
  for (int i = 0; i < nth; i++) sum += part[i];
  free(part);
  return sum;
}

static double normalize(double *x, size_t n) {
  double r = sqrt(kahan_dot(x, x, n));
  double f = 1.0 / r;
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; i++) x[i] *= f;
  return r;
}

/* Cyclic Jacobi eigen-solver of a symmetric n x n matrix (column-major, leading dim lda);
 * on return A holds eigenvectors in columns, E eigenvalues ascending. */
static void jacobi_sorted(int n, double *A, int lda, double *E) {
  double *V = calloc((size_t)n * n, sizeof(double));
  double *M = malloc((size_t)n * n * sizeof(double));
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) M[i + n * j] = A[i + lda * j];
  for (int i = 0; i < n; i++) V[i + n * i] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (int j = 0; j < n; j++)
      for (int i = 0; i < j; i++) off += M[i + n * j] * M[i + n * j];
    if (off < 1e-30) break;
    for (int p = 0; p < n; p++) {
      for (int q = p + 1; q < n; q++) {
        double apq = M[p + n * q];
        if (fabs(apq) < 1e-300) continue;
        double app = M[p + n * p], aqq = M[q + n * q];
        double theta = (aqq - app) / (2.0 * apq);
        double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(tt * tt + 1.0), s = tt * c;
        for (int k = 0; k < n; k++) {
          double mkp = M[k + n * p], mkq = M[k + n * q];
          M[k + n * p] = c * mkp - s * mkq;
          M[k + n * q] = s * mkp + c * mkq;
        }
        for (int k = 0; k < n; k++) {
          double mpk = M[p + n * k], mqk = M[q + n * k];
          M[p + n * k] = c * mpk - s * mqk;
          M[q + n * k] = s * mpk + c * mqk;
        }
        for (int k = 0; k < n; k++) {
          double vkp = V[k + n * p], vkq = V[k + n * q];
          V[k + n * p] = c * vkp - s * vkq;
          V[k + n * q] = s * vkp + c * vkq;
        }
      }
    }
  }
  int *ord = malloc(n * sizeof(int));
  for (int i = 0; i < n; i++) ord[i] = i;
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++)
      if (M[ord[j] + n * ord[j]] < M[ord[i] + n * ord[i]]) {
        int tmp = ord[i];
        ord[i] = ord[j];
        ord[j] = tmp;
      }
  for (int k = 0; k < n; k++) {
    E[k] = M[ord[k] + n * ord[k]];
    for (int i = 0; i < n; i++) A[i + lda * k] = V[i + n * ord[k]];
  }
  free(ord);
  free(V);
  free(M);
}

int orc_davidson(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                 const orc_tables *t, const orc_ham *h, const double *hii, double *W, int max_it,
                 int max_nb, double eps, int verbose, double *energy, double *resid) {
  const size_t n = na * nb;
  const double eps_reg = 1.0e-12;
  const int nbk = max_nb;
  double **C = malloc(nbk * sizeof(double *));
  double **HC = malloc(nbk * sizeof(double *));
  for (int b = 0; b < nbk; b++) {
    C[b] = malloc(n * sizeof(double));
    HC[b] = malloc(n * sizeof(double));
  }
  double *R = malloc(n * sizeof(double));
  double *H = calloc((size_t)nbk * nbk, sizeof(double));
  double *U = calloc((size_t)nbk * nbk, sizeof(double));
  double *E = calloc((size_t)nbk, sizeof(double));
  int nsigma = 0;
  double norm_R = 0.0;
  int done = 0;
  for (int it = 0; it < max_it && !done; it++) {
    memcpy(C[0], W, n * sizeof(double));
    for (int ib = 0; ib < nbk; ib++) {
      memset(HC[ib], 0, n * sizeof(double));
      orc_sigma(astr, na, bstr, nb, t, h, hii, C[ib], HC[ib]);
      nsigma++;
      for (int jb = 0; jb <= ib; jb++) {
        H[jb + nbk * ib] = kahan_dot(C[jb], HC[ib], n);
        H[ib + nbk * jb] = H[jb + nbk * ib];
      }
      for (int jb = 0; jb <= ib; jb++)
        for (int kb = 0; kb <= ib; kb++) U[jb + nbk * kb] = H[jb + nbk * kb];
      jacobi_sorted(ib + 1, U, nbk, E);
      /* W = sum_k U[k,0] C_k ; R = E0 W - sum_k U[k,0] HC_k (davidson.h:782-806) */
#pragma omp parallel for schedule(static)
      for (size_t s = 0; s < n; s++) {
        double w = C[0][s] * U[0];
        double r = HC[0][s] * (-U[0]);
        for (int kb = 1; kb <= ib; kb++) {
          w += C[kb][s] * U[kb];
          r += HC[kb][s] * (-U[kb]);
        }
        W[s] = w;
        R[s] = r + E[0] * w;
      }
      normalize(W, n);
      norm_R = normalize(R, n);
      if (verbose) {
        printf(" Davidson iteration %d.%d (tol=%.16g):", it, ib, norm_R);
        for (int p = 0; p < (ib + 1 < 4 ? ib + 1 : 4); p++) printf(" %.16g", E[p]);
        printf("\n");
      }
      if (norm_R < eps) {
        done = 1;
        break;
      }
      if (ib < nbk - 1) {
        /* t = R / (E0 - H_ii) with the 1e-12 regularisation (davidson.h:858-868) */
        double *Cn = C[ib + 1];
#pragma omp parallel for schedule(static)
        for (size_t s = 0; s < n; s++) {
          if (fabs(E[0] - hii[s]) > eps_reg) Cn[s] = R[s] / (E[0] - hii[s]);
          else Cn[s] = R[s] / (E[0] - hii[s] - eps_reg);
        }
        for (int kb = 0; kb < ib + 1; kb++) {
          double olap = -kahan_dot(C[kb], Cn, n);
#pragma omp parallel for schedule(static)
          for (size_t s = 0; s < n; s++) Cn[s] += C[kb][s] * olap;
        }
        normalize(Cn, n);
      }
    }
  }
  /* final energy <W|H|W> (sbdiag.h:431-469) */
  double *Cw = calloc(n, sizeof(double));
  orc_sigma(astr, na, bstr, nb, t, h, hii, W, Cw);
  *energy = kahan_dot(W, Cw, n);
  *resid = norm_R;
  free(Cw);
  for (int b = 0; b < nbk; b++) {
    free(C[b]);
    free(HC[b]);
  }
  free(C);
  free(HC);
  free(R);
  free(H);
  free(U);
  free(E);
  return nsigma;
}

int orc_lanczos(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                const orc_tables *t, const orc_ham *h, const double *hii, double *W,
                int max_it, int num_block, double eps, int verbose, double *energy, int *steps_printed,
                int *converged) {
  const size_t n = na * nb;
  const int lda = num_block;
  double *A = calloc((size_t)lda * lda, sizeof(double));
  double *U = calloc((size_t)lda * lda, sizeof(double));
  double *E = calloc((size_t)lda, sizeof(double));
  double *HC = malloc(n * sizeof(double));
  double **C = malloc((size_t)lda * sizeof(double *));
  for (int b = 0; b < lda; b++) C[b] = malloc(n * sizeof(double));
  int nsigma = 0, printed = 0, stop_it = 0;
  for (int it = 0; it < max_it; it++) {
    /* C[0] = W; HC = 0 (tpb/lanczos.h:204-214) */
    memcpy(C[0], W, n * sizeof(double));
    memset(HC, 0, n * sizeof(double));
    int m = 0;
    double E_old = 1.0e+8;
    stop_it = 0;
    for (int ib = 0; ib < num_block; ib++) {
      m++;
      /* HC += H C[ib]; A[ib][ib] = <C[ib], HC> (:216-226) */
      orc_sigma(astr, na, bstr, nb, t, h, hii, C[ib], HC);
      nsigma++;
      A[ib + lda * ib] = kahan_dot(C[ib], HC, n);
      for (int i = 0; i < m; i++)
        for (int j = 0; j < m; j++) U[i + lda * j] = A[i + lda * j];
      jacobi_sorted(m, U, lda, E);
      /* stop on a small eigenvalue change, or at the last block (:234-241) */
      if (fabs(E[0] - E_old) < eps) {
        stop_it = 1;
        break;
      }
      E_old = E[0];
      if (ib + 1 == num_block) break;
      /* C[ib+1] = normalised (HC - a C[ib]), b = its norm (:243-254) */
      const double a = A[ib + lda * ib];
#pragma omp parallel for schedule(static)
      for (size_t s = 0; s < n; s++) HC[s] -= a * C[ib][s];
      memcpy(C[ib + 1], HC, n * sizeof(double));
      const double b = normalize(C[ib + 1], n);
      A[ib + lda * (ib + 1)] = b;
      A[ib + 1 + lda * ib] = b;
      printed++;
      if (verbose) {
        printf(" Lanczos iteration %d, step %d: (A,B)=(%.16g,%.16g):", it, ib, a, b);
        for (int q = 0; q < (m < 4 ? m : 4); q++) printf(" %.16g", E[q]);
        printf("\n");
      }
      if (fabs(b) < eps) break;
      /* HC = -b C[ib] (:275-285, one rank) */
#pragma omp parallel for schedule(static)
      for (size_t s = 0; s < n; s++) HC[s] = -b * C[ib][s];
    }
    /* W = sum_k U[k][0] C[k] (:288-305) */
    for (int i = 0; i < m; i++)
      for (int j = 0; j < m; j++) U[i + lda * j] = A[i + lda * j];
    jacobi_sorted(m, U, lda, E);
#pragma omp parallel for schedule(static)
    for (size_t s = 0; s < n; s++) {
      double w = U[0] * C[0][s];
      for (int k = 1; k < m; k++) w += U[k] * C[k][s];
      W[s] = w;
    }
    if (stop_it) break;
  }
  double *Cw = calloc(n, sizeof(double));
  orc_sigma(astr, na, bstr, nb, t, h, hii, W, Cw);
  *energy = kahan_dot(W, Cw, n);
  if (steps_printed) *steps_printed = printed;
  if (converged) *converged = stop_it;
  free(Cw);
  for (int b = 0; b < lda; b++) free(C[b]);
  free(C);
  free(HC);
  free(A);
  free(U);
  free(E);
  return nsigma;
}

/* ------------------------------------------------------------------------------------------ */
/* RDMs (tpb/correlation.h:378-664, basic/correlation.h:16-231)                                */
/* ------------------------------------------------------------------------------------------ */

static void zero_diff(const det128 *d, double w, int L, double *one, double *two) {
  /* ZeroDiffCorrelation (basic/correlation.h:16-44) */
  size_t L2 = (size_t)L * L, L4 = L2 * L2;
  int closed[128], nc = 0;
  for (int x = 0; x < 2 * L; x++)
    if (getocc(d, x)) closed[nc++] = x;
  double ww = w * w;
  for (int i = 0; i < nc; i++) {
    int oi = closed[i] / 2, si = closed[i] % 2;
    one[si * L2 + oi + (size_t)L * oi] += ww;
    for (int j = i + 1; j < nc; j++) {
      int oj = closed[j] / 2, sj = closed[j] % 2;
      two[(si + 2 * sj) * L4 + oi + (size_t)L * oj + L2 * oi + L2 * L * oj] += ww;
      two[(sj + 2 * si) * L4 + oj + (size_t)L * oi + L2 * oj + L2 * L * oi] += ww;
      if (si == sj) {
        two[(si + 2 * sj) * L4 + oi + (size_t)L * oj + L2 * oj + L2 * L * oi] += -ww;
        two[(sj + 2 * si) * L4 + oj + (size_t)L * oi + L2 * oi + L2 * L * oj] += -ww;
      }
    }
  }
}

static void one_diff(const det128 *d, double wi, double wj, int L, int i, int a, double *one,
                     double *two) {
  /* OneDiffCorrelation (basic/correlation.h:97-133) */
  size_t L2 = (size_t)L * L, L4 = L2 * L2, L3 = L2 * L;
  double sgn = parity(d, i < a ? i : a, i < a ? a : i, 1.0);
  int oi = i / 2, si = i % 2, oa = a / 2;
  double v = wi * wj * sgn;
  one[si * L2 + oi + (size_t)L * oa] += v;
  for (int x = 0; x < 2; x++) {
    uint64_t bits = d->w[x];
    while (bits) {
      int pos = __builtin_ffsll((long long)bits);
      int soj = x * 64 + pos - 1;
      int oj = soj / 2, sj = soj % 2;
      two[(si + 2 * sj) * L4 + oa + (size_t)oj * L + oi * L2 + oj * L3] += v;
      two[(sj + 2 * si) * L4 + oj + (size_t)oa * L + oj * L2 + oi * L3] += v;
      if (si == sj) {
        two[(si + 2 * sj) * L4 + oa + (size_t)oj * L + oj * L2 + oi * L3] += -v;
        two[(sj + 2 * si) * L4 + oj + (size_t)oa * L + oi * L2 + oj * L3] += -v;
      }
      bits &= ~((uint64_t)1 << (pos - 1));
    }
  }
}

static void two_diff(const det128 *d, double wi, double wj, int L, int i, int j, int a, int b,
                     double *two) {
  /* TwoDiffCorrelation (basic/correlation.h:191-231) */
  size_t L2 = (size_t)L * L, L4 = L2 * L2;
  double sgn = 1.0;
  int I = i < j ? i : j, J = i < j ? j : i, A = a < b ? a : b, B = a < b ? b : a;
  sgn = parity(d, I < A ? I : A, I < A ? A : I, sgn);
  sgn = parity(d, J < B ? J : B, J < B ? B : J, sgn);
  if (A > J || B < I) sgn *= -1.0;
  int oi = I / 2, si = I % 2, oa = A / 2, sa = A % 2, oj = J / 2, sj = J % 2, ob = B / 2,
      sb = B % 2;
  (void)sa;
  double v = sgn * wi * wj;
  if (si == sa) {
    two[(si + 2 * sj) * L4 + oa + (size_t)L * ob + L2 * (oi + (size_t)L * oj)] += v;
    two[(sj + 2 * si) * L4 + ob + (size_t)L * oa + L2 * (oj + (size_t)L * oi)] += v;
  }
  if (si == sb) {
    two[(si + 2 * sj) * L4 + oa + (size_t)L * ob + L2 * (oj + (size_t)L * oi)] += -v;
    two[(sj + 2 * si) * L4 + ob + (size_t)L * oa + L2 * (oi + (size_t)L * oj)] += -v;
  }
}

void orc_rdm(const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
             const orc_tables *t, int L, const double *W, double *one, double *two) {
  size_t L2 = (size_t)L * L, L4 = L2 * L2;
  memset(one, 0, 2 * L2 * sizeof(double));
  memset(two, 0, 4 * L4 * sizeof(double));
  int nth = omp_get_max_threads();
  double *one_t = calloc((size_t)nth * 2 * L2, sizeof(double));
  double *two_t = calloc((size_t)nth * 4 * L4, sizeof(double));
#pragma omp parallel
  {
    int tid = omp_get_thread_num();
    double *o = one_t + (size_t)tid * 2 * L2, *w2 = two_t + (size_t)tid * 4 * L4;
#pragma omp for schedule(dynamic, 4)
    for (size_t ia = 0; ia < na; ia++) {
      for (size_t ib = 0; ib < nb; ib++) {
        size_t bra = ia * nb + ib;
        det128 d = interleave(astr[ia], bstr[ib]);
        zero_diff(&d, W[bra], L, o, w2);
        for (uint64_t j = t->sa_off[ia]; j < t->sa_off[ia + 1]; j++)
          one_diff(&d, W[bra], W[t->sa_ket[j] * nb + ib], L, t->sa_cran[2 * j],
                   t->sa_cran[2 * j + 1], o, w2);
        for (uint64_t j = t->da_off[ia]; j < t->da_off[ia + 1]; j++) {
          const int32_t *c = t->da_cran + 4 * j;
          two_diff(&d, W[bra], W[t->da_ket[j] * nb + ib], L, c[0], c[1], c[2], c[3], w2);
        }
        for (uint64_t j = t->sb_off[ib]; j < t->sb_off[ib + 1]; j++)
          one_diff(&d, W[bra], W[ia * nb + t->sb_ket[j]], L, t->sb_cran[2 * j],
                   t->sb_cran[2 * j + 1], o, w2);
        for (uint64_t j = t->db_off[ib]; j < t->db_off[ib + 1]; j++) {
          const int32_t *c = t->db_cran + 4 * j;
          two_diff(&d, W[bra], W[ia * nb + t->db_ket[j]], L, c[0], c[1], c[2], c[3], w2);
        }
        for (uint64_t j = t->sa_off[ia]; j < t->sa_off[ia + 1]; j++) {
          size_t ja = t->sa_ket[j];
          for (uint64_t k = t->sb_off[ib]; k < t->sb_off[ib + 1]; k++)
            two_diff(&d, W[bra], W[ja * nb + t->sb_ket[k]], L, t->sa_cran[2 * j],
                     t->sb_cran[2 * k], t->sa_cran[2 * j + 1], t->sb_cran[2 * k + 1], w2);
        }
      }
    }
  }
  for (int tid = 0; tid < nth; tid++) {
    for (size_t i = 0; i < 2 * L2; i++) one[i] += one_t[(size_t)tid * 2 * L2 + i];
    for (size_t i = 0; i < 4 * L4; i++) two[i] += two_t[(size_t)tid * 4 * L4 + i];
  }
  free(one_t);
  free(two_t);
}

void orc_rdm_energy(const orc_ham *h, const double *one, const double *two, double *out) {
  /* main.cc:264-317: E1 = sum I1(2i,2j) (g0+g1)[i+Lj]; E2 = 1/2 sum (i a|j b) G_s[i+Lj+L^2 a+L^3 b] */
  int L = h->L;
  size_t L2 = (size_t)L * L, L4 = L2 * L2;
  double e1 = 0.0, e2 = 0.0;
  for (int io = 0; io < L; io++)
    for (int jo = 0; jo < L; jo++)
      e1 += I1v(h, 2 * io, 2 * jo) * (one[io + L * jo] + one[L2 + io + L * jo]);
  for (int io = 0; io < L; io++)
    for (int jo = 0; jo < L; jo++)
      for (int ia = 0; ia < L; ia++)
        for (int ja = 0; ja < L; ja++) {
          double v = I2v(h, 2 * io, 2 * ia, 2 * jo, 2 * ja);
          size_t k = io + (size_t)L * jo + L2 * ia + L2 * L * ja;
          for (int s = 0; s < 4; s++) e2 += 0.5 * v * two[s * L4 + k];
        }
  out[0] = h->I0;
  out[1] = e1;
  out[2] = e2;
}

/* ------------------------------------------------------------------------------------------ */
/* MLP reference (learned preconditioner checks)                                               */
/* ------------------------------------------------------------------------------------------ */

static inline float gelu_f(float x) {
  const float k0 = 0.7978845608028654f, k1 = 0.044715f;
  return 0.5f * x * (1.0f + tanhf(k0 * (x + k1 * x * x * x)));
}

static inline double dgelu_d(double x) {
  const double k0 = 0.7978845608028654, k1 = 0.044715;
  double u = k0 * (x + k1 * x * x * x);
  double th = tanh(u);
  return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * k0 * (1.0 + 3.0 * k1 * x * x);
}

void orc_mlp_forward(int n, int din, int dh, const float *x, const float *W1, const float *b1,
                     const float *W2, const float *b2, const float *W3, const float *b3,
                     float *h1_out, float *h2_out, float *y) {
#pragma omp parallel for schedule(static)
  for (int r = 0; r < n; r++) {
    float *h1 = h1_out + (size_t)r * dh, *h2 = h2_out + (size_t)r * dh;
    for (int o = 0; o < dh; o++) {
      float s = b1[o];
      for (int i = 0; i < din; i++) s += W1[(size_t)o * din + i] * x[(size_t)r * din + i];
      h1[o] = s; /* pre-activation kept */
    }
    for (int o = 0; o < dh; o++) {
      float s = b2[o];
      for (int i = 0; i < dh; i++) s += W2[(size_t)o * dh + i] * gelu_f(h1[i]);
      h2[o] = s;
    }
    float s = b3[0];
    for (int i = 0; i < dh; i++) s += W3[i] * gelu_f(h2[i]);
    y[r] = s;
  }
}

double orc_mlp_backward(int n, int din, int dh, const float *x, const float *a, const float *b,
                        const float *w, const float *W1, const float *b1, const float *W2,
                        const float *b2, const float *W3, const float *b3, double *gW1, double *gb1,
                        double *gW2, double *gb2, double *gW3, double *gb3) {
  float *h1 = malloc((size_t)n * dh * sizeof(float));
  float *h2 = malloc((size_t)n * dh * sizeof(float));
  float *y = malloc((size_t)n * sizeof(float));
  orc_mlp_forward(n, din, dh, x, W1, b1, W2, b2, W3, b3, h1, h2, y);
  memset(gW1, 0, (size_t)dh * din * sizeof(double));
  memset(gb1, 0, (size_t)dh * sizeof(double));
  memset(gW2, 0, (size_t)dh * dh * sizeof(double));
  memset(gb2, 0, (size_t)dh * sizeof(double));
  memset(gW3, 0, (size_t)dh * sizeof(double));
  gb3[0] = 0.0;
  double *d2 = malloc((size_t)dh * sizeof(double)), *d1 = malloc((size_t)dh * sizeof(double));
  double loss = 0.0;
  for (int r = 0; r < n; r++) {
    /* bounded factor 1 + c tanh(y) of the learned correction */
    const double th = tanh((double)y[r]);
    const double e = (double)a[r] * (1.0 + ORC_MLP_BOUND * th) - (double)b[r];
    loss += 0.5 * w[r] * e * e / n;
    double dy = (double)w[r] * a[r] * e / n * ORC_MLP_BOUND * (1.0 - th * th);
    const float *a1 = h1 + (size_t)r * dh, *a2 = h2 + (size_t)r * dh;
    gb3[0] += dy;
    for (int i = 0; i < dh; i++) {
      gW3[i] += dy * gelu_f(a2[i]);
      d2[i] = dy * W3[i] * dgelu_d(a2[i]);
    }
    for (int o = 0; o < dh; o++) {
      gb2[o] += d2[o];
      for (int i = 0; i < dh; i++) gW2[(size_t)o * dh + i] += d2[o] * gelu_f(a1[i]);
    }
    for (int i = 0; i < dh; i++) {
      double s = 0.0;
      for (int o = 0; o < dh; o++) s += d2[o] * W2[(size_t)o * dh + i];
      d1[i] = s * dgelu_d(a1[i]);
    }
    for (int o = 0; o < dh; o++) {
      gb1[o] += d1[o];
      for (int i = 0; i < din; i++) gW1[(size_t)o * din + i] += d1[o] * x[(size_t)r * din + i];
    }
  }
  free(d1);
  free(d2);
  free(h1);
  free(h2);
  free(y);
  return loss;
}

/* ------------------------------------------------------------------------------------------ */
/* Carry-over strings (tpb/sbdiag.h:690-736, tpb/rdmat.h, tpb/extend.h)                        */
/* ------------------------------------------------------------------------------------------ */

void orc_string_weights(const double *W, size_t na, size_t nb, double cutoff, double *wa, double *wb,
                        uint64_t *ca, uint64_t *cb, double *total) {
  /* DiagonalAdetReducedDensityMatrix (tpb/rdmat.h:47-54): ib inner, in order */
  for (size_t ia = 0; ia < na; ia++) {
    double d = 0.0;
    for (size_t ib = 0; ib < nb; ib++) d += W[ia * nb + ib] * W[ia * nb + ib];
    wa[ia] = d;
  }
  /* DiagonalBdetReducedDensityMatrix (tpb/rdmat.h:174-181): ia inner, in order */
  for (size_t ib = 0; ib < nb; ib++) {
    double d = 0.0;
    for (size_t ia = 0; ia < na; ia++) d += W[ia * nb + ib] * W[ia * nb + ib];
    wb[ib] = d;
  }
  /* SinglesExtendHalfdets (tpb/extend.h:45-58): counts above the cutoff, their total weight */
  if (ca) memset(ca, 0, sizeof(uint64_t) * na);
  if (cb) memset(cb, 0, sizeof(uint64_t) * nb);
  double t = 0.0;
  for (size_t ia = 0; ia < na; ia++)
    for (size_t ib = 0; ib < nb; ib++) {
      const double x = W[ia * nb + ib] * W[ia * nb + ib];
      if (x > cutoff) {
        t += x;
        if (ca) ca[ia]++;
        if (cb) cb[ib]++;
      }
    }
  if (total) *total = t;
}

static const double *g_sel_w; /* weights seen by the comparator below */

static int cmp_weight_desc(const void *x, const void *y) {
  const size_t i = *(const size_t *)x, j = *(const size_t *)y;
  if (g_sel_w[i] > g_sel_w[j]) return -1;
  if (g_sel_w[i] < g_sel_w[j]) return 1;
  return (i > j) - (i < j);
}

size_t orc_carryover_select(const double *w, size_t n, double ratio, double threshold, size_t *order,
                            double *truncated) {
  for (size_t i = 0; i < n; i++) order[i] = i;
  g_sel_w = w;
  qsort(order, n, sizeof(size_t), cmp_weight_desc); /* tpb/rdmat.h:78-83 */
  if (ratio > 0.0) {
    /* n_kept = static_cast<size_t>(ratio * size) (tpb/sbdiag.h:703), weight summed in order */
    size_t kept = (size_t)(ratio * (double)n);
    if (kept > n) kept = n;
    double sum = 0.0;
    for (size_t i = 0; i < kept; i++) sum += w[order[i]];
    if (truncated) *truncated = 1.0 - sum;
    return kept;
  }
  /* running sums S, Imax = upper_bound(S, 1 - threshold) + 1 (tpb/rdmat.h:85-95) */
  const double target = 1.0 - threshold;
  double sum = 0.0;
  size_t le = 0;
  for (size_t i = 0; i < n; i++) {
    sum += w[order[i]];
    if (sum <= target) le = i + 1;
  }
  if (truncated) *truncated = 0.0;
  return le + 1 < n ? le + 1 : n;
}

size_t orc_singles_extend(const uint64_t *s, size_t n, int L, uint64_t *out) {
  size_t m = 0;
  for (size_t i = 0; i < n; i++) out[m++] = s[i];
  for (size_t i = 0; i < n; i++) {
    /* single_from_hdet (basic/excitation.h:9-29): remove closed j, add open k */
    for (int j = 0; j < L; j++) {
      if (!((s[i] >> j) & 1)) continue;
      const uint64_t base = s[i] & ~((uint64_t)1 << j);
      for (int k = 0; k < L; k++)
        if (!((s[i] >> k) & 1)) out[m++] = base | ((uint64_t)1 << k);
    }
  }
  qsort(out, m, sizeof(uint64_t), cmp_u64);
  size_t u = 0;
  for (size_t i = 0; i < m; i++)
    if (u == 0 || out[i] != out[u - 1]) out[u++] = out[i];
  return u;
}
