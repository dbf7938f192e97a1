/*
 * sbd_oracle.c: CPU restatement of the reference sbd tensor-product-basis
 * selected-CI path (walkup/sbd-ykt, include/sbd/...), written from the
 * reference's algorithm in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product, pinned against
 * golden vectors from the compiled reference (tests/golden/). The product
 * library never loads it.
 *
 * Every function names the reference lines it restates. The determinant is
 * handled exactly as the reference does: the alpha and beta strings are
 * interleaved into one 2L-bit word (alpha p -> bit 2p, beta p -> bit 2p+1,
 * chemistry/basic/determinants.h:97-119), held here in an unsigned __int128.
 */
#include "sbd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

static int popc128(u128 x) {
  return __builtin_popcountll((uint64_t)x) + __builtin_popcountll((uint64_t)(x >> 64));
}
static int ctz128(u128 x) {
  uint64_t lo = (uint64_t)x;
  return lo ? __builtin_ctzll(lo) : 64 + __builtin_ctzll((uint64_t)(x >> 64));
}
static u128 bit128(int p) { return ((u128)1) << p; }

/* DetFromAlphaBeta (determinants.h:97-119) on uint64 strings. */
static u128 interleave(uint64_t a, uint64_t b) {
  u128 d = 0;
  for (int p = 0; p < 64; ++p) {
    if ((a >> p) & 1ull) d |= bit128(2 * p);
    if ((b >> p) & 1ull) d |= bit128(2 * p + 1);
  }
  return d;
}

size_t sbo_eri_index(int p, int q, int r, int s) {
  size_t pq = p > q ? (size_t)p * (p + 1) / 2 + q : (size_t)q * (q + 1) / 2 + p;
  size_t rs = r > s ? (size_t)r * (r + 1) / 2 + s : (size_t)s * (s + 1) / 2 + r;
  return pq > rs ? pq * (pq + 1) / 2 + rs : rs * (rs + 1) / 2 + pq;
}

/* oneInt::Value on spin orbitals (integrals.h:19-21 with the spin-diagonal
 * fill of makeintegrals.h:108-112): zero across spins. */
static double h1(int L, const double* h, int i, int j) {
  if ((i & 1) != (j & 1)) return 0.0;
  return h[(size_t)(i >> 1) * L + (j >> 1)];
}

/* twoInt::Value (integrals.h:51-59): zero unless spins of (i,j) and (k,l) match. */
static double v2(const double* eri, int i, int j, int k, int l) {
  if (!(((i & 1) == (j & 1)) && ((k & 1) == (l & 1)))) return 0.0;
  return eri[sbo_eri_index(i >> 1, j >> 1, k >> 1, l >> 1)];
}

/* parity (determinants.h:228-279): sign of the bits in [start, end), flipped
 * once more when bit `start` is set. */
static double parity128(u128 det, int start, int end) {
  u128 hi = end >= 128 ? ~(u128)0 : bit128(end) - 1;
  u128 lo = bit128(start) - 1;
  int n = popc128(det & (hi ^ lo));
  double sgn = (n & 1) ? -1.0 : 1.0;
  if ((det >> start) & 1) sgn = -sgn;
  return sgn;
}

int sbo_parity(uint64_t alpha, uint64_t beta, int start, int end) {
  return parity128(interleave(alpha, beta), start, end) < 0 ? -1 : 1;
}

/* ZeroExcite (determinants.h:397-421). */
static double zero_excite(u128 det, int L, double I0, const double* h, const double* eri) {
  int closed[128], n = 0;
  for (int i = 0; i < 2 * L; ++i)
    if ((det >> i) & 1) closed[n++] = i;
  double e = 0.0;
  for (int x = 0; x < n; ++x) {
    int I = closed[x];
    e += h1(L, h, I, I);
    for (int y = x + 1; y < n; ++y) {
      int J = closed[y];
      e += eri[sbo_eri_index(I / 2, I / 2, J / 2, J / 2)]; /* DirectMat (makeintegrals.h:122) */
      if ((I % 2) == (J % 2)) e -= eri[sbo_eri_index(I / 2, J / 2, J / 2, I / 2)]; /* ExchangeMat :123 */
    }
  }
  return e + I0;
}

/* OneExcite (determinants.h:423-445); det is the ket. */
static double one_excite(u128 det, int L, const double* h, const double* eri, int i, int a) {
  double sgn = parity128(det, i < a ? i : a, i < a ? a : i);
  double e = h1(L, h, a, i);
  u128 bits = det;
  while (bits) {
    int j = ctz128(bits);
    e += (v2(eri, a, i, j, j) - v2(eri, a, j, j, i));
    bits &= ~bit128(j);
  }
  return e * sgn;
}

/* TwoExcite (determinants.h:447-465); det is the ket. */
static double two_excite(u128 det, const double* eri, int i, int j, int a, int b) {
  int I = i < j ? i : j, J = i < j ? j : i;
  int A = a < b ? a : b, B = a < b ? b : a;
  double sgn = 1.0;
  sgn *= parity128(det, I < A ? I : A, I < A ? A : I);
  sgn *= parity128(det, J < B ? J : B, J < B ? B : J);
  if (A > J || B < I) sgn *= -1.0;
  return sgn * (v2(eri, A, I, B, J) - v2(eri, A, J, B, I));
}

/* Hij (determinants.h:467-526): c = bra\ket, d = ket\bra, ascending. */
static double hij128(u128 DI, u128 DJ, int L, double I0, const double* h, const double* eri) {
  u128 c = DI & ~DJ, d = DJ & ~DI;
  int nc = popc128(c);
  if (nc == 0) return zero_excite(DJ, L, I0, h, eri);
  if (nc == 1) return one_excite(DJ, L, h, eri, ctz128(d), ctz128(c));
  if (nc == 2) {
    int c0 = ctz128(c), d0 = ctz128(d);
    int c1 = ctz128(c & ~bit128(c0)), d1 = ctz128(d & ~bit128(d0));
    return two_excite(DJ, eri, d0, d1, c0, c1);
  }
  return 0.0;
}

double sbo_hij(int L, double I0, const double* h, const double* eri, uint64_t bra_a, uint64_t bra_b,
               uint64_t ket_a, uint64_t ket_b) {
  return hij128(interleave(bra_a, bra_b), interleave(ket_a, ket_b), L, I0, h, eri);
}

/* GenerateExcitation (helper.h:132-197) for one spin, flattened like
 * MakeSmartHelper (helper.h:367-437): per bra, singles then doubles. */
long long sbo_connectivity(const uint64_t* s, size_t n, uint64_t* slen, uint64_t* dlen, uint64_t* idx) {
  long long total = 0;
  for (size_t r = 0; r < n; ++r) {
    uint64_t ns = 0, nd = 0;
    for (size_t k = 0; k < n; ++k) {
      int d = __builtin_popcountll(s[r] ^ s[k]);
      if (d == 2) ++ns;
      else if (d == 4) ++nd;
    }
    if (slen) slen[r] = ns;
    if (dlen) dlen[r] = nd;
    if (idx) {
      uint64_t* ps = idx + total;
      uint64_t* pd = idx + total + ns;
      for (size_t k = 0; k < n; ++k) {
        int d = __builtin_popcountll(s[r] ^ s[k]);
        if (d == 2) *ps++ = k;
        else if (d == 4) *pd++ = k;
      }
    }
    total += (long long)(ns + nd);
  }
  return total;
}

typedef struct {
  size_t n;
  uint64_t *slen, *dlen, *off; /* off[r] = start of bra r's singles */
  uint64_t* idx;
} conn_t;

static conn_t make_conn(const uint64_t* s, size_t n) {
  conn_t c;
  c.n = n;
  c.slen = (uint64_t*)calloc(n ? n : 1, sizeof(uint64_t));
  c.dlen = (uint64_t*)calloc(n ? n : 1, sizeof(uint64_t));
  c.off = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
  long long tot = sbo_connectivity(s, n, c.slen, c.dlen, NULL);
  c.idx = (uint64_t*)calloc(tot ? (size_t)tot : 1, sizeof(uint64_t));
  sbo_connectivity(s, n, c.slen, c.dlen, c.idx);
  for (size_t r = 0; r < n; ++r) c.off[r + 1] = c.off[r] + c.slen[r] + c.dlen[r];
  return c;
}
static void free_conn(conn_t* c) { free(c->slen); free(c->dlen); free(c->off); free(c->idx); }

/* makeQChamDiagTerms (qcham.h:314-366). */
void sbo_diag_terms(int L, double I0, const double* h, const double* eri, const uint64_t* a, size_t na,
                    const uint64_t* b, size_t nb, double* hii) {
#pragma omp parallel for schedule(static)
  for (long long ia = 0; ia < (long long)na; ++ia)
    for (size_t ib = 0; ib < nb; ++ib)
      hii[(size_t)ia * nb + ib] = zero_excite(interleave(a[ia], b[ib]), L, I0, h, eri);
}

/* mult (mult.h:376-632) at world size 1: diagonal, then task type 2 (alpha
 * singles, alpha doubles), type 1 (beta singles, beta doubles), type 0
 * (alpha single x beta single), accumulated per bra element in that order. */
/* Rows [ia0, ia1) of sigma into S[(ia - ia0) * nb + ib]; hii == NULL leaves
 * out the diagonal term. */
static void sigma_conn(int L, double I0, const double* h, const double* eri, const uint64_t* a, size_t na,
                       const uint64_t* b, size_t nb, const conn_t* ca, const conn_t* cb, const double* hii,
                       const double* C, double* S, size_t ia0, size_t ia1) {
  (void)na;
#pragma omp parallel for schedule(dynamic, 1)
  for (long long ia = (long long)ia0; ia < (long long)ia1; ++ia) {
    for (size_t ib = 0; ib < nb; ++ib) {
      size_t bra = (size_t)ia * nb + ib;
      u128 DI = interleave(a[ia], b[ib]);
      double acc = hii ? hii[bra] * C[bra] : 0.0;
      for (uint64_t k = ca->off[ia]; k < ca->off[ia + 1]; ++k) {
        size_t ja = ca->idx[k];
        acc += hij128(DI, interleave(a[ja], b[ib]), L, I0, h, eri) * C[ja * nb + ib];
      }
      for (uint64_t k = cb->off[ib]; k < cb->off[ib + 1]; ++k) {
        size_t jb = cb->idx[k];
        acc += hij128(DI, interleave(a[ia], b[jb]), L, I0, h, eri) * C[(size_t)ia * nb + jb];
      }
      for (uint64_t k = ca->off[ia]; k < ca->off[ia] + ca->slen[ia]; ++k) {
        size_t ja = ca->idx[k];
        for (uint64_t m = cb->off[ib]; m < cb->off[ib] + cb->slen[ib]; ++m) {
          size_t jb = cb->idx[m];
          acc += hij128(DI, interleave(a[ja], b[jb]), L, I0, h, eri) * C[ja * nb + jb];
        }
      }
      S[bra - ia0 * nb] = acc;
    }
  }
}

void sbo_sigma(int L, double I0, const double* h, const double* eri, const uint64_t* a, size_t na,
               const uint64_t* b, size_t nb, const double* hii, const double* C, double* S) {
  conn_t ca = make_conn(a, na), cb = make_conn(b, nb);
  double* d = NULL;
  if (!hii) {
    d = (double*)malloc(sizeof(double) * na * nb);
    sbo_diag_terms(L, I0, h, eri, a, na, b, nb, d);
    hii = d;
  }
  sigma_conn(L, I0, h, eri, a, na, b, nb, &ca, &cb, hii, C, S, 0, na);
  free(d);
  free_conn(&ca);
  free_conn(&cb);
}

/* Off-diagonal part of the bra alpha rows [row0, row0 + rows) of sigma (all
 * kets), rows x nb values: what the reference mult computes for a bra block
 * with a zero diagonal (checks of large problems one block of rows at a
 * time). */
void sbo_sigma_rows(int L, double I0, const double* h, const double* eri, const uint64_t* a, size_t na,
                    const uint64_t* b, size_t nb, const double* C, size_t row0, size_t rows, double* S) {
  if (row0 >= na) return;
  if (rows > na - row0) rows = na - row0;
  conn_t ca = make_conn(a, na), cb = make_conn(b, nb);
  sigma_conn(L, I0, h, eri, a, na, b, nb, &ca, &cb, NULL, C, S, row0, row0 + rows);
  free_conn(&ca);
  free_conn(&cb);
}

/* InnerProduct with Kahan summation (dm_vector.h:20-48), one thread. */
static double kdot(const double* x, const double* y, size_t n) {
  double sum = 0.0, eps = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double val = x[i] * y[i] - eps;
    double tmp = sum + val;
    eps = (tmp - sum) - val;
    sum = tmp;
  }
  return sum;
}

/* Normalize (dm_vector.h:50-84). Returns the norm before scaling. */
static double knormalize(double* x, size_t n) {
  double r = sqrt(kdot(x, x, n));
  double f = 1.0 / r;
  for (size_t i = 0; i < n; ++i) x[i] *= f;
  return r;
}

/* Symmetric eigen-solver standing in for LAPACK dsyev('V','U')
 * (hp_numeric.h:497-516): cyclic Jacobi, eigenvalues ascending, eigenvectors
 * in the columns of A (column-major, leading dimension lda). */
static void jacobi_eig(int n, double* A, int lda, double* w) {
  double* a = (double*)malloc(sizeof(double) * n * n);
  double* v = (double*)calloc((size_t)n * n, sizeof(double));
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) a[i + n * j] = A[(i <= j ? i : j) + lda * (i <= j ? j : i)];
  for (int i = 0; i < n; ++i) v[i + n * i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < j; ++i) off += a[i + n * j] * a[i + n * j];
    if (off < 1e-300) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = a[p + n * q];
        if (fabs(apq) < 1e-300) continue;
        double app = a[p + n * p], aqq = a[q + n * q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = a[k + n * p], akq = a[k + n * q];
          a[k + n * p] = c * akp - s * akq;
          a[k + n * q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = a[p + n * k], aqk = a[q + n * k];
          a[p + n * k] = c * apk - s * aqk;
          a[q + n * k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = v[k + n * p], vkq = v[k + n * q];
          v[k + n * p] = c * vkp - s * vkq;
          v[k + n * q] = s * vkp + c * vkq;
        }
      }
  }
  int* ord = (int*)malloc(sizeof(int) * n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  for (int i = 1; i < n; ++i) {
    int x = ord[i], j = i - 1;
    while (j >= 0 && a[ord[j] + n * ord[j]] > a[x + n * x]) { ord[j + 1] = ord[j]; --j; }
    ord[j + 1] = x;
  }
  for (int k = 0; k < n; ++k) {
    w[k] = a[ord[k] + n * ord[k]];
    for (int i = 0; i < n; ++i) A[i + lda * k] = v[i + n * ord[k]];
  }
  free(ord); free(a); free(v);
}

/* Davidson, max_time overload (davidson.h:661-924), at world size 1, followed
 * by the energy evaluation of tpb::diag (sbdiag.h:250-273). */
double sbo_davidson(int L, double I0, const double* h, const double* eri, const uint64_t* a, size_t na,
                    const uint64_t* b, size_t nb, int max_it, int max_nb, double eps, double* W,
                    int* n_sigma) {
  size_t D = na * nb;
  const double eps_reg = 1.0e-12;
  int nbk = max_nb, nsig = 0;
  conn_t ca = make_conn(a, na), cb = make_conn(b, nb);
  double* hii = (double*)malloc(sizeof(double) * D);
  sbo_diag_terms(L, I0, h, eri, a, na, b, nb, hii);
  double* C = (double*)calloc(D * (size_t)nbk, sizeof(double));
  double* HC = (double*)calloc(D * (size_t)nbk, sizeof(double));
  double* R = (double*)calloc(D, sizeof(double));
  double* Hs = (double*)calloc((size_t)nbk * nbk, sizeof(double));
  double* U = (double*)calloc((size_t)nbk * nbk, sizeof(double));
  double* E = (double*)calloc((size_t)nbk, sizeof(double));
  double* w = W;
  if (!w) return 0.0;
  int done = 0;
  for (int it = 0; it < max_it; ++it) {
    memcpy(C, w, sizeof(double) * D);
    for (int ib = 0; ib < nbk; ++ib) {
      double* Cb = C + (size_t)ib * D;
      double* HCb = HC + (size_t)ib * D;
      sigma_conn(L, I0, h, eri, a, na, b, nb, &ca, &cb, hii, Cb, HCb, 0, na);
      ++nsig;
      for (int jb = 0; jb <= ib; ++jb) {
        Hs[jb + nbk * ib] = kdot(C + (size_t)jb * D, HCb, D);
        Hs[ib + nbk * jb] = Hs[jb + nbk * ib];
      }
      for (int jb = 0; jb <= ib; ++jb)
        for (int kb = 0; kb <= ib; ++kb) U[jb + nbk * kb] = Hs[jb + nbk * kb];
      jacobi_eig(ib + 1, U, nbk, E);
      double x = U[0];
      for (size_t s = 0; s < D; ++s) w[s] = C[s] * x;
      x = -1.0 * U[0];
      for (size_t s = 0; s < D; ++s) R[s] = HC[s] * x;
      for (int kb = 1; kb <= ib; ++kb) {
        x = U[kb];
        for (size_t s = 0; s < D; ++s) w[s] += C[(size_t)kb * D + s] * x;
        x = -1.0 * U[kb];
        for (size_t s = 0; s < D; ++s) R[s] += HC[(size_t)kb * D + s] * x;
      }
      for (size_t s = 0; s < D; ++s) R[s] += E[0] * w[s];
      knormalize(w, D);
      double norm_R = knormalize(R, D);
      if (norm_R < eps) { done = 1; break; }
      if (ib < nbk - 1) {
        double* Cn = C + (size_t)(ib + 1) * D;
        for (size_t s = 0; s < D; ++s) {
          if (fabs(E[0] - hii[s]) > eps_reg) Cn[s] = R[s] / (E[0] - hii[s]);
          else Cn[s] = R[s] / (E[0] - hii[s] - eps_reg);
        }
        for (int kb = 0; kb < ib + 1; ++kb) {
          double olap = kdot(C + (size_t)kb * D, Cn, D);
          olap *= -1.0;
          for (size_t s = 0; s < D; ++s) Cn[s] += C[(size_t)kb * D + s] * olap;
        }
        knormalize(Cn, D);
      }
    }
    if (done) break;
    memcpy(C, w, sizeof(double) * D);
  }
  double* S = HC; /* reuse */
  sigma_conn(L, I0, h, eri, a, na, b, nb, &ca, &cb, hii, w, S, 0, na);
  ++nsig;
  double Efin = kdot(w, S, D);
  if (n_sigma) *n_sigma = nsig;
  free(C); free(HC); free(R); free(Hs); free(U); free(E); free(hii);
  free_conn(&ca); free_conn(&cb);
  return Efin;
}

/* ZeroDiffCorrelation (correlation.h:15-44). */
static void rdm_zero(u128 det, int L, double wi, double* one, double* two) {
  size_t L2 = (size_t)L * L, L3 = L2 * L, L4 = L3 * L;
  int closed[128], n = 0;
  for (int i = 0; i < 2 * L; ++i)
    if ((det >> i) & 1) closed[n++] = i;
  for (int x = 0; x < n; ++x) {
    int oi = closed[x] / 2, si = closed[x] % 2;
    one[si * L2 + oi + L * oi] += wi * wi;
    for (int y = x + 1; y < n; ++y) {
      int oj = closed[y] / 2, sj = closed[y] % 2;
      two[(si + 2 * sj) * L4 + oi + L * oj + L2 * oi + L3 * oj] += wi * wi;
      two[(sj + 2 * si) * L4 + oj + L * oi + L2 * oj + L3 * oi] += wi * wi;
      if (si == sj) {
        two[(si + 2 * sj) * L4 + oi + L * oj + L2 * oj + L3 * oi] += -wi * wi;
        two[(sj + 2 * si) * L4 + oj + L * oi + L2 * oi + L3 * oj] += -wi * wi;
      }
    }
  }
}

/* OneDiffCorrelation (correlation.h:49-86); phase on the bra. */
static void rdm_one(u128 DI, int L, double wi, double wj, int i, int a, double* one, double* two) {
  size_t L2 = (size_t)L * L, L3 = L2 * L, L4 = L3 * L;
  double sgn = parity128(DI, i < a ? i : a, i < a ? a : i);
  int oi = i / 2, si = i % 2, oa = a / 2;
  double v = wi * wj * sgn;
  one[si * L2 + oi + L * oa] += v;
  u128 bits = DI;
  while (bits) {
    int soj = ctz128(bits);
    int oj = soj / 2, sj = soj % 2;
    two[(si + 2 * sj) * L4 + oa + oj * L + oi * L2 + oj * L3] += v;
    two[(sj + 2 * si) * L4 + oj + oa * L + oj * L2 + oi * L3] += v;
    if (si == sj) {
      two[(si + 2 * sj) * L4 + oa + oj * L + oj * L2 + oi * L3] += wi * wj * (-sgn);
      two[(sj + 2 * si) * L4 + oj + oa * L + oi * L2 + oj * L3] += wi * wj * (-sgn);
    }
    bits &= ~bit128(soj);
  }
}

/* TwoDiffCorrelation (correlation.h:91-130); phase on the bra. */
static void rdm_two(u128 DI, int L, double wi, double wj, int i, int j, int a, int b, double* two) {
  size_t L2 = (size_t)L * L, L4 = L2 * L2;
  int I = i < j ? i : j, J = i < j ? j : i, A = a < b ? a : b, B = a < b ? b : a;
  double sgn = 1.0;
  sgn *= parity128(DI, I < A ? I : A, I < A ? A : I);
  sgn *= parity128(DI, J < B ? J : B, J < B ? B : J);
  if (A > J || B < I) sgn *= -1.0;
  int oi = I / 2, si = I % 2, oa = A / 2, sa = A % 2, oj = J / 2, sj = J % 2, ob = B / 2, sb = B % 2;
  if (si == sa) {
    two[(si + 2 * sj) * L4 + oa + L * ob + L2 * (oi + L * oj)] += sgn * wi * wj;
    two[(sj + 2 * si) * L4 + ob + L * oa + L2 * (oj + L * oi)] += sgn * wi * wj;
  }
  if (si == sb) {
    two[(si + 2 * sj) * L4 + oa + L * ob + L2 * (oj + L * oi)] += (-sgn) * wi * wj;
    two[(sj + 2 * si) * L4 + ob + L * oa + L2 * (oi + L * oj)] += (-sgn) * wi * wj;
  }
}

/* CorrelationTermAddition (correlation.h:135-189). */
static void rdm_pair(u128 DI, u128 DJ, int L, double wi, double wj, double* one, double* two) {
  u128 c = DI & ~DJ, d = DJ & ~DI;
  int nc = popc128(c);
  if (nc == 0) rdm_zero(DI, L, wi, one, two);
  else if (nc == 1) rdm_one(DI, L, wi, wj, ctz128(c), ctz128(d), one, two);
  else if (nc == 2) {
    int c0 = ctz128(c), d0 = ctz128(d);
    int c1 = ctz128(c & ~bit128(c0)), d1 = ctz128(d & ~bit128(d0));
    rdm_two(DI, L, wi, wj, c0, c1, d0, d1, two);
  }
}

/* Correlation (correlation.h:194-444) at world size 1, one thread. */
void sbo_rdm(int L, const uint64_t* a, size_t na, const uint64_t* b, size_t nb, const double* W,
             double* one, double* two) {
  size_t L2 = (size_t)L * L, L4 = L2 * L2;
  memset(one, 0, sizeof(double) * 2 * L2);
  memset(two, 0, sizeof(double) * 4 * L4);
  conn_t ca = make_conn(a, na), cb = make_conn(b, nb);
  for (size_t ia = 0; ia < na; ++ia)
    for (size_t ib = 0; ib < nb; ++ib) rdm_zero(interleave(a[ia], b[ib]), L, W[ia * nb + ib], one, two);
  for (size_t ia = 0; ia < na; ++ia)
    for (size_t ib = 0; ib < nb; ++ib) {
      size_t bra = ia * nb + ib;
      u128 DI = interleave(a[ia], b[ib]);
      for (uint64_t k = ca.off[ia]; k < ca.off[ia + 1]; ++k) {
        size_t ja = ca.idx[k];
        rdm_pair(DI, interleave(a[ja], b[ib]), L, W[bra], W[ja * nb + ib], one, two);
      }
    }
  for (size_t ia = 0; ia < na; ++ia)
    for (size_t ib = 0; ib < nb; ++ib) {
      size_t bra = ia * nb + ib;
      u128 DI = interleave(a[ia], b[ib]);
      for (uint64_t k = cb.off[ib]; k < cb.off[ib + 1]; ++k) {
        size_t jb = cb.idx[k];
        rdm_pair(DI, interleave(a[ia], b[jb]), L, W[bra], W[ia * nb + jb], one, two);
      }
    }
  for (size_t ia = 0; ia < na; ++ia)
    for (size_t ib = 0; ib < nb; ++ib) {
      size_t bra = ia * nb + ib;
      u128 DI = interleave(a[ia], b[ib]);
      for (uint64_t k = ca.off[ia]; k < ca.off[ia] + ca.slen[ia]; ++k) {
        size_t ja = ca.idx[k];
        for (uint64_t m = cb.off[ib]; m < cb.off[ib] + cb.slen[ib]; ++m) {
          size_t jb = cb.idx[m];
          rdm_pair(DI, interleave(a[ja], b[jb]), L, W[bra], W[ja * nb + jb], one, two);
        }
      }
    }
  free_conn(&ca);
  free_conn(&cb);
}

/* OccupationDensity (occupation.h:10-95) for all orbitals, density[2p+s]. */
void sbo_occupation(int L, const uint64_t* a, size_t na, const uint64_t* b, size_t nb, const double* W,
                    double* density) {
  for (int p = 0; p < 2 * L; ++p) density[p] = 0.0;
  for (size_t ia = 0; ia < na; ++ia)
    for (size_t ib = 0; ib < nb; ++ib) {
      double w2 = W[ia * nb + ib] * W[ia * nb + ib];
      for (int p = 0; p < L; ++p) {
        if ((a[ia] >> p) & 1ull) density[2 * p] += w2;
        if ((b[ib] >> p) & 1ull) density[2 * p + 1] += w2;
      }
    }
}

static const double* g_sort_key;
static int cmp_desc(const void* x, const void* y) {
  uint64_t i = *(const uint64_t*)x, j = *(const uint64_t*)y;
  double di = g_sort_key[i], dj = g_sort_key[j];
  if (di > dj) return -1;
  if (di < dj) return 1;
  return i < j ? -1 : (i > j ? 1 : 0);
}

/* CarryOverAlphaDet (rdmat.h:99-196) with DiagonalReducedDensityMatrix
 * (rdmat.h:10-57). Ties in weight are broken by ascending alpha index (the
 * reference's std::sort leaves their order unspecified). */
long long sbo_carryover(const double* W, size_t na, size_t nb, double ratio, double threshold,
                        uint64_t* order, double* truncated) {
  double* Dw = (double*)calloc(na ? na : 1, sizeof(double));
  for (size_t ia = 0; ia < na; ++ia) {
    double s = 0.0;
    for (size_t ib = 0; ib < nb; ++ib) s += W[ia * nb + ib] * W[ia * nb + ib];
    Dw[ia] = s;
  }
  uint64_t* idx = (uint64_t*)malloc(sizeof(uint64_t) * (na ? na : 1));
  for (size_t i = 0; i < na; ++i) idx[i] = i;
  g_sort_key = Dw;
  qsort(idx, na, sizeof(uint64_t), cmp_desc);
  long long kept;
  if (ratio == 0.0) {
    double target = 1.0 - threshold, sum = 0.0;
    size_t first_above = na;
    for (size_t i = 0; i < na; ++i) {
      sum += Dw[idx[i]];
      if (sum > target) { first_above = i; break; }
    }
    kept = (long long)first_above + 1;
    if (kept > (long long)na) kept = (long long)na;
    if (truncated) *truncated = 0.0;
  } else {
    kept = (long long)(size_t)(ratio * (double)na);
    if (kept > (long long)na) kept = (long long)na;
    double sum = 0.0;
    for (long long i = 0; i < kept; ++i) sum += Dw[idx[i]];
    if (truncated) *truncated = 1.0 - sum;
  }
  for (long long i = 0; i < kept; ++i) order[i] = idx[i];
  free(idx);
  free(Dw);
  return kept;
}

/* E1 + E2 + I0 from the RDMs, as the sample driver checks it (main.cc:166-216). */
double sbo_rdm_energy(int L, double I0, const double* h, const double* eri, const double* one,
                      const double* two) {
  size_t L2 = (size_t)L * L, L4 = L2 * L2;
  double e1 = 0.0, e2 = 0.0;
  for (int io = 0; io < L; ++io)
    for (int jo = 0; jo < L; ++jo)
      e1 += h[(size_t)io * L + jo] * (one[io + L * jo] + one[L2 + io + L * jo]);
  for (int io = 0; io < L; ++io)
    for (int jo = 0; jo < L; ++jo)
      for (int ia = 0; ia < L; ++ia)
        for (int ja = 0; ja < L; ++ja) {
          double v = eri[sbo_eri_index(io, ia, jo, ja)];
          size_t k = io + (size_t)L * jo + L2 * ia + L2 * L * ja;
          for (int s = 0; s < 4; ++s) e2 += 0.5 * v * two[s * L4 + k];
        }
  return I0 + e1 + e2;
}
