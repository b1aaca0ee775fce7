/*
 * sbd_oracle.c -- CPU restatement of the reference's tensor-product-basis
 * Davidson hot path (r-ccs-cms/sbd), written from the reference's algorithm in
 * plain C.  TEST INFRASTRUCTURE ONLY: the product never links, loads or calls
 * this file; tests and the bench's CPU-baseline leg use it as the checker.
 *
 * Parity is pinned by comparing this restatement with the compiled reference
 * (oracle/_ref/libsbdref.so) and with golden vectors that the reference itself
 * produced (tests/golden/).
 *
 * Conventions follow the reference exactly: determinants interleave spin
 * orbitals (alpha orbital p -> bit 2p, beta orbital p -> bit 2p+1,
 * chemistry/basic/determinants.h:98-119); the wavefunction is row-major
 * W[ia*nb + ib]; fermionic signs count occupied spin orbitals strictly between
 * the two indices in that interleaved order (determinants.h:205-256).
 * Strings are packed one bit per orbital into a uint64 (norb <= 64).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

typedef struct {
  int L;
  size_t na, nb;
  uint64_t* a;   /* alpha strings, ascending */
  uint64_t* b;   /* beta strings, ascending */
  double ecore;
  double* h;     /* [L*L] */
  double* eri;   /* [L^4], (pq|rs) at ((p*L+q)*L+r)*L+s */
  /* excitation tables (helper.h:132-182): per bra string, ascending kets */
  uint64_t *sa_off, *sa_idx, *da_off, *da_idx;
  uint64_t *sb_off, *sb_idx, *db_off, *db_idx;
} orc_sys;

static inline int popc128(u128 x) {
  return __builtin_popcountll((uint64_t)x) + __builtin_popcountll((uint64_t)(x >> 64));
}

/* DetFromAlphaBeta, determinants.h:98-119 */
static inline u128 interleave(uint64_t a, uint64_t b, int L) {
  u128 d = 0;
  for (int i = 0; i < L; i++) {
    if ((a >> i) & 1) d |= (u128)1 << (2 * i);
    if ((b >> i) & 1) d |= (u128)1 << (2 * i + 1);
  }
  return d;
}

static inline double I1v(const orc_sys* s, int i, int j) { /* integrals.h:10-22 + makeintegrals.h:108-112 */
  if ((i & 1) != (j & 1)) return 0.0;
  return s->h[(i >> 1) * s->L + (j >> 1)];
}
static inline double I2v(const orc_sys* s, int i, int j, int k, int l) { /* integrals.h:51-59 */
  if (!(((i & 1) == (j & 1)) && ((k & 1) == (l & 1)))) return 0.0;
  int L = s->L;
  return s->eri[(((size_t)(i >> 1) * L + (j >> 1)) * L + (k >> 1)) * L + (l >> 1)];
}
static inline double direct(const orc_sys* s, int i, int j) { /* (ii|jj), makeintegrals.h:122 */
  int L = s->L;
  return s->eri[(((size_t)i * L + i) * L + j) * L + j];
}
static inline double exchange(const orc_sys* s, int i, int j) { /* (ij|ji), makeintegrals.h:123 */
  int L = s->L;
  return s->eri[(((size_t)i * L + j) * L + j) * L + i];
}

/* parity, determinants.h:205-256: sign (-1)^(occupied strictly between). */
static inline double parity(u128 det, int start, int end) {
  int lo = start < end ? start : end, hi = start < end ? end : start;
  if (hi - lo < 2) return 1.0;
  u128 mask = (((u128)1 << hi) - 1) ^ (((u128)1 << (lo + 1)) - 1);
  return (popc128(det & mask) & 1) ? -1.0 : 1.0;
}

/* ZeroExcite, determinants.h:374-398 */
static double zero_excite(const orc_sys* s, u128 det) {
  int closed[128];
  int n = 0;
  for (int i = 0; i < 2 * s->L; i++)
    if ((det >> i) & 1) closed[n++] = i;
  double e = 0.0;
  for (int i = 0; i < n; i++) {
    int I = closed[i];
    e += I1v(s, I, I);
    for (int j = i + 1; j < n; j++) {
      int J = closed[j];
      e += direct(s, I / 2, J / 2);
      if ((I % 2) == (J % 2)) e -= exchange(s, I / 2, J / 2);
    }
  }
  return e + s->ecore;
}

/* OneExcite, determinants.h:400-422 (det = ket, i annihilated, a created) */
static double one_excite(const orc_sys* s, u128 det, int i, int a) {
  double sgn = parity(det, i, a);
  double e = I1v(s, a, i);
  for (int j = 0; j < 2 * s->L; j++)
    if ((det >> j) & 1) e += (I2v(s, a, i, j, j) - I2v(s, a, j, j, i));
  return e * sgn;
}

/* TwoExcite, determinants.h:424-442 */
static double two_excite(const orc_sys* s, u128 det, int i, int j, int a, int b) {
  int I = i < j ? i : j, J = i < j ? j : i;
  int A = a < b ? a : b, B = a < b ? b : a;
  double sgn = parity(det, I, A) * parity(det, J, B);
  if (A > J || B < I) sgn *= -1.0;
  return sgn * (I2v(s, A, I, B, J) - I2v(s, A, J, B, I));
}

/* Hij, determinants.h:505-564 (DetA = bra, DetB = ket) */
static double hij(const orc_sys* s, u128 bra, u128 ket) {
  u128 cm = bra & ~ket, dm = ket & ~bra;
  int c[2], d[2], nc = 0, nd = 0;
  for (int i = 0; i < 2 * s->L; i++) {
    if ((cm >> i) & 1) { if (nc < 2) c[nc] = i; nc++; }
    if ((dm >> i) & 1) { if (nd < 2) d[nd] = i; nd++; }
  }
  if (nc == 0) return zero_excite(s, ket);
  if (nc == 1) return one_excite(s, ket, d[0], c[0]);
  if (nc == 2) return two_excite(s, ket, d[0], d[1], c[0], c[1]);
  return 0.0;
}

/* ---------------------------------------------------------------- tables */

/* GenerateExcitation, helper.h:132-182: for each bra string, the ascending kets
 * at popcount(bra ^ ket) == 2 (singles) or 4 (doubles). */
static void build_table(size_t n, const uint64_t* str, int dist, uint64_t** off_out, uint64_t** idx_out) {
  uint64_t* off = (uint64_t*)malloc((n + 1) * sizeof(uint64_t));
  off[0] = 0;
#pragma omp parallel for schedule(dynamic, 16)
  for (size_t i = 0; i < n; i++) {
    uint64_t c = 0;
    for (size_t j = 0; j < n; j++) c += (__builtin_popcountll(str[i] ^ str[j]) == dist);
    off[i + 1] = c;
  }
  for (size_t i = 0; i < n; i++) off[i + 1] += off[i];
  uint64_t* idx = (uint64_t*)malloc((off[n] ? off[n] : 1) * sizeof(uint64_t));
#pragma omp parallel for schedule(dynamic, 16)
  for (size_t i = 0; i < n; i++) {
    uint64_t k = off[i];
    for (size_t j = 0; j < n; j++)
      if (__builtin_popcountll(str[i] ^ str[j]) == dist) idx[k++] = j;
  }
  *off_out = off;
  *idx_out = idx;
}

void* orc_create(int L, size_t na, size_t nb, const uint64_t* a, const uint64_t* b, double ecore,
                 const double* h, const double* eri) {
  orc_sys* s = (orc_sys*)calloc(1, sizeof(orc_sys));
  s->L = L;
  s->na = na;
  s->nb = nb;
  s->a = (uint64_t*)malloc(na * sizeof(uint64_t));
  s->b = (uint64_t*)malloc(nb * sizeof(uint64_t));
  memcpy(s->a, a, na * sizeof(uint64_t));
  memcpy(s->b, b, nb * sizeof(uint64_t));
  s->ecore = ecore;
  size_t L2 = (size_t)L * L, L4 = L2 * L2;
  s->h = (double*)malloc(L2 * sizeof(double));
  s->eri = (double*)malloc(L4 * sizeof(double));
  memcpy(s->h, h, L2 * sizeof(double));
  memcpy(s->eri, eri, L4 * sizeof(double));
  build_table(na, s->a, 2, &s->sa_off, &s->sa_idx);
  build_table(na, s->a, 4, &s->da_off, &s->da_idx);
  build_table(nb, s->b, 2, &s->sb_off, &s->sb_idx);
  build_table(nb, s->b, 4, &s->db_off, &s->db_idx);
  return s;
}

void orc_destroy(void* p) {
  orc_sys* s = (orc_sys*)p;
  if (!s) return;
  free(s->a); free(s->b); free(s->h); free(s->eri);
  free(s->sa_off); free(s->sa_idx); free(s->da_off); free(s->da_idx);
  free(s->sb_off); free(s->sb_idx); free(s->db_off); free(s->db_idx);
  free(s);
}

/* kind 0 singles, 1 doubles; returns total; copies when out pointers non-null */
uint64_t orc_table(void* p, int spin, int kind, uint64_t* off, uint64_t* idx) {
  orc_sys* s = (orc_sys*)p;
  size_t n = spin == 0 ? s->na : s->nb;
  uint64_t* o = spin == 0 ? (kind == 0 ? s->sa_off : s->da_off) : (kind == 0 ? s->sb_off : s->db_off);
  uint64_t* x = spin == 0 ? (kind == 0 ? s->sa_idx : s->da_idx) : (kind == 0 ? s->sb_idx : s->db_idx);
  if (off) memcpy(off, o, (n + 1) * sizeof(uint64_t));
  if (idx) memcpy(idx, x, o[n] * sizeof(uint64_t));
  return o[n];
}

double orc_hij(void* p, uint64_t ia, uint64_t ib, uint64_t ja, uint64_t jb) {
  orc_sys* s = (orc_sys*)p;
  return hij(s, interleave(ia, ib, s->L), interleave(ja, jb, s->L));
}

/* makeQChamDiagTerms, qcham.h:314-366 */
void orc_hii(void* p, double* hii) {
  orc_sys* s = (orc_sys*)p;
#pragma omp parallel for schedule(static)
  for (size_t ia = 0; ia < s->na; ia++)
    for (size_t ib = 0; ib < s->nb; ib++)
      hii[ia * s->nb + ib] = zero_excite(s, interleave(s->a[ia], s->b[ib], s->L));
}

/* direct mult, mult.h:387-648, for bra alpha rows [r0, r1); out holds
 * (r1-r0)*nb values.  Per element the terms are accumulated in the reference's
 * task order: diagonal, alpha singles, alpha doubles, beta singles, beta
 * doubles, alpha-beta. */
void orc_sigma(void* p, const double* C, double* out, size_t r0, size_t r1) {
  orc_sys* s = (orc_sys*)p;
  size_t nb = s->nb;
  int L = s->L;
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t ia = r0; ia < r1; ia++) {
    for (size_t ib = 0; ib < nb; ib++) {
      u128 I = interleave(s->a[ia], s->b[ib], L);
      double acc = zero_excite(s, I) * C[ia * nb + ib];
      for (uint64_t k = s->sa_off[ia]; k < s->sa_off[ia + 1]; k++) {
        size_t ja = s->sa_idx[k];
        acc += hij(s, I, interleave(s->a[ja], s->b[ib], L)) * C[ja * nb + ib];
      }
      for (uint64_t k = s->da_off[ia]; k < s->da_off[ia + 1]; k++) {
        size_t ja = s->da_idx[k];
        acc += hij(s, I, interleave(s->a[ja], s->b[ib], L)) * C[ja * nb + ib];
      }
      for (uint64_t k = s->sb_off[ib]; k < s->sb_off[ib + 1]; k++) {
        size_t jb = s->sb_idx[k];
        acc += hij(s, I, interleave(s->a[ia], s->b[jb], L)) * C[ia * nb + jb];
      }
      for (uint64_t k = s->db_off[ib]; k < s->db_off[ib + 1]; k++) {
        size_t jb = s->db_idx[k];
        acc += hij(s, I, interleave(s->a[ia], s->b[jb], L)) * C[ia * nb + jb];
      }
      for (uint64_t k = s->sa_off[ia]; k < s->sa_off[ia + 1]; k++) {
        size_t ja = s->sa_idx[k];
        for (uint64_t m = s->sb_off[ib]; m < s->sb_off[ib + 1]; m++) {
          size_t jb = s->sb_idx[m];
          acc += hij(s, I, interleave(s->a[ja], s->b[jb], L)) * C[ja * nb + jb];
        }
      }
      out[(ia - r0) * nb + ib] = acc;
    }
  }
}

/* ---------------------------------------------------------------- Davidson */

static double dot(const double* x, const double* y, size_t n) {
  double sum = 0.0;
#pragma omp parallel for reduction(+ : sum) schedule(static)
  for (size_t i = 0; i < n; i++) sum += x[i] * y[i];
  return sum;
}

static double normalize(double* x, size_t n) { /* dm_vector.h:268-286 */
  double r = sqrt(dot(x, x, n));
  double f = 1.0 / r;
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; i++) x[i] *= f;
  return r;
}

/* Cyclic Jacobi eigen-solver for the small projected matrix (the reference
 * solves the same problem with LAPACK dsyev, hp_numeric.h:500-517, or its own
 * Jacobi routine, jacobi.h:18-95).  A is n x n column-major with leading
 * dimension lda; on return A holds eigenvectors (columns) sorted by ascending
 * eigenvalue, w the eigenvalues. */
static void jacobi_eig(int n, double* A, int lda, double* w) {
  double V[32 * 32], M[32 * 32];
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      M[i + j * n] = A[i + j * lda];
      V[i + j * n] = (i == j) ? 1.0 : 0.0;
    }
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (int j = 0; j < n; j++)
      for (int i = 0; i < j; i++) off += M[i + j * n] * M[i + j * n];
    if (off < 1e-300) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        double apq = M[p + q * n];
        if (fabs(apq) < 1e-300) continue;
        double app = M[p + p * n], aqq = M[q + q * n];
        double theta = 0.5 * (aqq - app) / apq;
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < n; k++) {
          double mkp = M[k + p * n], mkq = M[k + q * n];
          M[k + p * n] = c * mkp - sn * mkq;
          M[k + q * n] = sn * mkp + c * mkq;
        }
        for (int k = 0; k < n; k++) {
          double mpk = M[p + k * n], mqk = M[q + k * n];
          M[p + k * n] = c * mpk - sn * mqk;
          M[q + k * n] = sn * mpk + c * mqk;
        }
        for (int k = 0; k < n; k++) {
          double vkp = V[k + p * n], vkq = V[k + q * n];
          V[k + p * n] = c * vkp - sn * vkq;
          V[k + q * n] = sn * vkp + c * vkq;
        }
      }
  }
  int order[32];
  for (int i = 0; i < n; i++) order[i] = i;
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++)
      if (M[order[j] + order[j] * n] < M[order[i] + order[i] * n]) {
        int t = order[i]; order[i] = order[j]; order[j] = t;
      }
  for (int k = 0; k < n; k++) {
    int src = order[k];
    w[k] = M[src + src * n];
    for (int i = 0; i < n; i++) A[i + k * lda] = V[i + src * n];
  }
}

/* Davidson with wall-time budget, davidson.h:661-923, followed by the extra
 * sigma for E = <W|HW> (sbdiag.h:239-262).  W: in = initial vector, out = Ritz
 * vector.  Per step k: trace_e[k] = lowest Ritz value, trace_tol[k] = residual
 * norm.  Returns E; *nsteps receives the step count. */
double orc_davidson(void* p, double* W, int max_it, int nbk, double eps, double* trace_e,
                    double* trace_tol, int max_trace, int* nsteps) {
  orc_sys* s = (orc_sys*)p;
  size_t n = s->na * s->nb;
  double eps_reg = 1.0e-12;
  double* hii = (double*)malloc(n * sizeof(double));
  orc_hii(p, hii);
  double** C = (double**)malloc(nbk * sizeof(double*));
  double** HC = (double**)malloc(nbk * sizeof(double*));
  for (int k = 0; k < nbk; k++) {
    C[k] = (double*)malloc(n * sizeof(double));
    HC[k] = (double*)malloc(n * sizeof(double));
  }
  double* R = (double*)malloc(n * sizeof(double));
  double* H = (double*)calloc(nbk * nbk, sizeof(double));
  double* U = (double*)calloc(nbk * nbk, sizeof(double));
  double* E = (double*)malloc(nbk * sizeof(double));
  int steps = 0;
  int done = 0;
  for (int it = 0; it < max_it && !done; it++) {
    memcpy(C[0], W, n * sizeof(double));
    for (int ib = 0; ib < nbk; ib++) {
      orc_sigma(p, C[ib], HC[ib], 0, s->na);
      for (int jb = 0; jb <= ib; jb++) {
        H[jb + nbk * ib] = dot(C[jb], HC[ib], n);
        H[ib + nbk * jb] = H[jb + nbk * ib];
      }
      for (int jb = 0; jb <= ib; jb++)
        for (int kb = 0; kb <= ib; kb++) U[jb + nbk * kb] = H[jb + nbk * kb];
      jacobi_eig(ib + 1, U, nbk, E);
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < n; i++) {
        double w = 0.0, r = 0.0;
        for (int kb = 0; kb <= ib; kb++) {
          w += C[kb][i] * U[kb];
          r -= HC[kb][i] * U[kb];
        }
        W[i] = w;
        R[i] = r + E[0] * w;
      }
      normalize(W, n);
      double tol = normalize(R, n);
      if (steps < max_trace) {
        trace_e[steps] = E[0];
        trace_tol[steps] = tol;
      }
      steps++;
      if (tol < eps) { done = 1; break; }
      if (ib < nbk - 1) {
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < n; i++) {
          double den = E[0] - hii[i];
          C[ib + 1][i] = fabs(den) > eps_reg ? R[i] / den : R[i] / (den - eps_reg);
        }
        for (int kb = 0; kb < ib + 1; kb++) {
          double olap = -dot(C[kb], C[ib + 1], n);
#pragma omp parallel for schedule(static)
          for (size_t i = 0; i < n; i++) C[ib + 1][i] += C[kb][i] * olap;
        }
        normalize(C[ib + 1], n);
      }
    }
  }
  orc_sigma(p, W, R, 0, s->na);
  double energy = dot(W, R, n);
  *nsteps = steps;
  for (int k = 0; k < nbk; k++) { free(C[k]); free(HC[k]); }
  free(C); free(HC); free(R); free(H); free(U); free(E); free(hii);
  return energy;
}

/* ---------------------------------------------------------------- RDMs */

/* ZeroDiffCorrelation, correlation.h:15-44 */
static void zero_diff(const orc_sys* s, u128 det, double w, double* one, double* two) {
  int L = s->L;
  size_t L2 = (size_t)L * L, L3 = L2 * L, L4 = L3 * L;
  int cl[128], n = 0;
  for (int i = 0; i < 2 * L; i++)
    if ((det >> i) & 1) cl[n++] = i;
  for (int i = 0; i < n; i++) {
    int oi = cl[i] / 2, si = cl[i] % 2;
    one[si * L2 + oi + L * oi] += w * w;
    for (int j = i + 1; j < n; j++) {
      int oj = cl[j] / 2, sj = cl[j] % 2;
      two[(si + 2 * sj) * L4 + oi + L * oj + L2 * oi + L3 * oj] += w * w;
      two[(sj + 2 * si) * L4 + oj + L * oi + L2 * oj + L3 * oi] += w * w;
      if (si == sj) {
        two[(si + 2 * sj) * L4 + oi + L * oj + L2 * oj + L3 * oi] -= w * w;
        two[(sj + 2 * si) * L4 + oj + L * oi + L2 * oi + L3 * oj] -= w * w;
      }
    }
  }
}

/* OneDiffCorrelation, correlation.h:49-86 (det = bra, i = c0, a = d0) */
static void one_diff(const orc_sys* s, u128 det, double wi, double wj, int i, int a, double* one,
                     double* two) {
  int L = s->L;
  size_t L2 = (size_t)L * L, L3 = L2 * L, L4 = L3 * L;
  double sgn = parity(det, i, a);
  int oi = i / 2, si = i % 2, oa = a / 2;
  double v = wi * wj * sgn;
  one[si * L2 + oi + L * oa] += v;
  for (int soj = 0; soj < 2 * L; soj++) {
    if (!((det >> soj) & 1)) continue;
    int oj = soj / 2, sj = soj % 2;
    two[(si + 2 * sj) * L4 + oa + oj * L + oi * L2 + oj * L3] += v;
    two[(sj + 2 * si) * L4 + oj + oa * L + oj * L2 + oi * L3] += v;
    if (si == sj) {
      two[(si + 2 * sj) * L4 + oa + oj * L + oj * L2 + oi * L3] -= v;
      two[(sj + 2 * si) * L4 + oj + oa * L + oi * L2 + oj * L3] -= v;
    }
  }
}

/* TwoDiffCorrelation, correlation.h:91-130 (det = bra; i,j = c; a,b = d) */
static void two_diff(const orc_sys* s, u128 det, double wi, double wj, int i, int j, int a, int b,
                     double* two) {
  int L = s->L;
  size_t L2 = (size_t)L * L, L4 = L2 * L2;
  int I = i < j ? i : j, J = i < j ? j : i, A = a < b ? a : b, B = a < b ? b : a;
  double sgn = parity(det, I, A) * parity(det, J, B);
  if (A > J || B < I) sgn *= -1.0;
  int oi = I / 2, si = I % 2, oa = A / 2, sa = A % 2, oj = J / 2, sj = J % 2, ob = B / 2, sb = B % 2;
  double v = sgn * wi * wj;
  if (si == sa) {
    two[(si + 2 * sj) * L4 + oa + L * ob + L2 * (oi + L * oj)] += v;
    two[(sj + 2 * si) * L4 + ob + L * oa + L2 * (oj + L * oi)] += v;
  }
  if (si == sb) {
    two[(si + 2 * sj) * L4 + oa + L * ob + L2 * (oj + L * oi)] -= v;
    two[(sj + 2 * si) * L4 + ob + L * oa + L2 * (oi + L * oj)] -= v;
  }
}

/* CorrelationTermAddition, correlation.h:135-189 */
static void term(const orc_sys* s, u128 bra, u128 ket, double wi, double wj, double* one, double* two) {
  u128 cm = bra & ~ket, dm = ket & ~bra;
  int c[2], d[2], nc = 0, nd = 0;
  for (int i = 0; i < 2 * s->L; i++) {
    if ((cm >> i) & 1) { if (nc < 2) c[nc] = i; nc++; }
    if ((dm >> i) & 1) { if (nd < 2) d[nd] = i; nd++; }
  }
  if (nc == 1) one_diff(s, bra, wi, wj, c[0], d[0], one, two);
  else if (nc == 2) two_diff(s, bra, wi, wj, c[0], c[1], d[0], d[1], two);
}

/* Correlation, correlation.h:194-443.  one: [2][L*L], two: [4][L^4]. */
void orc_correlation(void* p, const double* W, double* one, double* two) {
  orc_sys* s = (orc_sys*)p;
  int L = s->L;
  size_t nb = s->nb, L2 = (size_t)L * L, L4 = L2 * L2;
  memset(one, 0, 2 * L2 * sizeof(double));
  memset(two, 0, 4 * L4 * sizeof(double));
#pragma omp parallel
  {
    double* o = (double*)calloc(2 * L2, sizeof(double));
    double* t = (double*)calloc(4 * L4, sizeof(double));
#pragma omp for schedule(dynamic, 1)
    for (size_t ia = 0; ia < s->na; ia++) {
      for (size_t ib = 0; ib < nb; ib++) {
        u128 I = interleave(s->a[ia], s->b[ib], L);
        double wi = W[ia * nb + ib];
        zero_diff(s, I, wi, o, t);
        for (int kind = 0; kind < 2; kind++) {
          uint64_t* off = kind == 0 ? s->sa_off : s->da_off;
          uint64_t* idx = kind == 0 ? s->sa_idx : s->da_idx;
          for (uint64_t k = off[ia]; k < off[ia + 1]; k++) {
            size_t ja = idx[k];
            term(s, I, interleave(s->a[ja], s->b[ib], L), wi, W[ja * nb + ib], o, t);
          }
        }
        for (int kind = 0; kind < 2; kind++) {
          uint64_t* off = kind == 0 ? s->sb_off : s->db_off;
          uint64_t* idx = kind == 0 ? s->sb_idx : s->db_idx;
          for (uint64_t k = off[ib]; k < off[ib + 1]; k++) {
            size_t jb = idx[k];
            term(s, I, interleave(s->a[ia], s->b[jb], L), wi, W[ia * nb + jb], o, t);
          }
        }
        for (uint64_t k = s->sa_off[ia]; k < s->sa_off[ia + 1]; k++) {
          size_t ja = s->sa_idx[k];
          for (uint64_t m = s->sb_off[ib]; m < s->sb_off[ib + 1]; m++) {
            size_t jb = s->sb_idx[m];
            term(s, I, interleave(s->a[ja], s->b[jb], L), wi, W[ja * nb + jb], o, t);
          }
        }
      }
    }
#pragma omp critical
    {
      for (size_t i = 0; i < 2 * L2; i++) one[i] += o[i];
      for (size_t i = 0; i < 4 * L4; i++) two[i] += t[i];
    }
    free(o);
    free(t);
  }
}

/* OccupationDensity, occupation.h:10-95: dens[2p] alpha, dens[2p+1] beta */
void orc_occupation(void* p, const double* W, double* dens) {
  orc_sys* s = (orc_sys*)p;
  int L = s->L;
  for (int i = 0; i < 2 * L; i++) dens[i] = 0.0;
  for (size_t ia = 0; ia < s->na; ia++)
    for (size_t ib = 0; ib < s->nb; ib++) {
      double w2 = W[ia * s->nb + ib] * W[ia * s->nb + ib];
      for (int o = 0; o < L; o++) {
        if ((s->a[ia] >> o) & 1) dens[2 * o] += w2;
        if ((s->b[ib] >> o) & 1) dens[2 * o + 1] += w2;
      }
    }
}
