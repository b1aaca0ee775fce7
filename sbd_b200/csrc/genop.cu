// The generic path: a second-quantised operator (basic/generalop.h GeneralOp)
// applied to a vector on a basis of bit strings (basic/basis.h Basis), and the
// Lanczos and Davidson solvers built on it (basic/out_of_place_func/mult.h,
// lanczos.h, davidson.h), at one rank on one GPU.
//
// Layout in HBM:
//   states      [n][nw] uint64 in the caller's order (site q at bit q%64 of
//               word q/64), nw = 1, 2 or 4
//   hash table  open addressing with linear probing over a power-of-two
//               table of at least twice the states: key words and the
//               caller's index (-1 marks an empty slot); the target of every
//               off-diagonal term is found in one to three probes
//   terms       the off-diagonal list as fixed-size records: annihilation and
//               creation masks (the sites of the first n_dag operators and of
//               the rest), the coefficient and the operator sites in order
//               (for the fermionic sign), sorted by annihilation mask, with one
//               bucket record per distinct mask; the diagonal list is folded
//               into one number per state at set-up (hdiag)
//
// mult: one warp per bra state.  The warp walks the buckets (warp-uniform),
// skips every bucket whose annihilated sites are not all occupied in the
// state, and splits the terms of the others over its lanes.  A term applies
// when its created sites are empty after the annihilation, which with the
// bucket's test is the reference's sequential test (mult.h:213-240) for terms
// whose annihilated sites are distinct and whose created sites are distinct
// (a term that repeats a site in either part never applies there and is
// dropped at set-up).  The lanes' sums are reduced in the warp, so no
// atomics.  For a chemistry operator a state's occupation admits about one
// bucket in ten.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <iostream>
#include <numeric>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "internal.cuh"

using sbdgpu::Error;

struct sbdgpu_genop {
  sbdgpu_ctx base;  // device, stream, reduction scratch and the error string
  int nw = 1;
  size_t n = 0;
  int sign = 1;
  uint64_t* states = nullptr;
  uint64_t* hkeys = nullptr;  // hash table: [slots][nw] key words
  int64_t* hidx = nullptr;    // [slots] caller index, -1 = empty
  uint64_t hmask = 0;         // slots - 1
  void* terms = nullptr;       // off-diagonal records, sorted by annihilation mask
  void* buckets = nullptr;     // one record per distinct annihilation mask
  size_t n_buckets = 0;
  size_t n_terms = 0;
  void* self_terms = nullptr;  // off-diagonal records that map a state onto itself
  size_t n_self = 0;
  double* hdiag = nullptr;     // diagonal list, per state (caller order)
  bool ready = false;
};

namespace {

constexpr int kMaxOps = SBDGPU_GENOP_MAX_OPS;
constexpr int kThreads = 256;

template <int NW>
struct Term {
  uint64_t ann[NW];
  uint64_t cre[NW];
  double coef;
  int32_t nops, ndag;
  uint8_t site[kMaxOps];
};

template <int NW>
struct DiagTerm {
  uint64_t mask[NW];
  double coef;
};

template <int NW>
struct Bucket {
  uint64_t ann[NW];
  int64_t start, end;  // its terms in the sorted term array
};

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

template <int NW>
__host__ __device__ __forceinline__ uint64_t hash_state(const uint64_t* w) {
  uint64_t h = 0x9e3779b97f4a7c15ull;
  for (int x = 0; x < NW; x++) h = mix64(h ^ w[x]);
  return h;
}

// caller index of state w, or -1
template <int NW>
__device__ __forceinline__ int64_t find_state(const uint64_t* __restrict__ hkeys, const int64_t* __restrict__ hidx,
                                              uint64_t hmask, const uint64_t* w) {
  uint64_t h = hash_state<NW>(w) & hmask;
  // the table is at most half full, so an empty slot ends every probe
  // sequence; the bound keeps the loop finite regardless
  for (uint64_t probe = 0; probe <= hmask; probe++) {
    const int64_t id = __ldg(&hidx[h]);
    if (id < 0) return -1;
    bool eq = true;
#pragma unroll
    for (int x = 0; x < NW; x++) eq &= __ldg(&hkeys[h * NW + x]) == w[x];
    if (eq) return id;
    h = (h + 1) & hmask;
  }
  return -1;
}

// parity of the occupied sites below q
template <int NW>
__device__ __forceinline__ int parity_below(const uint64_t* w, int q) {
  int c = 0;
  const int r = q >> 6;
#pragma unroll
  for (int x = 0; x < NW; x++) {
    if (x < r) c += __popcll(w[x]);
    else if (x == r) c += __popcll(w[x] & ((1ull << (q & 63)) - 1ull));
  }
  return c & 1;
}

// Apply term t to state v: false when it does not apply; else the target in
// w and the sign (+1 or -1; +1 when sign is off).
template <int NW>
__device__ __forceinline__ bool apply_term(const Term<NW>& t, const uint64_t* v, int sign, uint64_t* w, double* s) {
  bool ok = true;
#pragma unroll
  for (int x = 0; x < NW; x++) {
    ok &= (v[x] & t.ann[x]) == t.ann[x];
    ok &= ((v[x] & ~t.ann[x]) & t.cre[x]) == 0ull;
  }
  if (!ok) return false;
  int par = 0;
  if (sign) {
#pragma unroll
    for (int x = 0; x < NW; x++) w[x] = v[x];
    for (int k = 0; k < t.nops; k++) {
      const int q = t.site[k];
      const uint64_t b = 1ull << (q & 63);
      if (k < t.ndag) w[q >> 6] &= ~b;
      else w[q >> 6] |= b;
      par ^= parity_below<NW>(w, q);
    }
  } else {
#pragma unroll
    for (int x = 0; x < NW; x++) w[x] = (v[x] & ~t.ann[x]) | t.cre[x];
  }
  *s = par ? -1.0 : 1.0;
  return true;
}

// W[i] += hdiag[i] C[i] + sum over off-diagonal terms of coef * sign * C[j]:
// one warp per state, its lanes over the terms of each applicable bucket
constexpr int kMultWarps = kThreads / 32;
template <int NW>
__global__ void __launch_bounds__(kThreads) mult_kernel(const uint64_t* __restrict__ states, size_t n,
                                                       const uint64_t* __restrict__ hkeys,
                                                       const int64_t* __restrict__ hidx, uint64_t hmask,
                                                       const Bucket<NW>* __restrict__ buckets, size_t n_buckets,
                                                       const Term<NW>* __restrict__ terms, int sign,
                                                       const double* __restrict__ hdiag,
                                                       const double* __restrict__ C, double* __restrict__ W) {
  const int lane = threadIdx.x & 31;
  const size_t warps = (size_t)gridDim.x * kMultWarps;
  for (size_t i = (size_t)blockIdx.x * kMultWarps + (threadIdx.x >> 5); i < n; i += warps) {
    uint64_t v[NW];
#pragma unroll
    for (int x = 0; x < NW; x++) v[x] = __ldg(&states[i * NW + x]);
    double acc = 0.0;
    for (size_t b = 0; b < n_buckets; b++) {
      bool ok = true;
#pragma unroll
      for (int x = 0; x < NW; x++) {
        const uint64_t m = __ldg(&buckets[b].ann[x]);
        ok &= (v[x] & m) == m;
      }
      if (!ok) continue;  // warp-uniform: the same state in every lane
      const int64_t t1 = __ldg(&buckets[b].end);
      for (int64_t t = __ldg(&buckets[b].start) + lane; t < t1; t += 32) {
        uint64_t w[NW];
        double s;
        if (!apply_term<NW>(terms[t], v, sign, w, &s)) continue;
        const int64_t j = find_state<NW>(hkeys, hidx, hmask, w);
        if (j >= 0) acc += __ldg(&terms[t].coef) * s * __ldg(&C[j]);
      }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) W[i] = W[i] + hdiag[i] * C[i] + acc;
  }
}

// hdiag[i] = sum of the diagonal terms whose sites are all occupied in state i
template <int NW>
__global__ void __launch_bounds__(kThreads) diag_kernel(const uint64_t* __restrict__ states, size_t n,
                                                       const DiagTerm<NW>* __restrict__ terms, size_t n_terms,
                                                       double* __restrict__ hdiag) {
  const size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  uint64_t v[NW];
#pragma unroll
  for (int x = 0; x < NW; x++) v[x] = states[i * NW + x];
  double acc = 0.0;
  for (size_t k = 0; k < n_terms; k++) {
    bool ok = true;
#pragma unroll
    for (int x = 0; x < NW; x++) ok &= (v[x] & terms[k].mask[x]) == terms[k].mask[x];
    if (ok) acc += terms[k].coef;
  }
  hdiag[i] = acc;
}

// out[i] = hdiag[i] + sum of the self-mapping off-diagonal terms that apply
template <int NW>
__global__ void __launch_bounds__(kThreads) self_kernel(const uint64_t* __restrict__ states, size_t n,
                                                       const Term<NW>* __restrict__ terms, size_t n_terms, int sign,
                                                       const double* __restrict__ hdiag, double* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  uint64_t v[NW];
#pragma unroll
  for (int x = 0; x < NW; x++) v[x] = states[i * NW + x];
  double acc = hdiag[i];
  for (size_t k = 0; k < n_terms; k++) {
    uint64_t w[NW];
    double s;
    if (apply_term<NW>(terms[k], v, sign, w, &s)) acc += terms[k].coef * s;
  }
  out[i] = acc;
}

unsigned blocks_for(size_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

template <class F>
int guarded(sbdgpu_genop* g, F&& f) {
  if (!g) return SBDGPU_ERR_ARG;
  try {
    cudaError_t e = cudaSetDevice(g->base.device);
    if (e != cudaSuccess) throw Error{SBDGPU_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e)};
    f();
    g->base.err.clear();
    return SBDGPU_OK;
  } catch (const Error& e) {
    g->base.err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g->base.err = "host allocation failed";
    return SBDGPU_ERR_ALLOC;
  } catch (const std::exception& e) {
    g->base.err = e.what();
    return SBDGPU_ERR_STATE;
  }
}

// One list's terms as host records.  Off-diagonal terms that repeat a site
// among their annihilated or among their created operators never apply
// (the reference's sequential test fails at the repeat) and are left out.
template <int NW>
void build_terms(int nw, size_t n_terms, const int64_t* off, const int32_t* ops, const int32_t* ndag,
                 const double* coef, std::vector<Term<NW>>& all, std::vector<Term<NW>>& self) {
  const int max_site = 64 * nw;
  for (size_t k = 0; k < n_terms; k++) {
    const int64_t a = off[k], b = off[k + 1];
    if (b < a) throw Error{SBDGPU_ERR_ARG, "term offsets must not decrease"};
    const int nops = (int)(b - a);
    if (nops > kMaxOps) throw Error{SBDGPU_ERR_ARG, "more than " + std::to_string(kMaxOps) + " operators in a term"};
    if (ndag[k] < 0 || ndag[k] > nops) throw Error{SBDGPU_ERR_ARG, "n_dag out of range"};
    Term<NW> t;
    std::memset(&t, 0, sizeof(t));
    t.coef = coef[k];
    t.nops = nops;
    t.ndag = ndag[k];
    bool repeat = false;
    for (int j = 0; j < nops; j++) {
      const int q = ops[a + j] & 0xFFFF;
      if (q >= max_site) throw Error{SBDGPU_ERR_ARG, "site " + std::to_string(q) + " beyond the state width"};
      t.site[j] = (uint8_t)q;
      uint64_t* m = j < t.ndag ? t.ann : t.cre;
      const uint64_t bit = 1ull << (q & 63);
      if (m[q >> 6] & bit) repeat = true;
      m[q >> 6] |= bit;
    }
    if (repeat) continue;
    all.push_back(t);
    if (std::equal(t.ann, t.ann + NW, t.cre)) self.push_back(t);
  }
}

template <int NW>
void set_terms_nw(sbdgpu_genop* g, size_t n_diag, const int64_t* diag_off, const int32_t* diag_ops,
                  const int32_t* diag_ndag, const double* diag_coef, size_t n_off, const int64_t* off_off,
                  const int32_t* off_ops, const int32_t* off_ndag, const double* off_coef) {
  cudaStream_t st = g->base.stream;
  std::vector<DiagTerm<NW>> dt;
  dt.reserve(n_diag);
  for (size_t k = 0; k < n_diag; k++) {
    const int64_t a = diag_off[k], b = diag_off[k + 1];
    if (b < a) throw Error{SBDGPU_ERR_ARG, "term offsets must not decrease"};
    if (diag_ndag[k] < 0 || diag_ndag[k] > b - a) throw Error{SBDGPU_ERR_ARG, "n_dag out of range"};
    DiagTerm<NW> d;
    std::memset(&d, 0, sizeof(d));
    d.coef = diag_coef[k];
    for (int j = 0; j < diag_ndag[k]; j++) {  // the sites of the first n_dag operators (mult.h:130-139)
      const int q = diag_ops[a + j] & 0xFFFF;
      if (q >= 64 * NW) throw Error{SBDGPU_ERR_ARG, "site " + std::to_string(q) + " beyond the state width"};
      d.mask[q >> 6] |= 1ull << (q & 63);
    }
    dt.push_back(d);
  }
  std::vector<Term<NW>> all, self;
  build_terms<NW>(NW, n_off, off_off, off_ops, off_ndag, off_coef, all, self);
  // terms grouped by annihilation mask (stable), one bucket per mask
  std::stable_sort(all.begin(), all.end(), [](const Term<NW>& a, const Term<NW>& b) {
    return std::lexicographical_compare(a.ann, a.ann + NW, b.ann, b.ann + NW);
  });
  std::vector<Bucket<NW>> bk;
  for (size_t t = 0; t < all.size(); t++) {
    if (t == 0 || !std::equal(all[t].ann, all[t].ann + NW, all[t - 1].ann)) {
      Bucket<NW> b;
      std::memcpy(b.ann, all[t].ann, sizeof(b.ann));
      b.start = (int64_t)t;
      bk.push_back(b);
    }
    bk.back().end = (int64_t)t + 1;
  }
  cudaFree(g->terms);
  cudaFree(g->self_terms);
  cudaFree(g->buckets);
  g->terms = g->self_terms = g->buckets = nullptr;
  g->n_buckets = 0;
  g->ready = false;
  DiagTerm<NW>* d_dt = nullptr;
  try {
    if (!dt.empty()) {
      d_dt = (DiagTerm<NW>*)sbdgpu::dev_alloc(sizeof(DiagTerm<NW>) * dt.size());
      SBD_CUDA(cudaMemcpyAsync(d_dt, dt.data(), sizeof(DiagTerm<NW>) * dt.size(), cudaMemcpyHostToDevice, st));
    }
    if (!g->hdiag) g->hdiag = (double*)sbdgpu::dev_alloc(sizeof(double) * g->n);
    diag_kernel<NW><<<blocks_for(g->n), kThreads, 0, st>>>(g->states, g->n, d_dt, dt.size(), g->hdiag);
    SBD_CUDA(cudaGetLastError());
    if (!all.empty()) {
      g->terms = sbdgpu::dev_alloc(sizeof(Term<NW>) * all.size());
      SBD_CUDA(cudaMemcpyAsync(g->terms, all.data(), sizeof(Term<NW>) * all.size(), cudaMemcpyHostToDevice, st));
      g->buckets = sbdgpu::dev_alloc(sizeof(Bucket<NW>) * bk.size());
      SBD_CUDA(cudaMemcpyAsync(g->buckets, bk.data(), sizeof(Bucket<NW>) * bk.size(), cudaMemcpyHostToDevice, st));
    }
    if (!self.empty()) {
      g->self_terms = sbdgpu::dev_alloc(sizeof(Term<NW>) * self.size());
      SBD_CUDA(cudaMemcpyAsync(g->self_terms, self.data(), sizeof(Term<NW>) * self.size(), cudaMemcpyHostToDevice,
                               st));
    }
    SBD_CUDA(cudaStreamSynchronize(st));
  } catch (...) {
    cudaFree(d_dt);
    throw;
  }
  cudaFree(d_dt);
  g->n_terms = all.size();
  g->n_buckets = bk.size();
  g->n_self = self.size();
  g->ready = true;
}

template <int NW>
void mult_nw(sbdgpu_genop* g, const double* C, double* W) {
  const unsigned grid = (unsigned)std::min<size_t>((g->n + kMultWarps - 1) / kMultWarps, 148 * 16);
  mult_kernel<NW><<<grid, kThreads, 0, g->base.stream>>>(g->states, g->n, g->hkeys, g->hidx, g->hmask,
                                                        static_cast<const Bucket<NW>*>(g->buckets), g->n_buckets,
                                                        static_cast<const Term<NW>*>(g->terms), g->sign, g->hdiag,
                                                        C, W);
  SBD_CUDA(cudaGetLastError());
}

void mult(sbdgpu_genop* g, const double* C, double* W) {
  if (!g->ready) throw Error{SBDGPU_ERR_STATE, "no operator: call sbdgpu_genop_set_terms first"};
  switch (g->nw) {
    case 1: mult_nw<1>(g, C, W); break;
    case 2: mult_nw<2>(g, C, W); break;
    default: mult_nw<4>(g, C, W); break;
  }
}

void diagonal(sbdgpu_genop* g, double* out) {
  if (!g->ready) throw Error{SBDGPU_ERR_STATE, "no operator: call sbdgpu_genop_set_terms first"};
  cudaStream_t st = g->base.stream;
  switch (g->nw) {
    case 1:
      self_kernel<1><<<blocks_for(g->n), kThreads, 0, st>>>(g->states, g->n, static_cast<const Term<1>*>(g->self_terms),
                                                            g->n_self, g->sign, g->hdiag, out);
      break;
    case 2:
      self_kernel<2><<<blocks_for(g->n), kThreads, 0, st>>>(g->states, g->n, static_cast<const Term<2>*>(g->self_terms),
                                                            g->n_self, g->sign, g->hdiag, out);
      break;
    default:
      self_kernel<4><<<blocks_for(g->n), kThreads, 0, st>>>(g->states, g->n, static_cast<const Term<4>*>(g->self_terms),
                                                            g->n_self, g->sign, g->hdiag, out);
      break;
  }
  SBD_CUDA(cudaGetLastError());
}

struct DevVecs {
  std::vector<double*> p;
  cudaStream_t s;
  ~DevVecs() {
    cudaStreamSynchronize(s);
    for (auto x : p) cudaFree(x);
  }
  double* add(size_t n) {
    p.push_back((double*)sbdgpu::dev_alloc(sizeof(double) * n));
    return p.back();
  }
};

// swap of framework/dm_vector.h:89-101: X <- b Y, Y <- a X
__global__ void swap_kernel(double a, double* __restrict__ X, double b, double* __restrict__ Y, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double c = a * X[i];
    X[i] = b * Y[i];
    Y[i] = c;
  }
}

void lanczos(sbdgpu_genop* g, double* Wh, int max_it, double eps, double* energy, int* n_iter) {
  if (max_it < 1) throw Error{SBDGPU_ERR_ARG, "max_it must be positive"};
  const size_t n = g->n;
  cudaStream_t st = g->base.stream;
  sbdgpu_ctx* c = &g->base;
  DevVecs v{{}, st};
  double* W = v.add(n);
  double* C0 = v.add(n);
  double* C1 = v.add(n);
  SBD_CUDA(cudaMemcpyAsync(W, Wh, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  SBD_CUDA(cudaMemcpyAsync(C0, W, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  SBD_CUDA(cudaMemsetAsync(C1, 0, sizeof(double) * n, st));
  const int lda = max_it;
  std::vector<double> A((size_t)lda * lda, 0.0), U((size_t)lda * lda, 0.0), E(lda, 0.0);
  double e_old = 1.0e8;
  int it_stop = 0, steps = 0;
  const unsigned nblk = std::min<size_t>(blocks_for(n), 148 * 8);
  for (int it = 0; it < max_it; it++) {
    steps++;
    const int ii = it + lda * it, ij = it + lda * (it + 1), ji = it + 1 + lda * it;
    mult(g, C0, C1);
    const double aii = sbdgpu::dot(c, C0, C1, n);
    A[ii] = aii;
    for (int i = 0; i < steps; i++)
      for (int j = 0; j < steps; j++) U[i + lda * j] = A[i + lda * j];
    sbdgpu::jacobi_eig(steps, U.data(), lda, E.data());
    if (std::abs(E[0] - e_old) < eps || it + 1 == max_it) {
      it_stop = it;
      break;
    }
    e_old = E[0];
    sbdgpu::axpy(C1, C0, -aii, n, st);
    const double b = std::sqrt(sbdgpu::dot(c, C1, C1, n));
    sbdgpu::scale(C1, 1.0 / b, n, st);
    A[ij] = A[ji] = b;
    if (std::abs(b) < eps) {
      it_stop = it;
      break;
    }
    swap_kernel<<<nblk, kThreads, 0, st>>>(-b, C0, 1.0, C1, n);
    SBD_CUDA(cudaGetLastError());
  }
  // the Ritz vector from a second pass of the recurrence (lanczos.h:276-302)
  SBD_CUDA(cudaMemcpyAsync(C0, W, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  SBD_CUDA(cudaMemsetAsync(C1, 0, sizeof(double) * n, st));
  sbdgpu::scale(W, U[0], n, st);
  for (int it = 0; it < it_stop; it++) {
    const int ii = it + lda * it;
    mult(g, C0, C1);
    sbdgpu::axpy(C1, C0, -A[ii], n, st);
    const double b = std::sqrt(sbdgpu::dot(c, C1, C1, n));
    sbdgpu::scale(C1, 1.0 / b, n, st);
    sbdgpu::axpy(W, C1, U[it + 1], n, st);
    swap_kernel<<<nblk, kThreads, 0, st>>>(-b, C0, 1.0, C1, n);
    SBD_CUDA(cudaGetLastError());
  }
  SBD_CUDA(cudaMemcpyAsync(Wh, W, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  SBD_CUDA(cudaStreamSynchronize(st));
  if (energy) *energy = E[0];
  if (n_iter) *n_iter = steps;
}

void davidson(sbdgpu_genop* g, const sbdgpu_opts* o, double* Wh, double* energy, double* trace_e, double* trace_tol,
              int max_trace, int* n_steps) {
  const int nb = o->max_nb;
  if (nb < 1 || nb > 32) throw Error{SBDGPU_ERR_ARG, "max_nb must be in [1, 32]"};
  const size_t n = g->n;
  cudaStream_t st = g->base.stream;
  sbdgpu_ctx* c = &g->base;
  DevVecs v{{}, st};
  double* W = v.add(n);
  double* R = v.add(n);
  double* hii = v.add(n);
  std::vector<double*> C(nb), HC(nb);
  for (int k = 0; k < nb; k++) {
    C[k] = v.add(n);
    HC[k] = v.add(n);
  }
  diagonal(g, hii);
  SBD_CUDA(cudaMemcpyAsync(W, Wh, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  const double eps_reg = 1.0e-12;
  std::vector<double> H(nb * nb, 0.0), U(nb * nb, 0.0), E(nb, 0.0);
  int steps = 0;
  bool cont = true;
  for (int it = 0; it < o->max_it && cont; it++) {
    SBD_CUDA(cudaMemcpyAsync(C[0], W, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    for (int ib = 0; ib < nb; ib++) {
      SBD_CUDA(cudaMemsetAsync(HC[ib], 0, sizeof(double) * n, st));
      mult(g, C[ib], HC[ib]);
      for (int jb = 0; jb <= ib; jb++) {
        H[jb + nb * ib] = sbdgpu::dot(c, C[jb], HC[ib], n);
        H[ib + nb * jb] = H[jb + nb * ib];
      }
      for (int jb = 0; jb <= ib; jb++)
        for (int kb = 0; kb <= ib; kb++) U[jb + nb * kb] = H[jb + nb * kb];
      sbdgpu::jacobi_eig(ib + 1, U.data(), nb, E.data());
      sbdgpu::ritz_update(C.data(), HC.data(), U.data(), ib + 1, E[0], W, R, n, st);
      const double nw = std::sqrt(sbdgpu::dot(c, W, W, n));
      sbdgpu::scale(W, 1.0 / nw, n, st);
      const double tol = std::sqrt(sbdgpu::dot(c, R, R, n));
      sbdgpu::scale(R, 1.0 / tol, n, st);
      if (trace_e && steps < max_trace) trace_e[steps] = E[0];
      if (trace_tol && steps < max_trace) trace_tol[steps] = tol;
      steps++;
      if (o->verbose) {
        std::cout << " Davidson iteration " << it << "." << ib << " (tol = " << tol << "):";
        for (int p = 0; p < std::min(ib + 1, 4); p++) std::cout << " " << E[p];
        std::cout << std::endl;
      }
      if (tol < o->eps) {
        cont = false;
        break;
      }
      if (ib < nb - 1) {
        sbdgpu::precondition(R, hii, E[0], eps_reg, C[ib + 1], n, st);
        for (int kb = 0; kb < ib + 1; kb++) {
          const double olap = sbdgpu::dot(c, C[kb], C[ib + 1], n);
          sbdgpu::axpy(C[ib + 1], C[kb], -olap, n, st);
        }
        const double nc = std::sqrt(sbdgpu::dot(c, C[ib + 1], C[ib + 1], n));
        sbdgpu::scale(C[ib + 1], 1.0 / nc, n, st);
      }
    }
  }
  SBD_CUDA(cudaMemsetAsync(R, 0, sizeof(double) * n, st));
  mult(g, W, R);
  const double e = sbdgpu::dot(c, W, R, n);
  SBD_CUDA(cudaMemcpyAsync(Wh, W, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  SBD_CUDA(cudaStreamSynchronize(st));
  if (energy) *energy = e;
  if (n_steps) *n_steps = steps;
}


// ---------------------------------------------------------------- the expanded space
//
// MeasHamSquare and ExpandBasis (expand.h:10-366) look past the basis: every
// configuration an off-diagonal term reaches from a basis state, with weight
// coef * sign * W_i.  Here a count pass and a write pass lay those out (with
// the basis states themselves first), a least-significant-word-first radix
// sort of their indices (CUB) orders them by configuration, and head flags
// mark each distinct configuration.

constexpr int kGenThreads = 256;

// entries of state i: 1 (itself) + its applicable off-diagonal terms (with
// |coef sign W_i| > eps when select)
template <int NW>
__global__ void __launch_bounds__(kGenThreads) gen_count_kernel(const uint64_t* __restrict__ states, size_t n,
                                                               const Term<NW>* __restrict__ terms, size_t n_terms,
                                                               int sign, const double* __restrict__ W, double eps,
                                                               int select, int64_t* __restrict__ counts) {
  const size_t i = (size_t)blockIdx.x * kGenThreads + threadIdx.x;
  if (i >= n) return;
  uint64_t v[NW];
#pragma unroll
  for (int x = 0; x < NW; x++) v[x] = states[i * NW + x];
  const double wi = W[i];
  int64_t cnt = 1;
  for (size_t k = 0; k < n_terms; k++) {
    uint64_t w[NW];
    double s;
    if (!apply_term<NW>(terms[k], v, sign, w, &s)) continue;
    if (!select || fabs(terms[k].coef * s * wi) > eps) cnt++;
  }
  counts[i] = cnt;
}

template <int NW>
__global__ void __launch_bounds__(kGenThreads) gen_write_kernel(const uint64_t* __restrict__ states, size_t n,
                                                               const Term<NW>* __restrict__ terms, size_t n_terms,
                                                               int sign, const double* __restrict__ W,
                                                               const double* __restrict__ hdiag, double eps, int select,
                                                               const int64_t* __restrict__ offs,
                                                               uint64_t* __restrict__ keys, double* __restrict__ vals) {
  const size_t i = (size_t)blockIdx.x * kGenThreads + threadIdx.x;
  if (i >= n) return;
  uint64_t v[NW];
#pragma unroll
  for (int x = 0; x < NW; x++) v[x] = states[i * NW + x];
  const double wi = W[i];
  int64_t o = offs[i];
#pragma unroll
  for (int x = 0; x < NW; x++) keys[(size_t)o * NW + x] = v[x];
  vals[o++] = hdiag[i] * wi;  // the diagonal list's weight (expand.h:43-64)
  for (size_t k = 0; k < n_terms; k++) {
    uint64_t w[NW];
    double s;
    if (!apply_term<NW>(terms[k], v, sign, w, &s)) continue;
    const double val = terms[k].coef * s * wi;
    if (select && !(fabs(val) > eps)) continue;
#pragma unroll
    for (int x = 0; x < NW; x++) keys[(size_t)o * NW + x] = w[x];
    vals[o++] = val;
  }
}

__global__ void gather_word_kernel(const uint64_t* __restrict__ keys, int nw, int word,
                                   const int64_t* __restrict__ idx, uint64_t* __restrict__ out, size_t m) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
    out[i] = keys[(size_t)idx[i] * nw + word];
}

// head[i] = 1 where sorted entry i starts a new configuration
__global__ void head_kernel(const uint64_t* __restrict__ keys, int nw, const int64_t* __restrict__ idx,
                            int64_t* __restrict__ head, size_t m) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    int64_t h = i == 0;
    if (i > 0)
      for (int x = 0; x < nw; x++) h |= keys[(size_t)idx[i] * nw + x] != keys[(size_t)idx[i - 1] * nw + x];
    head[i] = h;
  }
}

// sums[seg[i]] += vals[idx[i]] (seg = inclusive scan of head - 1)
__global__ void seg_sum_kernel(const int64_t* __restrict__ seg, const int64_t* __restrict__ idx,
                               const double* __restrict__ vals, double* __restrict__ sums, size_t m) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
    atomicAdd(&sums[seg[i] - 1], vals[idx[i]]);
}

// out[seg[i]-1] = key of entry i for the heads
__global__ void compact_kernel(const uint64_t* __restrict__ keys, int nw, const int64_t* __restrict__ idx,
                               const int64_t* __restrict__ head, const int64_t* __restrict__ seg,
                               uint64_t* __restrict__ out, size_t m) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
    if (head[i])
      for (int x = 0; x < nw; x++) out[(size_t)(seg[i] - 1) * nw + x] = keys[(size_t)idx[i] * nw + x];
}

}  // namespace


namespace {

// The expanded space of W: sorted entry indices (idx), their configuration
// keys, weights, head flags and segment numbers (inclusive scan of the
// heads), all on the device; returns the number of distinct configurations.
struct Expanded {
  std::vector<void*> bufs;
  cudaStream_t s = nullptr;
  uint64_t* keys = nullptr;
  double* vals = nullptr;
  int64_t* idx = nullptr;
  int64_t* head = nullptr;
  int64_t* seg = nullptr;
  size_t m = 0, distinct = 0;
  void* alloc(size_t bytes) {
    bufs.push_back(sbdgpu::dev_alloc(std::max<size_t>(bytes, 16)));
    return bufs.back();
  }
  ~Expanded() {
    if (s) cudaStreamSynchronize(s);
    for (auto p : bufs) cudaFree(p);
  }
};

template <int NW>
void expand_nw(sbdgpu_genop* g, const double* dW, double eps, int select, Expanded& x) {
  cudaStream_t st = g->base.stream;
  x.s = st;
  const size_t n = g->n;
  const unsigned nblk = (unsigned)((n + kGenThreads - 1) / kGenThreads);
  const Term<NW>* terms = static_cast<const Term<NW>*>(g->terms);
  int64_t* counts = (int64_t*)x.alloc(sizeof(int64_t) * (n + 1));
  int64_t* offs = (int64_t*)x.alloc(sizeof(int64_t) * (n + 1));
  SBD_CUDA(cudaMemsetAsync(counts + n, 0, sizeof(int64_t), st));
  gen_count_kernel<NW><<<nblk, kGenThreads, 0, st>>>(g->states, n, terms, g->n_terms, g->sign, dW, eps, select,
                                                     counts);
  SBD_CUDA(cudaGetLastError());
  size_t tb = 0;
  SBD_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, counts, offs, n + 1, st));
  void* tmp = x.alloc(tb);
  SBD_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, counts, offs, n + 1, st));
  int64_t m = 0;
  SBD_CUDA(cudaMemcpyAsync(&m, offs + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  SBD_CUDA(cudaStreamSynchronize(st));
  x.m = (size_t)m;
  x.keys = (uint64_t*)x.alloc(sizeof(uint64_t) * x.m * NW);
  x.vals = (double*)x.alloc(sizeof(double) * x.m);
  gen_write_kernel<NW><<<nblk, kGenThreads, 0, st>>>(g->states, n, terms, g->n_terms, g->sign, dW, g->hdiag, eps,
                                                     select, offs, x.keys, x.vals);
  SBD_CUDA(cudaGetLastError());
  // sort the entry indices by configuration, least significant word first
  // (each radix pass is stable)
  int64_t* ia = (int64_t*)x.alloc(sizeof(int64_t) * x.m);
  int64_t* ib = (int64_t*)x.alloc(sizeof(int64_t) * x.m);
  uint64_t* ka = (uint64_t*)x.alloc(sizeof(uint64_t) * x.m);
  uint64_t* kb = (uint64_t*)x.alloc(sizeof(uint64_t) * x.m);
  std::vector<int64_t> iota(x.m);
  for (size_t i = 0; i < x.m; i++) iota[i] = (int64_t)i;
  SBD_CUDA(cudaMemcpyAsync(ia, iota.data(), sizeof(int64_t) * x.m, cudaMemcpyHostToDevice, st));
  const unsigned gb = (unsigned)std::min<size_t>((x.m + 255) / 256 + 1, 148 * 8);
  size_t tsort = 0;
  SBD_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tsort, ka, kb, ia, ib, x.m, 0, 64, st));
  void* tmp2 = x.alloc(tsort);
  for (int w = 0; w < NW; w++) {
    gather_word_kernel<<<gb, 256, 0, st>>>(x.keys, NW, w, ia, ka, x.m);
    SBD_CUDA(cudaGetLastError());
    SBD_CUDA(cub::DeviceRadixSort::SortPairs(tmp2, tsort, ka, kb, ia, ib, x.m, 0, 64, st));
    std::swap(ia, ib);
  }
  x.idx = ia;
  x.head = (int64_t*)x.alloc(sizeof(int64_t) * x.m);
  x.seg = (int64_t*)x.alloc(sizeof(int64_t) * x.m);
  head_kernel<<<gb, 256, 0, st>>>(x.keys, NW, x.idx, x.head, x.m);
  SBD_CUDA(cudaGetLastError());
  size_t ts = 0;
  SBD_CUDA(cub::DeviceScan::InclusiveSum(nullptr, ts, x.head, x.seg, x.m, st));
  void* tmp3 = x.alloc(ts);
  SBD_CUDA(cub::DeviceScan::InclusiveSum(tmp3, ts, x.head, x.seg, x.m, st));
  int64_t d = 0;
  SBD_CUDA(cudaMemcpyAsync(&d, x.seg + x.m - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  SBD_CUDA(cudaStreamSynchronize(st));
  x.distinct = (size_t)d;
}

void expand_space(sbdgpu_genop* g, const double* dW, double eps, int select, Expanded& x) {
  if (!g->ready) throw Error{SBDGPU_ERR_STATE, "no operator: call sbdgpu_genop_set_terms first"};
  switch (g->nw) {
    case 1: expand_nw<1>(g, dW, eps, select, x); break;
    case 2: expand_nw<2>(g, dW, eps, select, x); break;
    default: expand_nw<4>(g, dW, eps, select, x); break;
  }
}

}  // namespace

namespace sbdgpu {
void genop_set_error(sbdgpu_genop* g, const std::string& msg) { g->base.err = msg; }
}  // namespace sbdgpu

extern "C" {

int sbdgpu_genop_create(sbdgpu_genop** out, int device, int nwords, size_t nstates, const uint64_t* states,
                        int sign) {
  if (!out) return SBDGPU_ERR_ARG;
  *out = nullptr;
  auto* g = new (std::nothrow) sbdgpu_genop();
  if (!g) return SBDGPU_ERR_ALLOC;
  g->base.device = device;
  int rc = guarded(g, [&] {
    if (nwords != 1 && nwords != 2 && nwords != 4) throw Error{SBDGPU_ERR_ARG, "nwords must be 1, 2 or 4"};
    if (nstates == 0 || !states) throw Error{SBDGPU_ERR_ARG, "empty basis"};
    g->nw = nwords;
    g->n = nstates;
    g->sign = sign ? 1 : 0;
    SBD_CUDA(cudaStreamCreateWithFlags(&g->base.stream, cudaStreamNonBlocking));
    // the hash table: at least twice the states, a power of two
    size_t slots = 1024;
    while (slots < 2 * nstates) slots <<= 1;
    std::vector<uint64_t> hk(slots * nwords, 0);
    std::vector<int64_t> hi(slots, -1);
    const uint64_t hmask = slots - 1;
    for (size_t i = 0; i < nstates; i++) {
      const uint64_t* w = &states[i * nwords];
      uint64_t h = (nwords == 1 ? hash_state<1>(w) : nwords == 2 ? hash_state<2>(w) : hash_state<4>(w)) & hmask;
      while (hi[h] >= 0) {
        if (std::equal(w, w + nwords, &hk[h * nwords])) throw Error{SBDGPU_ERR_ARG, "repeated basis state"};
        h = (h + 1) & hmask;
      }
      hi[h] = (int64_t)i;
      std::memcpy(&hk[h * nwords], w, sizeof(uint64_t) * nwords);
    }
    const size_t bytes = sizeof(uint64_t) * nstates * nwords;
    g->states = (uint64_t*)sbdgpu::dev_alloc(bytes);
    g->hkeys = (uint64_t*)sbdgpu::dev_alloc(sizeof(uint64_t) * hk.size());
    g->hidx = (int64_t*)sbdgpu::dev_alloc(sizeof(int64_t) * slots);
    g->hmask = hmask;
    SBD_CUDA(cudaMemcpyAsync(g->states, states, bytes, cudaMemcpyHostToDevice, g->base.stream));
    SBD_CUDA(cudaMemcpyAsync(g->hkeys, hk.data(), sizeof(uint64_t) * hk.size(), cudaMemcpyHostToDevice,
                             g->base.stream));
    SBD_CUDA(cudaMemcpyAsync(g->hidx, hi.data(), sizeof(int64_t) * slots, cudaMemcpyHostToDevice, g->base.stream));
    SBD_CUDA(cudaStreamSynchronize(g->base.stream));
  });
  if (rc != SBDGPU_OK) {  // a bad argument, or no memory on the device
    sbdgpu_genop_destroy(g);
    return rc;
  }
  *out = g;
  return SBDGPU_OK;
}

int sbdgpu_genop_set_terms(sbdgpu_genop* g, size_t n_diag, const int64_t* diag_off, const int32_t* diag_ops,
                           const int32_t* diag_ndag, const double* diag_coef, size_t n_off, const int64_t* off_off,
                           const int32_t* off_ops, const int32_t* off_ndag, const double* off_coef) {
  return guarded(g, [&] {
    if ((n_diag && (!diag_off || !diag_ndag || !diag_coef)) || (n_off && (!off_off || !off_ndag || !off_coef)))
      throw Error{SBDGPU_ERR_ARG, "null term array"};
    switch (g->nw) {
      case 1:
        set_terms_nw<1>(g, n_diag, diag_off, diag_ops, diag_ndag, diag_coef, n_off, off_off, off_ops, off_ndag,
                        off_coef);
        break;
      case 2:
        set_terms_nw<2>(g, n_diag, diag_off, diag_ops, diag_ndag, diag_coef, n_off, off_off, off_ops, off_ndag,
                        off_coef);
        break;
      default:
        set_terms_nw<4>(g, n_diag, diag_off, diag_ops, diag_ndag, diag_coef, n_off, off_off, off_ops, off_ndag,
                        off_coef);
        break;
    }
  });
}

int sbdgpu_genop_mult_device(sbdgpu_genop* g, const double* dC, double* dW) {
  return guarded(g, [&] {
    if (!dC || !dW) throw Error{SBDGPU_ERR_ARG, "null vector"};
    mult(g, dC, dW);
    SBD_CUDA(cudaStreamSynchronize(g->base.stream));
  });
}

int sbdgpu_genop_mult(sbdgpu_genop* g, const double* C, double* W) {
  return guarded(g, [&] {
    if (!C || !W) throw Error{SBDGPU_ERR_ARG, "null vector"};
    cudaStream_t st = g->base.stream;
    DevVecs v{{}, st};
    double* dC = v.add(g->n);
    double* dW = v.add(g->n);
    SBD_CUDA(cudaMemcpyAsync(dC, C, sizeof(double) * g->n, cudaMemcpyHostToDevice, st));
    SBD_CUDA(cudaMemcpyAsync(dW, W, sizeof(double) * g->n, cudaMemcpyHostToDevice, st));
    mult(g, dC, dW);
    SBD_CUDA(cudaMemcpyAsync(W, dW, sizeof(double) * g->n, cudaMemcpyDeviceToHost, st));
    SBD_CUDA(cudaStreamSynchronize(st));
  });
}

int sbdgpu_genop_diagonal(sbdgpu_genop* g, double* hii) {
  return guarded(g, [&] {
    if (!hii) throw Error{SBDGPU_ERR_ARG, "null vector"};
    cudaStream_t st = g->base.stream;
    DevVecs v{{}, st};
    double* d = v.add(g->n);
    diagonal(g, d);
    SBD_CUDA(cudaMemcpyAsync(hii, d, sizeof(double) * g->n, cudaMemcpyDeviceToHost, st));
    SBD_CUDA(cudaStreamSynchronize(st));
  });
}

int sbdgpu_genop_lanczos(sbdgpu_genop* g, double* W, int max_it, double eps, double* energy, int* n_iter) {
  return guarded(g, [&] {
    if (!W) throw Error{SBDGPU_ERR_ARG, "null vector"};
    if (!g->ready) throw Error{SBDGPU_ERR_STATE, "no operator: call sbdgpu_genop_set_terms first"};
    lanczos(g, W, max_it, eps, energy, n_iter);
  });
}

int sbdgpu_genop_davidson(sbdgpu_genop* g, const sbdgpu_opts* opts, double* W, double* energy, double* trace_e,
                          double* trace_tol, int max_trace, int* n_steps) {
  return guarded(g, [&] {
    if (!opts || !W) throw Error{SBDGPU_ERR_ARG, "null argument"};
    if (!g->ready) throw Error{SBDGPU_ERR_STATE, "no operator: call sbdgpu_genop_set_terms first"};
    davidson(g, opts, W, energy, trace_e, trace_tol, max_trace, n_steps);
  });
}

int sbdgpu_genop_ham_square(sbdgpu_genop* g, const double* W, double* res) {
  return guarded(g, [&] {
    if (!W || !res) throw Error{SBDGPU_ERR_ARG, "null argument"};
    cudaStream_t st = g->base.stream;
    DevVecs v{{}, st};
    double* dW = v.add(g->n);
    SBD_CUDA(cudaMemcpyAsync(dW, W, sizeof(double) * g->n, cudaMemcpyHostToDevice, st));
    Expanded x;
    expand_space(g, dW, 0.0, 0, x);
    double* sums = v.add(x.distinct);
    SBD_CUDA(cudaMemsetAsync(sums, 0, sizeof(double) * x.distinct, st));
    const unsigned gb = (unsigned)std::min<size_t>((x.m + 255) / 256 + 1, 148 * 8);
    seg_sum_kernel<<<gb, 256, 0, st>>>(x.seg, x.idx, x.vals, sums, x.m);
    SBD_CUDA(cudaGetLastError());
    *res = sbdgpu::dot(&g->base, sums, sums, x.distinct);
  });
}

int sbdgpu_genop_expand(sbdgpu_genop* g, const double* W, double eps_hb, uint64_t* out, size_t capacity,
                        size_t* n_out) {
  return guarded(g, [&] {
    if (!W || !n_out) throw Error{SBDGPU_ERR_ARG, "null argument"};
    cudaStream_t st = g->base.stream;
    DevVecs v{{}, st};
    double* dW = v.add(g->n);
    SBD_CUDA(cudaMemcpyAsync(dW, W, sizeof(double) * g->n, cudaMemcpyHostToDevice, st));
    Expanded x;
    expand_space(g, dW, eps_hb, 1, x);
    *n_out = x.distinct;
    if (!out) return;
    if (capacity < x.distinct) throw Error{SBDGPU_ERR_LIMIT, "output holds fewer states than the expanded basis"};
    uint64_t* d = (uint64_t*)x.alloc(sizeof(uint64_t) * x.distinct * g->nw);
    const unsigned gb = (unsigned)std::min<size_t>((x.m + 255) / 256 + 1, 148 * 8);
    compact_kernel<<<gb, 256, 0, st>>>(x.keys, g->nw, x.idx, x.head, x.seg, d, x.m);
    SBD_CUDA(cudaGetLastError());
    SBD_CUDA(cudaMemcpyAsync(out, d, sizeof(uint64_t) * x.distinct * g->nw, cudaMemcpyDeviceToHost, st));
    SBD_CUDA(cudaStreamSynchronize(st));
  });
}

const char* sbdgpu_genop_last_error(sbdgpu_genop* g) { return g ? g->base.err.c_str() : "null object"; }

void sbdgpu_genop_destroy(sbdgpu_genop* g) {
  if (!g) return;
  cudaSetDevice(g->base.device);
  if (g->base.stream) cudaStreamSynchronize(g->base.stream);
  cudaFree(g->states);
  cudaFree(g->hkeys);
  cudaFree(g->hidx);
  cudaFree(g->buckets);
  cudaFree(g->terms);
  cudaFree(g->self_terms);
  cudaFree(g->hdiag);
  cudaFree(g->base.red);
  if (g->base.stream) cudaStreamDestroy(g->base.stream);
  g->base.red = nullptr;
  g->base.stream = nullptr;
  delete g;
}

}  // extern "C"
