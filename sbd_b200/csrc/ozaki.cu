// FP64-accurate same-spin terms of the FP64 sigma on the integer tensor cores.
//
// The string-only same-spin operator H0 (the reference's alpha-only and
// beta-only tasks, chemistry/tpb/mult.h:498-566, without the singles'
// Coulomb part and the diagonal) is ~9 % dense at 12,000 strings and applied
// as a dense product, sigma += H0_a C and sigma += C H0_b^T.  Each product is
// made exactly in integers (an Ozaki-type scheme with the Chinese remainder
// theorem):
//
//   1. the left factor is scaled per row and the right factor per column by
//      powers of two so that every entry rounds to an integer below 2^49;
//   2. both are reduced modulo 15 primes below 256 (symmetric residues, int8);
//   3. 15 INT8 GEMMs with exact INT32 sums (|residue| <= 125, K < 2^16)
//      give the integer product modulo each prime;
//   4. the CRT recovers the integer product (its magnitude is below
//      2^(98+16) < M/2, M = the product of the primes ~ 2^115.7) with 128-bit
//      integer arithmetic, and the power-of-two scales come off.
//
// The result differs from the exact product of the FP64 operands only by the
// rounding of the scaled operands to 49-bit integers: about 2^-49 of the row
// maximum times the column maximum per term.  The products are plain library
// GEMMs (cuBLAS, INT8 in, INT32 out); the scaling, the residues and the
// reconstruction are kernels here.
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>

#include "internal.cuh"

namespace sbdgpu {

namespace {

constexpr int kMods = 15;
constexpr int kBits = 49;
constexpr int kMaxExp = 1000;  // scale exponents lie in [kBits - 1024, kMaxExp]: 2^e is a normal double
constexpr int kT = 256;
constexpr int kNonFinite = 0x40000000;  // row exponent of a row holding a NaN or an infinity

// the primes, as compile-time constants wherever the index is one (the
// compiler then reduces by multiply-high and shift, not by a division)
__host__ __device__ constexpr unsigned prime_at(int l) {
  return l == 0 ? 251u : l == 1 ? 241u : l == 2 ? 239u : l == 3 ? 233u : l == 4 ? 229u : l == 5 ? 227u
       : l == 6 ? 223u : l == 7 ? 211u : l == 8 ? 199u : l == 9 ? 197u : l == 10 ? 193u : l == 11 ? 191u
       : l == 12 ? 181u : l == 13 ? 179u : 173u;
}
__host__ __device__ constexpr unsigned pow2_mod(int k, unsigned m) {
  unsigned r = 1;
  for (int i = 0; i < k; i++) r = (2 * r) % m;
  return r;
}
template <int L>
struct PrimeK {
  static constexpr unsigned m = prime_at(L);
  static constexpr unsigned p25 = pow2_mod(25, m);      // 2^25 mod m
  static constexpr unsigned off49 = m - pow2_mod(49, m);  // -2^49 mod m, in [1, m]
};

__constant__ unsigned c_w[kMods][4];          // CRT weights (< M) in 32-bit limbs, lowest first
__constant__ unsigned long long c_Mlo, c_Mhi;  // M
__constant__ double c_Minv;                    // 1 / M

// 2^k for -1022 <= k <= 1023, from its bit pattern
__device__ __forceinline__ double pow2(int k) { return __longlong_as_double((long long)(k + 1023) << 52); }

// exponent that scales a row (or column) with maximum |x| to below 2^kBits;
// at most kMaxExp, so that 2^e is a normal double (rows below 2^-951 keep
// fewer bits)
__device__ __forceinline__ int scale_exp(double amax) {
  if (!(amax > 0.0)) return 0;
  int ex;
  frexp(amax, &ex);  // amax = f * 2^ex, f in [0.5, 1)
  return min(kBits - ex, kMaxExp);
}

// per-row exponent of a row-major [rows][cols] matrix; kNonFinite for a row
// holding a NaN or an infinity (the product then carries a NaN into every
// entry that row feeds, as the FP64 product would carry it)
__global__ void __launch_bounds__(kT) row_exp_kernel(const double* __restrict__ X, size_t cols, int* __restrict__ e) {
  __shared__ double sh[kT / 32];
  __shared__ int bad_sh[kT / 32];
  const size_t r = blockIdx.x;
  double m = 0.0;
  bool bad = false;
  for (size_t c = threadIdx.x; c < cols; c += kT) {
    const double x = X[r * cols + c];
    bad |= !isfinite(x);
    m = fmax(m, fabs(x));
  }
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  bad = __any_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
    sh[threadIdx.x >> 5] = m;
    bad_sh[threadIdx.x >> 5] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kT / 32; w++) {
      m = fmax(m, sh[w]);
      bad |= bad_sh[w] != 0;
    }
    e[r] = bad ? kNonFinite : scale_exp(fmax(m, sh[0]));
  }
}

// The symmetric residue modulo prime L of y = hu 2^25 + lo - 2^49 (an
// integer of magnitude below 2^49 split so that every step is 32-bit).
template <int L>
__device__ __forceinline__ unsigned sym_residue_byte(unsigned hu, unsigned lo) {
  constexpr unsigned m = PrimeK<L>::m;
  const unsigned t = (hu % m) * PrimeK<L>::p25 + lo % m + PrimeK<L>::off49;  // < 2^17, = y mod m
  const int r = (int)(t % m);
  return (unsigned)(uint8_t)(int8_t)(r > (int)(m / 2) ? r - (int)m : r);
}

template <int L>
__device__ __forceinline__ void store_residues4(const unsigned (&hu)[4], const unsigned (&lo)[4], int8_t* out,
                                                size_t n, size_t at) {
  const unsigned packed = sym_residue_byte<L>(hu[0], lo[0]) | sym_residue_byte<L>(hu[1], lo[1]) << 8 |
                          sym_residue_byte<L>(hu[2], lo[2]) << 16 | sym_residue_byte<L>(hu[3], lo[3]) << 24;
  *reinterpret_cast<unsigned*>(out + (size_t)L * n + at) = packed;
}

template <size_t... L>
__device__ __forceinline__ void store_all_residues(std::index_sequence<L...>, const unsigned (&hu)[4],
                                                   const unsigned (&lo)[4], int8_t* out, size_t n, size_t at) {
  (store_residues4<(int)L>(hu, lo, out, n, at), ...);
}

// symmetric residues modulo the primes of round(X * 2^e_row), int8,
// [kMods][rows*cols]; one block per row, four consecutive entries per thread
// (cols a multiple of 4)
__global__ void __launch_bounds__(kT) residue_kernel(const double* __restrict__ X, size_t rows, size_t cols,
                                                    const int* __restrict__ e, int8_t* __restrict__ out) {
  const size_t n = rows * cols, row = blockIdx.x;
  const int er = e[row];
  const double scale = er == kNonFinite ? 0.0 : pow2(er);  // e <= kMaxExp; >= kBits - 1024
  const double* xr = X + row * cols;
  for (size_t c = 4 * (size_t)threadIdx.x; c < cols; c += 4 * kT) {
    double x[4];
    if (er == kNonFinite) {
      x[0] = x[1] = x[2] = x[3] = 0.0;  // residues 0: the reconstruction writes NaN for this row
    } else {
      const double2 x01 = *reinterpret_cast<const double2*>(xr + c);
      const double2 x23 = *reinterpret_cast<const double2*>(xr + c + 2);
      x[0] = x01.x;
      x[1] = x01.y;
      x[2] = x23.x;
      x[3] = x23.y;
    }
    unsigned hu[4], lo[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const long long y = __double2ll_rn(x[j] * scale);  // |y| < 2^kBits: the scaling is exact
      hu[j] = (unsigned)((y >> 25) + (1LL << 24));     // in [0, 2^25)
      lo[j] = (unsigned)(y & 0x1FFFFFFLL);
    }
    store_all_residues(std::make_index_sequence<kMods>{}, hu, lo, out, n, row * cols + c);
  }
}

template <int L>
__device__ __forceinline__ void crt_term(const int32_t* __restrict__ P, size_t n, size_t i,
                                         unsigned long long (&a)[4]) {
  constexpr int m = (int)PrimeK<L>::m;
  int r = __ldg(&P[(size_t)L * n + i]) % m;
  r += r < 0 ? m : 0;
#pragma unroll
  for (int q = 0; q < 4; q++) a[q] += (unsigned long long)c_w[L][q] * (unsigned)r;  // < 2^44 in all
}

template <size_t... L>
__device__ __forceinline__ void crt_all(std::index_sequence<L...>, const int32_t* __restrict__ P, size_t n, size_t i,
                                        unsigned long long (&a)[4]) {
  (crt_term<(int)L>(P, n, i, a), ...);
}

__device__ __forceinline__ double u128_to_double(unsigned __int128 x) {
  return (double)(unsigned long long)(x >> 64) * 18446744073709551616.0 + (double)(unsigned long long)x;
}

// S[row][col] += (integer product, from its residues) * 2^-(e_row + e_col);
// one block per row
__global__ void __launch_bounds__(kT) crt_add_kernel(const int32_t* __restrict__ P, size_t rows, size_t cols,
                                                    const int* __restrict__ e_row, const int* __restrict__ e_col,
                                                    double* __restrict__ S) {
  const size_t n = rows * cols, row = blockIdx.x;
  const int er = e_row[row];
  const unsigned __int128 M = ((unsigned __int128)c_Mhi << 64) | c_Mlo;
  for (size_t c = threadIdx.x; c < cols; c += kT) {
    const size_t i = row * cols + c;
    unsigned long long a[4] = {0, 0, 0, 0};
    crt_all(std::make_index_sequence<kMods>{}, P, n, i, a);
    // carries: acc = sum_l r_l w_l < kMods * 251 * M < 2^128
    a[1] += a[0] >> 32;
    a[2] += a[1] >> 32;
    a[3] += a[2] >> 32;
    const unsigned __int128 acc = ((unsigned __int128)a[3] << 96) | ((unsigned __int128)(a[2] & 0xFFFFFFFFull) << 64) |
                                  ((unsigned __int128)(a[1] & 0xFFFFFFFFull) << 32) | (a[0] & 0xFFFFFFFFull);
    // acc mod M: the quotient is below 2^12; estimate it in FP64, then correct
    unsigned long long q = (unsigned long long)(u128_to_double(acc) * c_Minv);
    unsigned __int128 qm = M * q;
    while (qm > acc) {
      qm -= M;
      q--;
    }
    unsigned __int128 x = acc - qm;
    while (x >= M) x -= M;
    const double v = x > (M >> 1) ? -u128_to_double(M - x) : u128_to_double(x);  // the symmetric representative
    const int ec = e_col[c];
    if (er == kNonFinite || ec == kNonFinite) {
      S[i] = __longlong_as_double(0x7FF8000000000000LL);  // NaN
      continue;
    }
    const int s = -(er + ec);
    S[i] += (s >= -1022 && s <= 1023) ? v * pow2(s) : ldexp(v, s);
  }
}

// the string-only same-spin operator of one spin, dense FP64 [n][n]
__global__ void __launch_bounds__(kT) dense_h0_kernel(size_t n, const int64_t* __restrict__ s_off,
                                                     const int32_t* __restrict__ s_idx,
                                                     const double* __restrict__ s_val,
                                                     const int64_t* __restrict__ d_off,
                                                     const int32_t* __restrict__ d_idx,
                                                     const double* __restrict__ d_val, double* __restrict__ H) {
  const size_t row = blockIdx.x;
  double* Hr = H + row * n;
  for (size_t j = threadIdx.x; j < n; j += kT) Hr[j] = 0.0;
  __syncthreads();
  for (int64_t k = s_off[row] + threadIdx.x; k < s_off[row + 1]; k += kT) Hr[s_idx[k]] = s_val[k];
  for (int64_t k = d_off[row] + threadIdx.x; k < d_off[row + 1]; k += kT) Hr[d_idx[k]] = d_val[k];
}

// S[row][col] (=) [hii C] + sum over the bra's singles of s J_pq[col] C[ket][col] (FP64);
// two consecutive columns per thread (ncols even)
template <bool kWithDiag>
__global__ void __launch_bounds__(kT) jsingles64_kernel(const double* __restrict__ C, double* __restrict__ S,
                                                       size_t ncols, const double* __restrict__ hii,
                                                       const int64_t* __restrict__ s_off,
                                                       const int32_t* __restrict__ s_idx,
                                                       const uint32_t* __restrict__ s_info,
                                                       const double* __restrict__ J) {
  const size_t row = blockIdx.x;
  const size_t col = 2 * ((size_t)blockIdx.y * kT + threadIdx.x);
  if (col >= ncols) return;
  double2 acc = {0.0, 0.0};
  if (kWithDiag) {
    const double2 h = *reinterpret_cast<const double2*>(hii + row * ncols + col);
    const double2 x = *reinterpret_cast<const double2*>(C + row * ncols + col);
    acc = {h.x * x.x, h.y * x.y};
  }
  const int64_t k1 = s_off[row + 1];
#pragma unroll 4
  for (int64_t k = s_off[row]; k < k1; k++) {
    const size_t j = (size_t)__ldg(&s_idx[k]);
    const uint32_t info = __ldg(&s_info[k]);
    const double2 jv = __ldg(reinterpret_cast<const double2*>(J + (size_t)((info >> 12) & 0xFFFu) * ncols + col));
    const double2 x = __ldg(reinterpret_cast<const double2*>(C + j * ncols + col));
    const double sg = (info & 0x80000000u) ? -1.0 : 1.0;
    acc.x = fma(sg * jv.x, x.x, acc.x);
    acc.y = fma(sg * jv.y, x.y, acc.y);
  }
  *reinterpret_cast<double2*>(S + row * ncols + col) = acc;
}

// the CRT constants in constant memory on the current device
void upload_crt_constants() {
  unsigned __int128 M = 1;
  for (int l = 0; l < kMods; l++) M *= prime_at(l);
  unsigned w32[kMods][4];
  for (int l = 0; l < kMods; l++) {
    const unsigned m = prime_at(l);
    const unsigned __int128 Ml = M / m;
    const unsigned r = (unsigned)(Ml % m);
    unsigned inv = 1;
    while ((unsigned long long)r * inv % m != 1) inv++;  // m < 256
    const unsigned __int128 w = (Ml * inv) % M;  // Ml * inv < M * 256 < 2^124
    for (int q = 0; q < 4; q++) w32[l][q] = (unsigned)(w >> (32 * q));
  }
  const unsigned long long mlo = (unsigned long long)M, mhi = (unsigned long long)(M >> 64);
  const double minv = 1.0 / ((double)mhi * 18446744073709551616.0 + (double)mlo);
  SBD_CUDA(cudaMemcpyToSymbol(c_w, w32, sizeof(w32)));
  SBD_CUDA(cudaMemcpyToSymbol(c_Mlo, &mlo, sizeof(mlo)));
  SBD_CUDA(cudaMemcpyToSymbol(c_Mhi, &mhi, sizeof(mhi)));
  SBD_CUDA(cudaMemcpyToSymbol(c_Minv, &minv, sizeof(minv)));
}

// INT8 GEMM, column-major: out (m x n, int32) = op(A) op(B); false when
// cuBLAS does not offer it
bool gemm_i8(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, const int8_t* A,
             int lda, const int8_t* B, int ldb, int32_t* out, int ldc) {
  const int32_t one = 1, zero = 0;
  return cublasGemmEx(h, ta, tb, m, n, k, &one, A, CUDA_R_8I, lda, B, CUDA_R_8I, ldb, &zero, out, CUDA_R_32I, ldc,
                      CUBLAS_COMPUTE_32I, CUBLAS_GEMM_DEFAULT) == CUBLAS_STATUS_SUCCESS;
}

}  // namespace

// Residues of both spins' operators, their row exponents and the per-sigma
// scratch; false (and the rows kernels stay in use) when they would not fit
// comfortably in device memory.
bool ensure_ozaki(sbdgpu_ctx* c) {
  if (c->oz.ready) return true;
  if (c->oz.failed) return false;
  const size_t na = c->na, nb = c->nb, N = c->N, nmax = std::max(na, nb);
  const size_t bytes = (size_t)kMods * (na * na + nb * nb) + 2 * (size_t)kMods * N + 4 * (size_t)kMods * N +
                       sizeof(double) * nmax * nmax;
  size_t free_b = 0, total_b = 0;
  SBD_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (bytes + (size_t(8) << 30) > free_b) {
    c->oz.failed = true;
    return false;
  }
  build_tables(c);
  ensure_scratch(c);
  upload_crt_constants();
  cudaStream_t st = c->stream;
  double* tmp = (double*)dev_alloc(sizeof(double) * nmax * nmax);
  try {
    for (int spin = 0; spin < 2; spin++) {
      const size_t n = spin == 0 ? na : nb;
      const SpinTables& t = c->tab[spin];
      dense_h0_kernel<<<(unsigned)n, kT, 0, st>>>(n, t.s_off, t.s_idx, t.s_val, t.d_off, t.d_idx, t.d_val, tmp);
      c->oz.h0e[spin] = (int*)dev_alloc(sizeof(int) * n);
      row_exp_kernel<<<(unsigned)n, kT, 0, st>>>(tmp, n, c->oz.h0e[spin]);
      c->oz.h0r[spin] = (int8_t*)dev_alloc((size_t)kMods * n * n);
      residue_kernel<<<(unsigned)n, kT, 0, st>>>(tmp, n, n, c->oz.h0e[spin], c->oz.h0r[spin]);
      SBD_CUDA(cudaGetLastError());
      SBD_CUDA(cudaStreamSynchronize(st));
    }
  } catch (...) {
    cudaFree(tmp);
    free_ozaki(c);
    throw;
  }
  cudaFree(tmp);
  try {
    c->oz.cr = (int8_t*)dev_alloc((size_t)kMods * N);
    c->oz.ctr = (int8_t*)dev_alloc((size_t)kMods * N);
    c->oz.ce = (int*)dev_alloc(sizeof(int) * na);
    c->oz.cte = (int*)dev_alloc(sizeof(int) * nb);
    c->oz.prod = (int32_t*)dev_alloc(sizeof(int32_t) * (size_t)kMods * N);
    if (!c->blas) {
      cublasHandle_t h = nullptr;
      if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) throw Error{SBDGPU_ERR_CUDA, "cublasCreate failed"};
      c->blas = h;
    }
  } catch (...) {
    free_ozaki(c);  // nothing half-built stays behind for a later call to overwrite
    throw;
  }
  cublasSetStream(static_cast<cublasHandle_t>(c->blas), st);
  c->oz.ready = true;
  return true;
}

void free_ozaki(sbdgpu_ctx* c) {
  for (int s = 0; s < 2; s++) {
    cudaFree(c->oz.h0r[s]);
    cudaFree(c->oz.h0e[s]);
    c->oz.h0r[s] = nullptr;
    c->oz.h0e[s] = nullptr;
  }
  cudaFree(c->oz.cr);
  cudaFree(c->oz.ctr);
  cudaFree(c->oz.ce);
  cudaFree(c->oz.cte);
  cudaFree(c->oz.prod);
  c->oz.cr = c->oz.ctr = nullptr;
  c->oz.ce = c->oz.cte = nullptr;
  c->oz.prod = nullptr;
  c->oz.ready = false;
}

// Whether the FP64 sigma takes its same-spin terms from the integer products:
// the context's choice (c->oz.mode: 0 automatic, 1 never), at least 1,024
// strings per spin, leading dimensions the INT8 GEMMs take (multiples of 4)
// and room in device memory.
bool use_ozaki(sbdgpu_ctx* c) {
  if (c->oz.mode == 1 || c->oz.failed || c->na < 1024 || c->nb < 1024 || c->na % 4 || c->nb % 4) return false;
  return ensure_ozaki(c);
}

// sigma (FP64) = hii C + same-spin terms (the alpha-beta term is added
// after); ct, st: FP64 scratch of N each.  Returns false, having written
// nothing, when cuBLAS refuses the INT8 products (the caller then uses the
// rows kernels, and this context stops asking).
bool same_spin_ozaki_fp64(sbdgpu_ctx* c, const double* C, double* S, double* ct, double* st, bool events) {
  cudaStream_t s = c->stream;
  const size_t na = c->na, nb = c->nb, N = c->N;
  const SpinTables& ta = c->tab[0];
  const SpinTables& tb = c->tab[1];
  cublasHandle_t h = static_cast<cublasHandle_t>(c->blas);
  if (((uintptr_t)C | (uintptr_t)S) & 15) return false;  // the kernels move pairs of doubles
  SBD_CUDA(cudaGetLastError());
  if (events) SBD_CUDA(cudaEventRecord(c->ev[0], s));
  // scaled residues of C (rows: for the beta product) and of C^T (for the alpha product)
  transpose(C, ct, na, nb, s);
  row_exp_kernel<<<(unsigned)na, kT, 0, s>>>(C, nb, c->oz.ce);
  row_exp_kernel<<<(unsigned)nb, kT, 0, s>>>(ct, na, c->oz.cte);
  residue_kernel<<<(unsigned)na, kT, 0, s>>>(C, na, nb, c->oz.ce, c->oz.cr);
  residue_kernel<<<(unsigned)nb, kT, 0, s>>>(ct, nb, na, c->oz.cte, c->oz.ctr);
  SBD_CUDA(cudaGetLastError());
  // alpha: sigma^T (nb x na, column-major) = (C^T)(H0a^T), one INT8 product per prime
  for (int l = 0; l < kMods; l++)
    if (!gemm_i8(h, CUBLAS_OP_T, CUBLAS_OP_N, (int)nb, (int)na, (int)na, c->oz.ctr + (size_t)l * N, (int)na,
                 c->oz.h0r[0] + (size_t)l * na * na, (int)na, c->oz.prod + (size_t)l * N, (int)nb)) {
      c->oz.failed = true;
      return false;
    }
  jsingles64_kernel<true><<<dim3((unsigned)na, (unsigned)((nb + 2 * kT - 1) / (2 * kT))), kT, 0, s>>>(
      C, S, nb, c->hii, ta.s_off, ta.s_idx, ta.s_info, c->jb);
  crt_add_kernel<<<(unsigned)na, kT, 0, s>>>(c->oz.prod, na, nb, c->oz.h0e[0], c->oz.cte, S);
  SBD_CUDA(cudaGetLastError());
  if (events) SBD_CUDA(cudaEventRecord(c->ev[1], s));
  // beta: sigma^T = H0b (C^T), with H0b's rows and C's rows scaled
  for (int l = 0; l < kMods; l++)
    if (!gemm_i8(h, CUBLAS_OP_T, CUBLAS_OP_N, (int)nb, (int)na, (int)nb, c->oz.h0r[1] + (size_t)l * nb * nb, (int)nb,
                 c->oz.cr + (size_t)l * N, (int)nb, c->oz.prod + (size_t)l * N, (int)nb))
      throw Error{SBDGPU_ERR_CUDA, "INT8 product refused after the alpha products ran"};
  crt_add_kernel<<<(unsigned)na, kT, 0, s>>>(c->oz.prod, na, nb, c->oz.ce, c->oz.h0e[1], S);
  jsingles64_kernel<false><<<dim3((unsigned)nb, (unsigned)((na + 2 * kT - 1) / (2 * kT))), kT, 0, s>>>(
      ct, st, na, nullptr, tb.s_off, tb.s_idx, tb.s_info, c->ja);
  SBD_CUDA(cudaGetLastError());
  transpose_add(st, S, nb, na, s);
  if (events) SBD_CUDA(cudaEventRecord(c->ev[2], s));
  return true;
}

}  // namespace sbdgpu
