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

#include "internal.cuh"

namespace sbdgpu {

namespace {

constexpr int kMods = 15;
constexpr int kBits = 49;
constexpr int kT = 256;
const int kPrimes[kMods] = {251, 241, 239, 233, 229, 227, 223, 211, 199, 197, 193, 191, 181, 179, 173};

__constant__ int c_mod[kMods];
__constant__ unsigned long long c_wlo[kMods], c_whi[kMods];  // CRT weights, < M
__constant__ unsigned long long c_Mlo, c_Mhi;                 // M
__constant__ double c_Mdbl;

// exponent that scales a row (or column) with maximum |x| to below 2^kBits
__device__ __forceinline__ int scale_exp(double amax) {
  if (!(amax > 0.0)) return 0;
  int ex;
  frexp(amax, &ex);  // amax = f * 2^ex, f in [0.5, 1)
  return kBits - ex;
}

// per-row exponent of a row-major [rows][cols] matrix
__global__ void __launch_bounds__(kT) row_exp_kernel(const double* __restrict__ X, size_t cols, int* __restrict__ e) {
  __shared__ double sh[kT / 32];
  const size_t r = blockIdx.x;
  double m = 0.0;
  for (size_t c = threadIdx.x; c < cols; c += kT) m = fmax(m, fabs(X[r * cols + c]));
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kT / 32; w++) m = fmax(m, sh[w]);
    e[r] = scale_exp(fmax(m, sh[0]));
  }
}

// symmetric residues modulo the primes of round(X * 2^e_row), int8, [kMods][rows*cols]
__global__ void __launch_bounds__(kT) residue_kernel(const double* __restrict__ X, size_t rows, size_t cols,
                                                    const int* __restrict__ e, int8_t* __restrict__ out) {
  const size_t n = rows * cols;
  for (size_t i = (size_t)blockIdx.x * kT + threadIdx.x; i < n; i += (size_t)gridDim.x * kT) {
    const double y = rint(ldexp(X[i], e[i / cols]));  // an integer, |y| < 2^kBits: exact in FP64
#pragma unroll
    for (int l = 0; l < kMods; l++) {
      const double m = (double)c_mod[l];
      double r = y - m * floor(y / m);  // m * floor(...) < 2^kBits: exact
      if (r < 0.0) r += m;
      if (r >= m) r -= m;
      int ri = (int)r;
      if (ri > c_mod[l] / 2) ri -= c_mod[l];
      out[(size_t)l * n + i] = (int8_t)ri;
    }
  }
}

// S[i] += (integer product, from its residues) * 2^-(e_row + e_col)
__global__ void __launch_bounds__(kT) crt_add_kernel(const int32_t* __restrict__ P, size_t rows, size_t cols,
                                                    const int* __restrict__ e_row, const int* __restrict__ e_col,
                                                    double* __restrict__ S) {
  const size_t n = rows * cols;
  for (size_t i = (size_t)blockIdx.x * kT + threadIdx.x; i < n; i += (size_t)gridDim.x * kT) {
    unsigned __int128 acc = 0;
#pragma unroll
    for (int l = 0; l < kMods; l++) {
      int r = P[(size_t)l * n + i] % c_mod[l];
      if (r < 0) r += c_mod[l];
      const unsigned __int128 w = ((unsigned __int128)c_whi[l] << 64) | c_wlo[l];
      acc += w * (unsigned)r;  // < kMods * 251 * M < 2^128
    }
    const unsigned __int128 M = ((unsigned __int128)c_Mhi << 64) | c_Mlo;
    // acc mod M: the quotient is below 2^12; estimate it in FP64, then correct
    const double accd = (double)(unsigned long long)(acc >> 64) * 18446744073709551616.0 +
                        (double)(unsigned long long)acc;
    unsigned long long q = (unsigned long long)(accd / c_Mdbl);
    unsigned __int128 qm = M * q;
    while (qm > acc) {
      qm -= M;
      q--;
    }
    unsigned __int128 x = acc - qm;
    while (x >= M) x -= M;
    double v;
    if (x > (M >> 1)) {  // negative: x - M
      const unsigned __int128 y = M - x;
      v = -((double)(unsigned long long)(y >> 64) * 18446744073709551616.0 + (double)(unsigned long long)y);
    } else {
      v = (double)(unsigned long long)(x >> 64) * 18446744073709551616.0 + (double)(unsigned long long)x;
    }
    S[i] += ldexp(v, -(e_row[i / cols] + e_col[i % cols]));
  }
}

unsigned grid_of(size_t n) { return (unsigned)std::min<size_t>((n + kT - 1) / kT, 148 * 8); }

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

// S[row][col] (=) [hii C] + sum over the bra's singles of s J_pq[col] C[ket][col] (FP64)
template <bool kWithDiag>
__global__ void __launch_bounds__(kT) jsingles64_kernel(const double* __restrict__ C, double* __restrict__ S,
                                                       size_t ncols, const double* __restrict__ hii,
                                                       const int64_t* __restrict__ s_off,
                                                       const int32_t* __restrict__ s_idx,
                                                       const uint32_t* __restrict__ s_info,
                                                       const double* __restrict__ J) {
  const size_t row = blockIdx.x;
  const size_t col = (size_t)blockIdx.y * kT + threadIdx.x;
  if (col >= ncols) return;
  double acc = kWithDiag ? hii[row * ncols + col] * C[row * ncols + col] : 0.0;
  for (int64_t k = s_off[row]; k < s_off[row + 1]; k++) {
    const size_t j = (size_t)__ldg(&s_idx[k]);
    const uint32_t info = __ldg(&s_info[k]);
    const double jv = __ldg(&J[(size_t)((info >> 12) & 0xFFFu) * ncols + col]);
    acc += ((info & 0x80000000u) ? -jv : jv) * __ldg(&C[j * ncols + col]);
  }
  S[row * ncols + col] = acc;
}

// the CRT constants in constant memory on the current device
void upload_crt_constants() {
  unsigned __int128 M = 1;
  for (int l = 0; l < kMods; l++) M *= (unsigned)kPrimes[l];
  unsigned long long wlo[kMods], whi[kMods];
  for (int l = 0; l < kMods; l++) {
    const unsigned m = (unsigned)kPrimes[l];
    const unsigned __int128 Ml = M / m;
    const unsigned r = (unsigned)(Ml % m);
    unsigned inv = 1;
    while ((unsigned long long)r * inv % m != 1) inv++;  // m < 256
    const unsigned __int128 w = (Ml * inv) % M;  // Ml * inv < M * 256 < 2^124
    wlo[l] = (unsigned long long)w;
    whi[l] = (unsigned long long)(w >> 64);
  }
  const unsigned long long mlo = (unsigned long long)M, mhi = (unsigned long long)(M >> 64);
  const double md = (double)mhi * 18446744073709551616.0 + (double)mlo;
  SBD_CUDA(cudaMemcpyToSymbol(c_mod, kPrimes, sizeof(kPrimes)));
  SBD_CUDA(cudaMemcpyToSymbol(c_wlo, wlo, sizeof(wlo)));
  SBD_CUDA(cudaMemcpyToSymbol(c_whi, whi, sizeof(whi)));
  SBD_CUDA(cudaMemcpyToSymbol(c_Mlo, &mlo, sizeof(mlo)));
  SBD_CUDA(cudaMemcpyToSymbol(c_Mhi, &mhi, sizeof(mhi)));
  SBD_CUDA(cudaMemcpyToSymbol(c_Mdbl, &md, sizeof(md)));
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
      residue_kernel<<<grid_of(n * n), kT, 0, st>>>(tmp, n, n, c->oz.h0e[spin], c->oz.h0r[spin]);
      SBD_CUDA(cudaGetLastError());
      SBD_CUDA(cudaStreamSynchronize(st));
    }
  } catch (...) {
    cudaFree(tmp);
    throw;
  }
  cudaFree(tmp);
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
  SBD_CUDA(cudaGetLastError());
  if (events) SBD_CUDA(cudaEventRecord(c->ev[0], s));
  // scaled residues of C (rows: for the beta product) and of C^T (for the alpha product)
  transpose(C, ct, na, nb, s);
  row_exp_kernel<<<(unsigned)na, kT, 0, s>>>(C, nb, c->oz.ce);
  row_exp_kernel<<<(unsigned)nb, kT, 0, s>>>(ct, na, c->oz.cte);
  residue_kernel<<<grid_of(N), kT, 0, s>>>(C, na, nb, c->oz.ce, c->oz.cr);
  residue_kernel<<<grid_of(N), kT, 0, s>>>(ct, nb, na, c->oz.cte, c->oz.ctr);
  SBD_CUDA(cudaGetLastError());
  // alpha: sigma^T (nb x na, column-major) = (C^T)(H0a^T), one INT8 product per prime
  for (int l = 0; l < kMods; l++)
    if (!gemm_i8(h, CUBLAS_OP_T, CUBLAS_OP_N, (int)nb, (int)na, (int)na, c->oz.ctr + (size_t)l * N, (int)na,
                 c->oz.h0r[0] + (size_t)l * na * na, (int)na, c->oz.prod + (size_t)l * N, (int)nb)) {
      c->oz.failed = true;
      return false;
    }
  jsingles64_kernel<true><<<dim3((unsigned)na, (unsigned)((nb + kT - 1) / kT)), kT, 0, s>>>(
      C, S, nb, c->hii, ta.s_off, ta.s_idx, ta.s_info, c->jb);
  crt_add_kernel<<<grid_of(N), kT, 0, s>>>(c->oz.prod, na, nb, c->oz.h0e[0], c->oz.cte, S);
  SBD_CUDA(cudaGetLastError());
  if (events) SBD_CUDA(cudaEventRecord(c->ev[1], s));
  // beta: sigma^T = H0b (C^T), with H0b's rows and C's rows scaled
  for (int l = 0; l < kMods; l++)
    if (!gemm_i8(h, CUBLAS_OP_T, CUBLAS_OP_N, (int)nb, (int)na, (int)nb, c->oz.h0r[1] + (size_t)l * nb * nb, (int)nb,
                 c->oz.cr + (size_t)l * N, (int)nb, c->oz.prod + (size_t)l * N, (int)nb))
      throw Error{SBDGPU_ERR_CUDA, "INT8 product refused after the alpha products ran"};
  crt_add_kernel<<<grid_of(N), kT, 0, s>>>(c->oz.prod, na, nb, c->oz.ce, c->oz.h0e[1], S);
  jsingles64_kernel<false><<<dim3((unsigned)nb, (unsigned)((na + kT - 1) / kT)), kT, 0, s>>>(
      ct, st, na, nullptr, tb.s_off, tb.s_idx, tb.s_info, c->ja);
  SBD_CUDA(cudaGetLastError());
  transpose_add(st, S, nb, na, s);
  if (events) SBD_CUDA(cudaEventRecord(c->ev[2], s));
  return true;
}

}  // namespace sbdgpu
