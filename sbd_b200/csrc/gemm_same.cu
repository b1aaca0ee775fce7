// Same-spin terms of the mixed-precision (FP32) sigma as dense tensor-core
// GEMMs.
//
// The reference's alpha-only and beta-only tasks (chemistry/tpb/mult.h:498-566)
// add, for every in-set single or double excitation of one spin,
//
//   sigma[ia,ib] += (v(ia,ja) + s J_pq[ib]) C[ja,ib]      (alpha; beta alike)
//
// where v is the string-only element (h_pq plus the same-spin Coulomb and
// exchange sums for a single, the two-electron element for a double) and
// J_pq[ib] = sum_{r in ib} (pq|rr) couples an alpha single to the beta
// occupation.  With 12,000 strings each string has ~1,100 in-set excitations
// of one spin, so the string-only operator H0 is ~9 % dense.  Applied as a
// dense product it runs on the tensor cores: sigma += H0_a C and
// sigma += C H0_b^T, each as three FP16 products of split operands (x = x_hi
// + x_lo, both FP16 after a power-of-two scaling, hi*hi + hi*lo + lo*hi, FP32
// accumulation), which keeps ~22 bits of every operand: FP32-class sums.  The
// products are plain library GEMMs (cuBLAS).  What depends on both strings,
// the diagonal and the J part of the singles (66 of the ~1,100 entries per
// row), is added by a rows kernel walking the singles only; the beta J part
// runs on the transposed vector as in the FP32 rows path.
#include <cublas_v2.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "internal.cuh"

namespace sbdgpu {

namespace {

constexpr int kJThreads = 256;

#define SBD_BLAS(x)                                                                                       \
  do {                                                                                                    \
    cublasStatus_t s_ = (x);                                                                              \
    if (s_ != CUBLAS_STATUS_SUCCESS)                                                                      \
      throw ::sbdgpu::Error{SBDGPU_ERR_CUDA, std::string(#x) + ": cuBLAS status " + std::to_string((int)s_)}; \
  } while (0)

// Dense string-only operator of one spin, row-major [n][n], FP32.
__global__ void dense_same_kernel(size_t n, const int64_t* __restrict__ s_off, const int32_t* __restrict__ s_idx,
                                  const double* __restrict__ s_val, const int64_t* __restrict__ d_off,
                                  const int32_t* __restrict__ d_idx, const double* __restrict__ d_val,
                                  float* __restrict__ H) {
  const size_t row = blockIdx.x;
  float* Hr = H + row * n;
  for (size_t j = threadIdx.x; j < n; j += blockDim.x) Hr[j] = 0.f;
  __syncthreads();
  for (int64_t k = s_off[row] + threadIdx.x; k < s_off[row + 1]; k += blockDim.x) Hr[s_idx[k]] = (float)s_val[k];
  for (int64_t k = d_off[row] + threadIdx.x; k < d_off[row + 1]; k += blockDim.x) Hr[d_idx[k]] = (float)d_val[k];
}

// x * scale split into FP16 hi + lo (hi = fp16(x*scale), lo = fp16(x*scale - hi))
__global__ void split_fp16_kernel(const float* __restrict__ x, size_t n, float scale, __half* __restrict__ hi,
                                  __half* __restrict__ lo) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float v = x[i] * scale;
    const __half h = __float2half_rn(v);
    hi[i] = h;
    lo[i] = __float2half_rn(v - __half2float(h));
  }
}

__global__ void absmax_kernel(const float* __restrict__ x, size_t n, unsigned int* __restrict__ out) {
  float m = 0.f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(x[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));  // non-negative floats order as integers
}

// S[row][col] (=) [hii * C] + sum over the bra's singles of s J_pq[col] C[ket][col];
// V consecutive columns per thread (V = 4: ncols a multiple of 4 and the
// arrays 16-byte aligned)
template <bool kWithDiag, int V>
__global__ void __launch_bounds__(kJThreads) jsingles_kernel(const float* __restrict__ C, float* __restrict__ S,
                                                             size_t ncols, const double* __restrict__ hii,
                                                             const int64_t* __restrict__ s_off,
                                                             const int32_t* __restrict__ s_idx,
                                                             const uint32_t* __restrict__ s_info,
                                                             const float* __restrict__ J) {
  using Vec = typename std::conditional<V == 4, float4, float>::type;
  const size_t row = blockIdx.x;
  const size_t col = V * ((size_t)blockIdx.y * kJThreads + threadIdx.x);
  if (col >= ncols) return;
  float acc[V];
#pragma unroll
  for (int v = 0; v < V; v++) acc[v] = 0.f;
  if (kWithDiag) {
#pragma unroll
    for (int v = 0; v < V; v++) acc[v] = (float)hii[row * ncols + col + v] * C[row * ncols + col + v];
  }
  const int64_t k1 = s_off[row + 1];
#pragma unroll 4
  for (int64_t k = s_off[row]; k < k1; k++) {
    const size_t j = (size_t)__ldg(&s_idx[k]);
    const uint32_t info = __ldg(&s_info[k]);
    const Vec jv = __ldg(reinterpret_cast<const Vec*>(J + (size_t)((info >> 12) & 0xFFFu) * ncols + col));
    const Vec x = __ldg(reinterpret_cast<const Vec*>(C + j * ncols + col));
    const float sg = (info & 0x80000000u) ? -1.f : 1.f;
    const float* jp = reinterpret_cast<const float*>(&jv);
    const float* xp = reinterpret_cast<const float*>(&x);
#pragma unroll
    for (int v = 0; v < V; v++) acc[v] = fmaf(sg * jp[v], xp[v], acc[v]);
  }
  if constexpr (V == 4) {
    *reinterpret_cast<float4*>(S + row * ncols + col) = make_float4(acc[0], acc[1], acc[2], acc[3]);
  } else {
    S[row * ncols + col] = acc[0];
  }
}

// one jsingles pass over rows x ncols, four columns per thread where the
// shapes and pointers allow
template <bool kWithDiag>
void launch_jsingles(const float* C, float* S, size_t rows, size_t ncols, const double* hii, const SpinTables& t,
                     const float* J, cudaStream_t s) {
  const bool vec4 = ncols % 4 == 0 && (((uintptr_t)C | (uintptr_t)S | (uintptr_t)J) & 15) == 0;
  if (vec4) {
    const unsigned gy = (unsigned)((ncols / 4 + kJThreads - 1) / kJThreads);
    jsingles_kernel<kWithDiag, 4><<<dim3((unsigned)rows, gy), kJThreads, 0, s>>>(C, S, ncols, hii, t.s_off, t.s_idx,
                                                                                 t.s_info, J);
  } else {
    const unsigned gy = (unsigned)((ncols + kJThreads - 1) / kJThreads);
    jsingles_kernel<kWithDiag, 1><<<dim3((unsigned)rows, gy), kJThreads, 0, s>>>(C, S, ncols, hii, t.s_off, t.s_idx,
                                                                                 t.s_info, J);
  }
  SBD_CUDA(cudaGetLastError());
}

constexpr float kHScale = 256.f;  // the string-only elements are O(1): 2^8 keeps their lo parts normal in FP16

}  // namespace

// Dense operators, the cuBLAS handle and the split-vector scratch (once per
// context); false when they would not fit comfortably in device memory.
bool ensure_dense_same(sbdgpu_ctx* c) {
  if (c->h0[0][0]) return true;
  const size_t bytes = 2 * sizeof(__half) * (c->na * c->na + c->nb * c->nb) + 2 * sizeof(__half) * c->N +
                       sizeof(float) * std::max(c->na, c->nb) * std::max(c->na, c->nb);
  size_t free_b = 0, total_b = 0;
  SBD_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (bytes + (size_t(4) << 30) > free_b) return false;
  build_tables(c);
  float* tmp = (float*)dev_alloc(sizeof(float) * std::max(c->na, c->nb) * std::max(c->na, c->nb));
  try {
    for (int spin = 0; spin < 2; spin++) {
      const size_t n = spin == 0 ? c->na : c->nb;
      const SpinTables& t = c->tab[spin];
      dense_same_kernel<<<(unsigned)n, 256, 0, c->stream>>>(n, t.s_off, t.s_idx, t.s_val, t.d_off, t.d_idx, t.d_val,
                                                             tmp);
      SBD_CUDA(cudaGetLastError());
      for (int part = 0; part < 2; part++) c->h0[spin][part] = dev_alloc(sizeof(__half) * n * n);
      split_fp16_kernel<<<592, 256, 0, c->stream>>>(tmp, n * n, kHScale, static_cast<__half*>(c->h0[spin][0]),
                                                    static_cast<__half*>(c->h0[spin][1]));
      SBD_CUDA(cudaGetLastError());
      SBD_CUDA(cudaStreamSynchronize(c->stream));
    }
  } catch (...) {
    cudaFree(tmp);
    throw;
  }
  cudaFree(tmp);
  for (int part = 0; part < 2; part++) c->c16[part] = dev_alloc(sizeof(__half) * c->N);
  if (!c->blas) {  // the INT8 same-spin products may have made the context's handle already
    cublasHandle_t h = nullptr;
    SBD_BLAS(cublasCreate(&h));
    c->blas = h;
  }
  SBD_BLAS(cublasSetStream(static_cast<cublasHandle_t>(c->blas), c->stream));
  return true;
}

void free_dense_same(sbdgpu_ctx* c) {
  for (int s = 0; s < 2; s++)
    for (int p = 0; p < 2; p++) {
      cudaFree(c->h0[s][p]);
      c->h0[s][p] = nullptr;
    }
  for (int p = 0; p < 2; p++) {
    cudaFree(c->c16[p]);
    c->c16[p] = nullptr;
  }
  if (c->blas) cublasDestroy(static_cast<cublasHandle_t>(c->blas));
  c->blas = nullptr;
}

// Whether the mixed-precision sigma takes its same-spin terms from the dense
// products: bases of at least 1,024 strings per spin (smaller ones are
// launch-bound either way) whose operators fit in device memory.
bool use_dense_same(sbdgpu_ctx* c) {
  if (c->dense_same_off || c->na < 1024 || c->nb < 1024) return false;
  return ensure_dense_same(c);
}

// sigma (FP32) = hii C + same-spin terms; the alpha-beta term is added after.
// ct, st: FP32 scratch of N each.
void same_spin_dense_fp32(sbdgpu_ctx* c, const float* C, float* S, float* ct, float* st, bool events) {
  cudaStream_t s = c->stream;
  const SpinTables& ta = c->tab[0];
  const SpinTables& tb = c->tab[1];
  const size_t na = c->na, nb = c->nb;
  if (events) SBD_CUDA(cudaEventRecord(c->ev[0], s));
  // diagonal and the alpha singles' J part
  launch_jsingles<true>(C, S, na, nb, c->hii, ta, c->jb32, s);
  // C split into FP16 hi + lo, scaled by a power of two that puts max|C| near 2^14
  unsigned int* amax = reinterpret_cast<unsigned int*>(c->red);
  SBD_CUDA(cudaMemsetAsync(amax, 0, sizeof(unsigned int), s));
  absmax_kernel<<<592, 256, 0, s>>>(C, c->N, amax);
  SBD_CUDA(cudaGetLastError());
  unsigned int bits = 0;
  SBD_CUDA(cudaMemcpyAsync(&bits, amax, sizeof(bits), cudaMemcpyDeviceToHost, s));
  SBD_CUDA(cudaStreamSynchronize(s));
  float cmax = 0.f;
  std::memcpy(&cmax, &bits, sizeof(float));
  // a NaN or an infinity in C keeps the scale at 1 and reaches sigma through the products
  const float cscale =
      cmax > 0.f && std::isfinite(cmax) ? std::ldexp(1.0f, 14 - (int)std::ceil(std::log2(cmax))) : 1.0f;
  __half* chi = static_cast<__half*>(c->c16[0]);
  __half* clo = static_cast<__half*>(c->c16[1]);
  split_fp16_kernel<<<592, 256, 0, s>>>(C, c->N, cscale, chi, clo);
  SBD_CUDA(cudaGetLastError());
  cublasHandle_t h = static_cast<cublasHandle_t>(c->blas);
  const float alpha = 1.0f / (kHScale * cscale), one = 1.0f;
  const __half* ha[2] = {static_cast<const __half*>(c->h0[0][0]), static_cast<const __half*>(c->h0[0][1])};
  const __half* hb[2] = {static_cast<const __half*>(c->h0[1][0]), static_cast<const __half*>(c->h0[1][1])};
  // column-major view: S^T (nb x na) += C^T (nb x na) * H0a^T, the three split products
  const __half* xa[3] = {chi, clo, chi};
  const __half* ya[3] = {ha[0], ha[0], ha[1]};
  for (int k = 0; k < 3; k++)
    SBD_BLAS(cublasGemmEx(h, CUBLAS_OP_N, CUBLAS_OP_N, (int)nb, (int)na, (int)na, &alpha, xa[k], CUDA_R_16F, (int)nb,
                          ya[k], CUDA_R_16F, (int)na, &one, S, CUDA_R_32F, (int)nb, CUBLAS_COMPUTE_32F,
                          CUBLAS_GEMM_DEFAULT));
  if (events) SBD_CUDA(cudaEventRecord(c->ev[1], s));
  // beta: S^T (nb x na) += H0b (nb x nb) * C^T, then the beta singles' J part on C^T
  const __half* xb[3] = {hb[0], hb[0], hb[1]};
  const __half* yb[3] = {chi, clo, chi};
  for (int k = 0; k < 3; k++)
    SBD_BLAS(cublasGemmEx(h, CUBLAS_OP_T, CUBLAS_OP_N, (int)nb, (int)na, (int)nb, &alpha, xb[k], CUDA_R_16F, (int)nb,
                          yb[k], CUDA_R_16F, (int)nb, &one, S, CUDA_R_32F, (int)nb, CUBLAS_COMPUTE_32F,
                          CUBLAS_GEMM_DEFAULT));
  transpose(C, ct, na, nb, s);
  launch_jsingles<false>(ct, st, nb, na, nullptr, tb, c->ja32, s);
  transpose_add(st, S, nb, na, s);
  if (events) SBD_CUDA(cudaEventRecord(c->ev[2], s));
}

}  // namespace sbdgpu
