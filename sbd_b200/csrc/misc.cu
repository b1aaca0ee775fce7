// Diagonal, sign phase, transposes, Davidson vector kernels, occupations and
// RDMs.  All HBM-bound; the vector kernels are grid-stride loops sized to the
// 148 SMs.
#include <cmath>
#include <cstring>

#include "internal.cuh"

namespace sbdgpu {

namespace {

constexpr int kRedBlocks = 592;  // 4 x 148 SMs
constexpr int kRedThreads = 256;

__device__ __forceinline__ int pair_index(int p, int q) {
  int a = p > q ? p : q, b = p > q ? q : p;
  return a * (a + 1) / 2 + b;
}

__global__ void jtable_kernel(const uint64_t* __restrict__ s, int n, const double* __restrict__ vf, int P,
                              double* __restrict__ J) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int pq = blockIdx.y;
  if (i >= n) return;
  uint64_t occ = s[i];
  double acc = 0.0;
  while (occ) {
    int r = __ffsll((long long)occ) - 1;
    occ &= occ - 1;
    acc += vf[(size_t)pq * P + pair_index(r, r)];
  }
  J[(size_t)pq * n + i] = acc;
}

// One-spin part of ZeroExcite (chemistry/basic/determinants.h:374-398).
__global__ void spin_energy_kernel(const uint64_t* __restrict__ s, int n, int L, const double* __restrict__ h1,
                                   const double* __restrict__ vf, int P, double* __restrict__ E) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t occ = s[i];
  double e = 0.0;
  for (uint64_t o1 = occ; o1; o1 &= o1 - 1) {
    int p = __ffsll((long long)o1) - 1;
    e += h1[p * L + p];
    for (uint64_t o2 = o1 & (o1 - 1); o2; o2 &= o2 - 1) {
      int q = __ffsll((long long)o2) - 1;
      e += vf[(size_t)pair_index(p, p) * P + pair_index(q, q)] - vf[(size_t)pair_index(p, q) * P + pair_index(p, q)];
    }
  }
  E[i] = e;
}

// H_ii = E_core + E_alpha(ia) + E_beta(ib) + sum_{p in a, r in b} (pp|rr)
__global__ void hii_kernel(const uint64_t* __restrict__ astr, size_t na, size_t nb, const double* __restrict__ Ea,
                           const double* __restrict__ Eb, const double* __restrict__ jb, int P, double ecore,
                           double* __restrict__ hii) {
  size_t ia = blockIdx.x;
  size_t ib = (size_t)blockIdx.y * blockDim.x + threadIdx.x;
  if (ib >= nb) return;
  uint64_t occ = astr[ia];
  double cross = 0.0;
  while (occ) {
    int p = __ffsll((long long)occ) - 1;
    occ &= occ - 1;
    cross += jb[(size_t)pair_index(p, p) * nb + ib];
  }
  hii[ia * nb + ib] = ecore + Ea[ia] + Eb[ib] + cross;
}

__global__ void phase_kernel(const uint64_t* __restrict__ astr, const uint64_t* __restrict__ bstr, size_t nb,
                             double* __restrict__ v) {
  size_t ia = blockIdx.x;
  size_t ib = (size_t)blockIdx.y * blockDim.x + threadIdx.x;
  if (ib >= nb) return;
  uint64_t a = astr[ia], b = bstr[ib];
  int cnt = 0;
  while (a) {
    int p = __ffsll((long long)a) - 1;
    a &= a - 1;
    cnt += __popcll(b & ((1ull << p) - 1ull));
  }
  if (cnt & 1) v[ia * nb + ib] = -v[ia * nb + ib];
}

template <typename T, bool kAdd>
__global__ void transpose_kernel(const T* __restrict__ in, T* __restrict__ out, size_t rows, size_t cols) {
  __shared__ T tile[32][33];
  size_t c0 = (size_t)blockIdx.x * 32, r0 = (size_t)blockIdx.y * 32;
  int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int k = ty; k < 32; k += 8) {
    size_t r = r0 + k, c = c0 + tx;
    if (r < rows && c < cols) tile[k][tx] = in[r * cols + c];
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {
    size_t c = c0 + k, r = r0 + tx;  // out[c][r]
    if (r < rows && c < cols) {
      if (kAdd)
        out[c * rows + r] += tile[tx][k];
      else
        out[c * rows + r] = tile[tx][k];
    }
  }
}

__global__ void dot_partial(const double* __restrict__ x, const double* __restrict__ y, size_t n,
                            double* __restrict__ part) {
  __shared__ double sh[kRedThreads / 32];
  double acc = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    acc += x[i] * y[i];
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kRedThreads / 32; w++) s += sh[w];
    part[blockIdx.x] = s;
  }
}

__global__ void dot_final(const double* __restrict__ part, int np, double* __restrict__ out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) acc += part[i];
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); w++) s += sh[w];
    *out = s;
  }
}

__global__ void scale_kernel(double* x, double a, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] *= a;
}

__global__ void axpy_kernel(double* y, const double* x, double a, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] += x[i] * a;
}

__global__ void dot_partial_f(const float* __restrict__ x, const float* __restrict__ y, const double* __restrict__ xd,
                              size_t n, double* __restrict__ part) {
  __shared__ double sh[kRedThreads / 32];
  double acc = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    acc += (xd ? xd[i] : (double)x[i]) * (double)y[i];
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kRedThreads / 32; w++) s += sh[w];
    part[blockIdx.x] = s;
  }
}

__global__ void axpy_df_kernel(double* y, const float* x, double a, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] += (double)x[i] * a;
}

__global__ void convert_kernel_df(const double* __restrict__ in, float* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

__global__ void convert_kernel_fd(const float* __restrict__ in, double* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

struct PtrPackF {
  const float* p[32];
};

// mixed path: W = sum_k U_k C_k ; R = E0*W - sum_k U_k HC_k, FP32 basis, FP64 result
__global__ void ritz_kernel_f(PtrPackF c, PtrPackF hc, const double* __restrict__ u, int nk, double e0,
                              double* __restrict__ W, double* __restrict__ R, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double w = 0.0, r = 0.0;
    for (int k = 0; k < nk; k++) {
      w += (double)c.p[k][i] * u[k];
      r -= (double)hc.p[k][i] * u[k];
    }
    W[i] = w;
    R[i] = r + e0 * w;
  }
}

// out = sum_k u_k in_k (FP32 vectors, FP64 accumulation)
__global__ void lincomb_kernel_f(PtrPackF in, const double* __restrict__ u, int nk, float* __restrict__ out,
                                 size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int k = 0; k < nk; k++) acc += (double)in.p[k][i] * u[k];
    out[i] = (float)acc;
  }
}

struct PtrPack {
  const double* p[32];
  double u[32];
};

// W = sum_k U_k C_k ; R = E0*W - sum_k U_k HC_k  (davidson.h:772-797)
__global__ void ritz_kernel(PtrPack c, PtrPack hc, int nk, double e0, double* __restrict__ W,
                            double* __restrict__ R, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double w = 0.0, r = 0.0;
    for (int k = 0; k < nk; k++) {
      w += c.p[k][i] * c.u[k];
      r -= hc.p[k][i] * c.u[k];
    }
    W[i] = w;
    R[i] = r + e0 * w;
  }
}

// C_new = R / (E0 - H_ii), regularised as davidson.h:855-862
__global__ void precond_kernel(const double* __restrict__ R, const double* __restrict__ hii, double e0,
                               double eps_reg, double* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double den = e0 - hii[i];
    out[i] = fabs(den) > eps_reg ? R[i] / den : R[i] / (den - eps_reg);
  }
}

// ---------------------------------------------------------------- RDMs

// Per alpha row: D[ia] = sum_ib W^2 and X[ia][r] = sum_ib W^2 n_r(beta string ib)
__global__ void row_weights_kernel(const double* __restrict__ W, const uint64_t* __restrict__ bstr, size_t nb,
                                   int L, double* __restrict__ D, double* __restrict__ X) {
  __shared__ double acc[65];
  size_t ia = blockIdx.x;
  for (int r = threadIdx.x; r < 65; r += blockDim.x) acc[r] = 0.0;
  __syncthreads();
  double tot = 0.0;
  for (size_t ib = threadIdx.x; ib < nb; ib += blockDim.x) {
    double w = W[ia * nb + ib];
    double w2 = w * w;
    if (w2 == 0.0) continue;
    tot += w2;
    if (X) {
      uint64_t occ = bstr[ib];
      while (occ) {
        int r = __ffsll((long long)occ) - 1;
        occ &= occ - 1;
        atomicAdd(&acc[r], w2);
      }
    }
  }
  for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&acc[64], tot);
  __syncthreads();
  if (threadIdx.x == 0) D[ia] = acc[64];
  if (X)
    for (int r = threadIdx.x; r < L; r += blockDim.x) X[ia * L + r] = acc[r];
}

__global__ void col_weights_kernel(const double* __restrict__ W, size_t na, size_t nb, double* __restrict__ D) {
  size_t ib = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ib >= nb) return;
  double acc = 0.0;
  for (size_t ia = 0; ia < na; ia++) {
    double w = W[ia * nb + ib];
    acc += w * w;
  }
  D[ib] = acc;
}

inline int grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)(b < 148 * 8 ? (b ? b : 1) : 148 * 8);
}

}  // namespace

void build_j_tables(sbdgpu_ctx* c) {
  if (c->ja) return;
  c->ja = (double*)dev_alloc(sizeof(double) * c->P * c->na);
  c->jb = (double*)dev_alloc(sizeof(double) * c->P * c->nb);
  dim3 ga((unsigned)((c->na + 255) / 256), (unsigned)c->P);
  jtable_kernel<<<ga, 256, 0, c->stream>>>(c->astr, (int)c->na, c->vf, c->P, c->ja);
  dim3 gb((unsigned)((c->nb + 255) / 256), (unsigned)c->P);
  jtable_kernel<<<gb, 256, 0, c->stream>>>(c->bstr, (int)c->nb, c->vf, c->P, c->jb);
  SBD_CUDA(cudaGetLastError());
}

void compute_hii(sbdgpu_ctx* c) {
  if (c->hii_ready) return;
  build_j_tables(c);
  double* Ea = (double*)dev_alloc(sizeof(double) * (c->na + c->nb));
  double* Eb = Ea + c->na;
  spin_energy_kernel<<<(unsigned)((c->na + 255) / 256), 256, 0, c->stream>>>(c->astr, (int)c->na, c->L, c->h1,
                                                                             c->vf, c->P, Ea);
  spin_energy_kernel<<<(unsigned)((c->nb + 255) / 256), 256, 0, c->stream>>>(c->bstr, (int)c->nb, c->L, c->h1,
                                                                             c->vf, c->P, Eb);
  if (!c->hii) c->hii = (double*)dev_alloc(sizeof(double) * c->N);
  dim3 g((unsigned)c->na, (unsigned)((c->nb + 255) / 256));
  hii_kernel<<<g, 256, 0, c->stream>>>(c->astr, c->na, c->nb, Ea, Eb, c->jb, c->P, c->ecore, c->hii);
  SBD_CUDA(cudaGetLastError());
  SBD_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(Ea);
  c->hii_ready = true;
}

void apply_phase(sbdgpu_ctx* c, double* v) {
  dim3 g((unsigned)c->na, (unsigned)((c->nb + 255) / 256));
  phase_kernel<<<g, 256, 0, c->stream>>>(c->astr, c->bstr, c->nb, v);
  SBD_CUDA(cudaGetLastError());
}

void apply_phase_rows(sbdgpu_ctx* c, double* v, size_t r0, size_t nrows) {
  if (nrows == 0) return;
  dim3 g((unsigned)nrows, (unsigned)((c->nb + 255) / 256));
  phase_kernel<<<g, 256, 0, c->stream>>>(c->astr + r0, c->bstr, c->nb, v);
  SBD_CUDA(cudaGetLastError());
}

template <typename T>
void transpose(const T* in, T* out, size_t rows, size_t cols, cudaStream_t s) {
  dim3 g((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
  transpose_kernel<T, false><<<g, dim3(32, 8), 0, s>>>(in, out, rows, cols);
  SBD_CUDA(cudaGetLastError());
}

template <typename T>
void transpose_add(const T* in, T* out, size_t rows, size_t cols, cudaStream_t s) {
  dim3 g((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
  transpose_kernel<T, true><<<g, dim3(32, 8), 0, s>>>(in, out, rows, cols);
  SBD_CUDA(cudaGetLastError());
}

// Loads this file's kernels of the FP64 sigma path (sign phase, transposes)
// on the current device now rather than at their first launch: with CUDA's
// lazy module loading, a first launch loads the module and may allocate.
void preload_fp64_sigma_misc() {
  cudaFuncAttributes fa{};
  SBD_CUDA(cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(phase_kernel)));
  SBD_CUDA(cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(transpose_kernel<double, false>)));
  SBD_CUDA(cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(transpose_kernel<double, true>)));
}

template void transpose<double>(const double*, double*, size_t, size_t, cudaStream_t);
template void transpose<float>(const float*, float*, size_t, size_t, cudaStream_t);
template void transpose_add<double>(const double*, double*, size_t, size_t, cudaStream_t);
template void transpose_add<float>(const float*, float*, size_t, size_t, cudaStream_t);

__global__ void to_float_kernel(const double* __restrict__ in, float* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

void ensure_fp32(sbdgpu_ctx* c) {
  if (c->vf32) return;
  build_j_tables(c);
  size_t nja = (size_t)c->P * c->na, njb = (size_t)c->P * c->nb, nvf = (size_t)c->P * c->P;
  c->ja32 = (float*)dev_alloc(sizeof(float) * nja);
  c->jb32 = (float*)dev_alloc(sizeof(float) * njb);
  c->vf32 = (float*)dev_alloc(sizeof(float) * nvf);
  to_float_kernel<<<592, 256, 0, c->stream>>>(c->ja, c->ja32, nja);
  to_float_kernel<<<592, 256, 0, c->stream>>>(c->jb, c->jb32, njb);
  to_float_kernel<<<592, 256, 0, c->stream>>>(c->vf, c->vf32, nvf);
  SBD_CUDA(cudaGetLastError());
}

double dot(sbdgpu_ctx* c, const double* x, const double* y, size_t n) {
  ensure_scratch(c);
  dot_partial<<<kRedBlocks, kRedThreads, 0, c->stream>>>(x, y, n, c->red);
  dot_final<<<1, 1024, 0, c->stream>>>(c->red, kRedBlocks, c->red + kRedBlocks);
  SBD_CUDA(cudaGetLastError());
  double r = 0.0;
  SBD_CUDA(cudaMemcpyAsync(&r, c->red + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SBD_CUDA(cudaStreamSynchronize(c->stream));
  return r;
}

// <x|y> into device memory *out, on the context's stream, without waiting
void dot_device(sbdgpu_ctx* c, const double* x, const double* y, size_t n, double* out) {
  dot_partial<<<kRedBlocks, kRedThreads, 0, c->stream>>>(x, y, n, c->red);
  dot_final<<<1, 1024, 0, c->stream>>>(c->red, kRedBlocks, out);
  SBD_CUDA(cudaGetLastError());
}

double dot_f(sbdgpu_ctx* c, const float* x, const double* xd, const float* y, size_t n) {
  ensure_scratch(c);
  dot_partial_f<<<kRedBlocks, kRedThreads, 0, c->stream>>>(x, y, xd, n, c->red);
  dot_final<<<1, 1024, 0, c->stream>>>(c->red, kRedBlocks, c->red + kRedBlocks);
  SBD_CUDA(cudaGetLastError());
  double r = 0.0;
  SBD_CUDA(cudaMemcpyAsync(&r, c->red + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SBD_CUDA(cudaStreamSynchronize(c->stream));
  return r;
}

void axpy_df(double* y, const float* x, double a, size_t n, cudaStream_t s) {
  axpy_df_kernel<<<grid_for(n), 256, 0, s>>>(y, x, a, n);
  SBD_CUDA(cudaGetLastError());
}

void convert(const double* in, float* out, size_t n, cudaStream_t s) {
  convert_kernel_df<<<grid_for(n), 256, 0, s>>>(in, out, n);
  SBD_CUDA(cudaGetLastError());
}

void convert(const float* in, double* out, size_t n, cudaStream_t s) {
  convert_kernel_fd<<<grid_for(n), 256, 0, s>>>(in, out, n);
  SBD_CUDA(cudaGetLastError());
}

void ritz_update_f(float* const* C, float* const* HC, const double* U, int nk, double e0, double* W, double* R,
                   size_t n, sbdgpu_ctx* c) {
  PtrPackF pc{}, ph{};
  for (int k = 0; k < nk; k++) {
    pc.p[k] = C[k];
    ph.p[k] = HC[k];
  }
  ensure_scratch(c);
  double* du = c->red + 600;  // 32 spare doubles after the 593 reduction slots
  SBD_CUDA(cudaMemcpyAsync(du, U, sizeof(double) * nk, cudaMemcpyHostToDevice, c->stream));
  ritz_kernel_f<<<grid_for(n), 256, 0, c->stream>>>(pc, ph, du, nk, e0, W, R, n);
  SBD_CUDA(cudaGetLastError());
  SBD_CUDA(cudaStreamSynchronize(c->stream));
}

void lincomb_f(float* const* in, const double* U, int nk, float* out, size_t n, sbdgpu_ctx* c) {
  PtrPackF p{};
  for (int k = 0; k < nk; k++) p.p[k] = in[k];
  ensure_scratch(c);
  double* du = c->red + 640;
  SBD_CUDA(cudaMemcpyAsync(du, U, sizeof(double) * nk, cudaMemcpyHostToDevice, c->stream));
  lincomb_kernel_f<<<grid_for(n), 256, 0, c->stream>>>(p, du, nk, out, n);
  SBD_CUDA(cudaGetLastError());
  SBD_CUDA(cudaStreamSynchronize(c->stream));
}

void scale(double* x, double a, size_t n, cudaStream_t s) {
  scale_kernel<<<grid_for(n), 256, 0, s>>>(x, a, n);
  SBD_CUDA(cudaGetLastError());
}

void axpy(double* y, const double* x, double a, size_t n, cudaStream_t s) {
  axpy_kernel<<<grid_for(n), 256, 0, s>>>(y, x, a, n);
  SBD_CUDA(cudaGetLastError());
}

void ritz_update(double* const* C, double* const* HC, const double* U, int nk, double e0, double* W, double* R,
                 size_t n, cudaStream_t s) {
  PtrPack pc{}, ph{};
  for (int k = 0; k < nk; k++) {
    pc.p[k] = C[k];
    ph.p[k] = HC[k];
    pc.u[k] = U[k];
  }
  ritz_kernel<<<grid_for(n), 256, 0, s>>>(pc, ph, nk, e0, W, R, n);
  SBD_CUDA(cudaGetLastError());
}

void precondition(const double* R, const double* hii, double e0, double eps_reg, double* out, size_t n,
                  cudaStream_t s) {
  precond_kernel<<<grid_for(n), 256, 0, s>>>(R, hii, e0, eps_reg, out, n);
  SBD_CUDA(cudaGetLastError());
}

void alpha_weights(sbdgpu_ctx* c, const double* dW, double* D) {
  row_weights_kernel<<<(unsigned)c->na, 256, 0, c->stream>>>(dW, c->bstr, c->nb, c->L, D, nullptr);
  SBD_CUDA(cudaGetLastError());
}

void occupation(sbdgpu_ctx* c, const double* dW, double* dens) {
  double* Da = (double*)dev_alloc(sizeof(double) * (c->na + c->nb));
  double* Db = Da + c->na;
  alpha_weights(c, dW, Da);
  col_weights_kernel<<<(unsigned)((c->nb + 255) / 256), 256, 0, c->stream>>>(dW, c->na, c->nb, Db);
  SBD_CUDA(cudaGetLastError());
  std::vector<double> hd(c->na + c->nb);
  SBD_CUDA(cudaMemcpyAsync(hd.data(), Da, sizeof(double) * hd.size(), cudaMemcpyDeviceToHost, c->stream));
  SBD_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(Da);
  int L = c->L;
  for (int i = 0; i < 2 * L; i++) dens[i] = 0.0;
  for (size_t ia = 0; ia < c->na; ia++)
    for (int p = 0; p < L; p++)
      if ((c->h_astr[ia] >> p) & 1) dens[2 * p] += hd[ia];
  for (size_t ib = 0; ib < c->nb; ib++)
    for (int p = 0; p < L; p++)
      if ((c->h_bstr[ib] >> p) & 1) dens[2 * p + 1] += hd[c->na + ib];
}

void rdm(sbdgpu_ctx* c, const double* dW, double* one, double* two) {
  int L = c->L;
  size_t L2 = (size_t)L * L, L4 = L2 * L2;
  double* d_one = (double*)dev_alloc(sizeof(double) * (2 * L2 + 4 * L4));
  double* d_two = d_one + 2 * L2;
  SBD_CUDA(cudaMemsetAsync(d_one, 0, sizeof(double) * (2 * L2 + 4 * L4), c->stream));
  rdm_offdiag(c, dW, d_one, d_two);
  // diagonal contributions (ZeroDiffCorrelation, correlation.h:15-44) from the
  // alpha-row weights, beta-column weights and the alpha x beta occupation moment
  double* Da = (double*)dev_alloc(sizeof(double) * (c->na + c->nb + c->na * L));
  double* Db = Da + c->na;
  double* X = Db + c->nb;
  row_weights_kernel<<<(unsigned)c->na, 256, 0, c->stream>>>(dW, c->bstr, c->nb, L, Da, X);
  col_weights_kernel<<<(unsigned)((c->nb + 255) / 256), 256, 0, c->stream>>>(dW, c->na, c->nb, Db);
  SBD_CUDA(cudaGetLastError());
  std::vector<double> h(c->na + c->nb + c->na * L);
  SBD_CUDA(cudaMemcpyAsync(h.data(), Da, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
  SBD_CUDA(cudaMemcpyAsync(one, d_one, sizeof(double) * 2 * L2, cudaMemcpyDeviceToHost, c->stream));
  SBD_CUDA(cudaMemcpyAsync(two, d_two, sizeof(double) * 4 * L4, cudaMemcpyDeviceToHost, c->stream));
  SBD_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(d_one);
  cudaFree(Da);
  const double* hDa = h.data();
  const double* hDb = hDa + c->na;
  const double* hX = hDb + c->nb;
  std::vector<double> Aaa(L2, 0.0), Abb(L2, 0.0), M(L2, 0.0), na1(L, 0.0), nb1(L, 0.0);
  for (size_t ia = 0; ia < c->na; ia++) {
    uint64_t a = c->h_astr[ia];
    for (int p = 0; p < L; p++) {
      if (!((a >> p) & 1)) continue;
      na1[p] += hDa[ia];
      for (int r = 0; r < L; r++) M[p * L + r] += hX[ia * L + r];
      for (int q = 0; q < L; q++)
        if (q != p && ((a >> q) & 1)) Aaa[p * L + q] += hDa[ia];
    }
  }
  for (size_t ib = 0; ib < c->nb; ib++) {
    uint64_t b = c->h_bstr[ib];
    for (int p = 0; p < L; p++) {
      if (!((b >> p) & 1)) continue;
      nb1[p] += hDb[ib];
      for (int q = 0; q < L; q++)
        if (q != p && ((b >> q) & 1)) Abb[p * L + q] += hDb[ib];
    }
  }
  size_t L3 = L2 * L;
  for (int p = 0; p < L; p++) {
    one[0 * L2 + p + (size_t)L * p] += na1[p];
    one[1 * L2 + p + (size_t)L * p] += nb1[p];
    for (int q = 0; q < L; q++) {
      // same-spin pairs (each unordered pair contributes both orders)
      two[0 * L4 + p + L * q + L2 * p + L3 * q] += Aaa[p * L + q];
      two[0 * L4 + p + L * q + L2 * q + L3 * p] -= Aaa[p * L + q];
      two[3 * L4 + p + L * q + L2 * p + L3 * q] += Abb[p * L + q];
      two[3 * L4 + p + L * q + L2 * q + L3 * p] -= Abb[p * L + q];
      // opposite-spin pairs (alpha p, beta q)
      two[2 * L4 + p + L * q + L2 * p + L3 * q] += M[p * L + q];
      two[1 * L4 + q + L * p + L2 * q + L3 * p] += M[p * L + q];
    }
  }
}

}  // namespace sbdgpu
