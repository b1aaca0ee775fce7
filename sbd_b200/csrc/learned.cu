// Learned Davidson preconditioner: a small BF16 network that shifts the
// diagonal correction's denominator per determinant.
//
// The reference's Davidson takes the correction t_i = r_i / (E0 - H_ii)
// (chemistry/tpb/davidson.h:853-862).  Here
//
//   x_i  = features of determinant i: asinh(H_ii - E0), asinh(|r_i| sqrt(N)) / 4,
//          and per spin the holes in the 8 orbitals below the Fermi level, the
//          particles in the 8 above it and the excitation rank / electrons
//          (36 values, padded to kF = 48; independent of norb, so a network
//          trained on one system applies to another)
//   h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2)   (128 units, BF16 weights)
//   s_i = S tanh(w3 . h2 + b3)
//   t_i = r_i / (E0 - H_ii - s_i)                 (regularised like the diagonal)
//
// Training data are (Ritz vector u, residual r, correction t) triples the
// method generates itself: at restart points of a Davidson run on the training
// system, t solves the Jacobi-Davidson correction equation
// (I - uu^T)(H - E0)(I - uu^T) t = -r by MINRES on this library's own sigma.  (The unprojected (H - E0)^-1 r is u itself, so it
// carries no new direction.)  The loss of one triple is 1 - cos^2(P t_hat, t)
// over a weighted sample of its determinants, P the projection orthogonal to
// u.  Training runs on hand-written FP32 kernels (forward, loss, backward,
// Adam) with BF16-rounded weights; inference over all determinants runs on
// the tensor cores (tcgen05, BF16 operands, FP32 accumulation in TMEM).
#include <cuda_bf16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <random>
#include <vector>

#include "internal.cuh"

namespace sbdgpu {

namespace {

constexpr int kHid = 128;
constexpr int kWin = 8;
constexpr int kF = 48;
constexpr int oW1 = 0, ob1 = oW1 + kHid * kF, oW2 = ob1 + kHid, ob2 = oW2 + kHid * kHid, ow3 = ob2 + kHid,
              ob3 = ow3 + kHid;
constexpr int kNParams = ob3 + 1;
constexpr int kGroup = 32;  // samples per block iteration in the training kernels

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// One spin's window features into x[0 .. 2*kWin]: holes below the Fermi level,
// particles above it, excitation rank / ne.
__device__ __forceinline__ void spin_features(uint64_t s, int ne, float* x) {
#pragma unroll
  for (int j = 0; j < kWin; j++) {
    const int ph = ne - 1 - j, pp = ne + j;
    x[j] = ph >= 0 ? (float)(1 - (int)((s >> ph) & 1ull)) : 0.f;
    x[kWin + j] = pp < 64 ? (float)((s >> pp) & 1ull) : 0.f;
  }
  const uint64_t aufbau = ne >= 64 ? ~0ull : ((1ull << ne) - 1);
  x[2 * kWin] = (float)__popcll(s & ~aufbau) / (float)(ne > 0 ? ne : 1);
}

__device__ __forceinline__ void det_features(uint64_t a, uint64_t b, int nea, int neb, double hii_minus_e0,
                                             double r, double sqrt_n, float* x) {
  x[0] = asinhf((float)hii_minus_e0);
  x[1] = asinhf((float)(fabs(r) * sqrt_n)) * 0.25f;  // magnitude: t_i flips sign with r_i
  spin_features(a, nea, x + 2);
  spin_features(b, neb, x + 2 + 2 * kWin + 1);
#pragma unroll
  for (int f = 2 + 2 * (2 * kWin + 1); f < kF; f++) x[f] = 0.f;
}

// ---------------------------------------------------------------- training

// Features of sampled determinants: X[k][*] for sample k (determinant idx[k]).
__global__ void feat_batch_kernel(const int64_t* __restrict__ idx, const double* __restrict__ den,
                                  const double* __restrict__ r, const uint64_t* __restrict__ astr,
                                  const uint64_t* __restrict__ bstr, size_t nb, int nea, int neb, double sqrt_n, int B,
                                  float* __restrict__ X) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= B) return;
  const int64_t i = idx[k];
  float x[kF];
  // den = E0 - H_ii, so H_ii - E0 = -den
  det_features(astr[i / nb], bstr[i % nb], nea, neb, -den[k], r[k], sqrt_n, x);
#pragma unroll
  for (int f = 0; f < kF; f++) X[(size_t)k * kF + f] = x[f];
}

// Forward pass for B samples: H1, H2 (after relu) and z.  128 threads = hidden
// units; each block iteration takes kGroup samples.
__global__ void __launch_bounds__(kHid) mlp_fwd_kernel(const float* __restrict__ X, const float* __restrict__ we,
                                                       int B, float* __restrict__ H1, float* __restrict__ H2,
                                                       float* __restrict__ Z) {
  extern __shared__ float sm[];
  float* W1T = sm;                  // [kF][kHid]
  float* W2T = W1T + kF * kHid;     // [kHid][kHid], W2T[k][j] = W2[j][k]
  float* Xs = W2T + kHid * kHid;    // [kGroup][kF]
  float* H1s = Xs + kGroup * kF;    // [kGroup][kHid]
  float* red = H1s + kGroup * kHid; // [4][kGroup]
  const int j = threadIdx.x, lane = j & 31, warp = j >> 5;
  for (int i = j; i < kHid * kF; i += kHid) {
    const int jj = i / kF, f = i - jj * kF;
    W1T[f * kHid + jj] = we[oW1 + i];
  }
  for (int i = j; i < kHid * kHid; i += kHid) {
    const int jj = i / kHid, k = i - jj * kHid;
    W2T[k * kHid + jj] = we[oW2 + i];
  }
  const float b1 = we[ob1 + j], b2 = we[ob2 + j], w3 = we[ow3 + j], b3 = we[ob3];
  __syncthreads();
  const int ngroups = (B + kGroup - 1) / kGroup;
  for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
    const int s0 = g * kGroup;
    for (int i = j; i < kGroup * kF; i += kHid) {
      const int s = i / kF;
      Xs[i] = s0 + s < B ? X[(size_t)s0 * kF + i] : 0.f;
    }
    __syncthreads();
    float acc[kGroup];
#pragma unroll
    for (int s = 0; s < kGroup; s++) acc[s] = b1;
    for (int f = 0; f < kF; f++) {
      const float w = W1T[f * kHid + j];
#pragma unroll
      for (int s = 0; s < kGroup; s++) acc[s] += w * Xs[s * kF + f];
    }
#pragma unroll
    for (int s = 0; s < kGroup; s++) {
      const float h = fmaxf(acc[s], 0.f);
      H1s[s * kHid + j] = h;
      if (s0 + s < B) H1[(size_t)(s0 + s) * kHid + j] = h;
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < kGroup; s++) acc[s] = b2;
    for (int k = 0; k < kHid; k++) {
      const float w = W2T[k * kHid + j];
#pragma unroll
      for (int s = 0; s < kGroup; s++) acc[s] += w * H1s[s * kHid + k];
    }
#pragma unroll
    for (int s = 0; s < kGroup; s++) {
      const float h = fmaxf(acc[s], 0.f);
      if (s0 + s < B) H2[(size_t)(s0 + s) * kHid + j] = h;
      float p = w3 * h;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
      if (lane == 0) red[warp * kGroup + s] = p;
    }
    __syncthreads();
    if (j < kGroup && s0 + j < B) Z[s0 + j] = red[j] + red[kGroup + j] + red[2 * kGroup + j] + red[3 * kGroup + j] + b3;
    __syncthreads();
  }
}

// Per-sample correction and the six weighted sums of the loss:
// sums = [sum w u th, sum w u u, sum w th t, sum w th th, sum w u t, sum w t t]
__global__ void loss_sums_kernel(const float* __restrict__ Z, const double* __restrict__ r,
                                 const double* __restrict__ den, const double* __restrict__ u,
                                 const double* __restrict__ t, const double* __restrict__ wt, int B, double S,
                                 double eps_reg, double* __restrict__ th_out, double* __restrict__ dd_out,
                                 double* __restrict__ sums) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B; k += gridDim.x * blockDim.x) {
    const double s = S * tanh((double)Z[k]);
    double dd = den[k] - s;
    if (!(fabs(dd) > eps_reg)) dd -= eps_reg;
    const double th = r[k] / dd;
    th_out[k] = th;
    dd_out[k] = dd;
    const double w = wt[k];
    acc[0] += w * u[k] * th;
    acc[1] += w * u[k] * u[k];
    acc[2] += w * th * t[k];
    acc[3] += w * th * th;
    acc[4] += w * u[k] * t[k];
    acc[5] += w * t[k] * t[k];
  }
  __shared__ double red[6][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 6; i++) {
    double v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[i][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[threadIdx.x][w];
    atomicAdd(&sums[threadIdx.x], v);
  }
}

// Loss and the coefficients of dL/dth from the sums (one thread):
// coef = [loss, K1 = 2c/(ab), c/a, p/uu, K2 = 2cq/(ab uu)]
__global__ void loss_scalars_kernel(const double* __restrict__ sums, double* __restrict__ coef,
                                    double* __restrict__ loss_trace, int step) {
  const double p = sums[0], uu = sums[1], tht = sums[2], thth = sums[3], q = sums[4], b = sums[5];
  const double c = tht - (p / uu) * q;
  const double a = thth - p * p / uu;
  const double loss = 1.0 - c * c / (a * b);
  coef[0] = loss;
  coef[1] = 2.0 * c / (a * b);
  coef[2] = c / a;
  coef[3] = p / uu;
  coef[4] = 2.0 * c * q / (a * b * uu);
  if (loss_trace) loss_trace[step] = loss;
}

// dL/dz per sample
__global__ void grad_z_kernel(const float* __restrict__ Z, const double* __restrict__ th,
                              const double* __restrict__ dd, const double* __restrict__ u,
                              const double* __restrict__ t, const double* __restrict__ wt,
                              const double* __restrict__ coef, int B, double S, float* __restrict__ gz) {
  const double K1 = coef[1], ca = coef[2], pu = coef[3], K2 = coef[4];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B; k += gridDim.x * blockDim.x) {
    const double tp = th[k] - pu * u[k];
    const double g_th = wt[k] * K1 * (ca * tp - t[k]) + wt[k] * u[k] * K2;
    const double g_s = g_th * th[k] / dd[k];
    const double tz = tanh((double)Z[k]);
    gz[k] = (float)(g_s * S * (1.0 - tz * tz));
  }
}

// Hidden-layer gradients: G2 = gz w3 [h2 > 0], G1 = (G2 W2) [h1 > 0].
__global__ void __launch_bounds__(kHid) mlp_bwd_kernel(const float* __restrict__ we, const float* __restrict__ H1,
                                                       const float* __restrict__ H2, const float* __restrict__ gz,
                                                       int B, float* __restrict__ G1, float* __restrict__ G2) {
  extern __shared__ float sm[];
  float* W2 = sm;                     // [kHid][kHid], W2[j][k]
  float* G2s = W2 + kHid * kHid;      // [kGroup][kHid]
  const int k = threadIdx.x;
  for (int i = k; i < kHid * kHid; i += kHid) W2[i] = we[oW2 + i];
  const float w3 = we[ow3 + k];
  __syncthreads();
  const int ngroups = (B + kGroup - 1) / kGroup;
  for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
    const int s0 = g * kGroup;
    for (int s = 0; s < kGroup; s++) {
      float v = 0.f;
      if (s0 + s < B) {
        const float h2 = H2[(size_t)(s0 + s) * kHid + k];
        v = h2 > 0.f ? gz[s0 + s] * w3 : 0.f;
        G2[(size_t)(s0 + s) * kHid + k] = v;
      }
      G2s[s * kHid + k] = v;
    }
    __syncthreads();
    float acc[kGroup];
#pragma unroll
    for (int s = 0; s < kGroup; s++) acc[s] = 0.f;
    for (int j = 0; j < kHid; j++) {
      const float w = W2[j * kHid + k];
#pragma unroll
      for (int s = 0; s < kGroup; s++) acc[s] += w * G2s[s * kHid + j];
    }
#pragma unroll
    for (int s = 0; s < kGroup; s++)
      if (s0 + s < B) {
        const float h1 = H1[(size_t)(s0 + s) * kHid + k];
        G1[(size_t)(s0 + s) * kHid + k] = h1 > 0.f ? acc[s] : 0.f;
      }
    __syncthreads();
  }
}

// out[i][j] += sum_s A[s][i] Bm[s][j] over samples (one 32 x 32 tile per block
// and a chunk of samples per blockIdx.z); colsum[i] += sum_s A[s][i] when
// given (from the blocks of the first tile column only).
__global__ void outer_accum_kernel(const float* __restrict__ A, int m, const float* __restrict__ Bm, int n, int B,
                                   int chunk, float* __restrict__ out, float* __restrict__ colsum) {
  __shared__ float As[32][33];
  __shared__ float Bs[32][33];
  const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 256 threads: ty 0..7
  const int sb = blockIdx.z * chunk, se = min(B, sb + chunk);
  float acc[4] = {0, 0, 0, 0};
  float cs = 0.f;
  for (int s0 = sb; s0 < se; s0 += 32) {
    for (int r = ty; r < 32; r += 8) {
      const int s = s0 + r;
      As[r][tx] = (s < se && i0 + tx < m) ? A[(size_t)s * m + i0 + tx] : 0.f;
      Bs[r][tx] = (s < se && j0 + tx < n) ? Bm[(size_t)s * n + j0 + tx] : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int r = 0; r < 32; r++) {
      const float b = Bs[r][tx];
#pragma unroll
      for (int q = 0; q < 4; q++) acc[q] += As[r][ty + 8 * q] * b;
    }
    if (colsum && blockIdx.x == 0 && ty == 0)
      for (int r = 0; r < 32; r++) cs += As[r][tx];
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = i0 + ty + 8 * q, j = j0 + tx;
    if (i < m && j < n) atomicAdd(&out[(size_t)i * n + j], acc[q]);
  }
  if (colsum && blockIdx.x == 0 && ty == 0 && i0 + tx < m) atomicAdd(&colsum[i0 + tx], cs);
}

// Adam step on the FP32 master weights, then the BF16-rounded effective copy
// (FP32 for the training kernels, BF16 for inference).
__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, int n, float lr, float b1, float b2, float eps, int step,
                            float* __restrict__ we, __nv_bfloat16* __restrict__ w16) {
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    we[i] = bf16_round(wi);
    w16[i] = __float2bfloat16_rn(wi);
  }
}

__global__ void round_weights_kernel(const float* __restrict__ w, int n, float* __restrict__ we,
                                     __nv_bfloat16* __restrict__ w16) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    we[i] = bf16_round(w[i]);
    w16[i] = __float2bfloat16_rn(w[i]);
  }
}

size_t fwd_smem() { return sizeof(float) * (kF * kHid + kHid * kHid + kGroup * kF + kGroup * kHid + 4 * kGroup); }
size_t bwd_smem() { return sizeof(float) * (kHid * kHid + kGroup * kHid); }

}  // namespace

// Device buffers of one training minibatch (B samples).
struct MlpBatch {
  int cap = 0;
  float *X = nullptr, *H1 = nullptr, *H2 = nullptr, *Z = nullptr, *G1 = nullptr, *G2 = nullptr, *gz = nullptr;
  double *th = nullptr, *dd = nullptr, *sums = nullptr, *coef = nullptr;
  void ensure(int B) {
    if (B <= cap) return;
    release();
    X = (float*)dev_alloc(sizeof(float) * (size_t)B * kF);
    H1 = (float*)dev_alloc(sizeof(float) * (size_t)B * kHid);
    H2 = (float*)dev_alloc(sizeof(float) * (size_t)B * kHid);
    G1 = (float*)dev_alloc(sizeof(float) * (size_t)B * kHid);
    G2 = (float*)dev_alloc(sizeof(float) * (size_t)B * kHid);
    Z = (float*)dev_alloc(sizeof(float) * B);
    gz = (float*)dev_alloc(sizeof(float) * B);
    th = (double*)dev_alloc(sizeof(double) * B);
    dd = (double*)dev_alloc(sizeof(double) * B);
    sums = (double*)dev_alloc(sizeof(double) * 8);
    coef = (double*)dev_alloc(sizeof(double) * 8);
    cap = B;
  }
  void release() {
    for (void* p : {(void*)X, (void*)H1, (void*)H2, (void*)G1, (void*)G2, (void*)Z, (void*)gz, (void*)th, (void*)dd,
                    (void*)sums, (void*)coef})
      cudaFree(p);
    X = H1 = H2 = G1 = G2 = Z = gz = nullptr;
    th = dd = sums = coef = nullptr;
    cap = 0;
  }
};

// Loss and gradient of one minibatch whose features X (device, [B][kF]) are
// already in mb.X.  grad (device, kNParams) is accumulated into.
void mlp_loss_grad(MlpBatch& mb, const float* we, int B, const double* r, const double* den, const double* u,
                   const double* t, const double* wt, double S, double eps_reg, float* grad, double* loss_trace,
                   int step, cudaStream_t st) {
  int dev = 0;
  SBD_CUDA(cudaGetDevice(&dev));
  allow_dynamic_smem(reinterpret_cast<const void*>(mlp_fwd_kernel), dev);
  allow_dynamic_smem(reinterpret_cast<const void*>(mlp_bwd_kernel), dev);
  const int ngroups = (B + kGroup - 1) / kGroup;
  const int grid = std::min(ngroups, 296);
  mlp_fwd_kernel<<<grid, kHid, fwd_smem(), st>>>(mb.X, we, B, mb.H1, mb.H2, mb.Z);
  SBD_CUDA(cudaGetLastError());
  SBD_CUDA(cudaMemsetAsync(mb.sums, 0, sizeof(double) * 8, st));
  loss_sums_kernel<<<std::min((B + 255) / 256, 296), 256, 0, st>>>(mb.Z, r, den, u, t, wt, B, S, eps_reg, mb.th,
                                                                    mb.dd, mb.sums);
  SBD_CUDA(cudaGetLastError());
  loss_scalars_kernel<<<1, 1, 0, st>>>(mb.sums, mb.coef, loss_trace, step);
  SBD_CUDA(cudaGetLastError());
  grad_z_kernel<<<std::min((B + 255) / 256, 296), 256, 0, st>>>(mb.Z, mb.th, mb.dd, u, t, wt, mb.coef, B, S, mb.gz);
  SBD_CUDA(cudaGetLastError());
  mlp_bwd_kernel<<<grid, kHid, bwd_smem(), st>>>(we, mb.H1, mb.H2, mb.gz, B, mb.G1, mb.G2);
  SBD_CUDA(cudaGetLastError());
  const int chunk = 2048;
  const int nz = (B + chunk - 1) / chunk;
  // dW1 = G1^T X, db1 = colsum G1; dW2 = G2^T H1, db2 = colsum G2; dw3 = gz^T H2, db3 = sum gz
  outer_accum_kernel<<<dim3((kF + 31) / 32, kHid / 32, nz), 256, 0, st>>>(mb.G1, kHid, mb.X, kF, B, chunk,
                                                                          grad + oW1, grad + ob1);
  outer_accum_kernel<<<dim3(kHid / 32, kHid / 32, nz), 256, 0, st>>>(mb.G2, kHid, mb.H1, kHid, B, chunk, grad + oW2,
                                                                     grad + ob2);
  outer_accum_kernel<<<dim3(kHid / 32, 1, nz), 256, 0, st>>>(mb.gz, 1, mb.H2, kHid, B, chunk, grad + ow3,
                                                             grad + ob3);
  SBD_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------- inference

namespace {

constexpr int kInfThreads = 128;  // 4 warps: warp w owns TMEM lanes 32w..32w+31 (determinants)
constexpr uint32_t kSboF = (kF / 8) * 128;    // 8-row group stride of a K = kF operand
constexpr uint32_t kSboH = (kHid / 8) * 128;  // 8-row group stride of a K = 128 operand
constexpr uint32_t kW1Bytes = kHid * kF * 2, kW2Bytes = kHid * kHid * 2, kXBytes = 128 * kF * 2,
                   kH1Bytes = 128 * kHid * 2;
// kind::f16, BF16 x BF16 -> F32, A and B K-major, M = 128, N = 128
constexpr uint32_t kIdescInf = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kHid >> 3) << 17) | ((128u >> 4) << 24);
constexpr long long kInfSpin = kMaxSpinLimit;
constexpr uint64_t kInfWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t sm_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major core-matrix layout: element (row, k) of an operand whose 8-row
// groups are sbo bytes apart
__device__ __forceinline__ uint32_t kmaj(int row, int k, uint32_t sbo) {
  return (uint32_t)(row >> 3) * sbo + (uint32_t)(k >> 3) * 128u + (uint32_t)(row & 7) * 16u + (uint32_t)(k & 7) * 2u;
}

__device__ __forceinline__ uint64_t desc(uint32_t start, uint32_t sbo) {
  return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
         (1ull << 46);
}

__device__ __forceinline__ void mma_inf(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdescInf), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool wait_bar(uint32_t mbar, uint32_t parity) {
  const uint64_t t0 = gtimer();
  for (long long i = 0; i < kInfSpin; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 1023) == 1023 && gtimer() - t0 > kInfWaitNs) return false;
  }
  return false;
}

__device__ __forceinline__ void ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

struct InfArgs {
  const __nv_bfloat16* w16;  // effective weights (BF16), packed as the master weights
  const float* we;           // effective weights (FP32 copy): biases and w3 are read from here
  const double* R;           // residual
  const double* hii;
  const uint64_t* astr;
  const uint64_t* bstr;
  double* out;               // correction
  size_t n, nb;
  int nea, neb;
  double e0, eps_reg, S, sqrt_n;
  int* err;
};

// out_i = R_i / (E0 - H_ii - S tanh(net(x_i))) for all determinants, 128 per
// tile: features -> BF16 A tile (K-major) -> tcgen05.mma with W1 (B, K-major)
// into TMEM -> bias, relu, BF16 -> second A tile -> tcgen05.mma with W2 ->
// bias, relu, dot with w3 in registers.
__global__ void __launch_bounds__(kInfThreads) mlp_infer_kernel(InfArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* W1s = smem_raw;
  unsigned char* W2s = W1s + kW1Bytes;
  unsigned char* Xs = W2s + kW2Bytes;
  unsigned char* H1s = Xs + kXBytes;
  float* b1 = reinterpret_cast<float*>(H1s + kH1Bytes);
  float* b2 = b1 + kHid;
  float* w3 = b2 + kHid;
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t mbar = sm_addr(&s_bar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sm_addr(&s_tmem)),
                 "r"(kHid));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  // weights into the K-major B operands, 8 consecutive k per 16-byte store
  for (int task = tid; task < kHid * (kF / 8); task += kInfThreads) {
    const int nrow = task / (kF / 8), k8 = task - nrow * (kF / 8);
    *reinterpret_cast<uint4*>(W1s + kmaj(nrow, 8 * k8, kSboF)) =
        *reinterpret_cast<const uint4*>(a.w16 + oW1 + nrow * kF + 8 * k8);
  }
  for (int task = tid; task < kHid * (kHid / 8); task += kInfThreads) {
    const int nrow = task / (kHid / 8), k8 = task - nrow * (kHid / 8);
    *reinterpret_cast<uint4*>(W2s + kmaj(nrow, 8 * k8, kSboH)) =
        *reinterpret_cast<const uint4*>(a.w16 + oW2 + nrow * kHid + 8 * k8);
  }
  b1[tid] = a.we[ob1 + tid];
  b2[tid] = a.we[ob2 + tid];
  w3[tid] = a.we[ow3 + tid];
  const float b3 = a.we[ob3];
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
  const uint32_t x0 = sm_addr(Xs), h0 = sm_addr(H1s), w10 = sm_addr(W1s), w20 = sm_addr(W2s);
  uint32_t phase = 0;
  const size_t ntiles = (a.n + 127) / 128;
  for (size_t tile = blockIdx.x; tile < ntiles && !s_fail; tile += gridDim.x) {
    const size_t i = tile * 128 + tid;
    const bool valid = i < a.n;
    double r = 0.0, den = -1.0;
    {
      float x[kF];
      if (valid) {
        r = a.R[i];
        den = a.e0 - a.hii[i];
        det_features(a.astr[i / a.nb], a.bstr[i % a.nb], a.nea, a.neb, -den, r, a.sqrt_n, x);
      } else {
#pragma unroll
        for (int f = 0; f < kF; f++) x[f] = 0.f;
      }
#pragma unroll
      for (int k8 = 0; k8 < kF / 8; k8++)
        *reinterpret_cast<uint4*>(Xs + kmaj(tid, 8 * k8, kSboF)) =
            make_uint4(pack_bf16(x[8 * k8], x[8 * k8 + 1]), pack_bf16(x[8 * k8 + 2], x[8 * k8 + 3]),
                       pack_bf16(x[8 * k8 + 4], x[8 * k8 + 5]), pack_bf16(x[8 * k8 + 6], x[8 * k8 + 7]));
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int ks = 0; ks < kF / 16; ks++)
        mma_inf(tmem, desc(x0 + ks * 256, kSboF), desc(w10 + ks * 256, kSboF), ks > 0 ? 1u : 0u);
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                   : "memory");
    }
    if (!wait_bar(mbar, phase)) {
      s_fail = 1;
      atomicExch(a.err, 1);
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // layer 1 epilogue: this thread's row of D, 16 columns at a time
#pragma unroll 1
    for (int c = 0; c < kHid / 16; c++) {
      float v[16];
      ld16(trow + 16 * c, v);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      uint32_t p[8];
#pragma unroll
      for (int j = 0; j < 8; j++)
        p[j] = pack_bf16(fmaxf(v[2 * j] + b1[16 * c + 2 * j], 0.f), fmaxf(v[2 * j + 1] + b1[16 * c + 2 * j + 1], 0.f));
      *reinterpret_cast<uint4*>(H1s + kmaj(tid, 16 * c, kSboH)) = make_uint4(p[0], p[1], p[2], p[3]);
      *reinterpret_cast<uint4*>(H1s + kmaj(tid, 16 * c + 8, kSboH)) = make_uint4(p[4], p[5], p[6], p[7]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0 && !s_fail) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int ks = 0; ks < kHid / 16; ks++)
        mma_inf(tmem, desc(h0 + ks * 256, kSboH), desc(w20 + ks * 256, kSboH), ks > 0 ? 1u : 0u);
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                   : "memory");
    }
    if (!s_fail && !wait_bar(mbar, phase)) {
      s_fail = 1;
      atomicExch(a.err, 1);
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float z = b3;
#pragma unroll 1
    for (int c = 0; c < kHid / 16; c++) {
      float v[16];
      ld16(trow + 16 * c, v);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 16; j++) z += w3[16 * c + j] * fmaxf(v[j] + b2[16 * c + j], 0.f);
    }
    if (valid) {
      double dd = den - a.S * tanh((double)z);
      if (!(fabs(dd) > a.eps_reg)) dd -= a.eps_reg;
      a.out[i] = r / dd;
    }
    // TMEM and the A tiles are reused by the next tile
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kHid));
}

constexpr size_t kInfSmem = kW1Bytes + kW2Bytes + kXBytes + kH1Bytes + 3 * kHid * sizeof(float);

// |t|^2 + |r|^2 of each determinant, and a histogram of its binary exponent
__global__ void score_hist_kernel(const double* __restrict__ t, const double* __restrict__ r, size_t n,
                                  unsigned long long* __restrict__ hist) {
  __shared__ unsigned int h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double sc = t[i] * t[i] + r[i] * r[i];
    int e = sc > 0 ? ilogb(sc) : -1000;
    e = min(max(e + 200, 0), 255);
    atomicAdd(&h[e], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
}

// indices of determinants whose score's exponent bin is >= bin_min (up to cap)
__global__ void select_top_kernel(const double* __restrict__ t, const double* __restrict__ r, size_t n, int bin_min,
                                  int cap, int64_t* __restrict__ out, int* __restrict__ count) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double sc = t[i] * t[i] + r[i] * r[i];
    int e = sc > 0 ? ilogb(sc) : -1000;
    e = min(max(e + 200, 0), 255);
    if (e >= bin_min) {
      const int k = atomicAdd(count, 1);
      if (k < cap) out[k] = (int64_t)i;
    }
  }
}

// sample values of one harvested triple
__global__ void gather_samples_kernel(const int64_t* __restrict__ idx, int m, const double* __restrict__ r,
                                      const double* __restrict__ u, const double* __restrict__ t,
                                      const double* __restrict__ hii, double e0, double* __restrict__ sr,
                                      double* __restrict__ su, double* __restrict__ stt, double* __restrict__ sden) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int64_t i = idx[k];
  sr[k] = r[i];
  su[k] = u[i];
  stt[k] = t[i];
  sden[k] = e0 - hii[i];
}

__global__ void sub_scaled_kernel(double* __restrict__ y, const double* __restrict__ x, double a, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] -= a * x[i];
}

}  // namespace

// Network state of one context.
struct Learned {
  float *w = nullptr, *we = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
  __nv_bfloat16* w16 = nullptr;
  bool trained = false;
  double S = 0.5;
  int adam_step = 0;
  MlpBatch mb;
  void alloc() {
    if (w) return;
    w = (float*)dev_alloc(sizeof(float) * kNParams);
    we = (float*)dev_alloc(sizeof(float) * kNParams);
    m = (float*)dev_alloc(sizeof(float) * kNParams);
    v = (float*)dev_alloc(sizeof(float) * kNParams);
    g = (float*)dev_alloc(sizeof(float) * kNParams);
    w16 = (__nv_bfloat16*)dev_alloc(sizeof(__nv_bfloat16) * kNParams);
  }
  ~Learned() {
    mb.release();
    for (void* p : {(void*)w, (void*)we, (void*)m, (void*)v, (void*)g, (void*)w16}) cudaFree(p);
  }
};

void free_learned(sbdgpu_ctx* c) {
  delete c->learned;
  c->learned = nullptr;
}

bool learned_ready(const sbdgpu_ctx* c) { return c->learned && c->learned->trained; }

// The learned correction of the residual R into out (the network sees |R_i|,
// so out has R's sign convention).
void learned_precondition(sbdgpu_ctx* c, const double* R, double e0, double eps_reg, double* out) {
  Learned* L = c->learned;
  if (!L || !L->trained) throw Error{SBDGPU_ERR_STATE, "no trained preconditioner network on this context"};
  if (!c->tc_err) {
    c->tc_err = (int*)dev_alloc(sizeof(int));
    SBD_CUDA(cudaMemset(c->tc_err, 0, sizeof(int)));
  }
  InfArgs a;
  a.w16 = L->w16;
  a.we = L->we;
  a.R = R;
  a.hii = c->hii;
  a.astr = c->astr;
  a.bstr = c->bstr;
  a.out = out;
  a.n = c->N;
  a.nb = c->nb;
  a.nea = __builtin_popcountll(c->h_astr[0]);
  a.neb = __builtin_popcountll(c->h_bstr[0]);
  a.e0 = e0;
  a.eps_reg = eps_reg;
  a.S = L->S;
  a.sqrt_n = std::sqrt((double)c->N);
  a.err = c->tc_err;
  allow_dynamic_smem(reinterpret_cast<const void*>(mlp_infer_kernel), c->device);
  int sms = 148;
  SBD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  const size_t ntiles = (c->N + 127) / 128;
  const int grid = (int)std::min<size_t>(ntiles, (size_t)2 * sms);
  mlp_infer_kernel<<<grid, kInfThreads, kInfSmem, c->stream>>>(a);
  SBD_CUDA(cudaGetLastError());
}

// Harvest (u, r, t) triples on this context's system and train the network.
void train_learned(sbdgpu_ctx* c, const sbdgpu_learn_opts* o, double* loss_trace, double* seconds) {
  if (o->pairs < 1 || o->cycle < 1 || o->cycle > 32 || o->cg_iters < 1 || o->samples < 64 || o->steps < 0)
    throw Error{SBDGPU_ERR_ARG, "learn options: pairs >= 1, 1 <= cycle <= 32, cg_iters >= 1, samples >= 64"};
  build_tables(c);
  compute_hii(c);
  ensure_scratch(c);
  if (!c->learned) c->learned = new Learned();
  Learned* L = c->learned;
  L->alloc();
  cudaStream_t st = c->stream;
  const size_t n = c->N;
  auto t_start = std::chrono::steady_clock::now();
  // working vectors: u, Hu / Lanczos, Lanczos (2), solution t, r, two MINRES directions
  std::vector<double*> vec(8, nullptr);
  struct FreeV {
    std::vector<double*>* v;
    cudaStream_t s;
    ~FreeV() {
      cudaStreamSynchronize(s);
      for (auto p : *v) cudaFree(p);
    }
  } guard{&vec, st};
  for (auto& p : vec) p = (double*)dev_alloc(sizeof(double) * n);
  double *u = vec[0], *q = vec[1], *res = vec[2], *p = vec[3], *tt = vec[4], *r = vec[5];
  const int m_top = o->samples / 2, m_rand = o->samples - o->samples / 2;
  const int ms = m_top + m_rand;
  // harvested samples, [pair][sample]
  int64_t* s_idx = (int64_t*)dev_alloc(sizeof(int64_t) * (size_t)o->pairs * ms);
  double* s_val = (double*)dev_alloc(sizeof(double) * (size_t)o->pairs * ms * 5);  // r, u, t, den, wt
  float* s_X = (float*)dev_alloc(sizeof(float) * (size_t)o->pairs * ms * kF);
  unsigned long long* hist = (unsigned long long*)dev_alloc(sizeof(unsigned long long) * 256);
  int* cnt = (int*)dev_alloc(sizeof(int));
  struct FreeS {
    void* a[5];
    ~FreeS() {
      for (auto x : a) cudaFree(x);
    }
  } guard_s{{s_idx, s_val, s_X, hist, cnt}};
  std::mt19937_64 rng(o->seed);
  const int nea = __builtin_popcountll(c->h_astr[0]), neb = __builtin_popcountll(c->h_bstr[0]);
  const double sqrt_n = std::sqrt((double)n);
  // the Davidson run that generates the triples: FP64, the reference's
  // algorithm, restarted every `cycle` steps from the aufbau determinant
  std::vector<double> Wh(n, 0.0);
  Wh[0] = 1.0;
  sbdgpu_opts dopt{};
  dopt.max_it = 1;
  dopt.max_nb = o->cycle;
  dopt.eps = 0.0;
  dopt.max_time = 1e30;
  dopt.precision = SBDGPU_FP64;
  auto dot = [&](const double* x, const double* y) { return sbdgpu::dot(c, x, y, n); };
  for (int k = 0; k < o->pairs; k++) {
    double e = 0.0;
    int steps = 0;
    const int rc = sbdgpu_davidson(c, &dopt, Wh.data(), &e, nullptr, nullptr, 0, &steps);
    if (rc != SBDGPU_OK) throw Error{rc, "harvest Davidson cycle: " + c->err};
    SBD_CUDA(cudaMemcpyAsync(u, Wh.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
    apply_phase(c, u);
    scale(u, 1.0 / std::sqrt(dot(u, u)), n, st);
    sigma_fp64(c, u, q);
    const double theta = dot(u, q);
    // r = Hu - theta u, normalised (the Davidson loop normalises its residual)
    SBD_CUDA(cudaMemcpyAsync(r, q, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    sub_scaled_kernel<<<592, 256, 0, st>>>(r, u, theta, n);
    SBD_CUDA(cudaGetLastError());
    const double rn = std::sqrt(dot(r, r));
    if (!(rn > 0.0)) throw Error{SBDGPU_ERR_STATE, "harvest: zero residual (converged before the first triple)"};
    scale(r, 1.0 / rn, n, st);
    // MINRES on (I - uu^T)(H - theta)(I - uu^T) t = -r, t _|_ u: the operator
    // is symmetric but indefinite while theta is above the lowest eigenvalue,
    // so conjugate gradients would stop at the first negative curvature.
    // Lanczos vectors (kept orthogonal to u), the tridiagonal factored by
    // Givens rotations, t updated along the rotated directions (Paige and
    // Saunders, SIAM J. Numer. Anal. 12, 1975).  Buffers: vprev, v, p (the
    // Lanczos recurrence) and w1, w2 (the last two directions); tt holds t.
    double *vprev = res, *v = p, *pv = q, *w1 = vec[6], *w2 = vec[7];
    SBD_CUDA(cudaMemsetAsync(tt, 0, sizeof(double) * n, st));
    SBD_CUDA(cudaMemsetAsync(vprev, 0, sizeof(double) * n, st));
    SBD_CUDA(cudaMemsetAsync(w1, 0, sizeof(double) * n, st));
    SBD_CUDA(cudaMemsetAsync(w2, 0, sizeof(double) * n, st));
    SBD_CUDA(cudaMemcpyAsync(v, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    scale(v, -1.0, n, st);  // b = -r (already orthogonal to u), |b| = 1
    const double beta1 = std::sqrt(dot(v, v));
    double beta = beta1, phibar = beta1;
    double c1 = 1.0, s1 = 0.0, c2 = 1.0, s2 = 0.0;  // rotations k-1 and k-2
    scale(v, 1.0 / beta1, n, st);
    for (int it = 0; it < o->cg_iters; it++) {
      sigma_fp64(c, v, pv);
      sub_scaled_kernel<<<592, 256, 0, st>>>(pv, v, theta, n);
      sub_scaled_kernel<<<592, 256, 0, st>>>(pv, u, dot(u, pv), n);
      if (it > 0) sub_scaled_kernel<<<592, 256, 0, st>>>(pv, vprev, beta, n);
      const double alpha = dot(v, pv);
      sub_scaled_kernel<<<592, 256, 0, st>>>(pv, v, alpha, n);
      const double beta_next = std::sqrt(dot(pv, pv));
      // column it of the tridiagonal: (beta above, alpha, beta_next below)
      const double b_above = it > 0 ? beta : 0.0;
      const double eps_k = s2 * b_above, dbar = c2 * b_above;
      const double delta = c1 * dbar + s1 * alpha;
      const double gbar = -s1 * dbar + c1 * alpha;
      const double gamma = std::sqrt(gbar * gbar + beta_next * beta_next);
      if (!(gamma > 0.0)) break;
      const double ck = gbar / gamma, sk = beta_next / gamma;
      const double tau = ck * phibar;
      phibar = -sk * phibar;
      // w_new = (v - delta w1 - eps_k w2) / gamma, built in w2's buffer
      scale(w2, -eps_k, n, st);
      axpy(w2, v, 1.0, n, st);
      axpy(w2, w1, -delta, n, st);
      scale(w2, 1.0 / gamma, n, st);
      axpy(tt, w2, tau, n, st);
      std::swap(w1, w2);
      c2 = c1;
      s2 = s1;
      c1 = ck;
      s1 = sk;
      if (std::fabs(phibar) < 1e-4 * beta1 || !(beta_next > 1e-300)) break;
      // next Lanczos vector
      scale(pv, 1.0 / beta_next, n, st);
      std::swap(vprev, v);
      std::swap(v, pv);
      beta = beta_next;
    }
    const double tn = std::sqrt(dot(tt, tt));
    if (!(tn > 0.0)) throw Error{SBDGPU_ERR_STATE, "harvest: the correction solve made no progress"};
    scale(tt, 1.0 / tn, n, st);
    // samples: the determinants with the largest |t|^2 + |r|^2 (weight 1), and
    // uniform ones (weight n / their count, the rest of the vector's estimate)
    SBD_CUDA(cudaMemsetAsync(hist, 0, sizeof(unsigned long long) * 256, st));
    score_hist_kernel<<<592, 256, 0, st>>>(tt, r, n, hist);
    SBD_CUDA(cudaGetLastError());
    std::vector<unsigned long long> hh(256);
    SBD_CUDA(cudaMemcpyAsync(hh.data(), hist, sizeof(unsigned long long) * 256, cudaMemcpyDeviceToHost, st));
    SBD_CUDA(cudaStreamSynchronize(st));
    int bin_min = 255;
    unsigned long long acc = 0;
    while (bin_min > 0 && acc + hh[bin_min] <= (unsigned long long)m_top) acc += hh[bin_min--];
    bin_min++;
    int64_t* idx_k = s_idx + (size_t)k * ms;
    SBD_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), st));
    select_top_kernel<<<592, 256, 0, st>>>(tt, r, n, bin_min, m_top, idx_k, cnt);
    SBD_CUDA(cudaGetLastError());
    int ntop = 0;
    SBD_CUDA(cudaMemcpyAsync(&ntop, cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
    SBD_CUDA(cudaStreamSynchronize(st));
    ntop = std::min(ntop, m_top);
    std::vector<int64_t> ridx(ms - ntop);
    std::uniform_int_distribution<int64_t> pick(0, (int64_t)n - 1);
    for (auto& x : ridx) x = pick(rng);
    SBD_CUDA(cudaMemcpy(idx_k + ntop, ridx.data(), sizeof(int64_t) * ridx.size(), cudaMemcpyHostToDevice));
    double* sv = s_val + (size_t)k * ms * 5;
    gather_samples_kernel<<<(ms + 255) / 256, 256, 0, st>>>(idx_k, ms, r, u, tt, c->hii, theta, sv, sv + ms,
                                                           sv + 2 * ms, sv + 3 * ms);
    SBD_CUDA(cudaGetLastError());
    std::vector<double> wts(ms, 1.0);
    for (int i = ntop; i < ms; i++) wts[i] = (double)n / (double)(ms - ntop);
    SBD_CUDA(cudaMemcpy(sv + 4 * ms, wts.data(), sizeof(double) * ms, cudaMemcpyHostToDevice));
    feat_batch_kernel<<<(ms + 255) / 256, 256, 0, st>>>(idx_k, sv + 3 * ms, sv, c->astr, c->bstr, c->nb, nea, neb,
                                                       sqrt_n, ms, s_X + (size_t)k * ms * kF);
    SBD_CUDA(cudaGetLastError());
    SBD_CUDA(cudaStreamSynchronize(st));
  }
  auto t_harvest = std::chrono::steady_clock::now();
  // training: Adam over the triples in turn, one whole triple per step
  {
    std::vector<double> w0(kNParams);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (int i = 0; i < kNParams; i++) {
      double sdev = 0.0;
      if (i < ob1) sdev = std::sqrt(2.0 / kF);
      else if (i >= oW2 && i < ob2) sdev = std::sqrt(2.0 / kHid);
      else if (i >= ow3 && i < ob3) sdev = 0.01;
      w0[i] = sdev * nd(rng);
    }
    std::vector<float> wf(w0.begin(), w0.end());
    SBD_CUDA(cudaMemcpy(L->w, wf.data(), sizeof(float) * kNParams, cudaMemcpyHostToDevice));
    SBD_CUDA(cudaMemset(L->m, 0, sizeof(float) * kNParams));
    SBD_CUDA(cudaMemset(L->v, 0, sizeof(float) * kNParams));
    round_weights_kernel<<<64, 256, 0, st>>>(L->w, kNParams, L->we, L->w16);
    SBD_CUDA(cudaGetLastError());
    L->adam_step = 0;
  }
  L->mb.ensure(ms);
  double* d_trace = nullptr;
  if (loss_trace && o->steps > 0) d_trace = (double*)dev_alloc(sizeof(double) * o->steps);
  struct FreeT {
    double* p;
    ~FreeT() { cudaFree(p); }
  } guard_t{d_trace};
  for (int step = 0; step < o->steps; step++) {
    const int k = step % o->pairs;
    const double* sv = s_val + (size_t)k * ms * 5;
    SBD_CUDA(cudaMemcpyAsync(L->mb.X, s_X + (size_t)k * ms * kF, sizeof(float) * (size_t)ms * kF,
                             cudaMemcpyDeviceToDevice, st));
    SBD_CUDA(cudaMemsetAsync(L->g, 0, sizeof(float) * kNParams, st));
    mlp_loss_grad(L->mb, L->we, ms, sv, sv + 3 * ms, sv + ms, sv + 2 * ms, sv + 4 * ms, L->S, 1e-12, L->g, d_trace,
                  step, st);
    L->adam_step++;
    adam_kernel<<<64, 256, 0, st>>>(L->w, L->m, L->v, L->g, kNParams, o->lr, 0.9f, 0.999f, 1e-8f, L->adam_step,
                                    L->we, L->w16);
    SBD_CUDA(cudaGetLastError());
  }
  if (d_trace) SBD_CUDA(cudaMemcpyAsync(loss_trace, d_trace, sizeof(double) * o->steps, cudaMemcpyDeviceToHost, st));
  SBD_CUDA(cudaStreamSynchronize(st));
  L->trained = true;
  auto t_end = std::chrono::steady_clock::now();
  if (seconds) {
    seconds[0] = std::chrono::duration<double>(t_harvest - t_start).count();
    seconds[1] = std::chrono::duration<double>(t_end - t_harvest).count();
  }
}

void learned_get(sbdgpu_ctx* c, float* w, int* n) {
  if (n) *n = kNParams;
  if (!w) return;
  if (!learned_ready(c)) throw Error{SBDGPU_ERR_STATE, "no trained preconditioner network on this context"};
  SBD_CUDA(cudaMemcpy(w, c->learned->w, sizeof(float) * kNParams, cudaMemcpyDeviceToHost));
}

void learned_set(sbdgpu_ctx* c, const float* w, int n) {
  if (!w || n != kNParams) throw Error{SBDGPU_ERR_ARG, "network weights: expected " + std::to_string(kNParams)};
  if (!c->learned) c->learned = new Learned();
  Learned* L = c->learned;
  L->alloc();
  SBD_CUDA(cudaMemcpy(L->w, w, sizeof(float) * kNParams, cudaMemcpyHostToDevice));
  SBD_CUDA(cudaMemset(L->m, 0, sizeof(float) * kNParams));
  SBD_CUDA(cudaMemset(L->v, 0, sizeof(float) * kNParams));
  round_weights_kernel<<<64, 256, 0, c->stream>>>(L->w, kNParams, L->we, L->w16);
  SBD_CUDA(cudaGetLastError());
  SBD_CUDA(cudaStreamSynchronize(c->stream));
  L->trained = true;
}

}  // namespace sbdgpu

// Gradient check entry point: loss and gradient of the training kernels for
// given master weights and features, on `device`.
extern "C" int sbdgpu_mlp_loss_grad(int device, const float* w, int B, const float* X, const double* r,
                                    const double* den, const double* u, const double* t, const double* wt, double S,
                                    double eps_reg, double* loss, float* grad) {
  using namespace sbdgpu;
  if (!w || B < 1 || !X || !r || !den || !u || !t || !wt || !loss || !grad) return SBDGPU_ERR_ARG;
  MlpBatch mb;
  std::vector<void*> bufs;
  auto alloc = [&](size_t bytes) {
    void* p = dev_alloc(bytes);
    bufs.push_back(p);
    return p;
  };
  int rc = SBDGPU_OK;
  cudaStream_t st = nullptr;
  try {
    SBD_CUDA(cudaSetDevice(device));
    SBD_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    mb.ensure(B);
    float* dw = (float*)alloc(sizeof(float) * kNParams);
    float* we = (float*)alloc(sizeof(float) * kNParams);
    __nv_bfloat16* w16 = (__nv_bfloat16*)alloc(sizeof(__nv_bfloat16) * kNParams);
    float* dg = (float*)alloc(sizeof(float) * kNParams);
    double* dv[5];
    const double* hv[5] = {r, den, u, t, wt};
    for (int i = 0; i < 5; i++) {
      dv[i] = (double*)alloc(sizeof(double) * B);
      SBD_CUDA(cudaMemcpyAsync(dv[i], hv[i], sizeof(double) * B, cudaMemcpyHostToDevice, st));
    }
    double* dloss = (double*)alloc(sizeof(double));
    SBD_CUDA(cudaMemcpyAsync(dw, w, sizeof(float) * kNParams, cudaMemcpyHostToDevice, st));
    SBD_CUDA(cudaMemcpyAsync(mb.X, X, sizeof(float) * (size_t)B * kF, cudaMemcpyHostToDevice, st));
    SBD_CUDA(cudaMemsetAsync(dg, 0, sizeof(float) * kNParams, st));
    round_weights_kernel<<<64, 256, 0, st>>>(dw, kNParams, we, w16);
    SBD_CUDA(cudaGetLastError());
    mlp_loss_grad(mb, we, B, dv[0], dv[1], dv[2], dv[3], dv[4], S, eps_reg, dg, dloss, 0, st);
    SBD_CUDA(cudaMemcpyAsync(grad, dg, sizeof(float) * kNParams, cudaMemcpyDeviceToHost, st));
    SBD_CUDA(cudaMemcpyAsync(loss, dloss, sizeof(double), cudaMemcpyDeviceToHost, st));
    SBD_CUDA(cudaStreamSynchronize(st));
  } catch (const Error& e) {
    rc = e.code;
  }
  if (st) cudaStreamSynchronize(st);
  mb.release();
  for (void* p : bufs) cudaFree(p);
  if (st) cudaStreamDestroy(st);
  return rc;
}
