// FP64 sigma build, sigma = H*C on the alpha x beta product basis.
//
// Replaces the direct mult of chemistry/tpb/mult.h:387-648.  The reference
// evaluates every matrix element with Hij on interleaved determinants; here the
// Hamiltonian is split by the spin structure of the excitation, in the
// alpha-string-major sign convention (identical to the reference's up to the
// diagonal phase applied at the C ABI):
//
//  rows kernel (alpha)   sigma[ia,:]  = hii[ia,:] C[ia,:] + sum_{ja in D(ia)} d C[ja,:]
//                                       + sum_{ja in S(ia)} s (F + Jb_pq[:]) C[ja,:]
//                        (task type 2 of the reference: alpha singles/doubles)
//  rows kernel (beta)    the same kernel on the transposed vector C^T, with the
//                        beta tables and Ja (task type 1), added back transposed
//  alpha-beta kernel     sigma[ia,ib] += sum_{ja in S(ia)} sum_{jb in S(ib)}
//                                        s_a s_b (pq|rs) C[ja,jb]   (task type 0)
//
// The rows kernel streams whole rows of C (coalesced) for every table entry of
// its bra row.  The alpha-beta kernel holds one source row C[ja,:] and the
// integral rows (pq|.) of a group of ja's singles in shared memory, streams the
// beta singles (sliced ELL, coalesced) once per group, and adds each group's
// contributions to sigma rows ia with FP64 atomics.
#include <algorithm>

#include "internal.cuh"

namespace sbdgpu {

namespace {

constexpr int kRowsThreads = 256;
constexpr int kRowsCols = 2;  // columns per thread

// sigma_row[ia][cols] (=) diag + sum over the bra's table entries, in the
// vector type T (double: plain path; float: mixed path, FP32 accumulation).
// J: [P][ncols] Coulomb coupling to the other spin's occupation.
template <typename T, bool kWithDiag>
__global__ void __launch_bounds__(kRowsThreads) rows_kernel(
    const T* __restrict__ C, T* __restrict__ S, size_t ncols, const double* __restrict__ hii,
    const int64_t* __restrict__ s_off, const int32_t* __restrict__ s_idx, const uint32_t* __restrict__ s_info,
    const double* __restrict__ s_val, const int64_t* __restrict__ d_off, const int32_t* __restrict__ d_idx,
    const double* __restrict__ d_val, const T* __restrict__ J) {
  size_t row = blockIdx.x;
  size_t c0 = (size_t)blockIdx.y * (kRowsThreads * kRowsCols) + threadIdx.x;
  T acc[kRowsCols];
  bool ok[kRowsCols];
#pragma unroll
  for (int u = 0; u < kRowsCols; u++) {
    size_t col = c0 + (size_t)u * kRowsThreads;
    ok[u] = col < ncols;
    acc[u] = (kWithDiag && ok[u]) ? (T)hii[row * ncols + col] * C[row * ncols + col] : (T)0;
  }
  int64_t b = s_off[row], e = s_off[row + 1];
  for (int64_t k = b; k < e; k++) {
    size_t j = (size_t)__ldg(&s_idx[k]);
    uint32_t info = __ldg(&s_info[k]);
    T v = (T)__ldg(&s_val[k]);
    T sg = (info & 0x80000000u) ? (T)-1 : (T)1;
    const T* Jr = J + (size_t)((info >> 12) & 0xFFFu) * ncols;
    const T* Cr = C + j * ncols;
#pragma unroll
    for (int u = 0; u < kRowsCols; u++) {
      size_t col = c0 + (size_t)u * kRowsThreads;
      if (ok[u]) acc[u] += (v + sg * Jr[col]) * Cr[col];
    }
  }
  b = d_off[row];
  e = d_off[row + 1];
  for (int64_t k = b; k < e; k++) {
    size_t j = (size_t)__ldg(&d_idx[k]);
    T v = (T)__ldg(&d_val[k]);
    const T* Cr = C + j * ncols;
#pragma unroll
    for (int u = 0; u < kRowsCols; u++) {
      size_t col = c0 + (size_t)u * kRowsThreads;
      if (ok[u]) acc[u] += v * Cr[col];
    }
  }
#pragma unroll
  for (int u = 0; u < kRowsCols; u++) {
    size_t col = c0 + (size_t)u * kRowsThreads;
    if (ok[u]) S[row * ncols + col] = acc[u];
  }
}

constexpr int kAbThreads = 512;

// One CTA per (source alpha string ja, group of G of its singles).
template <typename T, int G>
__global__ void __launch_bounds__(kAbThreads) ab_kernel(
    const T* __restrict__ C, T* __restrict__ S, size_t nb, int P, const T* __restrict__ vf,
    const int64_t* __restrict__ a_off, const int32_t* __restrict__ a_idx, const uint32_t* __restrict__ a_info,
    const int64_t* __restrict__ sell_off, const int32_t* __restrict__ sell_w, const uint32_t* __restrict__ sell,
    size_t nslice) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* crow = reinterpret_cast<T*>(smem_raw);  // [nb]
  T* vsub = crow + nb;                       // [G][P]
  __shared__ int tgt[G];
  __shared__ T sgn[G];
  size_t ja = blockIdx.x;
  int64_t k0 = a_off[ja] + (int64_t)blockIdx.y * G;
  int64_t k1 = min(k0 + G, a_off[ja + 1]);
  if (k0 >= k1) return;
  int gcount = (int)(k1 - k0);
  for (size_t i = threadIdx.x; i < nb; i += blockDim.x) crow[i] = C[ja * nb + i];
  for (int g = 0; g < G; g++) {
    if (g < gcount) {
      uint32_t info = a_info[k0 + g];
      int pq = (info >> 12) & 0xFFFu;
      for (int i = threadIdx.x; i < P; i += blockDim.x) vsub[g * P + i] = vf[(size_t)pq * P + i];
      if (threadIdx.x == 0) {
        tgt[g] = a_idx[k0 + g];
        sgn[g] = (info & 0x80000000u) ? (T)-1 : (T)1;
      }
    } else {
      for (int i = threadIdx.x; i < P; i += blockDim.x) vsub[g * P + i] = (T)0;
    }
  }
  __syncthreads();
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (size_t sl = warp; sl < nslice; sl += nwarp) {
    size_t ib = sl * 32 + lane;
    int w = sell_w[sl];
    const uint32_t* ent = sell + sell_off[sl] + lane;
    T y[G];
#pragma unroll
    for (int g = 0; g < G; g++) y[g] = (T)0;
    for (int t = 0; t < w; t++) {
      uint32_t e = __ldg(&ent[(size_t)t * 32]);
      if (e == kSellInvalid) continue;
      T x = crow[e & 0xFFFFu];
      if (e & 0x80000000u) x = -x;
      const T* vr = vsub + ((e >> 16) & 0xFFFu);
#pragma unroll
      for (int g = 0; g < G; g++) y[g] += vr[g * P] * x;
    }
    if (ib < nb) {
#pragma unroll
      for (int g = 0; g < G; g++)
        if (g < gcount) atomicAdd(&S[(size_t)tgt[g] * nb + ib], sgn[g] * y[g]);
    }
  }
}

template <typename T, int G>
void launch_ab(sbdgpu_ctx* c, const T* C, T* S, const T* vf, size_t smem) {
  const SpinTables& ta = c->tab[0];
  const SpinTables& tb = c->tab[1];
  SBD_CUDA(cudaFuncSetAttribute(ab_kernel<T, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((unsigned)c->na, (unsigned)((ta.max_s + G - 1) / G));
  if (grid.y == 0) return;
  ab_kernel<T, G><<<grid, kAbThreads, smem, c->stream>>>(C, S, c->nb, c->P, vf, ta.s_off, ta.s_idx, ta.s_info,
                                                          tb.sell_off, tb.sell_w, tb.sell, tb.nslice);
  SBD_CUDA(cudaGetLastError());
}

// The full kernel sequence of one sigma on given scratch (ct, st: na*nb of T).
template <typename T>
void sigma_launch(sbdgpu_ctx* c, const T* C, T* S, T* ct, T* st, const T* ja, const T* jb, const T* vf,
                  bool events) {
  const SpinTables& ta = c->tab[0];
  const SpinTables& tb = c->tab[1];
  cudaStream_t s = c->stream;
  if (events) SBD_CUDA(cudaEventRecord(c->ev[0], s));
  {
    dim3 g((unsigned)c->na, (unsigned)((c->nb + kRowsThreads * kRowsCols - 1) / (kRowsThreads * kRowsCols)));
    rows_kernel<T, true><<<g, kRowsThreads, 0, s>>>(C, S, c->nb, c->hii, ta.s_off, ta.s_idx, ta.s_info, ta.s_val,
                                                    ta.d_off, ta.d_idx, ta.d_val, jb);
    SBD_CUDA(cudaGetLastError());
  }
  if (events) SBD_CUDA(cudaEventRecord(c->ev[1], s));
  transpose(C, ct, c->na, c->nb, s);
  {
    dim3 g((unsigned)c->nb, (unsigned)((c->na + kRowsThreads * kRowsCols - 1) / (kRowsThreads * kRowsCols)));
    rows_kernel<T, false><<<g, kRowsThreads, 0, s>>>(ct, st, c->na, nullptr, tb.s_off, tb.s_idx, tb.s_info,
                                                     tb.s_val, tb.d_off, tb.d_idx, tb.d_val, ja);
    SBD_CUDA(cudaGetLastError());
  }
  transpose_add(st, S, c->nb, c->na, s);
  if (events) SBD_CUDA(cudaEventRecord(c->ev[2], s));
  int dev_smem = 0;
  SBD_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
  size_t budget = (size_t)dev_smem - 1024;
  size_t base = sizeof(T) * c->nb;
  size_t per = sizeof(T) * c->P;
  if (c->nb > 65536) throw Error{SBDGPU_ERR_LIMIT, "alpha-beta kernel: more than 65536 beta strings"};
  if (base + per > budget)
    throw Error{SBDGPU_ERR_LIMIT, "alpha-beta kernel: one beta row and integral row exceed shared memory"};
  size_t gmax = (budget - base) / per;
  if (gmax >= 16)
    launch_ab<T, 16>(c, C, S, vf, base + 16 * per);
  else if (gmax >= 8)
    launch_ab<T, 8>(c, C, S, vf, base + 8 * per);
  else if (gmax >= 4)
    launch_ab<T, 4>(c, C, S, vf, base + 4 * per);
  else if (gmax >= 2)
    launch_ab<T, 2>(c, C, S, vf, base + 2 * per);
  else
    launch_ab<T, 1>(c, C, S, vf, base + per);
  if (events) SBD_CUDA(cudaEventRecord(c->ev[3], s));
}

}  // namespace

void sigma_fp64(sbdgpu_ctx* c, const double* C, double* S) {
  build_tables(c);
  compute_hii(c);
  ensure_scratch(c);
  sigma_launch<double>(c, C, S, c->ct, c->st, c->ja, c->jb, c->vf, true);
}

void sigma_fp64_prepared(sbdgpu_ctx* c, const double* C, double* S, double* ct, double* st) {
  sigma_launch<double>(c, C, S, ct, st, c->ja, c->jb, c->vf, false);
}

void sigma_fp32(sbdgpu_ctx* c, const float* C, float* S) {
  build_tables(c);
  compute_hii(c);
  ensure_scratch(c);
  ensure_fp32(c);
  // the FP64 scratch vectors hold the FP32 transposes (half their size)
  sigma_launch<float>(c, C, S, reinterpret_cast<float*>(c->ct), reinterpret_cast<float*>(c->st), c->ja32, c->jb32,
                      c->vf32, true);
}

}  // namespace sbdgpu
