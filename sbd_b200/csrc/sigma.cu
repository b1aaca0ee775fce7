// FP64 sigma build, sigma = H*C on the alpha x beta product basis.
//
// Replaces the direct mult of chemistry/tpb/mult.h:387-648.  The reference
// evaluates every matrix element with Hij on interleaved determinants; here the
// Hamiltonian is split by the spin structure of the excitation, in the
// alpha-string-major sign convention (identical to the reference's up to the
// diagonal phase applied at the C ABI):
//
//  same-spin (alpha)     sigma[ia,:]  = hii[ia,:] C[ia,:] + sum_{ja in D(ia)} d C[ja,:]
//                                       + sum_{ja in S(ia)} s (F + Jb_pq[:]) C[ja,:]
//                        (task type 2 of the reference: alpha singles/doubles)
//  same-spin (beta)      the same kernel on the transposed vector C^T, with the
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


// 16-byte vector of T: VW = 16 / sizeof(T) consecutive columns per thread.
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using V = float4;
  static constexpr int W = 4;
  __device__ static void get(const V& v, float (&x)[4]) { x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w; }
  __device__ static V make(const float (&x)[4]) { return make_float4(x[0], x[1], x[2], x[3]); }
};
template <>
struct Vec16<double> {
  using V = double2;
  static constexpr int W = 2;
  __device__ static void get(const V& v, double (&x)[2]) { x[0] = v.x; x[1] = v.y; }
  __device__ static V make(const double (&x)[2]) { return make_double2(x[0], x[1]); }
};

// The rows kernel with one 16-byte vector of columns per thread: the same sums
// in the same order per column as rows_kernel, with a quarter (FP32) or half
// (FP64) of its load instructions, which bound it in the L1/TEX pipe.  Needs
// ncols % (16 / sizeof(T)) == 0 and 16-byte aligned C, S and J rows.
template <typename T, bool kWithDiag>
__global__ void __launch_bounds__(kRowsThreads) rows_vec_kernel(
    const T* __restrict__ C, T* __restrict__ S, size_t ncols, const double* __restrict__ hii,
    const int64_t* __restrict__ s_off, const int32_t* __restrict__ s_idx, const uint32_t* __restrict__ s_info,
    const double* __restrict__ s_val, const int64_t* __restrict__ d_off, const int32_t* __restrict__ d_idx,
    const double* __restrict__ d_val, const T* __restrict__ J) {
  using VT = Vec16<T>;
  using V = typename VT::V;
  constexpr int W = VT::W;
  const size_t row = blockIdx.x;
  const size_t col = ((size_t)blockIdx.y * kRowsThreads + threadIdx.x) * W;
  if (col >= ncols) return;
  T acc[W];
  if (kWithDiag) {
    V c = *reinterpret_cast<const V*>(C + row * ncols + col);
    T x[W];
    VT::get(c, x);
#pragma unroll
    for (int u = 0; u < W; u++) acc[u] = (T)hii[row * ncols + col + u] * x[u];
  } else {
#pragma unroll
    for (int u = 0; u < W; u++) acc[u] = (T)0;
  }
  int64_t b = s_off[row], e = s_off[row + 1];
  for (int64_t k = b; k < e; k++) {
    const size_t j = (size_t)__ldg(&s_idx[k]);
    const uint32_t info = __ldg(&s_info[k]);
    const T v = (T)__ldg(&s_val[k]);
    const T sg = (info & 0x80000000u) ? (T)-1 : (T)1;
    T jr[W], cr[W];
    VT::get(__ldg(reinterpret_cast<const V*>(J + (size_t)((info >> 12) & 0xFFFu) * ncols + col)), jr);
    VT::get(__ldg(reinterpret_cast<const V*>(C + j * ncols + col)), cr);
#pragma unroll
    for (int u = 0; u < W; u++) acc[u] += (v + sg * jr[u]) * cr[u];
  }
  b = d_off[row];
  e = d_off[row + 1];
  for (int64_t k = b; k < e; k++) {
    const size_t j = (size_t)__ldg(&d_idx[k]);
    const T v = (T)__ldg(&d_val[k]);
    T cr[W];
    VT::get(__ldg(reinterpret_cast<const V*>(C + j * ncols + col)), cr);
#pragma unroll
    for (int u = 0; u < W; u++) acc[u] += v * cr[u];
  }
  *reinterpret_cast<V*>(S + row * ncols + col) = VT::make(acc);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// Same-spin rows: the vector kernel when the rows allow it, else rows_kernel.
template <typename T, bool kWithDiag>
void launch_rows(const T* C, T* S, size_t nrows, size_t ncols, const double* hii, const SpinTables& t, const T* J,
                 cudaStream_t s) {
  constexpr int W = Vec16<T>::W;
  if (ncols % W == 0 && aligned16(C) && aligned16(S) && aligned16(J) && (!kWithDiag || aligned16(hii))) {
    dim3 g((unsigned)nrows, (unsigned)((ncols / W + kRowsThreads - 1) / kRowsThreads));
    rows_vec_kernel<T, kWithDiag><<<g, kRowsThreads, 0, s>>>(C, S, ncols, hii, t.s_off, t.s_idx, t.s_info, t.s_val,
                                                             t.d_off, t.d_idx, t.d_val, J);
  } else {
    dim3 g((unsigned)nrows, (unsigned)((ncols + kRowsThreads * kRowsCols - 1) / (kRowsThreads * kRowsCols)));
    rows_kernel<T, kWithDiag><<<g, kRowsThreads, 0, s>>>(C, S, ncols, hii, t.s_off, t.s_idx, t.s_info, t.s_val,
                                                         t.d_off, t.d_idx, t.d_val, J);
  }
  SBD_CUDA(cudaGetLastError());
}

// Row stride (elements) of the integral block in shared memory: G values per
// beta pair index rs, padded by 16 bytes so that the 16-byte vector loads of a
// warp (random rs per lane) spread over 8 different 4-bank windows.
template <typename T, int G>
__host__ __device__ constexpr int ab_vstride() {
  return G * (int)sizeof(T) >= 16 ? G + 16 / (int)sizeof(T) : G;
}

template <typename T, int G>
__device__ __forceinline__ void ab_accumulate(const T* __restrict__ vr, T x, T (&y)[G]) {
  if constexpr (G * sizeof(T) >= 16) {
    constexpr int W = 16 / sizeof(T);
#pragma unroll
    for (int g = 0; g < G; g += W) {
      if constexpr (sizeof(T) == 4) {
        float4 v = *reinterpret_cast<const float4*>(vr + g);
        y[g] += v.x * x;
        y[g + 1] += v.y * x;
        y[g + 2] += v.z * x;
        y[g + 3] += v.w * x;
      } else {
        double2 v = *reinterpret_cast<const double2*>(vr + g);
        y[g] += v.x * x;
        y[g + 1] += v.y * x;
      }
    }
  } else {
#pragma unroll
    for (int g = 0; g < G; g++) y[g] += vr[g] * x;
  }
}

// One CTA per (source alpha string ja, group of G of its singles).  Shared
// memory: the source row C[ja,:] and, for every folded beta pair index rs, the
// G integrals (pq_g|rs) of the group's alpha singles, contiguous.
template <typename T, int G, int NT>
__global__ void __launch_bounds__(NT) ab_kernel(
    const T* __restrict__ C, T* __restrict__ S, size_t nb, int P, const T* __restrict__ vf,
    const int64_t* __restrict__ a_off, const int32_t* __restrict__ a_idx, const uint32_t* __restrict__ a_info,
    const int64_t* __restrict__ sell_off, const int32_t* __restrict__ sell_w, const uint32_t* __restrict__ sell,
    size_t nslice) {
  constexpr int VS = ab_vstride<T, G>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* crow = reinterpret_cast<T*>(smem_raw);  // [nb], padded to 16 bytes
  T* vsub = reinterpret_cast<T*>(smem_raw + ((nb * sizeof(T) + 15) & ~size_t(15)));  // [P][VS]
  __shared__ int tgt[G];
  __shared__ T sgn[G];
  __shared__ int pqs[G];
  size_t ja = blockIdx.x;
  int64_t k0 = a_off[ja] + (int64_t)blockIdx.y * G;
  int64_t k1 = min(k0 + G, a_off[ja + 1]);
  if (k0 >= k1) return;
  int gcount = (int)(k1 - k0);
  if (threadIdx.x < G) {
    int g = threadIdx.x;
    if (g < gcount) {
      uint32_t info = a_info[k0 + g];
      pqs[g] = (info >> 12) & 0xFFFu;
      tgt[g] = a_idx[k0 + g];
      sgn[g] = (info & 0x80000000u) ? (T)-1 : (T)1;
    } else {
      pqs[g] = -1;
      tgt[g] = 0;
      sgn[g] = (T)0;
    }
  }
  for (size_t i = threadIdx.x; i < nb; i += blockDim.x) crow[i] = C[ja * nb + i];
  __syncthreads();
  for (int i = threadIdx.x; i < P * G; i += blockDim.x) {
    int g = i / P, rs = i - g * P;  // consecutive threads read consecutive rs of one integral row
    int pq = pqs[g];
    vsub[rs * VS + g] = pq >= 0 ? vf[(size_t)pq * P + rs] : (T)0;
  }
  __syncthreads();
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (size_t sl = warp; sl < nslice; sl += nwarp) {
    size_t ib = sl * 32 + lane;
    if (ib >= nb) continue;  // padding lane of the last slice (no warp-wide operation below)
    int w = sell_w[sl];
    const uint32_t* ent = sell + sell_off[sl] + lane;
    T y[G];
#pragma unroll
    for (int g = 0; g < G; g++) y[g] = (T)0;
    // four entries in flight per lane: the global loads of the sliced-ELL
    // entries and the dependent shared-memory loads overlap
    int t = 0;
    for (; t + 4 <= w; t += 4) {
      uint32_t e[4];
#pragma unroll
      for (int u = 0; u < 4; u++) e[u] = __ldg(&ent[(size_t)(t + u) * 32]);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        if (e[u] == kSellInvalid) continue;
        T x = crow[e[u] & 0xFFFFu];
        if (e[u] & 0x80000000u) x = -x;
        ab_accumulate<T, G>(vsub + ((e[u] >> 16) & 0xFFFu) * VS, x, y);
      }
    }
    for (; t < w; t++) {
      uint32_t e = __ldg(&ent[(size_t)t * 32]);
      if (e == kSellInvalid) continue;
      T x = crow[e & 0xFFFFu];
      if (e & 0x80000000u) x = -x;
      ab_accumulate<T, G>(vsub + ((e >> 16) & 0xFFFu) * VS, x, y);
    }
    if (ib < nb) {
#pragma unroll
      for (int g = 0; g < G; g++)
        if (g < gcount) atomicAdd(&S[(size_t)tgt[g] * nb + ib], sgn[g] * y[g]);
    }
  }
}

template <typename T, int G>
size_t ab_smem(size_t nb, int P) {
  return ((nb * sizeof(T) + 15) & ~size_t(15)) + (size_t)P * ab_vstride<T, G>() * sizeof(T);
}

// 512 threads while two CTAs fit in shared memory, else 1024 so that one CTA
// still keeps 32 warps resident per SM.
template <typename T, int G>
void launch_ab(sbdgpu_ctx* c, const T* C, T* S, const T* vf, size_t smem) {
  const SpinTables& ta = c->tab[0];
  const SpinTables& tb = c->tab[1];
  dim3 grid((unsigned)c->na, (unsigned)((ta.max_s + G - 1) / G));
  if (grid.y == 0) return;
  if (2 * (smem + 1024) <= 228 * 1024) {
    allow_dynamic_smem(reinterpret_cast<const void*>(ab_kernel<T, G, 512>), c->device);
    ab_kernel<T, G, 512><<<grid, 512, smem, c->stream>>>(C, S, c->nb, c->P, vf, ta.s_off, ta.s_idx, ta.s_info,
                                                         tb.sell_off, tb.sell_w, tb.sell, tb.nslice);
  } else {
    allow_dynamic_smem(reinterpret_cast<const void*>(ab_kernel<T, G, 1024>), c->device);
    ab_kernel<T, G, 1024><<<grid, 1024, smem, c->stream>>>(C, S, c->nb, c->P, vf, ta.s_off, ta.s_idx, ta.s_info,
                                                           tb.sell_off, tb.sell_w, tb.sell, tb.nslice);
  }
  SBD_CUDA(cudaGetLastError());
}

// The full kernel sequence of one sigma on given scratch (ct, st: na*nb of T).
template <typename T>
void sigma_launch(sbdgpu_ctx* c, const T* C, T* S, T* ct, T* st, const T* ja, const T* jb, const T* vf,
                  bool events) {
  cudaStream_t s = c->stream;
  const SpinTables& ta = c->tab[0];
  const SpinTables& tb = c->tab[1];
  if (events) SBD_CUDA(cudaEventRecord(c->ev[0], s));
  launch_rows<T, true>(C, S, c->na, c->nb, c->hii, ta, jb, s);
  if (events) SBD_CUDA(cudaEventRecord(c->ev[1], s));
  transpose(C, ct, c->na, c->nb, s);
  launch_rows<T, false>(ct, st, c->nb, c->na, nullptr, tb, ja, s);
  transpose_add(st, S, c->nb, c->na, s);
  if (events) SBD_CUDA(cudaEventRecord(c->ev[2], s));
  int dev_smem = 0;
  SBD_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
  size_t budget = (size_t)dev_smem - 1024;
  if (c->nb > 65536) throw Error{SBDGPU_ERR_LIMIT, "alpha-beta kernel: more than 65536 beta strings"};
  size_t nb = c->nb;
  int P = c->P;
  if (ab_smem<T, 16>(nb, P) <= budget)
    launch_ab<T, 16>(c, C, S, vf, ab_smem<T, 16>(nb, P));
  else if (ab_smem<T, 8>(nb, P) <= budget)
    launch_ab<T, 8>(c, C, S, vf, ab_smem<T, 8>(nb, P));
  else if (ab_smem<T, 4>(nb, P) <= budget)
    launch_ab<T, 4>(c, C, S, vf, ab_smem<T, 4>(nb, P));
  else if (ab_smem<T, 2>(nb, P) <= budget)
    launch_ab<T, 2>(c, C, S, vf, ab_smem<T, 2>(nb, P));
  else if (ab_smem<T, 1>(nb, P) <= budget)
    launch_ab<T, 1>(c, C, S, vf, ab_smem<T, 1>(nb, P));
  else
    throw Error{SBDGPU_ERR_LIMIT, "alpha-beta kernel: one beta row and integral row exceed shared memory"};
  if (events) SBD_CUDA(cudaEventRecord(c->ev[3], s));
}

template <int G>
void preload_ab(int device) {
  allow_dynamic_smem(reinterpret_cast<const void*>(ab_kernel<double, G, 512>), device);
  allow_dynamic_smem(reinterpret_cast<const void*>(ab_kernel<double, G, 1024>), device);
}

}  // namespace

// Loads every kernel that an FP64 sigma build can launch on the current
// device now (and sets the alpha-beta kernels' shared-memory limit), instead
// of at first launch, where CUDA's lazy module loading may allocate.
void preload_fp64_sigma(int device) {
  cudaFuncAttributes fa{};
  SBD_CUDA(cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(rows_kernel<double, true>)));
  SBD_CUDA(cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(rows_kernel<double, false>)));
  SBD_CUDA(cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(rows_vec_kernel<double, true>)));
  SBD_CUDA(cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(rows_vec_kernel<double, false>)));
  preload_ab<16>(device);
  preload_ab<8>(device);
  preload_ab<4>(device);
  preload_ab<2>(device);
  preload_ab<1>(device);
  preload_fp64_sigma_misc();
}

void sigma_fp64(sbdgpu_ctx* c, const double* C, double* S) {
  build_tables(c);
  compute_hii(c);
  if (c->stored) {  // method 1: the product with the stored Hamiltonian
    spmv_stored(c, C, S);
    return;
  }
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

// FP32 sigma with the alpha-beta term on the tensor cores (BF16 operands,
// FP32 accumulation); the same-spin terms as in sigma_fp32.
void sigma_fp32_tc(sbdgpu_ctx* c, const float* C, float* S) {
  build_tables(c);
  compute_hii(c);
  ensure_scratch(c);
  ensure_fp32(c);
  build_tc_buckets(c);
  if (!tc_ab_supported(c)) throw Error{SBDGPU_ERR_LIMIT, "tensor-core alpha-beta kernel: basis or norb too large"};
  const SpinTables& ta = c->tab[0];
  const SpinTables& tb = c->tab[1];
  cudaStream_t s = c->stream;
  float* ct = reinterpret_cast<float*>(c->ct);
  float* st = reinterpret_cast<float*>(c->st);
  SBD_CUDA(cudaEventRecord(c->ev[0], s));
  launch_rows<float, true>(C, S, c->na, c->nb, c->hii, ta, c->jb32, s);
  SBD_CUDA(cudaEventRecord(c->ev[1], s));
  transpose(C, ct, c->na, c->nb, s);
  launch_rows<float, false>(ct, st, c->nb, c->na, nullptr, tb, c->ja32, s);
  transpose_add(st, S, c->nb, c->na, s);
  SBD_CUDA(cudaEventRecord(c->ev[2], s));
  tc_alpha_beta(c, ct, st);
  transpose_add(st, S, c->nb, c->na, s);
  SBD_CUDA(cudaEventRecord(c->ev[3], s));
}

}  // namespace sbdgpu
