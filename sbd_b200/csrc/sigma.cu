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
#include <vector>

#include "internal.cuh"

namespace sbdgpu {

namespace {

constexpr int kRowsThreads = 256;
constexpr int kRowsCols = 2;  // columns per thread

// sigma_row[ia][cols] (=) diag + sum over the bra's table entries, in the
// vector type T (double: plain path; float: mixed path, FP32 accumulation).
// J: [P][jstride] Coulomb coupling to the other spin's occupation.
// Bra row row0 + blockIdx.x; sigma row blockIdx.x of S (a block of rows when
// row0 > 0); J rows jstride apart.
template <typename T, bool kWithDiag>
__global__ void __launch_bounds__(kRowsThreads) rows_kernel(
    const T* __restrict__ C, T* __restrict__ S, size_t ncols, const double* __restrict__ hii,
    const int64_t* __restrict__ s_off, const int32_t* __restrict__ s_idx, const uint32_t* __restrict__ s_info,
    const double* __restrict__ s_val, const int64_t* __restrict__ d_off, const int32_t* __restrict__ d_idx,
    const double* __restrict__ d_val, const T* __restrict__ J, size_t row0, size_t jstride) {
  const size_t row = row0 + blockIdx.x;
  T* Srow = S + (size_t)blockIdx.x * ncols;
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
    const T* Jr = J + (size_t)((info >> 12) & 0xFFFu) * jstride;
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
    if (ok[u]) Srow[col] = acc[u];
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
    const double* __restrict__ d_val, const T* __restrict__ J, size_t row0, size_t jstride) {
  using VT = Vec16<T>;
  using V = typename VT::V;
  constexpr int W = VT::W;
  const size_t row = row0 + blockIdx.x;
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
    VT::get(__ldg(reinterpret_cast<const V*>(J + (size_t)((info >> 12) & 0xFFFu) * jstride + col)), jr);
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
  *reinterpret_cast<V*>(S + (size_t)blockIdx.x * ncols + col) = VT::make(acc);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// Same-spin rows: the vector kernel when the rows allow it, else rows_kernel.
// Bra rows row0 .. row0 + nrows of the table t into the nrows x ncols block S
// (row0 = 0 and jstride = ncols for a whole vector).
template <typename T, bool kWithDiag>
void launch_rows(const T* C, T* S, size_t nrows, size_t ncols, const double* hii, const SpinTables& t, const T* J,
                 cudaStream_t s, size_t row0 = 0, size_t jstride = 0) {
  constexpr int W = Vec16<T>::W;
  if (jstride == 0) jstride = ncols;
  if (nrows == 0) return;
  if (ncols % W == 0 && jstride % W == 0 && aligned16(C) && aligned16(S) && aligned16(J) &&
      (!kWithDiag || aligned16(hii))) {
    dim3 g((unsigned)nrows, (unsigned)((ncols / W + kRowsThreads - 1) / kRowsThreads));
    rows_vec_kernel<T, kWithDiag><<<g, kRowsThreads, 0, s>>>(C, S, ncols, hii, t.s_off, t.s_idx, t.s_info, t.s_val,
                                                             t.d_off, t.d_idx, t.d_val, J, row0, jstride);
  } else {
    dim3 g((unsigned)nrows, (unsigned)((ncols + kRowsThreads * kRowsCols - 1) / (kRowsThreads * kRowsCols)));
    rows_kernel<T, kWithDiag><<<g, kRowsThreads, 0, s>>>(C, S, ncols, hii, t.s_off, t.s_idx, t.s_info, t.s_val,
                                                         t.d_off, t.d_idx, t.d_val, J, row0, jstride);
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
    size_t nslice, size_t ia0) {
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
        if (g < gcount) atomicAdd(&S[((size_t)tgt[g] - ia0) * nb + ib], sgn[g] * y[g]);
    }
  }
}

template <typename T, int G>
size_t ab_smem(size_t nb, int P) {
  return ((nb * sizeof(T) + 15) & ~size_t(15)) + (size_t)P * ab_vstride<T, G>() * sizeof(T);
}

// 512 threads while two CTAs fit in shared memory, else 1024 so that one CTA
// still keeps 32 warps resident per SM.
// The alpha singles the kernel walks: CSR by source string ja (all targets, or
// only those of one block of target rows, ia0 .. ia0 + rows).
struct AlphaSingles {
  const int64_t* off;
  const int32_t* idx;
  const uint32_t* info;
  int max_s;
  size_t ia0;
};

template <typename T, int G, int NT>
void launch_ab_nt(sbdgpu_ctx* c, const T* C, T* S, const T* vf, size_t smem, const AlphaSingles& as) {
  const SpinTables& tb = c->tab[1];
  dim3 grid((unsigned)c->na, (unsigned)((as.max_s + G - 1) / G));
  if (grid.y == 0) return;
  allow_dynamic_smem(reinterpret_cast<const void*>(ab_kernel<T, G, NT>), c->device);
  ab_kernel<T, G, NT><<<grid, NT, smem, c->stream>>>(C, S, c->nb, c->P, vf, as.off, as.idx, as.info, tb.sell_off,
                                                     tb.sell_w, tb.sell, tb.nslice, as.ia0);
  SBD_CUDA(cudaGetLastError());
}

// threads per CTA: the tuned choice, else 512 while two CTAs fit an SM's
// shared memory and 1024 when only one does, halved (down to 128) while the
// warps would outnumber the 32-string slices of beta strings they loop over
template <typename T, int G>
void launch_ab(sbdgpu_ctx* c, const T* C, T* S, const T* vf, size_t smem, const AlphaSingles& as, int nt) {
  if (nt == 0) {
    nt = 2 * (smem + 1024) <= 228 * 1024 ? 512 : 1024;
    while (nt > 128 && (size_t)(nt / 2) >= c->tab[1].nslice * 32) nt /= 2;
  }
  switch (nt) {
    case 128: launch_ab_nt<T, G, 128>(c, C, S, vf, smem, as); break;
    case 256: launch_ab_nt<T, G, 256>(c, C, S, vf, smem, as); break;
    case 512: launch_ab_nt<T, G, 512>(c, C, S, vf, smem, as); break;
    default: launch_ab_nt<T, G, 1024>(c, C, S, vf, smem, as); break;
  }
}

}  // namespace

// Alpha-beta launch shapes an FP64 sigma of this context can take: group
// sizes whose integral block fits in shared memory next to one row of C,
// times 128 / 256 / 512 / 1024 threads per CTA.
std::vector<std::pair<int, int>> ab_shapes(sbdgpu_ctx* c) {
  int dev_smem = 0;
  SBD_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
  const size_t budget = (size_t)dev_smem - 1024;
  std::vector<std::pair<int, int>> out;
  const int groups[5] = {16, 8, 4, 2, 1};
  const size_t sm[5] = {ab_smem<double, 16>(c->nb, c->P), ab_smem<double, 8>(c->nb, c->P),
                        ab_smem<double, 4>(c->nb, c->P), ab_smem<double, 2>(c->nb, c->P),
                        ab_smem<double, 1>(c->nb, c->P)};
  for (int k = 0; k < 5; k++)
    if (sm[k] <= budget)
      for (int nt : {128, 256, 512, 1024}) out.emplace_back(groups[k], nt);
  return out;
}

namespace {

// The alpha-beta term: the context's tuned group size and threads for FP64
// when set (sbdgpu_set_tuning / sbdgpu_autotune), else the largest group of
// alpha singles per CTA whose integral block fits in shared memory next to
// one row of C.
template <typename T>
void alpha_beta(sbdgpu_ctx* c, const T* C, T* S, const T* vf, const AlphaSingles& as) {
  int dev_smem = 0;
  SBD_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
  size_t budget = (size_t)dev_smem - 1024;
  if (c->nb > 65536) throw Error{SBDGPU_ERR_LIMIT, "alpha-beta kernel: more than 65536 beta strings"};
  size_t nb = c->nb;
  int P = c->P;
  const bool tuned = sizeof(T) == 8 && c->ab_group > 0;
  const int g = tuned ? c->ab_group : 0, nt = tuned ? c->ab_threads : 0;
  if ((g == 0 || g == 16) && ab_smem<T, 16>(nb, P) <= budget)
    launch_ab<T, 16>(c, C, S, vf, ab_smem<T, 16>(nb, P), as, nt);
  else if ((g == 0 || g == 8) && ab_smem<T, 8>(nb, P) <= budget)
    launch_ab<T, 8>(c, C, S, vf, ab_smem<T, 8>(nb, P), as, nt);
  else if ((g == 0 || g == 4) && ab_smem<T, 4>(nb, P) <= budget)
    launch_ab<T, 4>(c, C, S, vf, ab_smem<T, 4>(nb, P), as, nt);
  else if ((g == 0 || g == 2) && ab_smem<T, 2>(nb, P) <= budget)
    launch_ab<T, 2>(c, C, S, vf, ab_smem<T, 2>(nb, P), as, nt);
  else if ((g == 0 || g == 1) && ab_smem<T, 1>(nb, P) <= budget)
    launch_ab<T, 1>(c, C, S, vf, ab_smem<T, 1>(nb, P), as, nt);
  else
    throw Error{SBDGPU_ERR_LIMIT, "alpha-beta kernel: one beta row and integral row exceed shared memory"};
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
  const SpinTables& tas = c->tab[0];
  alpha_beta(c, C, S, vf, AlphaSingles{tas.s_off, tas.s_idx, tas.s_info, tas.max_s, 0});
  if (events) SBD_CUDA(cudaEventRecord(c->ev[3], s));
}

template <int G>
void preload_ab(int device) {
  allow_dynamic_smem(reinterpret_cast<const void*>(ab_kernel<double, G, 128>), device);
  allow_dynamic_smem(reinterpret_cast<const void*>(ab_kernel<double, G, 256>), device);
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
  if (use_ozaki(c) && same_spin_ozaki_fp64(c, C, S, c->ct, c->st, true)) {
    const SpinTables& ta = c->tab[0];
    alpha_beta<double>(c, C, S, c->vf, AlphaSingles{ta.s_off, ta.s_idx, ta.s_info, ta.max_s, 0});
    SBD_CUDA(cudaEventRecord(c->ev[3], c->stream));
    return;
  }
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
  float* ct = reinterpret_cast<float*>(c->ct);
  float* st = reinterpret_cast<float*>(c->st);
  if (use_dense_same(c)) {
    same_spin_dense_fp32(c, C, S, ct, st, true);
    const SpinTables& ta = c->tab[0];
    alpha_beta<float>(c, C, S, c->vf32, AlphaSingles{ta.s_off, ta.s_idx, ta.s_info, ta.max_s, 0});
    SBD_CUDA(cudaEventRecord(c->ev[3], c->stream));
    return;
  }
  sigma_launch<float>(c, C, S, ct, st, c->ja32, c->jb32, c->vf32, true);
}

// Alpha singles whose target lies in rows [r0, r1), CSR by source string
// (kept for the last block asked for).
void ensure_row_block_singles(sbdgpu_ctx* c, size_t r0, size_t r1) {
  if (c->blk_off && c->blk_r0 == r0 && c->blk_r1 == r1) return;
  cudaFree(c->blk_off);
  cudaFree(c->blk_idx);
  cudaFree(c->blk_info);
  c->blk_off = nullptr;
  c->blk_idx = nullptr;
  c->blk_info = nullptr;
  const SpinTables& ta = c->tab[0];
  std::vector<int32_t> idx(ta.ns);
  std::vector<uint32_t> info(ta.ns);
  if (ta.ns) {
    SBD_CUDA(cudaMemcpy(idx.data(), ta.s_idx, sizeof(int32_t) * ta.ns, cudaMemcpyDeviceToHost));
    SBD_CUDA(cudaMemcpy(info.data(), ta.s_info, sizeof(uint32_t) * ta.ns, cudaMemcpyDeviceToHost));
  }
  std::vector<int64_t> off(c->na + 1, 0);
  std::vector<int32_t> bidx;
  std::vector<uint32_t> binfo;
  int max_s = 0;
  for (size_t ja = 0; ja < c->na; ja++) {
    for (int64_t k = ta.h_s_off[ja]; k < ta.h_s_off[ja + 1]; k++)
      if ((size_t)idx[k] >= r0 && (size_t)idx[k] < r1) {
        bidx.push_back(idx[k]);
        binfo.push_back(info[k]);
      }
    off[ja + 1] = (int64_t)bidx.size();
    max_s = std::max(max_s, (int)(off[ja + 1] - off[ja]));
  }
  c->blk_off = (int64_t*)dev_alloc(sizeof(int64_t) * off.size());
  c->blk_idx = (int32_t*)dev_alloc(sizeof(int32_t) * std::max<size_t>(bidx.size(), 1));
  c->blk_info = (uint32_t*)dev_alloc(sizeof(uint32_t) * std::max<size_t>(binfo.size(), 1));
  SBD_CUDA(cudaMemcpy(c->blk_off, off.data(), sizeof(int64_t) * off.size(), cudaMemcpyHostToDevice));
  if (!bidx.empty()) {
    SBD_CUDA(cudaMemcpy(c->blk_idx, bidx.data(), sizeof(int32_t) * bidx.size(), cudaMemcpyHostToDevice));
    SBD_CUDA(cudaMemcpy(c->blk_info, binfo.data(), sizeof(uint32_t) * binfo.size(), cudaMemcpyHostToDevice));
  }
  c->blk_max = max_s;
  c->blk_r0 = r0;
  c->blk_r1 = r1;
}

// FP64 sigma rows [r0, r1) of H C for the full vector C (device, reference
// convention) into S_rows ((r1 - r0) x nb, reference convention): the work of
// one rank when W and sigma are split into blocks of alpha rows (the
// reference's adet_comm blocks, chemistry/tpb/helper.h:505-540 with
// get_mpi_range, framework/mpi_utility.h:14-36).  Every term of a target row
// is summed on this device: alpha rows from C's rows, beta rows from the
// block's own rows, alpha-beta pairs from the source rows with the singles
// restricted to the block's targets.
void sigma_rows_fp64(sbdgpu_ctx* c, const double* dC, double* S, size_t r0, size_t r1) {
  build_tables(c);
  compute_hii(c);
  ensure_scratch(c);
  ensure_io(c);
  const size_t nrows = r1 - r0, nb = c->nb;
  cudaStream_t s = c->stream;
  const SpinTables& ta = c->tab[0];
  const SpinTables& tb = c->tab[1];
  SBD_CUDA(cudaMemcpyAsync(c->io_a, dC, sizeof(double) * c->N, cudaMemcpyDeviceToDevice, s));
  apply_phase(c, c->io_a);
  if (nrows == 0) return;
  launch_rows<double, true>(c->io_a, S, nrows, nb, c->hii, ta, c->jb, s, r0, nb);
  transpose(c->io_a + r0 * nb, c->ct, nrows, nb, s);
  launch_rows<double, false>(c->ct, c->st, nb, nrows, nullptr, tb, c->ja + r0, s, 0, c->na);
  transpose_add(c->st, S, nb, nrows, s);
  ensure_row_block_singles(c, r0, r1);
  alpha_beta<double>(c, c->io_a, S, c->vf, AlphaSingles{c->blk_off, c->blk_idx, c->blk_info, c->blk_max, r0});
  apply_phase_rows(c, S, r0, nrows);
  SBD_CUDA(cudaStreamSynchronize(s));
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
  if (use_dense_same(c)) {
    same_spin_dense_fp32(c, C, S, ct, st, true);  // leaves C^T in ct
  } else {
    SBD_CUDA(cudaEventRecord(c->ev[0], s));
    launch_rows<float, true>(C, S, c->na, c->nb, c->hii, ta, c->jb32, s);
    SBD_CUDA(cudaEventRecord(c->ev[1], s));
    transpose(C, ct, c->na, c->nb, s);
    launch_rows<float, false>(ct, st, c->nb, c->na, nullptr, tb, c->ja32, s);
    transpose_add(st, S, c->nb, c->na, s);
    SBD_CUDA(cudaEventRecord(c->ev[2], s));
  }
  tc_alpha_beta(c, ct, st);
  transpose_add(st, S, c->nb, c->na, s);
  SBD_CUDA(cudaEventRecord(c->ev[3], s));
}

}  // namespace sbdgpu
