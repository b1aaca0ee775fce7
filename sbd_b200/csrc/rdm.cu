// Off-diagonal part of the one- and two-particle RDMs (Correlation,
// chemistry/tpb/correlation.h:194-443; the diagonal part is in misc.cu).
//
// The reference walks every determinant and each of its connected
// determinants and adds OneDiff/TwoDiffCorrelation terms (correlation.h:
// 49-130) one pair at a time.  Every such term is W_bra W_ket times a sign
// that counts the bra's occupied spin orbitals between two spin-orbital
// indices of the interleaved order, and that count splits into an alpha part
// and a beta part over two fixed orbital ranges:
//   spin orbitals strictly between x and y = alpha orbitals [lo/2+1, (hi+1)/2)
//                                          + beta orbitals  [(lo+1)/2, hi/2)
// So the terms of one excitation pair of one spin are summed over the other
// spin's string first, with that string's part of the sign, and added to the
// RDM arrays once per pair:
//
//   same-spin singles (i <- j of one spin, the other string k free):
//     S0 = sum_k V[i,k] V[j,k] s_k, S1[r] = sum_k V[i,k] V[j,k] s_k n_r(k)
//     (S1 carries the other spin's spectators of OneDiffCorrelation)
//   same-spin doubles: S = sum_k V[i,k] V[j,k] s_k
//   alpha single x beta single: per alpha pair (ia <- ja), per beta
//     excitation bin (r <- s), X = sum over the bin's beta pairs of
//     W[ia,ib] W[ja,jb] s_ib
//
// with V = W for alpha pairs and V = W^T for beta pairs.  Each pair is one
// warp's dot product over rows held in shared memory (rows kernel), and each
// alpha single one CTA pass over the beta pairs grouped by excitation (the
// alpha-beta kernel): no per-term global atomics.  The alpha-beta part does
// 2 N s_a s_b multiply-adds with two shared-memory reads each, like the
// alpha-beta sigma term.
#include <algorithm>
#include <vector>

#include "internal.cuh"

namespace sbdgpu {

namespace {

constexpr int kRowThreads = 256;
constexpr int kAbThreads = 1024;

__device__ __forceinline__ uint64_t range_mask(int a, int b) {  // orbitals [a, b)
  if (b <= a) return 0ull;
  const uint64_t hi = b >= 64 ? ~0ull : ((1ull << b) - 1ull);
  const uint64_t lo = a >= 64 ? ~0ull : ((1ull << a) - 1ull);
  return hi & ~lo;
}

// alpha / beta orbitals whose spin orbitals lie strictly between spin orbitals x and y
__device__ __forceinline__ uint64_t mask_a(int x, int y) {
  const int lo = min(x, y), hi = max(x, y);
  return range_mask((lo >> 1) + 1, (hi + 1) >> 1);
}
__device__ __forceinline__ uint64_t mask_b(int x, int y) {
  const int lo = min(x, y), hi = max(x, y);
  return range_mask((lo + 1) >> 1, hi >> 1);
}
template <int S>
__device__ __forceinline__ uint64_t mask_s(int x, int y) {
  return S == 0 ? mask_a(x, y) : mask_b(x, y);
}

__device__ __forceinline__ double psign(uint64_t s, uint64_t m) { return (__popcll(s & m) & 1) ? -1.0 : 1.0; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// TwoDiffCorrelation's entries (correlation.h:91-130) for spin orbitals
// I < J (bra) and A < B (ket), v = the signed product
__device__ void two_add(double* two, int L, int I, int J, int A, int B, double v) {
  const size_t L2 = (size_t)L * L, L4 = L2 * L2;
  const int oi = I >> 1, si = I & 1, oj = J >> 1, sj = J & 1, oa = A >> 1, sa = A & 1, ob = B >> 1, sb = B & 1;
  if (si == sa) {
    atomicAdd(&two[(si + 2 * sj) * L4 + oa + L * ob + L2 * (oi + (size_t)L * oj)], v);
    atomicAdd(&two[(sj + 2 * si) * L4 + ob + L * oa + L2 * (oj + (size_t)L * oi)], v);
  }
  if (si == sb) {
    atomicAdd(&two[(si + 2 * sj) * L4 + oa + L * ob + L2 * (oj + (size_t)L * oi)], -v);
    atomicAdd(&two[(sj + 2 * si) * L4 + ob + L * oa + L2 * (oi + (size_t)L * oj)], -v);
  }
}

// I, J, A, B, the flip of TwoDiffCorrelation and the two strings' sign masks
// for creation spin orbitals c0, c1 (in the bra) and d0, d1 (in the ket)
struct Quad {
  int I, J, A, B;
  double flip;
  uint64_t ma, mb;
};
__device__ __forceinline__ Quad quad(int c0, int c1, int d0, int d1) {
  Quad q;
  q.I = min(c0, c1);
  q.J = max(c0, c1);
  q.A = min(d0, d1);
  q.B = max(d0, d1);
  q.flip = (q.A > q.J || q.B < q.I) ? -1.0 : 1.0;
  q.ma = mask_a(q.I, q.A) ^ mask_a(q.J, q.B);
  q.mb = mask_b(q.I, q.A) ^ mask_b(q.J, q.B);
  return q;
}

__device__ __forceinline__ int low_bit(uint64_t x) { return __ffsll((long long)x) - 1; }

// Same-spin pairs of spin S.  V: [n_own][n_oth] (W for S = 0, W^T for S = 1);
// one CTA per bra string i, one warp per excitation pair.  kStr: the other
// spin's strings staged in shared memory beside the row (when both fit).
template <int S, bool kStr>
__global__ void __launch_bounds__(kRowThreads) rdm_rows_kernel(const double* __restrict__ V, size_t n_oth,
                                                              const uint64_t* __restrict__ own,
                                                              const uint64_t* __restrict__ oth, int L,
                                                              const int64_t* __restrict__ s_off,
                                                              const int32_t* __restrict__ s_idx,
                                                              const uint32_t* __restrict__ s_info,
                                                              const int64_t* __restrict__ d_off,
                                                              const int32_t* __restrict__ d_idx, double* one,
                                                              double* two) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* vi = reinterpret_cast<double*>(smem_raw);
  uint64_t* os = reinterpret_cast<uint64_t*>(smem_raw + sizeof(double) * n_oth);
  const size_t i = blockIdx.x;
  for (size_t c = threadIdx.x; c < n_oth; c += kRowThreads) {
    vi[c] = V[i * n_oth + c];
    if (kStr) os[c] = oth[c];
  }
  __syncthreads();
  const uint64_t* ostr = kStr ? os : oth;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int nwarp = kRowThreads / 32;
  const size_t L2 = (size_t)L * L, L3 = L2 * L, L4 = L3 * L;
  const uint64_t si_str = own[i];
  const int64_t ns0 = s_off[i], ns = s_off[i + 1] - ns0;
  const int64_t nd0 = d_off[i], nd = d_off[i + 1] - nd0;
  for (int64_t k = warp; k < ns + nd; k += nwarp) {
    if (k < ns) {
      // OneDiffCorrelation summed over the other spin (correlation.h:49-86)
      const size_t j = (size_t)s_idx[ns0 + k];
      const uint32_t info = s_info[ns0 + k];
      const int oi = info & 63, oa = (info >> 6) & 63;  // in the bra / in the ket
      const int x = 2 * oi + S, y = 2 * oa + S;
      const double pown = psign(si_str, mask_s<S>(x, y));
      const uint64_t moth = mask_s<1 - S>(x, y);
      const double* vj = V + j * n_oth;
      for (int r0 = 0; r0 < L; r0 += 32) {
        double s0 = 0.0, acc[32];
#pragma unroll
        for (int r = 0; r < 32; r++) acc[r] = 0.0;
        for (size_t c = lane; c < n_oth; c += 32) {
          const uint64_t o = ostr[c];
          const double t = vi[c] * __ldg(&vj[c]) * psign(o, moth);
          s0 += t;
          const uint64_t ob = r0 ? (o >> 32) : o;
#pragma unroll
          for (int r = 0; r < 32; r++) acc[r] += ((ob >> r) & 1ull) ? t : 0.0;
        }
        double mine = 0.0;
#pragma unroll
        for (int r = 0; r < 32; r++) {
          const double tot = warp_sum(acc[r]);
          if (lane == r) mine = tot;
        }
        // the other spin's spectators r = r0 + lane
        const int r = r0 + lane;
        if (r < L && mine != 0.0) {
          const double v = pown * mine;
          atomicAdd(&two[(S + 2 * (1 - S)) * L4 + oa + (size_t)r * L + oi * L2 + (size_t)r * L3], v);
          atomicAdd(&two[((1 - S) + 2 * S) * L4 + r + (size_t)oa * L + (size_t)r * L2 + oi * L3], v);
        }
        if (r0 == 0) {
          const double v = pown * warp_sum(s0);
          if (lane == 0) atomicAdd(&one[S * L2 + oi + (size_t)L * oa], v);
          // this spin's spectators: the bra's occupied orbitals, one per lane
          if (lane < L && ((si_str >> lane) & 1ull)) {
            const size_t oj = lane, b = (size_t)(3 * S) * L4;
            atomicAdd(&two[b + oa + oj * L + oi * L2 + oj * L3], v);
            atomicAdd(&two[b + oj + oa * L + oj * L2 + oi * L3], v);
            atomicAdd(&two[b + oa + oj * L + oj * L2 + oi * L3], -v);
            atomicAdd(&two[b + oj + oa * L + oi * L2 + oj * L3], -v);
          }
          if (L > 32 && lane + 32 < L && ((si_str >> (lane + 32)) & 1ull)) {
            const size_t oj = lane + 32, b = (size_t)(3 * S) * L4;
            atomicAdd(&two[b + oa + oj * L + oi * L2 + oj * L3], v);
            atomicAdd(&two[b + oj + oa * L + oj * L2 + oi * L3], v);
            atomicAdd(&two[b + oa + oj * L + oj * L2 + oi * L3], -v);
            atomicAdd(&two[b + oj + oa * L + oi * L2 + oj * L3], -v);
          }
        }
      }
    } else {
      // TwoDiffCorrelation summed over the other spin (correlation.h:91-130)
      const size_t j = (size_t)d_idx[nd0 + (k - ns)];
      const uint64_t sj_str = own[j];
      const uint64_t cm = si_str & ~sj_str, dm = sj_str & ~si_str;
      const int c0 = low_bit(cm), c1 = low_bit(cm & (cm - 1)), d0 = low_bit(dm), d1 = low_bit(dm & (dm - 1));
      const Quad q = quad(2 * c0 + S, 2 * c1 + S, 2 * d0 + S, 2 * d1 + S);
      const uint64_t mown = S == 0 ? q.ma : q.mb, moth = S == 0 ? q.mb : q.ma;
      const double* vj = V + j * n_oth;
      double s = 0.0;
      for (size_t c = lane; c < n_oth; c += 32) s += vi[c] * __ldg(&vj[c]) * psign(ostr[c], moth);
      s = warp_sum(s);
      if (lane == 0) two_add(two, L, q.I, q.J, q.A, q.B, q.flip * psign(si_str, mown) * s);
    }
  }
}

// Alpha single x beta single (the opposite-spin branch of
// CorrelationTermAddition, correlation.h:135-189): one alpha pair per CTA
// pass, its two W rows in shared memory, one warp per beta excitation bin.
// kRows: the ket row fits beside the bra row (else it is read from L2).
template <bool kRows>
__global__ void __launch_bounds__(kAbThreads) rdm_ab_kernel(const double* __restrict__ W, size_t nb,
                                                           const uint64_t* __restrict__ astr,
                                                           const uint64_t* __restrict__ bstr, int L,
                                                           const int32_t* __restrict__ a_row,
                                                           const int32_t* __restrict__ a_idx,
                                                           const uint32_t* __restrict__ a_info, size_t n_pairs,
                                                           const int64_t* __restrict__ bin_off,
                                                           const uint32_t* __restrict__ bin_ent, double* two) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* wi = reinterpret_cast<double*>(smem_raw);
  double* wj = wi + nb;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int nwarp = kAbThreads / 32;
  const int nbin = L * L;
  for (size_t k = blockIdx.x; k < n_pairs; k += gridDim.x) {
    const size_t ia = (size_t)a_row[k], ja = (size_t)a_idx[k];
    const uint32_t info = a_info[k];
    const int oi = info & 63, oa = (info >> 6) & 63;
    __syncthreads();  // the previous pair's rows are no longer read
    for (size_t c = threadIdx.x; c < nb; c += kAbThreads) {
      wi[c] = W[ia * nb + c];
      if (kRows) wj[c] = W[ja * nb + c];
    }
    __syncthreads();
    const double* wjr = kRows ? wj : W + ja * nb;
    const uint64_t sa = astr[ia];
    for (int bin = warp; bin < nbin; bin += nwarp) {
      const int64_t e0 = bin_off[bin], e1 = bin_off[bin + 1];
      if (e0 == e1) continue;
      const int ri = bin / L, ra = bin - ri * L;  // in the beta bra / in the beta ket
      const Quad q = quad(2 * oi, 2 * ri + 1, 2 * oa, 2 * ra + 1);
      double x = 0.0;
      for (int64_t e = e0 + lane; e < e1; e += 32) {
        const uint32_t ent = __ldg(&bin_ent[e]);
        const uint32_t ib = ent & 0xFFFFu, jb = ent >> 16;
        x += wi[ib] * (kRows ? wjr[jb] : __ldg(&wjr[jb])) * psign(__ldg(&bstr[ib]), q.mb);
      }
      x = warp_sum(x);
      if (lane == 0 && x != 0.0) two_add(two, L, q.I, q.J, q.A, q.B, q.flip * psign(sa, q.ma) * x);
    }
  }
}

}  // namespace

// The beta singles grouped by excitation: bin ri * L + ra holds the pairs
// (ib, jb) with ri in beta string ib and ra in jb; and the bra row of every
// alpha single.  Built once per context.
void ensure_rdm_tables(sbdgpu_ctx* c) {
  if (c->rdm_bin_off) return;
  const int L = c->L;
  const SpinTables& ta = c->tab[0];
  const SpinTables& tb = c->tab[1];
  std::vector<int32_t> b_idx(tb.ns);
  std::vector<uint32_t> b_info(tb.ns);
  SBD_CUDA(cudaMemcpy(b_idx.data(), tb.s_idx, sizeof(int32_t) * tb.ns, cudaMemcpyDeviceToHost));
  SBD_CUDA(cudaMemcpy(b_info.data(), tb.s_info, sizeof(uint32_t) * tb.ns, cudaMemcpyDeviceToHost));
  std::vector<int64_t> off((size_t)L * L + 1, 0);
  for (size_t k = 0; k < tb.ns; k++) off[(b_info[k] & 63) * L + ((b_info[k] >> 6) & 63) + 1]++;
  for (size_t b = 0; b < (size_t)L * L; b++) off[b + 1] += off[b];
  std::vector<int64_t> pos(off.begin(), off.end() - 1);
  std::vector<uint32_t> ent(tb.ns);
  for (size_t ib = 0; ib < c->nb; ib++)
    for (int64_t k = tb.h_s_off[ib]; k < tb.h_s_off[ib + 1]; k++) {
      const size_t b = (b_info[k] & 63) * L + ((b_info[k] >> 6) & 63);
      ent[pos[b]++] = (uint32_t)ib | ((uint32_t)b_idx[k] << 16);
    }
  std::vector<int32_t> row(ta.ns);
  for (size_t ia = 0; ia < c->na; ia++)
    for (int64_t k = ta.h_s_off[ia]; k < ta.h_s_off[ia + 1]; k++) row[k] = (int32_t)ia;
  c->rdm_bin_off = (int64_t*)dev_alloc(sizeof(int64_t) * off.size());
  c->rdm_bin_ent = (uint32_t*)dev_alloc(sizeof(uint32_t) * std::max<size_t>(ent.size(), 1));
  c->rdm_a_row = (int32_t*)dev_alloc(sizeof(int32_t) * std::max<size_t>(row.size(), 1));
  SBD_CUDA(cudaMemcpy(c->rdm_bin_off, off.data(), sizeof(int64_t) * off.size(), cudaMemcpyHostToDevice));
  SBD_CUDA(cudaMemcpy(c->rdm_bin_ent, ent.data(), sizeof(uint32_t) * ent.size(), cudaMemcpyHostToDevice));
  SBD_CUDA(cudaMemcpy(c->rdm_a_row, row.data(), sizeof(int32_t) * row.size(), cudaMemcpyHostToDevice));
}

void free_rdm_tables(sbdgpu_ctx* c) {
  cudaFree(c->rdm_bin_off);
  cudaFree(c->rdm_bin_ent);
  cudaFree(c->rdm_a_row);
  c->rdm_bin_off = nullptr;
  c->rdm_bin_ent = nullptr;
  c->rdm_a_row = nullptr;
}

namespace {

template <int S>
void launch_rows(sbdgpu_ctx* c, const double* V, size_t n_own, size_t n_oth, const uint64_t* own,
                 const uint64_t* oth, const SpinTables& t, double* one, double* two, size_t smem_cap) {
  const size_t both = sizeof(double) * n_oth + sizeof(uint64_t) * n_oth;
  if (both <= smem_cap) {
    allow_dynamic_smem(reinterpret_cast<const void*>(rdm_rows_kernel<S, true>), c->device);
    rdm_rows_kernel<S, true><<<(unsigned)n_own, kRowThreads, both, c->stream>>>(
        V, n_oth, own, oth, c->L, t.s_off, t.s_idx, t.s_info, t.d_off, t.d_idx, one, two);
  } else {
    const size_t row = sizeof(double) * n_oth;
    if (row > smem_cap) throw Error{SBDGPU_ERR_LIMIT, "RDM: a row of the vector exceeds shared memory"};
    allow_dynamic_smem(reinterpret_cast<const void*>(rdm_rows_kernel<S, false>), c->device);
    rdm_rows_kernel<S, false><<<(unsigned)n_own, kRowThreads, row, c->stream>>>(
        V, n_oth, own, oth, c->L, t.s_off, t.s_idx, t.s_info, t.d_off, t.d_idx, one, two);
  }
  SBD_CUDA(cudaGetLastError());
}

}  // namespace

void rdm_offdiag(sbdgpu_ctx* c, const double* dW, double* one, double* two) {
  if (c->nb > 65535) throw Error{SBDGPU_ERR_LIMIT, "RDM: more than 65,535 beta strings"};
  ensure_rdm_tables(c);
  int optin = 0;
  SBD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
  const size_t cap = (size_t)optin;
  // alpha pairs on the rows of W, beta pairs on the rows of W^T
  launch_rows<0>(c, dW, c->na, c->nb, c->astr, c->bstr, c->tab[0], one, two, cap);
  double* wt = (double*)dev_alloc(sizeof(double) * c->N);
  try {
    transpose(dW, wt, c->na, c->nb, c->stream);
    launch_rows<1>(c, wt, c->nb, c->na, c->bstr, c->astr, c->tab[1], one, two, cap);
    SBD_CUDA(cudaStreamSynchronize(c->stream));
  } catch (...) {
    cudaStreamSynchronize(c->stream);
    cudaFree(wt);
    throw;
  }
  cudaFree(wt);
  const size_t n_pairs = c->tab[0].ns;
  if (n_pairs == 0 || c->tab[1].ns == 0) return;
  const size_t rows2 = 2 * sizeof(double) * c->nb;
  const unsigned grid = (unsigned)std::min<size_t>(n_pairs, 148 * 4);
  if (rows2 <= cap) {
    allow_dynamic_smem(reinterpret_cast<const void*>(rdm_ab_kernel<true>), c->device);
    rdm_ab_kernel<true><<<grid, kAbThreads, rows2, c->stream>>>(dW, c->nb, c->astr, c->bstr, c->L, c->rdm_a_row,
                                                                  c->tab[0].s_idx, c->tab[0].s_info, n_pairs,
                                                                  c->rdm_bin_off, c->rdm_bin_ent, two);
  } else {
    const size_t row = sizeof(double) * c->nb;
    if (row > cap) throw Error{SBDGPU_ERR_LIMIT, "RDM: a row of the vector exceeds shared memory"};
    allow_dynamic_smem(reinterpret_cast<const void*>(rdm_ab_kernel<false>), c->device);
    rdm_ab_kernel<false><<<grid, kAbThreads, row, c->stream>>>(dW, c->nb, c->astr, c->bstr, c->L, c->rdm_a_row,
                                                                 c->tab[0].s_idx, c->tab[0].s_info, n_pairs,
                                                                 c->rdm_bin_off, c->rdm_bin_ent, two);
  }
  SBD_CUDA(cudaGetLastError());
}

}  // namespace sbdgpu
