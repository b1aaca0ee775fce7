// Same-spin sigma with ket-row reuse across blocks of bra rows.
//
// The same-spin part sigma[i,:] += sum_{j in S(i) u D(i)} h_ij C[j,:] streams a
// row of C for every table entry.  Consecutive bra strings share many of their
// single/double neighbours (the union of the neighbour lists of 32 consecutive
// strings is ~3.5x smaller than their sum at 144M determinants), so a CTA
// takes a block of R bra rows and one column slice, loads each distinct ket
// row segment of the block once into shared memory (in batches of KB rows) and
// applies it to every bra row of the block that references it.
//
// Per block the entries are regrouped on the host after the table build:
//   kets      distinct ket rows of the block, in batches of KB (padding = -1)
//   entries   per (batch, bra row in block): {element, slot | single<<8 |
//             pair<<12 | neg<<31}; singles add sign * J[pair][col], the
//             Coulomb coupling to the other spin's occupation
#include <algorithm>
#include <numeric>

#include "internal.cuh"

namespace sbdgpu {

namespace {

constexpr int kBlockThreads = 256;  // 8 warps
constexpr int kWarps = kBlockThreads / 32;
constexpr int kSliceCols = 256;    // columns of C per CTA
constexpr int kColsPerLane = kSliceCols / 32;

// CTA = (block of R bra rows, slice of 256 columns).  Warp w owns the block's
// rows w, w+8, w+16, ...; lane l owns columns l, l+32, ..., so every entry
// (warp-uniform) feeds 8 FMAs per lane from conflict-free shared memory.
template <typename T, bool kWithDiag, int R>
__global__ void __launch_bounds__(kBlockThreads, 2) block_rows_kernel(
    const T* __restrict__ C, T* __restrict__ S, size_t nrows, size_t ncols, const double* __restrict__ hii,
    const int64_t* __restrict__ blk_batch0, const int32_t* __restrict__ kets, const int64_t* __restrict__ eoff,
    const RowEntry* __restrict__ ent, const T* __restrict__ J) {
  constexpr int RW = R / kWarps;  // rows per warp
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);  // [kRowBatch][kSliceCols]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t b = blockIdx.x;
  const size_t row0 = b * R;
  const size_t cbase = (size_t)blockIdx.y * kSliceCols;
  T acc[RW][kColsPerLane];
#pragma unroll
  for (int i = 0; i < RW; i++) {
    size_t row = row0 + warp + (size_t)i * kWarps;
#pragma unroll
    for (int k = 0; k < kColsPerLane; k++) {
      size_t col = cbase + lane + 32 * k;
      acc[i][k] = (kWithDiag && row < nrows && col < ncols) ? (T)hii[row * ncols + col] * C[row * ncols + col]
                                                           : (T)0;
    }
  }
  const int64_t g0 = blk_batch0[b], g1 = blk_batch0[b + 1];
  for (int64_t g = g0; g < g1; g++) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < kRowBatch * kSliceCols; idx += kBlockThreads) {
      int slot = idx / kSliceCols, cc = idx - slot * kSliceCols;
      int ket = __ldg(&kets[g * kRowBatch + slot]);
      size_t col = cbase + cc;
      sm[idx] = (ket >= 0 && col < ncols) ? C[(size_t)ket * ncols + col] : (T)0;
    }
    __syncthreads();
    const int64_t* eo = eoff + g * R;
#pragma unroll
    for (int i = 0; i < RW; i++) {
      const int r = warp + i * kWarps;
      const int64_t e0 = eo[r], e1 = eo[r + 1];
      for (int64_t e = e0; e < e1; e++) {
        RowEntry en = ent[e];
        const T* x = sm + (en.info & 0xFFu) * kSliceCols + lane;
        T v = (T)en.val;
        if (en.info & 0x100u) {
          const T* Jr = J + (size_t)((en.info >> 12) & 0xFFFu) * ncols + cbase + lane;
          T sg = (en.info & 0x80000000u) ? (T)-1 : (T)1;
#pragma unroll
          for (int k = 0; k < kColsPerLane; k++) {
            T jv = (cbase + lane + 32 * k < ncols) ? Jr[32 * k] : (T)0;
            acc[i][k] += (v + sg * jv) * x[32 * k];
          }
        } else {
#pragma unroll
          for (int k = 0; k < kColsPerLane; k++) acc[i][k] += v * x[32 * k];
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < RW; i++) {
    size_t row = row0 + warp + (size_t)i * kWarps;
#pragma unroll
    for (int k = 0; k < kColsPerLane; k++) {
      size_t col = cbase + lane + 32 * k;
      if (row < nrows && col < ncols) S[row * ncols + col] = acc[i][k];
    }
  }
}

template <typename T, bool kWithDiag, int R>
void launch_block_rows(const RowBlocks& rb, const T* C, T* S, size_t nrows, size_t ncols, const double* hii,
                       const T* J, cudaStream_t s) {
  size_t smem = sizeof(T) * kRowBatch * kSliceCols;
  SBD_CUDA(cudaFuncSetAttribute(block_rows_kernel<T, kWithDiag, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
  dim3 g((unsigned)rb.nblk, (unsigned)((ncols + kSliceCols - 1) / kSliceCols));
  block_rows_kernel<T, kWithDiag, R><<<g, kBlockThreads, smem, s>>>(C, S, nrows, ncols, hii, rb.blk_batch0,
                                                                    rb.kets, rb.eoff, rb.ent, J);
  SBD_CUDA(cudaGetLastError());
}

}  // namespace

// Regroup one spin's tables into row blocks of R bra rows (host side, once).
void build_row_blocks(sbdgpu_ctx* c, int spin, int R) {
  SpinTables& t = c->tab[spin];
  RowBlocks& rb = c->blocks[spin];
  if (rb.ent && rb.R == R) return;
  free_row_blocks(rb);
  size_t n = t.n;
  std::vector<int32_t> s_idx(t.ns), d_idx(t.nd);
  std::vector<uint32_t> s_info(t.ns);
  std::vector<double> s_val(t.ns), d_val(t.nd);
  if (t.ns) {
    SBD_CUDA(cudaMemcpy(s_idx.data(), t.s_idx, sizeof(int32_t) * t.ns, cudaMemcpyDeviceToHost));
    SBD_CUDA(cudaMemcpy(s_info.data(), t.s_info, sizeof(uint32_t) * t.ns, cudaMemcpyDeviceToHost));
    SBD_CUDA(cudaMemcpy(s_val.data(), t.s_val, sizeof(double) * t.ns, cudaMemcpyDeviceToHost));
  }
  if (t.nd) {
    SBD_CUDA(cudaMemcpy(d_idx.data(), t.d_idx, sizeof(int32_t) * t.nd, cudaMemcpyDeviceToHost));
    SBD_CUDA(cudaMemcpy(d_val.data(), t.d_val, sizeof(double) * t.nd, cudaMemcpyDeviceToHost));
  }
  rb.R = R;
  rb.nblk = (n + R - 1) / R;
  std::vector<int64_t> batch0(rb.nblk + 1, 0);
  std::vector<int32_t> kets;
  std::vector<int64_t> eoff;
  std::vector<RowEntry> ents;
  ents.reserve(t.ns + t.nd);
  struct Tmp {
    int32_t ket;
    int r;
    RowEntry e;
  };
  std::vector<Tmp> tmp;
  std::vector<int32_t> uniq;
  int64_t nbatch = 0;
  for (size_t b = 0; b < rb.nblk; b++) {
    tmp.clear();
    for (int r = 0; r < R; r++) {
      size_t i = b * R + r;
      if (i >= n) break;
      for (int64_t k = t.h_s_off[i]; k < t.h_s_off[i + 1]; k++)
        tmp.push_back({s_idx[k], r, RowEntry{s_val[k], 0x100u | (s_info[k] & 0xFFFFF000u)}});
      for (int64_t k = t.h_d_off[i]; k < t.h_d_off[i + 1]; k++) tmp.push_back({d_idx[k], r, RowEntry{d_val[k], 0u}});
    }
    uniq.resize(tmp.size());
    for (size_t k = 0; k < tmp.size(); k++) uniq[k] = tmp[k].ket;
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    int64_t nb_b = (int64_t)((uniq.size() + kRowBatch - 1) / kRowBatch);
    for (auto& x : tmp) {
      int64_t pos = std::lower_bound(uniq.begin(), uniq.end(), x.ket) - uniq.begin();
      x.e.info |= (uint32_t)(pos % kRowBatch);
      x.ket = (int32_t)(pos / kRowBatch);  // batch within the block
    }
    std::stable_sort(tmp.begin(), tmp.end(), [](const Tmp& a, const Tmp& b2) {
      return a.ket != b2.ket ? a.ket < b2.ket : a.r < b2.r;
    });
    for (int64_t g = 0; g < nb_b; g++)
      for (int s = 0; s < kRowBatch; s++) {
        size_t p = (size_t)(g * kRowBatch + s);
        kets.push_back(p < uniq.size() ? uniq[p] : -1);
      }
    size_t k = 0;
    for (int64_t g = 0; g < nb_b; g++)
      for (int r = 0; r < R; r++) {
        eoff.push_back((int64_t)ents.size());
        while (k < tmp.size() && tmp[k].ket == g && tmp[k].r == r) ents.push_back(tmp[k++].e);
      }
    nbatch += nb_b;
    batch0[b + 1] = nbatch;
  }
  eoff.push_back((int64_t)ents.size());
  rb.nbatch = nbatch;
  rb.blk_batch0 = (int64_t*)dev_alloc(sizeof(int64_t) * batch0.size());
  rb.kets = (int32_t*)dev_alloc(sizeof(int32_t) * std::max<size_t>(kets.size(), 1));
  rb.eoff = (int64_t*)dev_alloc(sizeof(int64_t) * eoff.size());
  rb.ent = (RowEntry*)dev_alloc(sizeof(RowEntry) * std::max<size_t>(ents.size(), 1));
  SBD_CUDA(cudaMemcpy(rb.blk_batch0, batch0.data(), sizeof(int64_t) * batch0.size(), cudaMemcpyHostToDevice));
  if (!kets.empty())
    SBD_CUDA(cudaMemcpy(rb.kets, kets.data(), sizeof(int32_t) * kets.size(), cudaMemcpyHostToDevice));
  SBD_CUDA(cudaMemcpy(rb.eoff, eoff.data(), sizeof(int64_t) * eoff.size(), cudaMemcpyHostToDevice));
  if (!ents.empty())
    SBD_CUDA(cudaMemcpy(rb.ent, ents.data(), sizeof(RowEntry) * ents.size(), cudaMemcpyHostToDevice));
}

void free_row_blocks(RowBlocks& rb) {
  cudaFree(rb.blk_batch0);
  cudaFree(rb.kets);
  cudaFree(rb.eoff);
  cudaFree(rb.ent);
  rb = RowBlocks();
}

template <typename T, bool kWithDiag>
void same_spin_blocked(const RowBlocks& rb, const T* C, T* S, size_t nrows, size_t ncols, const double* hii,
                       const T* J, cudaStream_t s) {
  launch_block_rows<T, kWithDiag, kRowBlock>(rb, C, S, nrows, ncols, hii, J, s);
}

template void same_spin_blocked<double, true>(const RowBlocks&, const double*, double*, size_t, size_t,
                                              const double*, const double*, cudaStream_t);
template void same_spin_blocked<double, false>(const RowBlocks&, const double*, double*, size_t, size_t,
                                               const double*, const double*, cudaStream_t);
template void same_spin_blocked<float, true>(const RowBlocks&, const float*, float*, size_t, size_t, const double*,
                                             const float*, cudaStream_t);
template void same_spin_blocked<float, false>(const RowBlocks&, const float*, float*, size_t, size_t,
                                              const double*, const float*, cudaStream_t);

}  // namespace sbdgpu
