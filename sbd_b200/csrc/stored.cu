// Stored Hamiltonian (method 1).
//
// Replaces makeQCham (chemistry/tpb/qcham.h:10-312), which keeps every
// off-diagonal element of the bra rows as (bra, ket, Hij) triplets per task and
// thread, and the stored mult (chemistry/tpb/mult.h:13-123), which adds
// hii*C and then Hij*C[ket] over the triplets.  Here the same elements are one
// CSR matrix in HBM, rows = bra determinants ia*nb + ib in the
// alpha-string-major sign convention, built from the excitation tables:
//
//   row (ia, ib):  alpha singles  (ja, ib)  s_a + sg_a * Jb[pq][ib]
//                  alpha doubles  (ja, ib)  d_a
//                  beta singles   (ia, jb)  s_b + sg_b * Ja[rs][ia]
//                  beta doubles   (ia, jb)  d_b
//                  alpha-beta     (ja, jb)  sg_a * sg_b * (pq|rs)   for every pair of singles
//
// which are the reference's task types 2, 1 and 0 (qcham.h:204-300) and the
// same element values the on-the-fly kernels use.  The row start has a closed
// form from the per-string table lengths, so the fill needs no scan:
//   off(ia, ib) = base[ia] + ib*(Sa+Da)(ia) + Bpre[ib] + Sa(ia)*SBpre[ib].
// The product is one warp per row: coalesced loads of (col, val), gathered C,
// a warp-shuffle reduction.  HBM bound: 12 bytes per stored element.
#include <algorithm>

#include "internal.cuh"

namespace sbdgpu {

namespace {

struct DevTab {
  const int64_t* s_off;
  const int32_t* s_idx;
  const uint32_t* s_info;
  const double* s_val;
  const int64_t* d_off;
  const int32_t* d_idx;
  const double* d_val;
};

DevTab view(const SpinTables& t) { return DevTab{t.s_off, t.s_idx, t.s_info, t.s_val, t.d_off, t.d_idx, t.d_val}; }

constexpr int kStoredThreads = 256;

__global__ void __launch_bounds__(kStoredThreads) fill_stored_kernel(
    size_t na, size_t nb, int P, const int64_t* __restrict__ abase, const int64_t* __restrict__ bpre,
    const int64_t* __restrict__ sbpre, DevTab ta, DevTab tb, const double* __restrict__ Ja,
    const double* __restrict__ Jb, const double* __restrict__ vf, int64_t* __restrict__ row,
    uint32_t* __restrict__ col, double* __restrict__ val) {
  const int lane = threadIdx.x & 31;
  const size_t nrows = na * nb;
  const size_t wstride = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t r = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nrows; r += wstride) {
    const size_t ia = r / nb, ib = r - ia * nb;
    const int64_t as0 = ta.s_off[ia], sa = ta.s_off[ia + 1] - as0;
    const int64_t ad0 = ta.d_off[ia], da = ta.d_off[ia + 1] - ad0;
    const int64_t bs0 = tb.s_off[ib], sb = tb.s_off[ib + 1] - bs0;
    const int64_t bd0 = tb.d_off[ib], db = tb.d_off[ib + 1] - bd0;
    int64_t o = abase[ia] + (int64_t)ib * (sa + da) + bpre[ib] + sa * sbpre[ib];
    if (lane == 0) row[r] = o;
    for (int64_t k = lane; k < sa; k += 32) {
      const int64_t e = as0 + k;
      const uint32_t info = ta.s_info[e];
      const double J = Jb[(size_t)((info >> 12) & 0xFFFu) * nb + ib];
      col[o + k] = (uint32_t)((size_t)ta.s_idx[e] * nb + ib);
      val[o + k] = ta.s_val[e] + ((info & 0x80000000u) ? -J : J);
    }
    o += sa;
    for (int64_t k = lane; k < da; k += 32) {
      const int64_t e = ad0 + k;
      col[o + k] = (uint32_t)((size_t)ta.d_idx[e] * nb + ib);
      val[o + k] = ta.d_val[e];
    }
    o += da;
    for (int64_t k = lane; k < sb; k += 32) {
      const int64_t e = bs0 + k;
      const uint32_t info = tb.s_info[e];
      const double J = Ja[(size_t)((info >> 12) & 0xFFFu) * na + ia];
      col[o + k] = (uint32_t)(ia * nb + (size_t)tb.s_idx[e]);
      val[o + k] = tb.s_val[e] + ((info & 0x80000000u) ? -J : J);
    }
    o += sb;
    for (int64_t k = lane; k < db; k += 32) {
      const int64_t e = bd0 + k;
      col[o + k] = (uint32_t)(ia * nb + (size_t)tb.d_idx[e]);
      val[o + k] = tb.d_val[e];
    }
    o += db;
    const int64_t nab = sa * sb;
    for (int64_t m = lane; m < nab; m += 32) {
      const int64_t t = m / sb, u = m - t * sb;
      const uint32_t ia_info = ta.s_info[as0 + t], ib_info = tb.s_info[bs0 + u];
      const double v = vf[(size_t)((ia_info >> 12) & 0xFFFu) * P + ((ib_info >> 12) & 0xFFFu)];
      col[o + m] = (uint32_t)((size_t)ta.s_idx[as0 + t] * nb + (size_t)tb.s_idx[bs0 + u]);
      val[o + m] = ((ia_info ^ ib_info) & 0x80000000u) ? -v : v;
    }
  }
}

// S[r] = hii[r] C[r] + sum_k val[k] C[col[k]] over row r's stored elements.
__global__ void __launch_bounds__(kStoredThreads) spmv_kernel(size_t nrows, const int64_t* __restrict__ row,
                                                              const uint32_t* __restrict__ col,
                                                              const double* __restrict__ val,
                                                              const double* __restrict__ hii,
                                                              const double* __restrict__ C, double* __restrict__ S) {
  const int lane = threadIdx.x & 31;
  const size_t wstride = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t r = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nrows; r += wstride) {
    const int64_t b = row[r], e = row[r + 1];
    double acc = 0.0;
#pragma unroll 4
    for (int64_t k = b + lane; k < e; k += 32) acc += __ldg(&val[k]) * __ldg(&C[__ldg(&col[k])]);
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) S[r] = hii[r] * C[r] + acc;
  }
}

unsigned warp_grid(size_t rows, int device) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  size_t want = (rows * 32 + kStoredThreads - 1) / kStoredThreads;
  return (unsigned)std::max<size_t>(1, std::min<size_t>(want, (size_t)sms * 8 * 16));
}

}  // namespace

void release_hamiltonian(sbdgpu_ctx* c) {
  cudaFree(c->hs_row);
  cudaFree(c->hs_col);
  cudaFree(c->hs_val);
  c->hs_row = nullptr;
  c->hs_col = nullptr;
  c->hs_val = nullptr;
  c->hs_nnz = 0;
  c->stored = false;
}

void store_hamiltonian(sbdgpu_ctx* c) {
  if (c->stored) return;
  build_tables(c);
  compute_hii(c);  // also builds the J tables
  if (c->N > 0xFFFFFFFFull)
    throw Error{SBDGPU_ERR_LIMIT, "stored Hamiltonian: more than 2^32 - 1 determinants"};
  const SpinTables& ta = c->tab[0];
  const SpinTables& tb = c->tab[1];
  const size_t na = c->na, nb = c->nb;
  // closed-form row starts from the per-string table lengths
  std::vector<int64_t> bpre(nb + 1, 0), sbpre(nb + 1, 0), abase(na + 1, 0);
  for (size_t ib = 0; ib < nb; ib++) {
    int64_t s = tb.h_s_off[ib + 1] - tb.h_s_off[ib], d = tb.h_d_off[ib + 1] - tb.h_d_off[ib];
    bpre[ib + 1] = bpre[ib] + s + d;
    sbpre[ib + 1] = sbpre[ib] + s;
  }
  for (size_t ia = 0; ia < na; ia++) {
    int64_t s = ta.h_s_off[ia + 1] - ta.h_s_off[ia], d = ta.h_d_off[ia + 1] - ta.h_d_off[ia];
    abase[ia + 1] = abase[ia] + (int64_t)nb * (s + d) + bpre[nb] + s * sbpre[nb];
  }
  const uint64_t nnz = (uint64_t)abase[na];
  const size_t need = nnz * (sizeof(uint32_t) + sizeof(double)) + sizeof(int64_t) * (c->N + 1);
  size_t free_b = 0, total_b = 0;
  SBD_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const size_t margin = (size_t)1 << 30;
  if (need + margin > free_b)
    throw Error{SBDGPU_ERR_LIMIT, "stored Hamiltonian: needs " + std::to_string(need >> 20) + " MiB, " +
                                      std::to_string(free_b >> 20) + " MiB free on the device"};
  int64_t* d_aux = (int64_t*)dev_alloc(sizeof(int64_t) * (na + 2 * nb));
  int64_t* d_abase = d_aux;
  int64_t* d_bpre = d_aux + na;
  int64_t* d_sbpre = d_aux + na + nb;
  cudaStream_t st = c->stream;
  try {
    SBD_CUDA(cudaMemcpyAsync(d_abase, abase.data(), sizeof(int64_t) * na, cudaMemcpyHostToDevice, st));
    SBD_CUDA(cudaMemcpyAsync(d_bpre, bpre.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, st));
    SBD_CUDA(cudaMemcpyAsync(d_sbpre, sbpre.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, st));
    c->hs_row = (int64_t*)dev_alloc(sizeof(int64_t) * (c->N + 1));
    c->hs_col = (uint32_t*)dev_alloc(sizeof(uint32_t) * std::max<uint64_t>(nnz, 1));
    c->hs_val = (double*)dev_alloc(sizeof(double) * std::max<uint64_t>(nnz, 1));
    int64_t total = (int64_t)nnz;
    SBD_CUDA(cudaMemcpyAsync(c->hs_row + c->N, &total, sizeof(int64_t), cudaMemcpyHostToDevice, st));
    if (c->N) {
      fill_stored_kernel<<<warp_grid(c->N, c->device), kStoredThreads, 0, st>>>(
          na, nb, c->P, d_abase, d_bpre, d_sbpre, view(ta), view(tb), c->ja, c->jb, c->vf, c->hs_row, c->hs_col,
          c->hs_val);
      SBD_CUDA(cudaGetLastError());
    }
    SBD_CUDA(cudaStreamSynchronize(st));
  } catch (...) {
    cudaFree(d_aux);
    release_hamiltonian(c);
    throw;
  }
  cudaFree(d_aux);
  c->hs_nnz = nnz;
  c->stored = true;
}

void spmv_stored(sbdgpu_ctx* c, const double* C, double* S) {
  cudaStream_t st = c->stream;
  SBD_CUDA(cudaEventRecord(c->ev[0], st));
  if (c->N) {
    spmv_kernel<<<warp_grid(c->N, c->device), kStoredThreads, 0, st>>>(c->N, c->hs_row, c->hs_col, c->hs_val, c->hii,
                                                                       C, S);
    SBD_CUDA(cudaGetLastError());
  }
  // one phase: the event pairs of the on-the-fly path's later phases are empty
  SBD_CUDA(cudaEventRecord(c->ev[1], st));
  SBD_CUDA(cudaEventRecord(c->ev[2], st));
  SBD_CUDA(cudaEventRecord(c->ev[3], st));
}

}  // namespace sbdgpu
