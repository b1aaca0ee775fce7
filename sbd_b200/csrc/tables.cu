// Excitation tables on the GPU.
//
// Replaces GenerateExcitation (chemistry/tpb/helper.h:132-182): for every bra
// string i, the ascending list of kets j with popcount(s_i ^ s_j) == 2 (single)
// or == 4 (double).  One warp per bra row scans all kets 32 at a time; a warp
// ballot compacts the hits in ascending j, so the lists are bit-exact with the
// reference's.  The same pass computes each entry's payload: the orbitals
// involved, the string-internal fermionic sign and the FP64 matrix element part
// that depends on this spin's strings only.
#include <algorithm>
#include <numeric>

#include "internal.cuh"

namespace sbdgpu {

namespace {

__device__ __forceinline__ int pair_index(int p, int q) {
  int a = p > q ? p : q, b = p > q ? q : p;
  return a * (a + 1) / 2 + b;
}

// (-1)^(occupied orbitals of s strictly between p and q)
__device__ __forceinline__ bool neg_between(uint64_t s, int p, int q) {
  int lo = p < q ? p : q, hi = p < q ? q : p;
  uint64_t mask = (hi - lo < 2) ? 0ull : (((1ull << hi) - 1ull) & ~((2ull << lo) - 1ull));
  return __popcll(s & mask) & 1;
}

__global__ void count_kernel(const uint64_t* __restrict__ s, int n, int* cs, int* cd) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= n) return;
  uint64_t si = s[warp];
  int a = 0, b = 0;
  for (int j = lane; j < n; j += 32) {
    int d = __popcll(si ^ s[j]);
    a += (d == 2);
    b += (d == 4);
  }
  for (int o = 16; o; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    cs[warp] = a;
    cd[warp] = b;
  }
}

__global__ void fill_kernel(const uint64_t* __restrict__ s, int n, int L, const int64_t* __restrict__ s_off,
                            const int64_t* __restrict__ d_off, const double* __restrict__ h1,
                            const double* __restrict__ vf, int P, int32_t* s_idx, uint32_t* s_info,
                            double* s_val, int32_t* d_idx, double* d_val) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= n) return;
  uint64_t si = s[warp];
  int64_t bs = s_off[warp], bd = d_off[warp];
  unsigned lt = (1u << lane) - 1u;
  for (int j0 = 0; j0 < n; j0 += 32) {
    int j = j0 + lane;
    uint64_t sj = j < n ? s[j] : si;
    uint64_t diff = si ^ sj;
    int d = __popcll(diff);
    unsigned ms = __ballot_sync(0xffffffffu, d == 2);
    unsigned md = __ballot_sync(0xffffffffu, d == 4);
    if (d == 2) {
      int64_t k = bs + __popc(ms & lt);
      int p = __ffsll((long long)(si & diff)) - 1;  // created (in bra)
      int q = __ffsll((long long)(sj & diff)) - 1;  // annihilated (in ket)
      bool neg = neg_between(sj, p, q);
      int pq = pair_index(p, q);
      // OneExcite, chemistry/basic/determinants.h:400-422, same-spin part
      double e = h1[p * L + q];
      uint64_t occ = sj;
      while (occ) {
        int r = __ffsll((long long)occ) - 1;
        occ &= occ - 1;
        e += vf[(size_t)pq * P + pair_index(r, r)] - vf[(size_t)pair_index(p, r) * P + pair_index(r, q)];
      }
      s_idx[k] = j;
      s_info[k] = (uint32_t)p | ((uint32_t)q << 6) | ((uint32_t)pq << 12) | (neg ? 0x80000000u : 0u);
      s_val[k] = neg ? -e : e;
    }
    if (d == 4) {
      int64_t k = bd + __popc(md & lt);
      uint64_t c = si & diff, a = sj & diff;
      int p1 = __ffsll((long long)c) - 1;
      c &= c - 1;
      int p2 = __ffsll((long long)c) - 1;
      int q1 = __ffsll((long long)a) - 1;
      a &= a - 1;
      int q2 = __ffsll((long long)a) - 1;
      // TwoExcite, chemistry/basic/determinants.h:424-442, restricted to one string
      bool neg = neg_between(sj, q1, p1) ^ neg_between(sj, q2, p2);
      if (p1 > q2 || p2 < q1) neg = !neg;
      double e = vf[(size_t)pair_index(p1, q1) * P + pair_index(p2, q2)] -
                 vf[(size_t)pair_index(p1, q2) * P + pair_index(p2, q1)];
      d_idx[k] = j;
      d_val[k] = neg ? -e : e;
    }
    bs += __popc(ms);
    bd += __popc(md);
  }
}

__global__ void sell_fill_kernel(int n, const int64_t* __restrict__ s_off, const int32_t* __restrict__ s_idx,
                                 const uint32_t* __restrict__ s_info, const int64_t* __restrict__ sell_off,
                                 const int32_t* __restrict__ sell_w, uint32_t* sell) {
  // every lane of every slice, the padding lanes past the last bra string
  // included: those get kSellInvalid entries, never uninitialised memory
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int nslice = (n + kSlice - 1) / kSlice;
  if (i >= nslice * kSlice) return;
  int slice = i / kSlice, lane = i % kSlice;
  int64_t base = sell_off[slice];
  int w = sell_w[slice];
  int64_t b = i < n ? s_off[i] : 0, e = i < n ? s_off[i + 1] : 0;
  for (int t = 0; t < w; t++) {
    uint32_t v = kSellInvalid;
    if (b + t < e) {
      uint32_t info = s_info[b + t];
      v = (uint32_t)s_idx[b + t] | (((info >> 12) & 0xFFFu) << 16) | (info & 0x80000000u);
    }
    sell[base + (int64_t)t * kSlice + lane] = v;
  }
}

}  // namespace

void free_tables(SpinTables& t) {
  cudaFree(t.s_off); cudaFree(t.d_off); cudaFree(t.s_idx); cudaFree(t.s_info); cudaFree(t.s_val);
  cudaFree(t.d_idx); cudaFree(t.d_val); cudaFree(t.sell_off); cudaFree(t.sell_w); cudaFree(t.sell);
  t = SpinTables();
}

static void build_one(sbdgpu_ctx* c, SpinTables& t, const uint64_t* dstr, size_t n) {
  cudaStream_t st = c->stream;
  t.n = n;
  int ni = (int)n;
  int *cs = nullptr, *cd = nullptr;
  cs = (int*)dev_alloc(sizeof(int) * (n + 1));
  cd = (int*)dev_alloc(sizeof(int) * (n + 1));
  int threads = 256;
  int blocks = (int)((n * 32 + threads - 1) / threads);
  count_kernel<<<blocks, threads, 0, st>>>(dstr, ni, cs, cd);
  SBD_CUDA(cudaGetLastError());
  std::vector<int> hs(n), hd(n);
  SBD_CUDA(cudaMemcpyAsync(hs.data(), cs, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  SBD_CUDA(cudaMemcpyAsync(hd.data(), cd, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  SBD_CUDA(cudaStreamSynchronize(st));
  cudaFree(cs);
  cudaFree(cd);
  t.h_s_off.assign(n + 1, 0);
  t.h_d_off.assign(n + 1, 0);
  for (size_t i = 0; i < n; i++) {
    t.h_s_off[i + 1] = t.h_s_off[i] + hs[i];
    t.h_d_off[i + 1] = t.h_d_off[i] + hd[i];
  }
  t.ns = (uint64_t)t.h_s_off[n];
  t.nd = (uint64_t)t.h_d_off[n];
  t.max_s = n ? *std::max_element(hs.begin(), hs.end()) : 0;
  t.s_off = (int64_t*)dev_alloc(sizeof(int64_t) * (n + 1));
  t.d_off = (int64_t*)dev_alloc(sizeof(int64_t) * (n + 1));
  SBD_CUDA(cudaMemcpyAsync(t.s_off, t.h_s_off.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st));
  SBD_CUDA(cudaMemcpyAsync(t.d_off, t.h_d_off.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st));
  size_t ns = std::max<uint64_t>(t.ns, 1), nd = std::max<uint64_t>(t.nd, 1);
  t.s_idx = (int32_t*)dev_alloc(sizeof(int32_t) * ns);
  t.s_info = (uint32_t*)dev_alloc(sizeof(uint32_t) * ns);
  t.s_val = (double*)dev_alloc(sizeof(double) * ns);
  t.d_idx = (int32_t*)dev_alloc(sizeof(int32_t) * nd);
  t.d_val = (double*)dev_alloc(sizeof(double) * nd);
  fill_kernel<<<blocks, threads, 0, st>>>(dstr, ni, c->L, t.s_off, t.d_off, c->h1, c->vf, c->P, t.s_idx,
                                          t.s_info, t.s_val, t.d_idx, t.d_val);
  SBD_CUDA(cudaGetLastError());
  // sliced ELL of the singles
  t.nslice = (n + kSlice - 1) / kSlice;
  std::vector<int32_t> w(t.nslice, 0);
  std::vector<int64_t> so(t.nslice + 1, 0);
  for (size_t i = 0; i < n; i++) w[i / kSlice] = std::max<int32_t>(w[i / kSlice], hs[i]);
  for (size_t s = 0; s < t.nslice; s++) so[s + 1] = so[s] + (int64_t)w[s] * kSlice;
  t.sell_off = (int64_t*)dev_alloc(sizeof(int64_t) * (t.nslice + 1));
  t.sell_w = (int32_t*)dev_alloc(sizeof(int32_t) * std::max<size_t>(t.nslice, 1));
  t.sell = (uint32_t*)dev_alloc(sizeof(uint32_t) * std::max<int64_t>(so[t.nslice], 1));
  SBD_CUDA(cudaMemcpyAsync(t.sell_off, so.data(), sizeof(int64_t) * (t.nslice + 1), cudaMemcpyHostToDevice, st));
  SBD_CUDA(cudaMemcpyAsync(t.sell_w, w.data(), sizeof(int32_t) * t.nslice, cudaMemcpyHostToDevice, st));
  if (n) {
    const int nlanes = (int)(t.nslice * kSlice);
    sell_fill_kernel<<<(nlanes + 255) / 256, 256, 0, st>>>(ni, t.s_off, t.s_idx, t.s_info, t.sell_off, t.sell_w,
                                                          t.sell);
    SBD_CUDA(cudaGetLastError());
  }
  SBD_CUDA(cudaStreamSynchronize(st));
}

void build_tables(sbdgpu_ctx* c) {
  if (c->tables_ready) return;
  build_one(c, c->tab[0], c->astr, c->na);
  build_one(c, c->tab[1], c->bstr, c->nb);
  c->tables_ready = true;
}

}  // namespace sbdgpu
