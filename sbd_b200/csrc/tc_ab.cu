// Alpha-beta sigma term on the 5th-generation tensor cores (tcgen05, BF16 in,
// FP32 accumulation in tensor memory).
//
//   sigma[ia,ib] += sum_{(ja,pq,sa) in S_a(ia)} sa * G_ib[pq][ja],
//   G_ib[pq][ja]  = sum_{(jb,rs,sb) in S_b(ib)} (pq|rs) * sb * C[ja,jb]
//
// For one beta string ib the second line is a dense GEMM: M = folded alpha
// pair index pq (P = L(L+1)/2 rows, tiles of 128), N = source alpha string ja
// (tiles of 64), K = the beta singles of ib (chunks of 80).  One CTA owns one
// ib at a time (persistent over ib), keeps the A operand sb_t (pq|rs_t) for
// the current K chunk in shared memory, streams B = C[ja, jb_t] tiles from the
// BF16 transposed vector with cp.async (double buffered), and issues
// tcgen05.mma from one thread into TMEM (one 128 x 64 FP32 accumulator per M
// tile).  The epilogue (16 warps, each reading one 32-lane x 16-column block
// of TMEM with tcgen05.ld) stages one M tile in shared memory and adds the
// entries that are real alpha singles, prefetched into registers while the
// MMAs ran, into the CTA's FP32 sigma column with shared-memory atomics; the
// column is written once per ib into a [nb][na] buffer.
//
// Layouts without swizzle: A is K-major (8-row x 16-byte core matrices,
// LBO = 128 B between core matrices along K, SBO = 10 x 128 B between 8-row
// groups); B is MN-major (core matrix = 8 K rows x 8 consecutive ja), so each
// 16-byte chunk is one cp.async from a row of the transposed vector.  Every
// wait on the MMA completion barrier is bounded; on timeout the kernel records
// an error, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "internal.cuh"

namespace sbdgpu {

namespace {

// 16 warps: warp w reads TMEM lane quarter w % 4 and the column group w / 4
// (kWarpCols columns) of each accumulator in the epilogue
constexpr int kTcThreads = 512;
constexpr int kTcN = 64;         // alpha strings (ja) per tile
constexpr int kTcK = 80;         // beta singles per K chunk (5 MMA steps of 16)
constexpr int kTcKSteps = kTcK / 16;
constexpr int kTcChunks = kTcK / 8;             // 16-byte core-matrix columns along K
constexpr uint32_t kLBO = 128;                  // bytes between K-adjacent core matrices
constexpr uint32_t kSBO = kTcChunks * 128;      // bytes between 8-row groups
constexpr int kTcMaxMTiles = 8;                 // 8 x 64 = 512 TMEM columns
constexpr int kWarpCols = kTcN * 4 / (kTcThreads / 32);  // accumulator columns per warp in the epilogue
static_assert(kWarpCols % 16 == 0 && kWarpCols >= 16, "epilogue reads 16-column groups");
constexpr int kGStride = kTcN + 4;  // epilogue staging row: 16-byte stores of 8 lanes hit distinct banks
constexpr long long kSpinLimit = kMaxSpinLimit;
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s: an MMA tile completes in microseconds
constexpr int kEntPerMt = 2;  // bucket entries per thread and M tile prefetched into registers

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t kmajor_offset(int row, int k) {
  return (uint32_t)(row >> 3) * kSBO + (uint32_t)(k >> 3) * kLBO + (uint32_t)(row & 7) * 16u + (uint32_t)(k & 7) * 2u;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t start) {
  return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((kLBO >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((kSBO >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16, BF16 x BF16 -> F32, A K-major, B MN-major (bit 16), M = 128, N = 64
constexpr uint32_t kIdesc =
    (1u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | ((uint32_t)(kTcN >> 3) << 17) | ((128u >> 4) << 24);

// MN-major canonical layout (no swizzle) of B = [K = t][N = ja]: core matrix =
// 8 K-rows x 16 bytes (8 consecutive ja); LBO between K groups, SBO between
// 8-ja groups.  Offsets are 16-byte aligned per 8-ja chunk, so each chunk is
// one cp.async from a row of the BF16 transposed vector.
__device__ __forceinline__ uint32_t mnmajor_chunk_offset(int n8, int t) {
  return (uint32_t)n8 * kSBO + (uint32_t)(t >> 3) * kLBO + (uint32_t)(t & 7) * 16u;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Polls the barrier at most `limit` times and for at most `max_ns`
// nanoseconds of the global timer (checked every 1024 polls), whichever ends
// first; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long long limit = kSpinLimit,
                                          uint64_t max_ns = kWaitNs) {
  const uint64_t t0 = global_ns();
  for (long long i = 0; i < limit; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 1023) == 1023 && global_ns() - t0 > max_ns) return false;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// One bucket entry: goff | neg<<14 | ia<<15, goff = row * kGStride + column of
// the staged tile.  sigma[ia] += (-1)^neg G[goff], the sign applied by
// flipping the float's sign bit.
__device__ __forceinline__ void tc_scatter(const float* G, float* sig, uint32_t en) {
  const uint32_t g = __float_as_uint(G[en & 0x3FFFu]) ^ ((en << 17) & 0x80000000u);
  atomicAdd(&sig[en >> 15], __uint_as_float(g));
}

struct TcArgs {
  const __nv_bfloat16* ct16;  // C^T in BF16, [nb][na_pad] (zero padded), alpha-string-major convention
  float* out;            // [nb][na] alpha-beta part of sigma, transposed
  const float* vf;       // (pq|rs) folded, [P][P]
  const int64_t* b_off;  // beta singles CSR by bra
  const int32_t* b_idx;
  const uint32_t* b_info;
  const int64_t* bk_off;   // alpha-pair buckets by (ja tile, M tile)
  const uint32_t* bk_ent;  // (pq_local * kGStride + ja_local) | neg<<14 | ia<<15
  int* err;
  int na, nb, P, mtiles, na_pad;
};

__global__ void __launch_bounds__(kTcThreads, 1) tc_ab_kernel(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  constexpr uint32_t kBBytes = (uint32_t)kTcN * kTcK * 2;
  unsigned char* A = smem_raw;                                      // mtiles x 128 x kTcK bf16, K-major
  unsigned char* Bb = A + (size_t)a.mtiles * 128 * kTcK * 2;        // 2 x (kTcK x kTcN bf16), MN-major
  float* G = reinterpret_cast<float*>(Bb + 2 * (size_t)kBBytes);    // 128 x kGStride
  float* sig = G + 128 * kGStride;                                  // na
  __shared__ int s_jb[kTcK];
  __shared__ int s_rs[kTcK];
  __shared__ float s_sb[kTcK];
  __shared__ int64_t s_bo[kTcMaxMTiles + 1];
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_mbar;
  __shared__ int s_fail;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quarter = warp & 3, cgroup = warp >> 2;
  const uint32_t mbar = smem_addr(&s_mbar);
  // TMEM columns: a power of two >= 64 per M tile, so small problems leave
  // room for other CTAs on the SM
  uint32_t ncols = 32;
  while (ncols < (uint32_t)(a.mtiles * kTcN)) ncols <<= 1;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  uint32_t phase = 0;
  const int ntiles = (a.na + kTcN - 1) / kTcN;
  const int Mrows = a.mtiles * 128;
  const uint32_t b_base = smem_addr(Bb);

  // B tile `tile` -> buffer `buf`: 8 chunks of 8 alpha strings per beta single t
  auto load_b = [&](int tile, int buf) {
    const int ja0 = tile * kTcN;
    for (int idx = tid; idx < kTcK * (kTcN / 8); idx += kTcThreads) {
      int t = idx >> 3, n8 = idx & 7;
      int jb = s_jb[t];
      const __nv_bfloat16* src = jb >= 0 ? a.ct16 + (size_t)jb * a.na_pad + ja0 + 8 * n8 : a.ct16;
      cp_async16(b_base + (uint32_t)buf * kBBytes + mnmajor_chunk_offset(n8, t), src, jb >= 0 ? 16u : 0u);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };

  for (int ib = blockIdx.x; ib < a.nb && !s_fail; ib += gridDim.x) {
    for (int i = tid; i < a.na; i += kTcThreads) sig[i] = 0.f;
    const int64_t t0 = a.b_off[ib], t1 = a.b_off[ib + 1];
    for (int64_t kc = t0; kc < t1 && !s_fail; kc += kTcK) {
      __syncthreads();
      for (int t = tid; t < kTcK; t += kTcThreads) {
        int64_t k = kc + t;
        if (k < t1) {
          uint32_t info = a.b_info[k];
          s_jb[t] = a.b_idx[k];
          s_rs[t] = (info >> 12) & 0xFFFu;
          s_sb[t] = (info & 0x80000000u) ? -1.f : 1.f;
        } else {
          s_jb[t] = -1;
          s_rs[t] = -1;
          s_sb[t] = 0.f;
        }
      }
      __syncthreads();
      load_b(0, 0);
      // A[m][t] = sb_t (pq_m | rs_t); (pq|rs) is symmetric, so row rs_t of Vf is
      // read; eight independent loads in flight per thread
      for (int base = 0; base < Mrows * kTcK; base += 8 * kTcThreads) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int idx = base + u * kTcThreads + tid;
          const int t = idx / Mrows, m = idx - t * Mrows;
          const int rs = idx < Mrows * kTcK ? s_rs[t] : -1;
          v[u] = (rs >= 0 && m < a.P) ? __ldg(&a.vf[(size_t)rs * a.P + m]) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int idx = base + u * kTcThreads + tid;
          if (idx < Mrows * kTcK) {
            const int t = idx / Mrows, m = idx - t * Mrows;
            *reinterpret_cast<__nv_bfloat16*>(A + kmajor_offset(m, t)) = __float2bfloat16_rn(s_sb[t] * v[u]);
          }
        }
      }
      // bucket offsets of the next tile's M tiles, fetched one tile ahead
      int64_t bo_next = tid <= a.mtiles ? __ldg(&a.bk_off[tid]) : 0;
      for (int tile = 0; tile < ntiles && !s_fail; tile++) {
        const int buf = tile & 1;
        // this tile's bucket offsets (the previous tile's epilogue ended with a
        // barrier, so nobody still reads the old ones)
        if (tid <= a.mtiles) s_bo[tid] = bo_next;
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_addr(A), b0 = b_base + (uint32_t)buf * kBBytes;
          for (int mt = 0; mt < a.mtiles; mt++)
#pragma unroll
            for (int ks = 0; ks < kTcKSteps; ks++)
              mma_bf16(tmem + (uint32_t)(mt * kTcN), smem_desc(a0 + (uint32_t)mt * 16u * kSBO + ks * 2 * kLBO),
                       smem_desc(b0 + ks * 2 * kLBO), ks > 0 ? 1u : 0u);
          mma_commit(mbar);
        }
        // the other buffer was read by the previous tile's MMAs, which completed
        if (tile + 1 < ntiles) load_b(tile + 1, buf ^ 1);
        if (tile + 1 < ntiles && tid <= a.mtiles) bo_next = __ldg(&a.bk_off[(size_t)(tile + 1) * a.mtiles + tid]);
        // this tile's bucket entries, loaded while the MMAs run: entry
        // e = s_bo[mt] + tid + u * kTcThreads of M tile mt in register [mt][u]
        uint32_t ent[kTcMaxMTiles][kEntPerMt];
#pragma unroll
        for (int mt = 0; mt < kTcMaxMTiles; mt++)
#pragma unroll
          for (int u = 0; u < kEntPerMt; u++) {
            const int64_t e = (mt < a.mtiles ? s_bo[mt] : 0) + tid + (int64_t)u * kTcThreads;
            ent[mt][u] = (mt < a.mtiles && e < s_bo[mt + 1]) ? __ldg(&a.bk_ent[e]) : 0xFFFFFFFFu;
          }
        if (!mbar_wait(mbar, phase)) {
          if (tid == 0) atomicExch(a.err, 1);
          s_fail = 1;
        }
        phase ^= 1u;
        __syncthreads();
        if (s_fail) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int mt = 0; mt < kTcMaxMTiles; mt++) {
          if (mt >= a.mtiles) break;
          // TMEM lanes 32q..32q+31 hold rows pq = 128 mt + 32 q + lane; this
          // warp stages columns [kWarpCols * cgroup, kWarpCols * (cgroup + 1))
          float v[kWarpCols];
          const uint32_t trow =
              tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(mt * kTcN + kWarpCols * cgroup);
#pragma unroll
          for (int c16 = 0; c16 < kWarpCols / 16; c16++) tmem_ld16(trow + 16u * c16, v + 16 * c16);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          float4* grow = reinterpret_cast<float4*>(G + (32 * quarter + lane) * kGStride + kWarpCols * cgroup);
#pragma unroll
          for (int i = 0; i < kWarpCols / 4; i++) grow[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
          __syncthreads();
#pragma unroll
          for (int u = 0; u < kEntPerMt; u++) {
            const uint32_t en = ent[mt][u];
            if (en != 0xFFFFFFFFu) tc_scatter(G, sig, en);
          }
          // entries beyond the prefetched ones
          for (int64_t e = s_bo[mt] + tid + (int64_t)kEntPerMt * kTcThreads; e < s_bo[mt + 1]; e += kTcThreads) {
            tc_scatter(G, sig, __ldg(&a.bk_ent[e]));
          }
          __syncthreads();
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      }
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    for (int i = tid; i < a.na; i += kTcThreads) a.out[(size_t)ib * a.na + i] = sig[i];
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// The bounded mbarrier wait of tc_ab_kernel on its own: one warp waits for
// phase 0 of a barrier that expects one arrival; with arrive = 0 nothing
// arrives, so the wait must give up after `limit` polls and report it.
__global__ void wait_probe_kernel(long long limit, int arrive, int* timed_out) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t mbar = smem_addr(&bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (arrive && threadIdx.x == 0)
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(mbar) : "memory");
  const bool ok = mbar_wait(mbar, 0u, limit);
  __syncthreads();
  if (threadIdx.x == 0) *timed_out = ok ? 0 : 1;
}

__global__ void to_bf16_padded_kernel(const float* __restrict__ in, __nv_bfloat16* __restrict__ out, size_t rows,
                                      size_t cols, size_t cols_pad) {
  size_t n = rows * cols_pad;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    size_t r = i / cols_pad, cc = i - r * cols_pad;
    out[i] = __float2bfloat16_rn(cc < cols ? in[r * cols + cc] : 0.f);
  }
}

size_t tc_smem_bytes(int mtiles, size_t na) {
  return (size_t)mtiles * 128 * kTcK * 2 + 2 * (size_t)kTcN * kTcK * 2 + 128 * kGStride * 4 + na * 4;
}

}  // namespace

// status[0]: the wait with no arrival timed out (expected 1); status[1]: the
// wait after one arrival timed out (expected 0)
void wait_selftest(sbdgpu_ctx* c, long long limit, int* status) {
  int* d = (int*)dev_alloc(2 * sizeof(int));
  try {
    SBD_CUDA(cudaMemsetAsync(d, 0xFF, 2 * sizeof(int), c->stream));
    wait_probe_kernel<<<1, 32, 0, c->stream>>>(limit, 0, d);
    SBD_CUDA(cudaGetLastError());
    wait_probe_kernel<<<1, 32, 0, c->stream>>>(limit, 1, d + 1);
    SBD_CUDA(cudaGetLastError());
    SBD_CUDA(cudaMemcpyAsync(status, d, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    SBD_CUDA(cudaStreamSynchronize(c->stream));
  } catch (...) {
    cudaFree(d);
    throw;
  }
  cudaFree(d);
}

bool tc_ab_supported(const sbdgpu_ctx* c) {
  int mtiles = (c->P + 127) / 128;
  // na < 2^17: ia takes bits 15..31 of an entry, and an entry of all ones is
  // the empty-register marker
  return mtiles <= kTcMaxMTiles && c->na < (1 << 17) - 1 && tc_smem_bytes(mtiles, c->na) <= 225 * 1024;
}

// Alpha singles bucketed by (tile of 64 source strings ja, M tile of 128 pq).
void build_tc_buckets(sbdgpu_ctx* c) {
  if (c->tc_bk_ent) return;
  const SpinTables& ta = c->tab[0];
  int mtiles = (c->P + 127) / 128;
  size_t na = c->na;
  std::vector<int32_t> idx(ta.ns);
  std::vector<uint32_t> info(ta.ns);
  if (ta.ns) {
    SBD_CUDA(cudaMemcpy(idx.data(), ta.s_idx, sizeof(int32_t) * ta.ns, cudaMemcpyDeviceToHost));
    SBD_CUDA(cudaMemcpy(info.data(), ta.s_info, sizeof(uint32_t) * ta.ns, cudaMemcpyDeviceToHost));
  }
  size_t ntiles = (na + kTcN - 1) / kTcN;
  std::vector<std::vector<uint32_t>> bucket(ntiles * mtiles);
  for (size_t ja = 0; ja < na; ja++) {
    for (int64_t k = ta.h_s_off[ja]; k < ta.h_s_off[ja + 1]; k++) {
      // row ja, ket ia: pair index and sign are those of the pair (ia <- ja)
      uint32_t pq = (info[k] >> 12) & 0xFFFu;
      uint32_t neg = (info[k] >> 31) & 1u;
      uint32_t ia = (uint32_t)idx[k];
      size_t tile = ja / kTcN;
      uint32_t goff = (pq % 128u) * (uint32_t)kGStride + (uint32_t)(ja % kTcN);  // < 2^14
      uint32_t e = goff | (neg << 14) | (ia << 15);
      bucket[tile * mtiles + pq / 128].push_back(e);
    }
  }
  std::vector<int64_t> off(bucket.size() + 1, 0);
  for (size_t i = 0; i < bucket.size(); i++) off[i + 1] = off[i] + (int64_t)bucket[i].size();
  std::vector<uint32_t> ent((size_t)off.back());
  for (size_t i = 0; i < bucket.size(); i++) std::copy(bucket[i].begin(), bucket[i].end(), ent.begin() + off[i]);
  c->tc_bk_off = (int64_t*)dev_alloc(sizeof(int64_t) * off.size());
  c->tc_bk_ent = (uint32_t*)dev_alloc(sizeof(uint32_t) * std::max<size_t>(ent.size(), 1));
  SBD_CUDA(cudaMemcpy(c->tc_bk_off, off.data(), sizeof(int64_t) * off.size(), cudaMemcpyHostToDevice));
  if (!ent.empty())
    SBD_CUDA(cudaMemcpy(c->tc_bk_ent, ent.data(), sizeof(uint32_t) * ent.size(), cudaMemcpyHostToDevice));
  if (!c->tc_err) {
    c->tc_err = (int*)dev_alloc(sizeof(int));
    SBD_CUDA(cudaMemset(c->tc_err, 0, sizeof(int)));
  }
}

// out[ib][ia] = alpha-beta part of sigma (FP32, transposed) from ct = C^T.
void tc_alpha_beta(sbdgpu_ctx* c, const float* ct, float* out) {
  const SpinTables& tb = c->tab[1];
  size_t na_pad = (c->na + kTcN - 1) / kTcN * kTcN;
  if (!c->ct16) c->ct16 = dev_alloc(sizeof(__nv_bfloat16) * na_pad * c->nb);
  __nv_bfloat16* ct16 = static_cast<__nv_bfloat16*>(c->ct16);
  to_bf16_padded_kernel<<<592, 256, 0, c->stream>>>(ct, ct16, c->nb, c->na, na_pad);
  SBD_CUDA(cudaGetLastError());
  TcArgs a;
  a.ct16 = ct16;
  a.na_pad = (int)na_pad;
  a.out = out;
  a.vf = c->vf32;
  a.b_off = tb.s_off;
  a.b_idx = tb.s_idx;
  a.b_info = tb.s_info;
  a.bk_off = c->tc_bk_off;
  a.bk_ent = c->tc_bk_ent;
  a.err = c->tc_err;
  a.na = (int)c->na;
  a.nb = (int)c->nb;
  a.P = c->P;
  a.mtiles = (c->P + 127) / 128;
  size_t smem = tc_smem_bytes(a.mtiles, c->na);
  allow_dynamic_smem(reinterpret_cast<const void*>(tc_ab_kernel), c->device);
  int sms = 148;
  SBD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  int grid = (int)std::min<size_t>((size_t)sms, c->nb);
  tc_ab_kernel<<<grid, kTcThreads, smem, c->stream>>>(a);
  SBD_CUDA(cudaGetLastError());
}

// Reads and clears the timeout flag: a timeout is reported once, and the
// context's later tensor-core sigma builds start clean.
int tc_error(sbdgpu_ctx* c) {
  if (!c->tc_err) return 0;
  int h = 0;
  SBD_CUDA(cudaMemcpyAsync(&h, c->tc_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  SBD_CUDA(cudaMemsetAsync(c->tc_err, 0, sizeof(int), c->stream));
  SBD_CUDA(cudaStreamSynchronize(c->stream));
  return h;
}

}  // namespace sbdgpu
