// Alpha-beta sigma term on the 5th-generation tensor cores (tcgen05, BF16 in,
// FP32 accumulation in tensor memory).
//
//   sigma[ia,ib] += sum_{(ja,pq,sa) in S_a(ia)} sa * G_ib[pq][ja],
//   G_ib[pq][ja]  = sum_{(jb,rs,sb) in S_b(ib)} (pq|rs) * sb * C[ja,jb]
//
// For one beta string ib the second line is a dense GEMM: M = folded alpha
// pair index pq (P = L(L+1)/2 rows, tiles of 128), N = source alpha string ja
// (tiles of 64), K = the beta singles of ib (chunks of up to 80).  One
// persistent CTA per SM takes one ib at a time and runs a warp-specialised
// pipeline:
//
//   warp 0 (one thread)   issues tcgen05.mma into a ring of 8 TMEM
//                         accumulator stages (one 128 x 64 FP32 tile each)
//   warps 1-3 (producers) build A = sb_t (pq|rs_t) in BF16 (K-major) once per
//                         ib and K chunk, and stream B = C[ja, jb_t] tiles
//                         from the BF16 transposed vector with cp.async into
//                         four slots (MN-major), completion on mbarriers
//   warps 4-19 (epilogue) each drain one 32-lane x 16-column block of a stage
//                         (tcgen05.ld), stage it in a private shared-memory
//                         tile, release the TMEM stage, and add the entries
//                         that are real alpha singles into the column ib of
//                         the [nb][na] output with global FP32 reductions
//                         (native in L2; the CTA's column stays in L2, while
//                         a float add on shared memory is a compare-and-swap
//                         loop and measured 1.6x slower for the whole kernel)
//
// so the MMAs of later tiles overlap the epilogue of earlier ones.  When the A
// operand of all M tiles does not fit in shared memory (norb 48), the M tiles
// are taken in groups and the B tiles are streamed once per group.
//
// Layouts without swizzle: A is K-major (8-row x 16-byte core matrices,
// LBO = 128 B between core matrices along K, SBO = 10 x 128 B between 8-row
// groups); B is MN-major (core matrix = 8 K rows x 8 consecutive ja), so each
// 16-byte chunk is one cp.async from a row of the transposed vector.  Every
// mbarrier wait is bounded by a poll count and by the global timer; on timeout
// the kernel records an error, every role stops at its next check, and the CTA
// frees its tensor memory and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "internal.cuh"

namespace sbdgpu {

namespace {

constexpr int kTcThreads = 640;  // warp 0 MMA, warps 1-3 producers, warps 4-19 epilogue
constexpr int kProdThreads = 96;
constexpr int kEpiWarps = 16;
constexpr int kEpiThreads = kEpiWarps * 32;
constexpr int kTcN = 64;         // alpha strings (ja) per tile
constexpr int kEpiCols = kTcN * 4 / kEpiWarps;  // accumulator columns per epilogue warp
constexpr int kTcK = 80;         // beta singles per K chunk (at most 5 MMA steps of 16)
constexpr int kTcChunks = kTcK / 8;             // 16-byte core-matrix columns along K
constexpr uint32_t kLBO = 128;                  // bytes between K-adjacent core matrices
constexpr uint32_t kSBO = kTcChunks * 128;      // bytes between 8-row groups
constexpr int kStages = 8;                      // TMEM accumulator ring: 8 x 64 = 512 columns
constexpr int kBSlots = 4;                      // B tiles in flight
constexpr uint32_t kABytesPerMt = 128u * kTcK * 2;   // one M tile of A
constexpr uint32_t kBBytes = (uint32_t)kTcN * kTcK * 2;  // one B slot
constexpr int kGS = kEpiCols;  // staging row stride (floats)
constexpr uint32_t kStgBytes = (uint32_t)kEpiWarps * 32 * kGS * 4;
constexpr long long kSpinLimit = kMaxSpinLimit;
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s: every wait here normally lasts microseconds
constexpr int kEntPref = 4;  // bucket entries per lane prefetched before a stage's wait

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

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(mbar) : "memory");
}

// arrives on the barrier once every cp.async this thread issued so far has
// landed (the barrier's expected count includes this arrival)
__device__ __forceinline__ void cp_async_arrive(uint32_t mbar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void named_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// One bucket entry: goff | neg<<11 | ia<<12, goff = row * kGS + column of the
// epilogue warp's 32 x kEpiCols staged block.  col[ia] += (-1)^neg G[goff],
// the sign applied by flipping the float's sign bit; the add is a global
// reduction (its result is not read).
__device__ __forceinline__ void tc_scatter(const float* G, float* col, uint32_t en) {
  const uint32_t g = __float_as_uint(G[en & 0x7FFu]) ^ ((en << 20) & 0x80000000u);
  atomicAdd(&col[en >> 12], __uint_as_float(g));
}

struct TcArgs {
  const __nv_bfloat16* ct16;  // C^T in BF16, [nb][na_pad] (zero padded), alpha-string-major convention
  float* out;            // [nb][na] alpha-beta part of sigma, transposed (zeroed before the launch)
  const float* vf;       // (pq|rs) folded, [P][P]
  const int64_t* b_off;  // beta singles CSR by bra
  const int32_t* b_idx;
  const uint32_t* b_info;
  const int64_t* bk_off;   // alpha singles bucketed by (ja tile, M tile, epilogue warp)
  const uint32_t* bk_ent;
  int* err;
  int na, nb, P, mtiles, na_pad, gsz;  // gsz: M tiles per group (A of a group fits in shared memory)
};

// The sequence of pipeline stages is the same for every role:
//   for ib (persistent) / K chunk c / M group g / ja tile / M tile in g.
__global__ void __launch_bounds__(kTcThreads, 1) tc_ab_kernel(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* A = smem_raw;                                           // gsz x 128 x kTcK bf16, K-major
  unsigned char* Bb = A + (size_t)a.gsz * kABytesPerMt;                  // kBSlots x (kTcK x kTcN bf16)
  float* stg = reinterpret_cast<float*>(Bb + (size_t)kBSlots * kBBytes); // kEpiWarps x 32 x kGS
  __shared__ int s_jb[kTcK];
  __shared__ int s_rs[kTcK];
  __shared__ float s_sb[kTcK];
  __shared__ __align__(8) uint64_t bar_a_full, bar_a_empty, bar_done;
  __shared__ __align__(8) uint64_t bar_b_full[kBSlots], bar_b_empty[kBSlots];
  __shared__ __align__(8) uint64_t bar_acc_full[kStages], bar_acc_empty[kStages];
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_fail;
  __shared__ int s_prod_stop, s_epi_stop;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                 "r"(kStages * kTcN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(smem_addr(&bar_a_full), kProdThreads);
    mbar_init(smem_addr(&bar_a_empty), 1);
    mbar_init(smem_addr(&bar_done), 1);
    for (int i = 0; i < kBSlots; i++) {
      mbar_init(smem_addr(&bar_b_full[i]), kProdThreads);
      mbar_init(smem_addr(&bar_b_empty[i]), 1);
    }
    for (int i = 0; i < kStages; i++) {
      mbar_init(smem_addr(&bar_acc_full[i]), 1);
      mbar_init(smem_addr(&bar_acc_empty[i]), kEpiWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
    s_prod_stop = 0;
    s_epi_stop = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const int ntiles = (a.na + kTcN - 1) / kTcN;
  const int ngroups = (a.mtiles + a.gsz - 1) / a.gsz;
  const uint32_t a_base = smem_addr(A), b_base = smem_addr(Bb);
  auto fail = [&]() {
    s_fail = 1;
    atomicExch(a.err, 1);
  };

  if (warp == 0) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      uint32_t stage = 0, tiles_used = 0, a_used = 0;
      for (int ib = blockIdx.x; ib < a.nb && !s_fail; ib += gridDim.x) {
        const int64_t nt = a.b_off[ib + 1] - a.b_off[ib];
        const int nchunk = (int)((nt + kTcK - 1) / kTcK);
        for (int c = 0; c < nchunk && !s_fail; c++) {
          const int kt = (int)min((int64_t)kTcK, nt - (int64_t)c * kTcK);
          const int ksteps = (kt + 15) / 16;
          for (int g = 0; g < ngroups && !s_fail; g++) {
            const int mt0 = g * a.gsz, mt1 = min(a.mtiles, mt0 + a.gsz);
            if (!mbar_wait(smem_addr(&bar_a_full), a_used & 1)) { fail(); break; }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int tile = 0; tile < ntiles && !s_fail; tile++) {
              const uint32_t slot = tiles_used % kBSlots;
              if (!mbar_wait(smem_addr(&bar_b_full[slot]), (tiles_used / kBSlots) & 1)) { fail(); break; }
              asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
              for (int mt = mt0; mt < mt1; mt++) {
                const uint32_t s = stage % kStages;
                if (!mbar_wait(smem_addr(&bar_acc_empty[s]), ((stage / kStages) & 1) ^ 1)) { fail(); break; }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a0 = a_base + (uint32_t)(mt - mt0) * kABytesPerMt;
                const uint32_t b0 = b_base + slot * kBBytes;
                for (int ks = 0; ks < ksteps; ks++)
                  mma_bf16(tmem + s * kTcN, smem_desc(a0 + ks * 2 * kLBO), smem_desc(b0 + ks * 2 * kLBO),
                           ks > 0 ? 1u : 0u);
                mma_commit(smem_addr(&bar_acc_full[s]));
                stage++;
              }
              mma_commit(smem_addr(&bar_b_empty[slot]));
              tiles_used++;
            }
            mma_commit(smem_addr(&bar_a_empty));
            a_used++;
          }
        }
      }
      // every MMA issued has completed before the tensor memory is freed
      mma_commit(smem_addr(&bar_done));
      if (!mbar_wait(smem_addr(&bar_done), 0)) fail();
    }
    __syncwarp();
  } else if (warp < 4) {
    // ---------------- producers: A per (ib, chunk, group), B per tile ----------------
    const int pt = tid - 32;
    uint32_t tiles_used = 0, a_used = 0;
    for (int ib = blockIdx.x; ib < a.nb; ib += gridDim.x) {
      const int64_t t0 = a.b_off[ib], nt = a.b_off[ib + 1] - t0;
      const int nchunk = (int)((nt + kTcK - 1) / kTcK);
      for (int c = 0; c < nchunk; c++) {
        const int kt = (int)min((int64_t)kTcK, nt - (int64_t)c * kTcK);
        const int krows = (kt + 15) / 16 * 16;
        named_sync(2, kProdThreads);  // the previous chunk's lists are no longer read
        for (int t = pt; t < kTcK; t += kProdThreads) {
          if (t < kt) {
            const int64_t k = t0 + (int64_t)c * kTcK + t;
            const uint32_t info = a.b_info[k];
            s_jb[t] = a.b_idx[k];
            s_rs[t] = (info >> 12) & 0xFFFu;
            s_sb[t] = (info & 0x80000000u) ? -1.f : 1.f;
          } else {
            s_jb[t] = -1;
            s_rs[t] = -1;
            s_sb[t] = 0.f;
          }
        }
        named_sync(2, kProdThreads);
        for (int g = 0; g < ngroups; g++) {
          const int mt0 = g * a.gsz, mt1 = min(a.mtiles, mt0 + a.gsz);
          const int mrows = (mt1 - mt0) * 128;
          if (!s_fail && !mbar_wait(smem_addr(&bar_a_empty), (a_used & 1) ^ 1)) fail();
          if (!s_fail) {
            // A[m][k] = sb_k (pq_m | rs_k): (pq|rs) is symmetric, so row rs_k of
            // Vf is read, coalesced over m; each task packs 8 consecutive k of
            // one row m into one 16-byte store
            const int tasks = mrows * (krows / 8);
            for (int task = pt; task < tasks; task += kProdThreads) {
              const int m = task % mrows, k8 = task / mrows;
              const int pq = mt0 * 128 + m;
              uint32_t w[4];
#pragma unroll
              for (int j = 0; j < 4; j++) {
                const int k0 = 8 * k8 + 2 * j;
                const int r0 = s_rs[k0], r1 = s_rs[k0 + 1];
                const float v0 = (r0 >= 0 && pq < a.P) ? s_sb[k0] * __ldg(&a.vf[(size_t)r0 * a.P + pq]) : 0.f;
                const float v1 = (r1 >= 0 && pq < a.P) ? s_sb[k0 + 1] * __ldg(&a.vf[(size_t)r1 * a.P + pq]) : 0.f;
                __nv_bfloat162 h2 = __floats2bfloat162_rn(v0, v1);
                w[j] = *reinterpret_cast<uint32_t*>(&h2);
              }
              *reinterpret_cast<uint4*>(A + kmajor_offset(m, 8 * k8)) = make_uint4(w[0], w[1], w[2], w[3]);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          }
          mbar_arrive(smem_addr(&bar_a_full));
          a_used++;
          for (int tile = 0; tile < ntiles; tile++) {
            const uint32_t slot = tiles_used % kBSlots;
            if (!s_fail && !mbar_wait(smem_addr(&bar_b_empty[slot]), ((tiles_used / kBSlots) & 1) ^ 1)) fail();
            if (!s_fail) {
              const int ja0 = tile * kTcN;
              for (int idx = pt; idx < krows * (kTcN / 8); idx += kProdThreads) {
                const int t = idx >> 3, n8 = idx & 7;
                const int jb = s_jb[t];
                const __nv_bfloat16* src = jb >= 0 ? a.ct16 + (size_t)jb * a.na_pad + ja0 + 8 * n8 : a.ct16;
                cp_async16(b_base + slot * kBBytes + mnmajor_chunk_offset(n8, t), src, jb >= 0 ? 16u : 0u);
              }
            }
            cp_async_arrive(smem_addr(&bar_b_full[slot]));
            tiles_used++;
          }
        }
      }
      // a uniform decision among the producers whether to go on
      named_sync(2, kProdThreads);
      if (pt == 0) s_prod_stop = s_fail;
      named_sync(2, kProdThreads);
      if (s_prod_stop) break;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else {
    // ---------------- epilogue ----------------
    const int e = warp - 4, q = e & 3, h = e >> 2;  // TMEM lane quarter = warp % 4, column block h
    float* my = stg + (size_t)e * 32 * kGS;
    const int et = tid - 128;
    uint32_t stage = 0;
    for (int ib = blockIdx.x; ib < a.nb; ib += gridDim.x) {
      const int64_t nt = a.b_off[ib + 1] - a.b_off[ib];
      const int nchunk = (int)((nt + kTcK - 1) / kTcK);
      float* col = a.out + (size_t)ib * a.na;
      for (int c = 0; c < nchunk; c++) {
        for (int g = 0; g < ngroups; g++) {
          const int mt0 = g * a.gsz, mt1 = min(a.mtiles, mt0 + a.gsz);
          // stages of this (chunk, group): sidx = tile * gm + (mt - mt0).  The
          // bucket offsets are loaded two stages ahead and the entries one
          // stage ahead, so their global-memory latency overlaps the work of
          // the stages before.
          const int gm = mt1 - mt0, nst = ntiles * gm;
          auto bk_of = [&](int sidx) {
            return ((size_t)(sidx / gm) * a.mtiles + mt0 + sidx % gm) * kEpiWarps + e;
          };
          int64_t eb = __ldg(&a.bk_off[bk_of(0)]), ee = __ldg(&a.bk_off[bk_of(0) + 1]);
          int64_t eb1 = 0, ee1 = 0;
          if (nst > 1) {
            eb1 = __ldg(&a.bk_off[bk_of(1)]);
            ee1 = __ldg(&a.bk_off[bk_of(1) + 1]);
          }
          uint32_t en[kEntPref];
#pragma unroll
          for (int j = 0; j < kEntPref; j++) {
            const int64_t i = eb + lane + 32 * j;
            en[j] = i < ee ? __ldg(&a.bk_ent[i]) : 0xFFFFFFFFu;
          }
          for (int sidx = 0; sidx < nst; sidx++) {
            {
              uint32_t en_next[kEntPref];
#pragma unroll
              for (int j = 0; j < kEntPref; j++) {
                const int64_t i = eb1 + lane + 32 * j;
                en_next[j] = (sidx + 1 < nst && i < ee1) ? __ldg(&a.bk_ent[i]) : 0xFFFFFFFFu;
              }
              int64_t eb2 = 0, ee2 = 0;
              if (sidx + 2 < nst) {
                eb2 = __ldg(&a.bk_off[bk_of(sidx + 2)]);
                ee2 = __ldg(&a.bk_off[bk_of(sidx + 2) + 1]);
              }
              const uint32_t s = stage % kStages;
              float v[kEpiCols];
              bool ok = !s_fail;
              if (ok && !mbar_wait(smem_addr(&bar_acc_full[s]), (stage / kStages) & 1)) {
                fail();
                ok = false;
              }
              if (ok) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + s * kTcN + kEpiCols * h;
#pragma unroll
                for (int c16 = 0; c16 < kEpiCols / 16; c16++) tmem_ld16(taddr + 16 * c16, v + 16 * c16);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
              }
              asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
              __syncwarp();
              if (lane == 0) mbar_arrive(smem_addr(&bar_acc_empty[s]));  // the stage is free again
              if (ok) {
                float4* row = reinterpret_cast<float4*>(my + lane * kGS);
#pragma unroll
                for (int i = 0; i < kEpiCols / 4; i++) row[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                __syncwarp();
#pragma unroll
                for (int j = 0; j < kEntPref; j++)
                  if (en[j] != 0xFFFFFFFFu) tc_scatter(my, col, en[j]);
                for (int64_t i = eb + lane + 32 * kEntPref; i < ee; i += 32) tc_scatter(my, col, __ldg(&a.bk_ent[i]));
                __syncwarp();  // the block is read before the next stage overwrites it
              }
              stage++;
              eb = eb1;
              ee = ee1;
              eb1 = eb2;
              ee1 = ee2;
#pragma unroll
              for (int j = 0; j < kEntPref; j++) en[j] = en_next[j];
            }
          }
        }
      }
      // a uniform decision among the epilogue warps whether to go on
      named_sync(1, kEpiThreads);
      if (et == 0) s_epi_stop = s_fail;
      named_sync(1, kEpiThreads);
      if (s_epi_stop) break;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kStages * kTcN));
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

// dynamic shared memory of the kernel with gsz M tiles of A resident
size_t tc_smem_bytes(int gsz) { return (size_t)gsz * kABytesPerMt + (size_t)kBSlots * kBBytes + kStgBytes; }

// static shared memory of the kernel (lists of one K chunk, barriers, flags)
constexpr size_t kTcStaticSmem = 3 * kTcK * 4 + (3 + 2 * kBSlots + 2 * kStages) * 8 + 64;

// M tiles per group: as many as fit next to the B slots and the staging
// blocks (0: not even one fits)
int tc_group_size(const sbdgpu_ctx* c) {
  const int mtiles = (c->P + 127) / 128;
  const size_t budget = 227 * 1024 - kTcStaticSmem - 1024;
  const size_t fixed = tc_smem_bytes(0);
  if (fixed + kABytesPerMt > budget) return 0;
  return (int)std::min<size_t>((size_t)mtiles, (budget - fixed) / kABytesPerMt);
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
  // na < 2^20: ia takes bits 12..31 of a bucket entry (all ones marks an
  // empty prefetch register); the beta-single pair index has 12 bits
  return c->na < (1u << 20) - 1 && c->P <= 4096 && tc_group_size(c) >= 1;
}

// Alpha singles bucketed by (tile of 64 source strings ja, M tile of 128 pq,
// epilogue warp: lane quarter q of the M tile and half h of the ja tile).
void build_tc_buckets(sbdgpu_ctx* c) {
  if (c->tc_bk_ent) return;
  const SpinTables& ta = c->tab[0];
  const int mtiles = (c->P + 127) / 128;
  const size_t na = c->na;
  std::vector<int32_t> idx(ta.ns);
  std::vector<uint32_t> info(ta.ns);
  if (ta.ns) {
    SBD_CUDA(cudaMemcpy(idx.data(), ta.s_idx, sizeof(int32_t) * ta.ns, cudaMemcpyDeviceToHost));
    SBD_CUDA(cudaMemcpy(info.data(), ta.s_info, sizeof(uint32_t) * ta.ns, cudaMemcpyDeviceToHost));
  }
  const size_t ntiles = (na + kTcN - 1) / kTcN;
  const size_t nbk = ntiles * mtiles * kEpiWarps;
  std::vector<int64_t> off(nbk + 1, 0);
  auto bucket_of = [&](size_t ja, uint32_t pq) {
    const uint32_t col = (uint32_t)(ja % kTcN), row = pq % 128u;
    const uint32_t e = (col / (uint32_t)kEpiCols) * 4u + row / 32u;
    return ((ja / kTcN) * mtiles + pq / 128u) * kEpiWarps + e;
  };
  for (size_t ja = 0; ja < na; ja++)
    for (int64_t k = ta.h_s_off[ja]; k < ta.h_s_off[ja + 1]; k++) off[bucket_of(ja, (info[k] >> 12) & 0xFFFu) + 1]++;
  for (size_t i = 0; i < nbk; i++) off[i + 1] += off[i];
  std::vector<uint32_t> ent((size_t)off.back());
  std::vector<int64_t> pos(off.begin(), off.end() - 1);
  for (size_t ja = 0; ja < na; ja++) {
    for (int64_t k = ta.h_s_off[ja]; k < ta.h_s_off[ja + 1]; k++) {
      // row ja, ket ia: pair index and sign are those of the pair (ia <- ja)
      const uint32_t pq = (info[k] >> 12) & 0xFFFu;
      const uint32_t neg = (info[k] >> 31) & 1u;
      const uint32_t ia = (uint32_t)idx[k];
      const uint32_t goff = (pq % 32u) * (uint32_t)kGS + (uint32_t)(ja % kEpiCols);  // < 2^11
      ent[(size_t)pos[bucket_of(ja, pq)]++] = goff | (neg << 11) | (ia << 12);
    }
  }
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
  SBD_CUDA(cudaMemsetAsync(out, 0, sizeof(float) * c->na * c->nb, c->stream));
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
  a.gsz = tc_group_size(c);
  if (a.gsz < 1) throw Error{SBDGPU_ERR_LIMIT, "tensor-core alpha-beta kernel: shared memory too small"};
  const size_t smem = tc_smem_bytes(a.gsz);
  allow_dynamic_smem(reinterpret_cast<const void*>(tc_ab_kernel), c->device);
  int sms = 148;
  SBD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  const int grid = (int)std::min<size_t>((size_t)sms, c->nb);
  tc_ab_kernel<<<grid, kTcThreads, smem, c->stream>>>(a);
  SBD_CUDA(cudaGetLastError());
}

int tc_error(sbdgpu_ctx* c) {
  if (!c->tc_err) return 0;
  int h = 0;
  SBD_CUDA(cudaMemcpyAsync(&h, c->tc_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  SBD_CUDA(cudaMemsetAsync(c->tc_err, 0, sizeof(int), c->stream));
  SBD_CUDA(cudaStreamSynchronize(c->stream));
  return h;
}

}  // namespace sbdgpu
