// Internal declarations of the sm_100a tensor-product-basis Davidson path.
//
// Data layout in HBM (one context, one device):
//   strings        uint64 per string, orbital i at bit i, in the caller's order
//   vectors        FP64 row-major [na][nb], alpha-string-major sign convention
//                  (the interleaved reference convention differs by the diagonal
//                  +-1 phase phi(a,b) = (-1)^#{(p in a, r in b): r < p}, applied
//                  only at the C ABI)
//   V              (pq|rs) folded over p<->q and r<->s: Vf[pair(p,q)*P + pair(r,s)],
//                  P = L(L+1)/2, pair(p,q) = max(max+1)/2 + min
//   tables         per spin, CSR by bra string: singles (ket, packed p/q/pair/sign,
//                  FP64 string-only matrix element) and doubles (ket, FP64 element);
//                  plus a sliced-ELL copy of the singles (32 bras per slice, column
//                  major) for the alpha-beta kernel
//   J tables       JX[pair(p,q)][i] = sum_{r in string i} (pq|rr): the Coulomb
//                  coupling of a same-spin single to the other spin's occupation
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "sbdgpu.h"

namespace sbdgpu {

struct Learned;  // learned.cu: the preconditioner network of a context

struct Error {
  int code;
  std::string msg;
};

#define SBD_CUDA(x)                                                                              \
  do {                                                                                           \
    cudaError_t e_ = (x);                                                                        \
    if (e_ != cudaSuccess)                                                                       \
      throw ::sbdgpu::Error{SBDGPU_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_) +   \
                                                 " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")"}; \
  } while (0)

constexpr uint32_t kSellInvalid = 0xFFFFFFFFu;
// polls of a bounded mbarrier wait (the tensor-core kernel's, and the largest
// limit sbdgpu_wait_selftest accepts)
constexpr long long kMaxSpinLimit = 1ll << 26;
constexpr int kSlice = 32;

struct SpinTables {
  size_t n = 0;
  int64_t* s_off = nullptr;   // [n+1]
  int64_t* d_off = nullptr;   // [n+1]
  int32_t* s_idx = nullptr;   // ket
  uint32_t* s_info = nullptr; // p | q<<6 | pair<<12 | neg<<31  (p created in bra, q annihilated)
  double* s_val = nullptr;    // sign * (h_pq + sum_{j in ket} ((pq|jj) - (pj|jq)))
  int32_t* d_idx = nullptr;
  double* d_val = nullptr;    // sign * ((p1q1|p2q2) - (p1q2|p2q1))
  uint64_t ns = 0, nd = 0;
  int max_s = 0;
  // sliced ELL of the singles, keyed by bra: ket | pair<<16 | neg<<31
  size_t nslice = 0;
  int64_t* sell_off = nullptr;  // [nslice+1]
  int32_t* sell_w = nullptr;    // [nslice]
  uint32_t* sell = nullptr;
  std::vector<int64_t> h_s_off, h_d_off;  // host copies of the offsets
};

}  // namespace sbdgpu

struct sbdgpu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int L = 0;
  int P = 0;
  size_t na = 0, nb = 0, N = 0;
  double ecore = 0.0;
  std::vector<uint64_t> h_astr, h_bstr;
  std::vector<double> h_h1, h_vf;  // host copies
  uint64_t* astr = nullptr;
  uint64_t* bstr = nullptr;
  double* h1 = nullptr;  // [L*L]
  double* vf = nullptr;  // [P*P]
  double* ja = nullptr;  // [P][na]
  double* jb = nullptr;  // [P][nb]
  double* hii = nullptr; // [N]
  float* ja32 = nullptr; // FP32 copies for the mixed path
  float* jb32 = nullptr;
  float* vf32 = nullptr;
  int64_t* tc_bk_off = nullptr;  // alpha singles bucketed for the tensor-core alpha-beta kernel
  uint32_t* tc_bk_ent = nullptr;
  int* tc_err = nullptr;
  void* ct16 = nullptr;  // BF16 copy of C^T, rows padded to 64 (tensor-core path)
  sbdgpu::Learned* learned = nullptr;  // learned preconditioner, created on first use
  // dense string-only same-spin operators (FP16 hi/lo, [spin][part]), split
  // vector scratch and the cuBLAS handle of the mixed-precision sigma
  void* h0[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  void* c16[2] = {nullptr, nullptr};
  void* blas = nullptr;
  bool dense_same_off = false;  // true: same-spin terms from the rows kernels instead
  // alpha singles restricted to the target rows [blk_r0, blk_r1) (row-block sigma)
  int64_t* blk_off = nullptr;
  int32_t* blk_idx = nullptr;
  uint32_t* blk_info = nullptr;
  int blk_max = 0;
  size_t blk_r0 = 0, blk_r1 = 0;
  sbdgpu::SpinTables tab[2];
  // same-spin terms of the FP64 sigma on the integer tensor cores (ozaki.cu)
  struct {
    int mode = 0;          // 0 automatic (the default), 1 the rows kernels only
    bool ready = false, failed = false;
    int8_t* h0r[2] = {nullptr, nullptr};  // residues of the string-only operators
    int* h0e[2] = {nullptr, nullptr};     // their row exponents
    int8_t* cr = nullptr;                 // residues of C (row-scaled)
    int8_t* ctr = nullptr;                // residues of C^T (row-scaled)
    int* ce = nullptr;
    int* cte = nullptr;
    int32_t* prod = nullptr;              // INT8 products, one per prime
  } oz;
  // alpha-beta launch shape of the FP64 sigma (0: the shared-memory heuristic)
  int ab_group = 0, ab_threads = 0;
  // RDM tables: beta singles grouped by excitation, bra row of every alpha single
  int64_t* rdm_bin_off = nullptr;
  uint32_t* rdm_bin_ent = nullptr;
  int32_t* rdm_a_row = nullptr;
  // stored Hamiltonian (method 1): off-diagonal elements, CSR by bra determinant
  int64_t* hs_row = nullptr;   // [N+1]
  uint32_t* hs_col = nullptr;  // ket determinant ja*nb + jb
  double* hs_val = nullptr;
  uint64_t hs_nnz = 0;
  bool stored = false;
  bool tables_ready = false;
  bool hii_ready = false;
  // scratch vectors (FP64, N each), allocated on first use
  double* io_a = nullptr;  // user I/O staging
  double* io_b = nullptr;
  float* io32 = nullptr;   // FP32 staging of C and sigma (mixed path), 2*N
  double* ct = nullptr;    // transposed C   [nb][na]
  double* st = nullptr;    // transposed sigma part [nb][na]
  double* red = nullptr;   // reduction scratch
  // ev[0..3]: kernel phases of one sigma; ev[4]/ev[5]: whole sigma incl. sign
  // phases; ev[6]/ev[7]: host-to-device copy start .. device-to-host copy end
  cudaEvent_t ev[8] = {};
  float last_ms[5] = {0, 0, 0, 0, 0};
  std::string err;
};

namespace sbdgpu {

// tables.cu
void build_tables(sbdgpu_ctx* c);
void free_tables(SpinTables& t);

// misc.cu
void build_j_tables(sbdgpu_ctx* c);
void compute_hii(sbdgpu_ctx* c);
void apply_phase(sbdgpu_ctx* c, double* v);
void apply_phase_rows(sbdgpu_ctx* c, double* v, size_t r0, size_t nrows);  // v: rows r0.. of a vector
template <typename T>
void transpose(const T* in, T* out, size_t rows, size_t cols, cudaStream_t s);
template <typename T>
void transpose_add(const T* in, T* out, size_t rows, size_t cols, cudaStream_t s);
void ensure_fp32(sbdgpu_ctx* c);
double dot(sbdgpu_ctx* c, const double* x, const double* y, size_t n);
void dot_device(sbdgpu_ctx* c, const double* x, const double* y, size_t n, double* out);  // needs ensure_scratch
void scale(double* x, double a, size_t n, cudaStream_t s);
double dot_f(sbdgpu_ctx* c, const float* x, const double* xd, const float* y, size_t n);
void axpy_df(double* y, const float* x, double a, size_t n, cudaStream_t s);
void lincomb_f(float* const* in, const double* U, int nk, float* out, size_t n, sbdgpu_ctx* c);
void convert(const double* in, float* out, size_t n, cudaStream_t s);
void convert(const float* in, double* out, size_t n, cudaStream_t s);
void ritz_update_f(float* const* C, float* const* HC, const double* U, int nk, double e0, double* W, double* R,
                   size_t n, sbdgpu_ctx* c);
void axpy(double* y, const double* x, double a, size_t n, cudaStream_t s);
void ritz_update(double* const* C, double* const* HC, const double* U, int nk, double e0, double* W,
                 double* R, size_t n, cudaStream_t s);
void precondition(const double* R, const double* hii, double e0, double eps_reg, double* out, size_t n,
                  cudaStream_t s);
void rdm(sbdgpu_ctx* c, const double* dW, double* one, double* two);
// rdm.cu: the off-diagonal terms, added into device arrays one [2][L*L] and two [4][L^4]
void rdm_offdiag(sbdgpu_ctx* c, const double* dW, double* one, double* two);
void ensure_rdm_tables(sbdgpu_ctx* c);
void free_rdm_tables(sbdgpu_ctx* c);
// sigma.cu: the alpha-beta launch shapes (group size, threads) open to this context's FP64 sigma
std::vector<std::pair<int, int>> ab_shapes(sbdgpu_ctx* c);
// ozaki.cu: the FP64 same-spin terms as exact INT8 products
bool ensure_ozaki(sbdgpu_ctx* c);
void free_ozaki(sbdgpu_ctx* c);
bool use_ozaki(sbdgpu_ctx* c);
bool same_spin_ozaki_fp64(sbdgpu_ctx* c, const double* C, double* S, double* ct, double* st, bool events);
// genop.cu: record an error message on a generic-path object
void genop_set_error(sbdgpu_genop* g, const std::string& msg);
void occupation(sbdgpu_ctx* c, const double* dW, double* dens);
void alpha_weights(sbdgpu_ctx* c, const double* dW, double* D);

// tc_ab.cu
bool tc_ab_supported(const sbdgpu_ctx* c);
void build_tc_buckets(sbdgpu_ctx* c);
void tc_alpha_beta(sbdgpu_ctx* c, const float* ct, float* out);
int tc_error(sbdgpu_ctx* c);
void wait_selftest(sbdgpu_ctx* c, long long limit, int* status);

// stored.cu
void store_hamiltonian(sbdgpu_ctx* c);
void release_hamiltonian(sbdgpu_ctx* c);
void spmv_stored(sbdgpu_ctx* c, const double* C, double* S);

// roots.cu
void davidson_roots(sbdgpu_ctx* c, const sbdgpu_opts* o, int nroots, double* Wh, double* energies, double* resid,
                    int* n_iter, int* n_sigma);

// sigma.cu
void preload_fp64_sigma(int device);
void preload_fp64_sigma_misc();  // misc.cu
void sigma_fp64(sbdgpu_ctx* c, const double* C, double* S);
void sigma_fp64_prepared(sbdgpu_ctx* c, const double* C, double* S, double* ct, double* st);
void sigma_fp32(sbdgpu_ctx* c, const float* C, float* S);
void sigma_fp32_tc(sbdgpu_ctx* c, const float* C, float* S);
void sigma_rows_fp64(sbdgpu_ctx* c, const double* dC, double* S, size_t r0, size_t r1);

// noalloc.cu
void noalloc_prepare(int device);

// gemm_same.cu
bool ensure_dense_same(sbdgpu_ctx* c);
bool use_dense_same(sbdgpu_ctx* c);
void free_dense_same(sbdgpu_ctx* c);
void same_spin_dense_fp32(sbdgpu_ctx* c, const float* C, float* S, float* ct, float* st, bool events);

// learned.cu
void free_learned(sbdgpu_ctx* c);
bool learned_ready(const sbdgpu_ctx* c);
void learned_precondition(sbdgpu_ctx* c, const double* R, double e0, double eps_reg, double* out);
void train_learned(sbdgpu_ctx* c, const sbdgpu_learn_opts* o, double* loss_trace, double* seconds);
void learned_get(sbdgpu_ctx* c, float* w, int* n);
void learned_set(sbdgpu_ctx* c, const float* w, int n);

// api.cu
void ensure_scratch(sbdgpu_ctx* c);
void ensure_io(sbdgpu_ctx* c);
void jacobi_eig(int n, double* A, int lda, double* w);
void* dev_alloc(size_t bytes);
void allow_dynamic_smem(const void* func, int device);

}  // namespace sbdgpu
