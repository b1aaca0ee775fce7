// C ABI (include/sbdgpu.h): context life cycle, host/device transfers and the
// Davidson driver.  No exception crosses the ABI; errors become status codes
// with a message kept in the context.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <mutex>
#include <new>
#include <set>
#include <utility>

#include "internal.cuh"

using sbdgpu::Error;

namespace sbdgpu {

void* dev_alloc(size_t bytes) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes ? bytes : 8);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error{SBDGPU_ERR_ALLOC, "device allocation of " + std::to_string(bytes) + " bytes failed: " +
                                      cudaGetErrorString(e)};
  }
  return p;
}

// The dynamic shared-memory limit of a kernel is one attribute per
// (function, device), shared by every host thread.  Setting it before each
// launch to that launch's size lets concurrent contexts undercut each other
// between the set and the launch, which the runtime then rejects.  It is set
// once instead, to the device's opt-in maximum; each launch still passes its
// own size.
void allow_dynamic_smem(const void* func, int device) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({func, device})) return;
  int optin = 0;
  SBD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  cudaFuncAttributes fa{};
  SBD_CUDA(cudaFuncGetAttributes(&fa, func));
  // dynamic + static shared memory may not pass the opt-in maximum
  SBD_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - (int)fa.sharedSizeBytes));
  done.insert({func, device});
}

void ensure_scratch(sbdgpu_ctx* c) {
  if (!c->red) c->red = (double*)dev_alloc(sizeof(double) * 1024);
  if (!c->ct) c->ct = (double*)dev_alloc(sizeof(double) * c->N);
  if (!c->st) c->st = (double*)dev_alloc(sizeof(double) * c->N);
}

void ensure_io(sbdgpu_ctx* c) {
  if (!c->io_a) c->io_a = (double*)dev_alloc(sizeof(double) * c->N);
  if (!c->io_b) c->io_b = (double*)dev_alloc(sizeof(double) * c->N);
}

// Cyclic Jacobi eigen-solver for the small projected matrix (the reference
// solves the same problem with LAPACK dsyev, framework/hp_numeric.h:500-517).
// A: n x n column-major, leading dimension lda; on return A holds the
// eigenvectors (columns) in ascending eigenvalue order, w the eigenvalues.
void jacobi_eig(int n, double* A, int lda, double* w) {
  std::vector<double> M(n * n), V(n * n, 0.0);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) M[i + j * n] = A[i + j * lda];
  for (int i = 0; i < n; i++) V[i + i * n] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (int j = 0; j < n; j++)
      for (int i = 0; i < j; i++) off += M[i + j * n] * M[i + j * n];
    if (off < 1e-300) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        double apq = M[p + q * n];
        if (std::fabs(apq) < 1e-300) continue;
        double theta = 0.5 * (M[q + q * n] - M[p + p * n]) / apq;
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < n; k++) {
          double a = M[k + p * n], b = M[k + q * n];
          M[k + p * n] = cs * a - sn * b;
          M[k + q * n] = sn * a + cs * b;
        }
        for (int k = 0; k < n; k++) {
          double a = M[p + k * n], b = M[q + k * n];
          M[p + k * n] = cs * a - sn * b;
          M[q + k * n] = sn * a + cs * b;
        }
        for (int k = 0; k < n; k++) {
          double a = V[k + p * n], b = V[k + q * n];
          V[k + p * n] = cs * a - sn * b;
          V[k + q * n] = sn * a + cs * b;
        }
      }
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return M[a + a * n] < M[b + b * n]; });
  for (int k = 0; k < n; k++) {
    int s = order[k];
    w[k] = M[s + s * n];
    for (int i = 0; i < n; i++) A[i + k * lda] = V[i + s * n];
  }
}

}  // namespace sbdgpu

namespace {

template <class F>
int guarded(sbdgpu_ctx* c, F&& f) {
  if (!c) return SBDGPU_ERR_ARG;
  try {
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) throw Error{SBDGPU_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e)};
    f();
    c->err.clear();
    return SBDGPU_OK;
  } catch (const Error& e) {
    c->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    c->err = "host allocation failed";
    return SBDGPU_ERR_ALLOC;
  } catch (const std::exception& e) {
    c->err = e.what();
    return SBDGPU_ERR_STATE;
  }
}

using sbdgpu::ensure_io;

void check_precision(int precision) {
  if (precision != SBDGPU_FP64 && precision != SBDGPU_MIXED && precision != SBDGPU_MIXED_TC)
    throw Error{SBDGPU_ERR_ARG, "unsupported precision " + std::to_string(precision)};
}

void sigma_ref_convention(sbdgpu_ctx* c, const double* dC, double* dS, int precision = SBDGPU_FP64) {
  // dC, dS in the reference (interleaved) sign convention
  ensure_io(c);
  sbdgpu::build_tables(c);
  sbdgpu::compute_hii(c);
  sbdgpu::ensure_scratch(c);
  if (precision != SBDGPU_FP64) sbdgpu::ensure_fp32(c);
  SBD_CUDA(cudaEventRecord(c->ev[4], c->stream));
  SBD_CUDA(cudaMemcpyAsync(c->io_a, dC, sizeof(double) * c->N, cudaMemcpyDeviceToDevice, c->stream));
  sbdgpu::apply_phase(c, c->io_a);
  if (precision != SBDGPU_FP64) {
    if (!c->io32) c->io32 = (float*)sbdgpu::dev_alloc(sizeof(float) * 2 * c->N);
    float* c32 = c->io32;
    float* s32 = c->io32 + c->N;
    sbdgpu::convert(c->io_a, c32, c->N, c->stream);
    if (precision == SBDGPU_MIXED_TC)
      sbdgpu::sigma_fp32_tc(c, c32, s32);
    else
      sbdgpu::sigma_fp32(c, c32, s32);
    sbdgpu::convert(s32, dS, c->N, c->stream);
  } else {
    sbdgpu::sigma_fp64(c, c->io_a, dS);
  }
  sbdgpu::apply_phase(c, dS);
  SBD_CUDA(cudaEventRecord(c->ev[5], c->stream));
  SBD_CUDA(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 3; k++) SBD_CUDA(cudaEventElapsedTime(&c->last_ms[k], c->ev[k], c->ev[k + 1]));
  SBD_CUDA(cudaEventElapsedTime(&c->last_ms[3], c->ev[4], c->ev[5]));
  c->last_ms[4] = 0.0f;
  if (precision == SBDGPU_MIXED_TC && sbdgpu::tc_error(c))
    throw Error{SBDGPU_ERR_CUDA, "tensor-core alpha-beta kernel: completion wait timed out"};
}

// Mixed-precision Davidson: FP32 basis and FP32 sigma; FP64 dot products,
// projected matrix, Ritz vector, residual, preconditioned correction and
// Gram-Schmidt; the energy is the FP64 Rayleigh quotient <W|H W> from one FP64
// refinement sigma of the final Ritz vector (the same final step as
// chemistry/tpb/sbdiag.h:239-262).  Vectors in the alpha-string-major convention.
// Restarts: the reference's collapse to W, or (restart_keep > 1) the lowest
// Ritz vectors with their sigma vectors, optionally (restart_prev) with the
// previous step's Ritz vector as well; with vectors carried over, the
// correction is orthogonalised in two Gram-Schmidt passes.
void davidson_mixed(sbdgpu_ctx* c, const sbdgpu_opts* o, double* W, double* R, double* energy, double* trace_e,
                    double* trace_tol, int max_trace, int* n_steps) {
  // SBDGPU_MIXED_TC: tensor-core sigma while the residual norm is above this,
  // then a restart from the current Ritz vector with FP32 sigma
  // (or when the BF16 operator stops improving the residual: a whole restart
  // cycle that gains less than 30 %, or 40 steps)
  const double tc_switch = 1.0e-2;
  bool use_tc = o->precision == SBDGPU_MIXED_TC && sbdgpu::tc_ab_supported(c);
  double tol_cycle = 1e300;
  int tc_steps = 0;
  int nb = o->max_nb;
  size_t n = c->N;
  cudaStream_t st = c->stream;
  sbdgpu::ensure_fp32(c);
  std::vector<float*> C(nb, nullptr), HC(nb, nullptr);
  double* X = nullptr;  // FP64 correction vector
  struct Free {
    std::vector<float*>* a;
    std::vector<float*>* b;
    double** x;
    cudaStream_t s;
    ~Free() {
      cudaStreamSynchronize(s);  // an error path may leave kernels queued on these buffers
      for (auto p : *a) cudaFree(p);
      for (auto p : *b) cudaFree(p);
      cudaFree(*x);
    }
  } guard{&C, &HC, &X, st};
  for (int k = 0; k < nb; k++) {
    C[k] = (float*)sbdgpu::dev_alloc(sizeof(float) * n);
    HC[k] = (float*)sbdgpu::dev_alloc(sizeof(float) * n);
  }
  X = (double*)sbdgpu::dev_alloc(sizeof(double) * n);
  // Olsen's correction needs P applied to the Ritz vector as well
  const bool olsen = o->precond == SBDGPU_PRECOND_OLSEN;
  double* Y = nullptr;
  struct FreeY {
    double** y;
    cudaStream_t s;
    ~FreeY() {
      cudaStreamSynchronize(s);
      cudaFree(*y);
    }
  } guard_y{&Y, st};
  if (olsen) Y = (double*)sbdgpu::dev_alloc(sizeof(double) * n);
  const double eps_reg = 1.0e-12;
  std::vector<double> H(nb * nb, 0.0), U(nb * nb, 0.0), E(nb, 0.0);
  std::vector<double> step_times;
  auto t_start = std::chrono::steady_clock::now();
  int steps = 0;
  bool cont = true;
  const bool keep_prev = o->restart_prev != 0 && nb > 2;
  const int keep_ritz = std::min(std::max(o->restart_keep, 1), nb - (keep_prev ? 2 : 1));
  // basis vectors carried over a restart: the keep_ritz lowest Ritz vectors,
  // plus the previous step's Ritz vector when keep_prev
  const int keep = keep_ritz + (keep_prev ? 1 : 0);
  std::vector<float*> T(keep, nullptr), TH(keep, nullptr);
  std::vector<double> u_last(nb, 0.0);  // Ritz coefficients of the previous step
  int u_last_len = 0, u_last_cycle = -1;
  struct FreeT {
    std::vector<float*>* a;
    std::vector<float*>* b;
    cudaStream_t s;
    ~FreeT() {
      cudaStreamSynchronize(s);
      for (auto p : *a) cudaFree(p);
      for (auto p : *b) cudaFree(p);
    }
  } guard_t{&T, &TH, st};
  if (keep > 1)
    for (int j = 0; j < keep; j++) {
      T[j] = (float*)sbdgpu::dev_alloc(sizeof(float) * n);
      TH[j] = (float*)sbdgpu::dev_alloc(sizeof(float) * n);
    }
  int kept = 0;  // basis vectors (with their sigma) carried into the next cycle
  // With Ritz vectors carried across restarts in FP32, one classical
  // Gram-Schmidt pass leaves the basis drifting out of orthogonality over the
  // cycles (the projected problem then loses its meaning); a second pass keeps
  // it orthonormal to FP32 rounding.  The collapse restart keeps one pass.
  const int gs_passes = keep > 1 ? 2 : 1;
  // learned correction while the context has a network and it keeps the
  // residual falling; the diagonal one otherwise
  bool use_learned = o->precond == SBDGPU_PRECOND_LEARNED && sbdgpu::learned_ready(c);
  double tol_learned_cycle = 1e300;
  double tol_thick_cycle = 1e300;
  auto add_correction = [&](int into, double e0) {
    if (use_learned) {
      sbdgpu::learned_precondition(c, R, e0, eps_reg, X);
    } else {
      sbdgpu::precondition(R, c->hii, e0, eps_reg, X, n, st);
      if (olsen) {
        // t = P r - eps P w with eps = <w|P r> / <w|P w>: the correction is
        // P-orthogonal to the Ritz vector w, so it does not fall back onto w
        // where P r is nearly parallel to it
        sbdgpu::precondition(W, c->hii, e0, eps_reg, Y, n, st);
        const double wpw = sbdgpu::dot(c, W, Y, n);
        if (std::fabs(wpw) > 0.0) sbdgpu::axpy(X, Y, -sbdgpu::dot(c, W, X, n) / wpw, n, st);
      }
    }
    for (int pass = 0; pass < gs_passes; pass++)
      for (int kb = 0; kb < into; kb++) {
        double olap = sbdgpu::dot_f(c, C[kb], X, C[kb], n);  // <X|C_kb> with X in FP64
        sbdgpu::axpy_df(X, C[kb], -olap, n, st);
      }
    double nc = std::sqrt(sbdgpu::dot(c, X, X, n));
    sbdgpu::scale(X, 1.0 / nc, n, st);
    sbdgpu::convert(X, C[into], n, st);
  };
  for (int it = 0; it < o->max_it && cont; it++) {
    int ib0 = kept;
    if (kept == 0) sbdgpu::convert(W, C[0], n, st);
    kept = 0;
    for (int ib = ib0; ib < nb; ib++) {
      auto t0 = std::chrono::steady_clock::now();
      if (use_tc)
        sbdgpu::sigma_fp32_tc(c, C[ib], HC[ib]);
      else
        sbdgpu::sigma_fp32(c, C[ib], HC[ib]);
      for (int jb = 0; jb <= ib; jb++) {
        H[jb + nb * ib] = sbdgpu::dot_f(c, C[jb], nullptr, HC[ib], n);
        H[ib + nb * jb] = H[jb + nb * ib];
      }
      for (int jb = 0; jb <= ib; jb++)
        for (int kb = 0; kb <= ib; kb++) U[jb + nb * kb] = H[jb + nb * kb];
      sbdgpu::jacobi_eig(ib + 1, U.data(), nb, E.data());
      sbdgpu::ritz_update_f(C.data(), HC.data(), U.data(), ib + 1, E[0], W, R, n, c);
      double nw = std::sqrt(sbdgpu::dot(c, W, W, n));
      sbdgpu::scale(W, 1.0 / nw, n, st);
      double tol = std::sqrt(sbdgpu::dot(c, R, R, n));
      sbdgpu::scale(R, 1.0 / tol, n, st);
      if (trace_e && steps < max_trace) trace_e[steps] = E[0];
      if (trace_tol && steps < max_trace) trace_tol[steps] = tol;
      steps++;
      if (o->verbose) {
        std::cout << " Davidson iteration " << it << "." << ib << " (tol=" << tol << "):";
        for (int p = 0; p < std::min(ib + 1, 4); p++) std::cout << " " << E[p];
        std::cout << std::endl;
      }
      if (tol < o->eps) {
        cont = false;
        break;
      }
      if (use_learned && ib == nb - 1) {
        // fallback: a whole cycle with the learned correction that cut the
        // residual norm by less than 10 % switches to the diagonal one
        if (tol > 0.9 * tol_learned_cycle) use_learned = false;
        tol_learned_cycle = tol;
      }
      if (use_tc) {
        tc_steps++;
        bool stalled = false;
        if (ib == nb - 1) {
          stalled = tol > 0.7 * tol_cycle;
          tol_cycle = tol;
        }
        if (tol < tc_switch || stalled || tc_steps >= 40) {
          if (sbdgpu::tc_error(c))
            throw Error{SBDGPU_ERR_CUDA, "tensor-core alpha-beta kernel: completion wait timed out"};
          use_tc = false;  // restart from W alone, so every sigma comes from the FP32 operator
          break;
        }
      }
      // the kept vectors' sigma are FP32 linear combinations carried from cycle
      // to cycle, so their rounding accumulates; a thick-restart cycle that cut
      // the residual norm by less than 10 % restarts from the Ritz vector alone
      // (its sigma computed afresh) instead
      bool drifted = false;
      if (ib == nb - 1 && keep > 1) {
        drifted = tol > 0.9 * tol_thick_cycle;
        tol_thick_cycle = drifted ? 1e300 : tol;
      }
      if (ib < nb - 1) {
        add_correction(ib + 1, E[0]);
      } else if (keep > 1 && !drifted) {
        // thick restart: the keep_ritz lowest Ritz vectors (and the previous
        // step's Ritz vector, orthonormalised against them in the small space)
        // with their sigma vectors, as linear combinations of the basis
        std::vector<std::vector<double>> Q;
        auto add_col = [&](std::vector<double> y) {
          for (int pass = 0; pass < 2; pass++)
            for (const auto& q : Q) {
              double d = 0.0;
              for (int i = 0; i < nb; i++) d += q[i] * y[i];
              for (int i = 0; i < nb; i++) y[i] -= d * q[i];
            }
          double nn = 0.0;
          for (int i = 0; i < nb; i++) nn += y[i] * y[i];
          nn = std::sqrt(nn);
          if (nn > 1e-8) {
            for (int i = 0; i < nb; i++) y[i] /= nn;
            Q.push_back(std::move(y));
          }
        };
        for (int j = 0; j < keep_ritz; j++) {
          std::vector<double> y(nb);
          for (int i = 0; i < nb; i++) y[i] = U[i + nb * j];
          add_col(std::move(y));
        }
        if (keep_prev && u_last_cycle == it) {
          std::vector<double> y(nb, 0.0);
          for (int i = 0; i < u_last_len; i++) y[i] = u_last[i];
          add_col(std::move(y));
        }
        const int kk = (int)Q.size();
        for (int j = 0; j < kk; j++) {
          sbdgpu::lincomb_f(C.data(), Q[j].data(), nb, T[j], n, c);
          sbdgpu::lincomb_f(HC.data(), Q[j].data(), nb, TH[j], n, c);
        }
        for (int j = 0; j < kk; j++) {
          std::swap(C[j], T[j]);
          std::swap(HC[j], TH[j]);
        }
        for (int j = 0; j < kk; j++)
          for (int i = 0; i <= j; i++) {
            H[i + nb * j] = sbdgpu::dot_f(c, C[i], nullptr, HC[j], n);
            H[j + nb * i] = H[i + nb * j];
          }
        add_correction(kk, E[0]);
        kept = kk;
      }
      // this step's Ritz coefficients, kept for the next restart of this cycle
      if (ib < nb - 1) {
        for (int i = 0; i <= ib; i++) u_last[i] = U[i];
        u_last_len = ib + 1;
        u_last_cycle = it;
      }
      SBD_CUDA(cudaStreamSynchronize(st));
      auto t1 = std::chrono::steady_clock::now();
      step_times.push_back(std::chrono::duration<double>(t1 - t0).count());
      double avg = 0.0;
      for (double x : step_times) avg += x;
      avg /= step_times.size();
      if (std::chrono::duration<double>(t1 - t_start).count() + avg > o->max_time) {
        cont = false;
        break;
      }
    }
  }
  if ((o->precision == SBDGPU_MIXED_TC || o->precond == SBDGPU_PRECOND_LEARNED) && sbdgpu::tc_error(c))
    throw Error{SBDGPU_ERR_CUDA, "tensor-core kernel: completion wait timed out"};
  sbdgpu::sigma_fp64(c, W, R);  // FP64 refinement sigma
  *energy = sbdgpu::dot(c, W, R, n);
  *n_steps = steps;
}

}  // namespace

extern "C" {

int sbdgpu_create(sbdgpu_ctx** out, int norb, size_t na, size_t nb, const uint64_t* astr, const uint64_t* bstr,
                  double ecore, const double* h1, const double* eri_packed, int device) {
  if (!out) return SBDGPU_ERR_ARG;
  *out = nullptr;
  if (norb < 1 || norb > 64 || na == 0 || nb == 0 || !astr || !bstr || !h1 || !eri_packed) return SBDGPU_ERR_ARG;
  for (size_t i = 0; i < na; i++)
    if (norb < 64 && (astr[i] >> norb)) return SBDGPU_ERR_ARG;
  for (size_t i = 0; i < nb; i++)
    if (norb < 64 && (bstr[i] >> norb)) return SBDGPU_ERR_ARG;
  if (na > (size_t)INT32_MAX || nb > (size_t)INT32_MAX) return SBDGPU_ERR_LIMIT;
  sbdgpu_ctx* c = new (std::nothrow) sbdgpu_ctx();
  if (!c) return SBDGPU_ERR_ALLOC;
  c->device = device;
  int rc = guarded(c, [&] {
    c->L = norb;
    c->P = norb * (norb + 1) / 2;
    c->na = na;
    c->nb = nb;
    c->N = na * nb;
    c->ecore = ecore;
    c->h_astr.assign(astr, astr + na);
    c->h_bstr.assign(bstr, bstr + nb);
    c->h_h1.assign(h1, h1 + (size_t)norb * norb);
    size_t P = c->P;
    c->h_vf.resize(P * P);
    for (size_t i = 0; i < P; i++)
      for (size_t j = 0; j < P; j++) {
        size_t a = std::max(i, j), b = std::min(i, j);
        c->h_vf[i * P + j] = eri_packed[a * (a + 1) / 2 + b];
      }
    SBD_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    for (int k = 0; k < 8; k++) SBD_CUDA(cudaEventCreate(&c->ev[k]));
    c->astr = (uint64_t*)sbdgpu::dev_alloc(sizeof(uint64_t) * na);
    c->bstr = (uint64_t*)sbdgpu::dev_alloc(sizeof(uint64_t) * nb);
    c->h1 = (double*)sbdgpu::dev_alloc(sizeof(double) * norb * norb);
    c->vf = (double*)sbdgpu::dev_alloc(sizeof(double) * P * P);
    SBD_CUDA(cudaMemcpyAsync(c->astr, astr, sizeof(uint64_t) * na, cudaMemcpyHostToDevice, c->stream));
    SBD_CUDA(cudaMemcpyAsync(c->bstr, bstr, sizeof(uint64_t) * nb, cudaMemcpyHostToDevice, c->stream));
    SBD_CUDA(cudaMemcpyAsync(c->h1, h1, sizeof(double) * norb * norb, cudaMemcpyHostToDevice, c->stream));
    SBD_CUDA(cudaMemcpyAsync(c->vf, c->h_vf.data(), sizeof(double) * P * P, cudaMemcpyHostToDevice, c->stream));
    SBD_CUDA(cudaStreamSynchronize(c->stream));
    // once per device: the no-allocation sigma's scratch address and kernels
    sbdgpu::noalloc_prepare(device);
  });
  if (rc != SBDGPU_OK) {
    std::fprintf(stderr, "sbdgpu_create: %s\n", c->err.c_str());
    sbdgpu_destroy(c);
    return rc;
  }
  *out = c;
  return SBDGPU_OK;
}

int sbdgpu_build_tables(sbdgpu_ctx* c) {
  return guarded(c, [&] { sbdgpu::build_tables(c); });
}

int sbdgpu_store_hamiltonian(sbdgpu_ctx* c, uint64_t* nnz) {
  return guarded(c, [&] {
    sbdgpu::store_hamiltonian(c);
    if (nnz) *nnz = c->hs_nnz;
  });
}

int sbdgpu_release_hamiltonian(sbdgpu_ctx* c) {
  return guarded(c, [&] {
    SBD_CUDA(cudaStreamSynchronize(c->stream));
    sbdgpu::release_hamiltonian(c);
  });
}

int sbdgpu_table_sizes(sbdgpu_ctx* c, int spin, uint64_t* ns, uint64_t* nd) {
  return guarded(c, [&] {
    if (spin < 0 || spin > 1) throw Error{SBDGPU_ERR_ARG, "spin must be 0 or 1"};
    sbdgpu::build_tables(c);
    if (ns) *ns = c->tab[spin].ns;
    if (nd) *nd = c->tab[spin].nd;
  });
}

int sbdgpu_get_tables(sbdgpu_ctx* c, int spin, uint64_t* s_off, uint64_t* s_idx, uint64_t* d_off, uint64_t* d_idx) {
  return guarded(c, [&] {
    if (spin < 0 || spin > 1) throw Error{SBDGPU_ERR_ARG, "spin must be 0 or 1"};
    sbdgpu::build_tables(c);
    const sbdgpu::SpinTables& t = c->tab[spin];
    if (s_off)
      for (size_t i = 0; i <= t.n; i++) s_off[i] = (uint64_t)t.h_s_off[i];
    if (d_off)
      for (size_t i = 0; i <= t.n; i++) d_off[i] = (uint64_t)t.h_d_off[i];
    std::vector<int32_t> tmp;
    if (s_idx && t.ns) {
      tmp.resize(t.ns);
      SBD_CUDA(cudaMemcpy(tmp.data(), t.s_idx, sizeof(int32_t) * t.ns, cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < t.ns; i++) s_idx[i] = (uint64_t)tmp[i];
    }
    if (d_idx && t.nd) {
      tmp.resize(t.nd);
      SBD_CUDA(cudaMemcpy(tmp.data(), t.d_idx, sizeof(int32_t) * t.nd, cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < t.nd; i++) d_idx[i] = (uint64_t)tmp[i];
    }
  });
}

int sbdgpu_diag(sbdgpu_ctx* c, double* hii) {
  return guarded(c, [&] {
    if (!hii) throw Error{SBDGPU_ERR_ARG, "null output"};
    sbdgpu::build_tables(c);
    sbdgpu::compute_hii(c);
    SBD_CUDA(cudaMemcpyAsync(hii, c->hii, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->stream));
    SBD_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int sbdgpu_sigma(sbdgpu_ctx* c, const double* C, double* S, int precision) {
  return guarded(c, [&] {
    if (!C || !S) throw Error{SBDGPU_ERR_ARG, "null vector"};
    check_precision(precision);
    ensure_io(c);
    sbdgpu::build_tables(c);
    sbdgpu::compute_hii(c);
    sbdgpu::ensure_scratch(c);
    SBD_CUDA(cudaEventRecord(c->ev[6], c->stream));
    SBD_CUDA(cudaMemcpyAsync(c->io_b, C, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
    // sigma_ref_convention stages the input in io_a, so io_b can take the result
    sigma_ref_convention(c, c->io_b, c->io_b, precision);
    SBD_CUDA(cudaMemcpyAsync(S, c->io_b, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->stream));
    SBD_CUDA(cudaEventRecord(c->ev[7], c->stream));
    SBD_CUDA(cudaStreamSynchronize(c->stream));
    SBD_CUDA(cudaEventElapsedTime(&c->last_ms[4], c->ev[6], c->ev[7]));
  });
}

int sbdgpu_sigma_device(sbdgpu_ctx* c, const double* dC, double* dS, int precision) {
  return guarded(c, [&] {
    if (!dC || !dS) throw Error{SBDGPU_ERR_ARG, "null vector"};
    check_precision(precision);
    sigma_ref_convention(c, dC, dS, precision);
  });
}

int sbdgpu_sigma_rows_device(sbdgpu_ctx* c, const double* dC, double* dS, size_t r0, size_t r1) {
  return guarded(c, [&] {
    if (!dC || !dS) throw Error{SBDGPU_ERR_ARG, "null vector"};
    if (r0 > r1 || r1 > c->na) throw Error{SBDGPU_ERR_ARG, "row block outside [0, na]"};
    if (c->stored) throw Error{SBDGPU_ERR_STATE, "row-block sigma runs on the fly; release the stored Hamiltonian"};
    sbdgpu::sigma_rows_fp64(c, dC, dS, r0, r1);
  });
}

int sbdgpu_last_sigma_ms(sbdgpu_ctx* c, float* ms5) {
  return guarded(c, [&] {
    for (int k = 0; k < 5; k++) ms5[k] = c->last_ms[k];
  });
}

int sbdgpu_davidson(sbdgpu_ctx* c, const sbdgpu_opts* o, double* Wh, double* energy, double* trace_e,
                    double* trace_tol, int max_trace, int* n_steps) {
  return guarded(c, [&] {
    if (!o || !Wh) throw Error{SBDGPU_ERR_ARG, "null argument"};
    check_precision(o->precision);
    if (o->precond != SBDGPU_PRECOND_DIAGONAL && o->precond != SBDGPU_PRECOND_LEARNED &&
        o->precond != SBDGPU_PRECOND_OLSEN)
      throw Error{SBDGPU_ERR_ARG, "unsupported precond " + std::to_string(o->precond)};
    int nb = o->max_nb;
    if (nb < 1 || nb > 32) throw Error{SBDGPU_ERR_ARG, "max_nb must be in [1, 32]"};
    size_t n = c->N;
    cudaStream_t st = c->stream;
    sbdgpu::build_tables(c);
    sbdgpu::compute_hii(c);
    sbdgpu::ensure_scratch(c);
    std::vector<double*> C(nb, nullptr), HC(nb, nullptr);
    double *W = nullptr, *R = nullptr;
    struct Free {
      std::vector<double*>* a;
      std::vector<double*>* b;
      double** w;
      double** r;
      cudaStream_t s;
      ~Free() {
        cudaStreamSynchronize(s);  // an error path may leave kernels queued on these buffers
        for (auto p : *a) cudaFree(p);
        for (auto p : *b) cudaFree(p);
        cudaFree(*w);
        cudaFree(*r);
      }
    } guard{&C, &HC, &W, &R, st};
    W = (double*)sbdgpu::dev_alloc(sizeof(double) * n);
    R = (double*)sbdgpu::dev_alloc(sizeof(double) * n);
    SBD_CUDA(cudaMemcpyAsync(W, Wh, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    sbdgpu::apply_phase(c, W);
    if (o->precision != SBDGPU_FP64) {
      double e = 0.0;
      int steps = 0;
      davidson_mixed(c, o, W, R, &e, trace_e, trace_tol, max_trace, &steps);
      sbdgpu::apply_phase(c, W);
      SBD_CUDA(cudaMemcpyAsync(Wh, W, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
      SBD_CUDA(cudaStreamSynchronize(st));
      if (energy) *energy = e;
      if (n_steps) *n_steps = steps;
      return;
    }
    for (int k = 0; k < nb; k++) {
      C[k] = (double*)sbdgpu::dev_alloc(sizeof(double) * n);
      HC[k] = (double*)sbdgpu::dev_alloc(sizeof(double) * n);
    }
    const double eps_reg = 1.0e-12;
    std::vector<double> H(nb * nb, 0.0), U(nb * nb, 0.0), E(nb, 0.0);
    std::vector<double> step_times;
    auto t_start = std::chrono::steady_clock::now();
    int steps = 0;
    bool cont = true;
    for (int it = 0; it < o->max_it && cont; it++) {
      SBD_CUDA(cudaMemcpyAsync(C[0], W, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      for (int ib = 0; ib < nb; ib++) {
        auto t0 = std::chrono::steady_clock::now();
        sbdgpu::sigma_fp64(c, C[ib], HC[ib]);
        for (int jb = 0; jb <= ib; jb++) {
          H[jb + nb * ib] = sbdgpu::dot(c, C[jb], HC[ib], n);
          H[ib + nb * jb] = H[jb + nb * ib];
        }
        for (int jb = 0; jb <= ib; jb++)
          for (int kb = 0; kb <= ib; kb++) U[jb + nb * kb] = H[jb + nb * kb];
        sbdgpu::jacobi_eig(ib + 1, U.data(), nb, E.data());
        sbdgpu::ritz_update(C.data(), HC.data(), U.data(), ib + 1, E[0], W, R, n, st);
        double nw = std::sqrt(sbdgpu::dot(c, W, W, n));
        sbdgpu::scale(W, 1.0 / nw, n, st);
        double tol = std::sqrt(sbdgpu::dot(c, R, R, n));
        sbdgpu::scale(R, 1.0 / tol, n, st);
        if (trace_e && steps < max_trace) trace_e[steps] = E[0];
        if (trace_tol && steps < max_trace) trace_tol[steps] = tol;
        steps++;
        if (o->verbose) {
          // the reference's log line, chemistry/tpb/davidson.h:837-842
          std::cout << " Davidson iteration " << it << "." << ib << " (tol=" << tol << "):";
          for (int p = 0; p < std::min(ib + 1, 4); p++) std::cout << " " << E[p];
          std::cout << std::endl;
        }
        if (tol < o->eps) {
          cont = false;
          break;
        }
        if (ib < nb - 1) {
          sbdgpu::precondition(R, c->hii, E[0], eps_reg, C[ib + 1], n, st);
          for (int kb = 0; kb < ib + 1; kb++) {
            double olap = sbdgpu::dot(c, C[kb], C[ib + 1], n);
            sbdgpu::axpy(C[ib + 1], C[kb], -olap, n, st);
          }
          double nc = std::sqrt(sbdgpu::dot(c, C[ib + 1], C[ib + 1], n));
          sbdgpu::scale(C[ib + 1], 1.0 / nc, n, st);
        }
        SBD_CUDA(cudaStreamSynchronize(st));
        auto t1 = std::chrono::steady_clock::now();
        step_times.push_back(std::chrono::duration<double>(t1 - t0).count());
        double avg = 0.0;
        for (double x : step_times) avg += x;
        avg /= step_times.size();
        double elapsed = std::chrono::duration<double>(t1 - t_start).count();
        if (elapsed + avg > o->max_time) {  // davidson.h:880-902
          cont = false;
          break;
        }
      }
    }
    // E = <W|HW>, chemistry/tpb/sbdiag.h:239-262
    sbdgpu::sigma_fp64(c, W, R);
    double e = sbdgpu::dot(c, W, R, n);
    sbdgpu::apply_phase(c, W);
    SBD_CUDA(cudaMemcpyAsync(Wh, W, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    SBD_CUDA(cudaStreamSynchronize(st));
    if (energy) *energy = e;
    if (n_steps) *n_steps = steps;
  });
}

int sbdgpu_davidson_roots(sbdgpu_ctx* c, const sbdgpu_opts* o, int nroots, double* W, double* energies,
                          double* resid, int* n_iter, int* n_sigma) {
  return guarded(c, [&] { sbdgpu::davidson_roots(c, o, nroots, W, energies, resid, n_iter, n_sigma); });
}

int sbdgpu_wait_selftest(sbdgpu_ctx* c, long long spin_limit, int* status) {
  return guarded(c, [&] {
    if (!status || spin_limit < 1 || spin_limit > sbdgpu::kMaxSpinLimit)
      throw Error{SBDGPU_ERR_ARG, "status must be non-null and spin_limit in [1, 2^26]"};
    sbdgpu::wait_selftest(c, spin_limit, status);
  });
}

int sbdgpu_rdm(sbdgpu_ctx* c, const double* Wh, double* one, double* two) {
  return guarded(c, [&] {
    if (!Wh || !one || !two) throw Error{SBDGPU_ERR_ARG, "null argument"};
    sbdgpu::build_tables(c);
    ensure_io(c);
    SBD_CUDA(cudaMemcpyAsync(c->io_a, Wh, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
    sbdgpu::rdm(c, c->io_a, one, two);
  });
}

int sbdgpu_occupation(sbdgpu_ctx* c, const double* Wh, double* dens) {
  return guarded(c, [&] {
    if (!Wh || !dens) throw Error{SBDGPU_ERR_ARG, "null argument"};
    ensure_io(c);
    SBD_CUDA(cudaMemcpyAsync(c->io_a, Wh, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
    sbdgpu::occupation(c, c->io_a, dens);
  });
}

int sbdgpu_alpha_weights(sbdgpu_ctx* c, const double* Wh, double* D) {
  return guarded(c, [&] {
    if (!Wh || !D) throw Error{SBDGPU_ERR_ARG, "null argument"};
    ensure_io(c);
    SBD_CUDA(cudaMemcpyAsync(c->io_a, Wh, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
    sbdgpu::alpha_weights(c, c->io_a, c->io_b);
    SBD_CUDA(cudaMemcpyAsync(D, c->io_b, sizeof(double) * c->na, cudaMemcpyDeviceToHost, c->stream));
    SBD_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int sbdgpu_precond_train(sbdgpu_ctx* c, const sbdgpu_learn_opts* o, double* loss_trace, double* seconds) {
  return guarded(c, [&] {
    if (!o) throw Error{SBDGPU_ERR_ARG, "null options"};
    sbdgpu::train_learned(c, o, loss_trace, seconds);
  });
}

int sbdgpu_precond_get(sbdgpu_ctx* c, float* w, int* n) {
  return guarded(c, [&] { sbdgpu::learned_get(c, w, n); });
}

int sbdgpu_precond_set(sbdgpu_ctx* c, const float* w, int n) {
  return guarded(c, [&] { sbdgpu::learned_set(c, w, n); });
}

int sbdgpu_precond_apply(sbdgpu_ctx* c, const double* Rh, double e0, double* out) {
  return guarded(c, [&] {
    if (!Rh || !out) throw Error{SBDGPU_ERR_ARG, "null argument"};
    sbdgpu::build_tables(c);
    sbdgpu::compute_hii(c);
    ensure_io(c);
    SBD_CUDA(cudaMemcpyAsync(c->io_a, Rh, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
    sbdgpu::learned_precondition(c, c->io_a, e0, 1e-12, c->io_b);
    SBD_CUDA(cudaMemcpyAsync(out, c->io_b, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->stream));
    SBD_CUDA(cudaStreamSynchronize(c->stream));
    if (sbdgpu::tc_error(c)) throw Error{SBDGPU_ERR_CUDA, "learned preconditioner kernel: wait timed out"};
  });
}

int sbdgpu_set_fp64_same_spin(sbdgpu_ctx* c, int method) {
  return guarded(c, [&] {
    if (method != 0 && method != 1) throw Error{SBDGPU_ERR_ARG, "method must be 0 or 1"};
    SBD_CUDA(cudaStreamSynchronize(c->stream));
    c->oz.mode = method;
    if (method == 1) sbdgpu::free_ozaki(c);  // the residues of the operators go back to the device
  });
}

const char* sbdgpu_last_error(sbdgpu_ctx* c) { return c ? c->err.c_str() : "null context"; }

void sbdgpu_destroy(sbdgpu_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  sbdgpu::release_hamiltonian(c);
  sbdgpu::free_learned(c);
  sbdgpu::free_dense_same(c);
  sbdgpu::free_rdm_tables(c);
  sbdgpu::free_ozaki(c);
  sbdgpu::free_tables(c->tab[0]);
  sbdgpu::free_tables(c->tab[1]);
  cudaFree(c->astr); cudaFree(c->bstr); cudaFree(c->h1); cudaFree(c->vf); cudaFree(c->ja); cudaFree(c->jb);
  cudaFree(c->blk_off); cudaFree(c->blk_idx); cudaFree(c->blk_info);
  cudaFree(c->hii); cudaFree(c->tc_bk_off); cudaFree(c->tc_bk_ent); cudaFree(c->tc_err); cudaFree(c->ct16); cudaFree(c->io32); cudaFree(c->ja32); cudaFree(c->jb32); cudaFree(c->vf32);
  cudaFree(c->io_a); cudaFree(c->io_b); cudaFree(c->ct); cudaFree(c->st); cudaFree(c->red);
  for (int k = 0; k < 8; k++)
    if (c->ev[k]) cudaEventDestroy(c->ev[k]);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

}  // extern "C"
