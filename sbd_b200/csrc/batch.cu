// Many independent problems at once: a device-resident Davidson.
//
// The single-problem Davidson (api.cu) keeps the projected matrix, its
// eigenvectors and every norm and overlap on the host, so each step waits on
// the GPU for every dot product.  For small problems those waits, not the
// kernels, take the time.  Here every quantity of a step stays on the device:
//
//   dots        the same two-stage reductions, written to a per-problem
//               scalar block instead of copied out
//   eigenproblem one thread per problem runs the cyclic Jacobi on the
//               (m <= 32) projected matrix (the reference uses LAPACK dsyev,
//               framework/hp_numeric.h:500-517)
//   Ritz vector, residual, the diagonal correction, Gram-Schmidt and the
//               normalisations read their coefficients from that block
//
// so a whole step of one problem -- the correction from the previous step,
// its orthogonalisation, the sigma, the projected row, the eigenproblem, the
// Ritz update and the norms -- is a fixed sequence of launches on the
// problem's stream with fixed pointers.  Each (problem, Krylov index) step is
// captured once into a CUDA graph and then replayed: one launch per problem
// per step.  One host thread drives all problems in rounds: it launches one
// step graph per unconverged problem, then waits once for the round and reads
// each problem's residual norm (8 bytes, copied to pinned memory inside the
// graph).  The vectors of all problems come from one device allocation made
// before the first round.  The algorithm is the reference's
// (chemistry/tpb/davidson.h:661-923): collapse restart to the Ritz vector,
// the diagonal correction regularised by 1e-12, modified Gram-Schmidt, and the
// final energy <W|HW>.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "internal.cuh"

namespace sbdgpu {

namespace {

constexpr int kMaxNb = 32;
constexpr int kVT = 256;

// scalar block of one problem (doubles)
constexpr int kH = 0;                       // projected matrix, column-major [kMaxNb][kMaxNb]
constexpr int kU = kH + kMaxNb * kMaxNb;    // eigenvectors
constexpr int kE = kU + kMaxNb * kMaxNb;    // eigenvalues
constexpr int kDot = kE + kMaxNb;           // scratch dot results
constexpr int kTol = kDot + 8;              // residual norm
constexpr int kEn = kTol + 1;               // final energy
constexpr int kScal = kEn + 7;

struct PtrPackD {
  const double* p[kMaxNb];
};

unsigned grid_n(size_t n) { return (unsigned)std::min<size_t>((n + kVT - 1) / kVT, 148 * 8); }

// Cyclic Jacobi (the host solver's algorithm, api.cu jacobi_eig) by one warp:
// lane 0 forms each rotation, the lanes apply it to rows / columns k = lane.
// H: the upper triangle of the leading m x m block of the projected matrix
// (column-major, leading dimension kMaxNb); U, E: eigenvectors and
// eigenvalues in ascending order.  The matrices live in shared memory.
__global__ void __launch_bounds__(32) eig_kernel(double* sc, int m) {
  __shared__ double M[kMaxNb * kMaxNb];
  __shared__ double V[kMaxNb * kMaxNb];
  __shared__ double rot[2];
  __shared__ int order[kMaxNb];
  const int k = threadIdx.x;
  const double* H = sc + kH;
  for (int j = 0; j < m; j++)
    if (k < m) {
      M[k + j * m] = k <= j ? H[k + j * kMaxNb] : H[j + k * kMaxNb];
      V[k + j * m] = k == j ? 1.0 : 0.0;
    }
  __syncwarp();
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (int j = 0; j < m; j++)
      if (k < j) off += M[k + j * m] * M[k + j * m];
    for (int o = 16; o; o >>= 1) off += __shfl_xor_sync(0xffffffffu, off, o);
    if (off < 1e-300) break;
    for (int p = 0; p < m; p++)
      for (int q = p + 1; q < m; q++) {
        const double apq = M[p + q * m];  // the same value in every lane
        if (fabs(apq) < 1e-300) continue;
        if (k == 0) {
          const double theta = 0.5 * (M[q + q * m] - M[p + p * m]) / apq;
          const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          rot[0] = 1.0 / sqrt(t * t + 1.0);
          rot[1] = t * rot[0];
        }
        __syncwarp();
        const double cs = rot[0], sn = rot[1];
        if (k < m) {
          const double a = M[k + p * m], b = M[k + q * m];
          M[k + p * m] = cs * a - sn * b;
          M[k + q * m] = sn * a + cs * b;
        }
        __syncwarp();
        if (k < m) {
          const double a = M[p + k * m], b = M[q + k * m];
          M[p + k * m] = cs * a - sn * b;
          M[q + k * m] = sn * a + cs * b;
          const double va = V[k + p * m], vb = V[k + q * m];
          V[k + p * m] = cs * va - sn * vb;
          V[k + q * m] = sn * va + cs * vb;
        }
        __syncwarp();
      }
  }
  if (k == 0) {
    for (int i = 0; i < m; i++) order[i] = i;
    for (int i = 1; i < m; i++)  // insertion sort by eigenvalue
      for (int j = i; j > 0 && M[order[j] * (m + 1)] < M[order[j - 1] * (m + 1)]; j--) {
        const int x = order[j];
        order[j] = order[j - 1];
        order[j - 1] = x;
      }
  }
  __syncwarp();
  for (int c = 0; c < m; c++) {
    const int s = order[c];
    if (k == 0) sc[kE + c] = M[s + s * m];
    if (k < m) sc[kU + k + c * kMaxNb] = V[k + s * m];
  }
}

// W = sum_k u_k C_k, R = E0 W - sum_k u_k HC_k (u = lowest eigenvector)
__global__ void ritz_dev_kernel(PtrPackD c, PtrPackD hc, int nk, const double* __restrict__ sc,
                                double* __restrict__ W, double* __restrict__ R, size_t n) {
  __shared__ double u[kMaxNb];
  __shared__ double e0;
  if (threadIdx.x < nk) u[threadIdx.x] = sc[kU + threadIdx.x];
  if (threadIdx.x == 0) e0 = sc[kE];
  __syncthreads();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double w = 0.0, r = 0.0;
    for (int k = 0; k < nk; k++) {
      w += c.p[k][i] * u[k];
      r -= hc.p[k][i] * u[k];
    }
    W[i] = w;
    R[i] = r + e0 * w;
  }
}

// x *= 1 / sqrt(*d)
__global__ void scale_rsqrt_kernel(double* __restrict__ x, const double* __restrict__ d, size_t n) {
  const double a = 1.0 / sqrt(*d);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] *= a;
}

// y -= (*a) x
__global__ void axpy_neg_kernel(double* __restrict__ y, const double* __restrict__ x, const double* __restrict__ a,
                                size_t n) {
  const double s = -*a;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] += x[i] * s;
}

// out = R / (E0 - H_ii), regularised as davidson.h:855-862, E0 = the lowest eigenvalue
__global__ void precond_dev_kernel(const double* __restrict__ R, const double* __restrict__ hii,
                                   const double* __restrict__ sc, double* __restrict__ out, size_t n) {
  const double e0 = sc[kE], eps_reg = 1.0e-12;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double den = e0 - hii[i];
    out[i] = fabs(den) > eps_reg ? R[i] / den : R[i] / (den - eps_reg);
  }
}

__global__ void sqrt_to_kernel(const double* __restrict__ d, double* __restrict__ out) { *out = sqrt(*d); }

// One problem of the batch: its context, vectors (slices of the batch's
// allocation), scalar block, pinned residual norm and step graphs.
struct Prob {
  sbdgpu_ctx* c = nullptr;
  size_t n = 0;
  int nb = 0;
  std::vector<double*> C, HC;
  double* W = nullptr;
  double* R = nullptr;
  double* sc = nullptr;
  double* host = nullptr;  // pinned: [tol, energy]
  std::vector<cudaGraphExec_t> step;  // step graph per Krylov index
  int it = 0, ib = 0, steps = 0;
  bool done = false;
};

// The launches of step ib: the correction of the previous step (or, at ib =
// 0, the copy W -> C[0] that opens a cycle), then the sigma, the projected
// row, the eigenproblem, the Ritz update, the norms and the copy of the
// residual norm to the host.
void enqueue_step(Prob& p, int ib) {
  sbdgpu_ctx* c = p.c;
  cudaStream_t st = c->stream;
  const size_t n = p.n;
  double* dot = p.sc + kDot;
  if (ib == 0) {
    SBD_CUDA(cudaMemcpyAsync(p.C[0], p.W, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  } else {
    precond_dev_kernel<<<grid_n(n), kVT, 0, st>>>(p.R, c->hii, p.sc, p.C[ib], n);
    SBD_CUDA(cudaGetLastError());
    for (int kb = 0; kb < ib; kb++) {  // modified Gram-Schmidt, davidson.h:864-875
      dot_device(c, p.C[kb], p.C[ib], n, dot);
      axpy_neg_kernel<<<grid_n(n), kVT, 0, st>>>(p.C[ib], p.C[kb], dot, n);
    }
    dot_device(c, p.C[ib], p.C[ib], n, dot);
    scale_rsqrt_kernel<<<grid_n(n), kVT, 0, st>>>(p.C[ib], dot, n);
    SBD_CUDA(cudaGetLastError());
  }
  sigma_fp64_prepared(c, p.C[ib], p.HC[ib], c->ct, c->st);
  for (int jb = 0; jb <= ib; jb++) dot_device(c, p.C[jb], p.HC[ib], n, p.sc + kH + jb + kMaxNb * ib);
  eig_kernel<<<1, 32, 0, st>>>(p.sc, ib + 1);
  PtrPackD pc{}, ph{};
  for (int k = 0; k <= ib; k++) {
    pc.p[k] = p.C[k];
    ph.p[k] = p.HC[k];
  }
  ritz_dev_kernel<<<grid_n(n), kVT, 0, st>>>(pc, ph, ib + 1, p.sc, p.W, p.R, n);
  SBD_CUDA(cudaGetLastError());
  dot_device(c, p.W, p.W, n, dot);
  scale_rsqrt_kernel<<<grid_n(n), kVT, 0, st>>>(p.W, dot, n);
  dot_device(c, p.R, p.R, n, dot + 1);
  sqrt_to_kernel<<<1, 1, 0, st>>>(dot + 1, p.sc + kTol);
  scale_rsqrt_kernel<<<grid_n(n), kVT, 0, st>>>(p.R, dot + 1, n);
  SBD_CUDA(cudaGetLastError());
  SBD_CUDA(cudaMemcpyAsync(p.host, p.sc + kTol, sizeof(double), cudaMemcpyDeviceToHost, st));
}

// Replays the step's graph, capturing it on first use.  If the capture or
// the instantiation is refused, the problem's steps are launched directly
// from then on.
void launch_step(Prob& p, int ib, bool& graphs) {
  cudaStream_t st = p.c->stream;
  if (graphs && !p.step[ib]) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      try {
        enqueue_step(p, ib);
      } catch (...) {
        ok = false;
      }
      ok = cudaStreamEndCapture(st, &g) == cudaSuccess && ok && g != nullptr;
      ok = ok && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
      if (g) cudaGraphDestroy(g);
    }
    if (!ok) {
      cudaGetLastError();  // the refused capture leaves no sticky error
      graphs = false;
    } else {
      p.step[ib] = ex;
    }
  }
  if (graphs && p.step[ib])
    SBD_CUDA(cudaGraphLaunch(p.step[ib], st));
  else
    enqueue_step(p, ib);
}

void davidson_batch_fp64(int nprob, sbdgpu_ctx* const* ctxs, const sbdgpu_opts* o, double* const* Wh,
                         double* energies, int* n_steps) {
  const int nb = o->max_nb;
  std::vector<Prob> P(nprob);
  size_t total = 0;
  for (int i = 0; i < nprob; i++) {
    sbdgpu_ctx* c = ctxs[i];
    build_tables(c);
    compute_hii(c);
    ensure_scratch(c);
    P[i].c = c;
    P[i].n = c->N;
    P[i].nb = nb;
    total += (size_t)(2 * nb + 2) * ((c->N + 1) & ~size_t(1)) + kScal;  // vectors start on 16 bytes
  }
  preload_fp64_sigma(ctxs[0]->device);
  // every vector of every problem in one allocation, made before the first round
  double* arena = (double*)dev_alloc(sizeof(double) * total);
  double* pinned = nullptr;
  struct Release {
    std::vector<Prob>* P;
    double* a;
    double** h;
    ~Release() {
      for (auto& p : *P) {
        if (p.c) cudaStreamSynchronize(p.c->stream);
        for (auto g : p.step)
          if (g) cudaGraphExecDestroy(g);
      }
      cudaFree(a);
      if (*h) cudaFreeHost(*h);
    }
  } release{&P, arena, &pinned};
  SBD_CUDA(cudaMallocHost(&pinned, sizeof(double) * 2 * std::max(nprob, 1)));
  size_t off = 0;
  for (int i = 0; i < nprob; i++) {
    Prob& p = P[i];
    const size_t stride = (p.n + 1) & ~size_t(1);
    p.C.resize(nb);
    p.HC.resize(nb);
    for (int k = 0; k < nb; k++) {
      p.C[k] = arena + off;
      off += stride;
      p.HC[k] = arena + off;
      off += stride;
    }
    p.W = arena + off;
    off += stride;
    p.R = arena + off;
    off += stride;
    p.sc = arena + off;
    off += kScal;
    p.host = pinned + 2 * i;
    p.step.assign(nb, nullptr);
    SBD_CUDA(cudaMemsetAsync(p.sc, 0, sizeof(double) * kScal, p.c->stream));
    SBD_CUDA(cudaMemcpyAsync(p.W, Wh[i], sizeof(double) * p.n, cudaMemcpyHostToDevice, p.c->stream));
    apply_phase(p.c, p.W);
  }
  const auto t0 = std::chrono::steady_clock::now();
  int active = nprob;
  bool graphs = true;
  while (active > 0) {
    for (auto& p : P)
      if (!p.done) launch_step(p, p.ib, graphs);
    for (auto& p : P) {
      if (p.done) continue;
      SBD_CUDA(cudaStreamSynchronize(p.c->stream));
      p.steps++;
      const double tol = p.host[0];
      bool stop = !(tol >= o->eps);  // a NaN residual stops the problem too
      if (!stop) {
        if (p.ib < nb - 1) {
          p.ib++;
        } else {
          p.ib = 0;
          p.it++;
          stop = p.it >= o->max_it;
        }
      }
      const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (stop || elapsed > o->max_time) {
        p.done = true;
        active--;
      }
    }
  }
  // E = <W|HW> (chemistry/tpb/sbdiag.h:239-262), W back in the caller's convention
  for (auto& p : P) {
    sigma_fp64_prepared(p.c, p.W, p.R, p.c->ct, p.c->st);
    dot_device(p.c, p.W, p.R, p.n, p.sc + kEn);
    SBD_CUDA(cudaMemcpyAsync(p.host + 1, p.sc + kEn, sizeof(double), cudaMemcpyDeviceToHost, p.c->stream));
    apply_phase(p.c, p.W);
  }
  for (int i = 0; i < nprob; i++) {
    Prob& p = P[i];
    SBD_CUDA(cudaMemcpyAsync(Wh[i], p.W, sizeof(double) * p.n, cudaMemcpyDeviceToHost, p.c->stream));
    SBD_CUDA(cudaStreamSynchronize(p.c->stream));
    energies[i] = p.host[1];
    if (n_steps) n_steps[i] = p.steps;
  }
}

}  // namespace

}  // namespace sbdgpu

using sbdgpu::Error;

namespace {

template <class F>
int guarded_ctx(sbdgpu_ctx* c, F&& f) {
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

}  // namespace

extern "C" int sbdgpu_davidson_batch(int nprob, sbdgpu_ctx* const* ctxs, const sbdgpu_opts* opts, double* const* W,
                                     double* energies, int* n_steps, int* status, int max_threads) {
  (void)max_threads;  // one host thread drives every problem
  if (nprob < 0 || (nprob > 0 && (!ctxs || !opts || !W || !energies))) return SBDGPU_ERR_ARG;
  for (int i = 0; i < nprob; i++)
    if (!ctxs[i] || !W[i]) return SBDGPU_ERR_ARG;
  if (nprob == 0) return SBDGPU_OK;
  {
    std::vector<sbdgpu_ctx*> seen(ctxs, ctxs + nprob);
    std::sort(seen.begin(), seen.end());
    if (std::adjacent_find(seen.begin(), seen.end()) != seen.end()) return SBDGPU_ERR_ARG;
  }
  bool engine = opts->precision == SBDGPU_FP64 && opts->max_nb >= 1 && opts->max_nb <= 32;
  for (int i = 0; i < nprob && engine; i++) engine = ctxs[i]->device == ctxs[0]->device && !ctxs[i]->stored;
  int first = SBDGPU_OK;
  if (engine) {
    const int rc = guarded_ctx(ctxs[0], [&] {
      sbdgpu::davidson_batch_fp64(nprob, ctxs, opts, W, energies, n_steps);
    });
    for (int i = 0; i < nprob; i++) {
      if (status) status[i] = rc;
      if (rc != SBDGPU_OK && i > 0) ctxs[i]->err = ctxs[0]->err;
    }
    return rc;
  }
  // other precisions, a stored Hamiltonian or several devices: each problem's
  // own Davidson in turn
  for (int i = 0; i < nprob; i++) {
    int steps = 0;
    double e = 0.0;
    const int rc = sbdgpu_davidson(ctxs[i], opts, W[i], &e, nullptr, nullptr, 0, &steps);
    energies[i] = e;
    if (n_steps) n_steps[i] = steps;
    if (status) status[i] = rc;
    if (first == SBDGPU_OK && rc != SBDGPU_OK) first = rc;
  }
  return first;
}

extern "C" int sbdgpu_set_tuning(sbdgpu_ctx* c, int ab_group, int ab_threads) {
  return guarded_ctx(c, [&] {
    if (ab_group == 0 && ab_threads == 0) {
      c->ab_group = c->ab_threads = 0;
      return;
    }
    sbdgpu::build_tables(c);
    const auto shapes = sbdgpu::ab_shapes(c);
    if (std::find(shapes.begin(), shapes.end(), std::make_pair(ab_group, ab_threads)) == shapes.end())
      throw Error{SBDGPU_ERR_ARG, "alpha-beta shape (" + std::to_string(ab_group) + ", " +
                                      std::to_string(ab_threads) + ") does not fit this basis"};
    c->ab_group = ab_group;
    c->ab_threads = ab_threads;
  });
}

extern "C" int sbdgpu_autotune(sbdgpu_ctx* c, int reps, int* ab_group, int* ab_threads, float* best_ms) {
  return guarded_ctx(c, [&] {
    if (reps < 1) throw Error{SBDGPU_ERR_ARG, "reps must be positive"};
    sbdgpu::build_tables(c);
    sbdgpu::compute_hii(c);
    sbdgpu::ensure_scratch(c);
    sbdgpu::ensure_io(c);
    sbdgpu::preload_fp64_sigma(c->device);
    cudaStream_t st = c->stream;
    // an input with no zeros: the diagonal
    SBD_CUDA(cudaMemcpyAsync(c->io_a, c->hii, sizeof(double) * c->N, cudaMemcpyDeviceToDevice, st));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    SBD_CUDA(cudaEventCreate(&e0));
    SBD_CUDA(cudaEventCreate(&e1));
    struct Ev {
      cudaEvent_t a, b;
      ~Ev() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
      }
    } ev{e0, e1};
    float best = 1e30f;
    std::pair<int, int> pick{0, 0};
    for (const auto& sh : sbdgpu::ab_shapes(c)) {
      c->ab_group = sh.first;
      c->ab_threads = sh.second;
      sbdgpu::sigma_fp64_prepared(c, c->io_a, c->io_b, c->ct, c->st);  // warm-up
      SBD_CUDA(cudaEventRecord(e0, st));
      for (int r = 0; r < reps; r++) sbdgpu::sigma_fp64_prepared(c, c->io_a, c->io_b, c->ct, c->st);
      SBD_CUDA(cudaEventRecord(e1, st));
      SBD_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      SBD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      ms /= reps;
      if (ms < best) {
        best = ms;
        pick = sh;
      }
    }
    c->ab_group = pick.first;
    c->ab_threads = pick.second;
    if (ab_group) *ab_group = pick.first;
    if (ab_threads) *ab_threads = pick.second;
    if (best_ms) *best_ms = best;
  });
}
