// Block Davidson for several of the lowest roots (FP64).
//
// The reference's Davidson (chemistry/tpb/davidson.h:661-923) follows the
// lowest root only.  This extends the same ingredients (the on-the-fly sigma,
// the diagonal preconditioner with eps_reg = 1e-12, Gram-Schmidt against the
// basis, the projected eigenproblem) to a block of roots, Davidson-Liu style:
//
//   basis V (m vectors, sigma HV kept), H_sub = V^T H V, H_sub u_k = E_k u_k
//   x_k = V u_k, r_k = E_k x_k - HV u_k for the nroots lowest k
//   each unconverged root adds t_k = r_k / (E_k - H_ii), orthogonalised
//   (two Gram-Schmidt passes) against V and the other new vectors
//   when m would pass max_nb: collapse (GD+k restart, Stathopoulos and Saad)
//   to the span of the current nroots Ritz vectors and the previous cycle's
//   nroots Ritz vectors, with their sigma vectors (linear combinations, no new
//   sigma).  Keeping the previous directions carries the convergence history
//   across the restart; in a numpy run of this loop on a 6,400-determinant
//   problem it cut the sigma builds for 8 roots from 2,171 (collapse to the
//   max_nb / 2 lowest Ritz vectors) to 569.
//
// Converged when every root's residual norm is below eps.  Vectors live in the
// alpha-string-major convention; the caller's W are in the reference's
// (interleaved) convention and go through the diagonal phase at entry and exit.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <iostream>
#include <numeric>

#include "internal.cuh"

namespace sbdgpu {

void davidson_roots(sbdgpu_ctx* c, const sbdgpu_opts* o, int nroots, double* Wh, double* energies, double* resid,
                    int* n_iter, int* n_sigma) {
  if (!o || !Wh || !energies) throw Error{SBDGPU_ERR_ARG, "null argument"};
  if (o->precision != SBDGPU_FP64) throw Error{SBDGPU_ERR_ARG, "several roots: FP64 only"};
  const size_t n = c->N;
  const int max_sub = o->max_nb;
  if (nroots < 1 || (size_t)nroots > n) throw Error{SBDGPU_ERR_ARG, "nroots must be in [1, na*nb]"};
  if (max_sub < 2 * nroots || max_sub > 32) throw Error{SBDGPU_ERR_ARG, "max_nb must be in [2*nroots, 32]"};
  cudaStream_t st = c->stream;
  build_tables(c);
  compute_hii(c);
  ensure_scratch(c);
  const int keep = 2 * nroots;  // collapsed basis: current and previous Ritz vectors
  std::vector<double*> C(max_sub, nullptr), HC(max_sub, nullptr), T(keep, nullptr), TH(keep, nullptr);
  double *X = nullptr, *R = nullptr;
  struct Free {
    std::vector<double*>* v[4];
    double** x[2];
    cudaStream_t s;
    ~Free() {
      cudaStreamSynchronize(s);  // an error path may leave kernels queued on these buffers
      for (auto* a : v)
        for (auto p : *a) cudaFree(p);
      for (auto* p : x) cudaFree(*p);
    }
  } guard{{&C, &HC, &T, &TH}, {&X, &R}, st};
  for (int k = 0; k < max_sub; k++) {
    C[k] = (double*)dev_alloc(sizeof(double) * n);
    HC[k] = (double*)dev_alloc(sizeof(double) * n);
  }
  for (int k = 0; k < keep; k++) {
    T[k] = (double*)dev_alloc(sizeof(double) * n);
    TH[k] = (double*)dev_alloc(sizeof(double) * n);
  }
  X = (double*)dev_alloc(sizeof(double) * n);
  R = (double*)dev_alloc(sizeof(double) * n);

  // orthonormalise v against C[0..m) (two passes); false if nothing is left
  auto orthonormalise = [&](double* v, int m) {
    double n0 = std::sqrt(dot(c, v, v, n));
    if (!(n0 > 0.0)) return false;
    for (int pass = 0; pass < 2; pass++)
      for (int j = 0; j < m; j++) axpy(v, C[j], -dot(c, C[j], v, n), n, st);
    double n1 = std::sqrt(dot(c, v, v, n));
    if (!(n1 > 1e-10 * n0)) return false;
    scale(v, 1.0 / n1, n, st);
    return true;
  };

  // initial basis: the caller's vectors, or determinant 0 (the reference's
  // start vector, davidson.h:120-135) and the lowest-H_ii determinants.  The
  // lowest-H_ii determinants alone can miss the ground state's symmetry
  // sector altogether (at 144M determinants they found a root 26 Eh above it).
  int m = 0;
  {
    double w2 = 0.0;
    for (size_t i = 0; i < (size_t)nroots * n; i++) w2 += Wh[i] * Wh[i];
    if (w2 > 0.0) {
      for (int k = 0; k < nroots; k++) {
        SBD_CUDA(cudaMemcpyAsync(C[m], Wh + (size_t)k * n, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        apply_phase(c, C[m]);
        if (orthonormalise(C[m], m)) m++;
      }
    }
    if (m < nroots) {
      std::vector<double> h(n);
      SBD_CUDA(cudaMemcpyAsync(h.data(), c->hii, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
      SBD_CUDA(cudaStreamSynchronize(st));
      std::vector<size_t> order(n);
      std::iota(order.begin(), order.end(), (size_t)0);
      std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return h[a] < h[b]; });
      const double one = 1.0;
      std::stable_partition(order.begin(), order.end(), [](size_t a) { return a == 0; });
      for (size_t q = 0; q < n && m < nroots; q++) {
        SBD_CUDA(cudaMemsetAsync(C[m], 0, sizeof(double) * n, st));
        SBD_CUDA(cudaMemcpyAsync(C[m] + order[q], &one, sizeof(double), cudaMemcpyHostToDevice, st));
        if (orthonormalise(C[m], m)) m++;
      }
    }
  }

  const double eps_reg = 1.0e-12;
  std::vector<double> H(max_sub * max_sub, 0.0), U(max_sub * max_sub, 0.0), E(max_sub, 0.0), rn(nroots, 0.0);
  std::vector<double> col(max_sub, 0.0);
  std::vector<double> Uprev((size_t)max_sub * nroots, 0.0);  // previous cycle's Ritz coefficients
  int m_prev = 0;
  int done = 0, iters = 0, sigmas = 0;
  auto t_start = std::chrono::steady_clock::now();
  // x_k = V u_k into X and r_k = E_k x_k - HV u_k into R
  auto ritz = [&](int k, int mm) {
    for (int i = 0; i < mm; i++) col[i] = U[i + max_sub * k];
    ritz_update(C.data(), HC.data(), col.data(), mm, E[k], X, R, n, st);
  };
  auto solve = [&](int mm) {
    for (int j = 0; j < mm; j++)
      for (int i = 0; i < mm; i++) U[i + max_sub * j] = H[i + max_sub * j];
    jacobi_eig(mm, U.data(), max_sub, E.data());
  };
  for (int it = 0; it < o->max_it; it++) {
    for (; done < m; done++) {
      sigma_fp64(c, C[done], HC[done]);
      sigmas++;
      for (int i = 0; i <= done; i++) {
        H[i + max_sub * done] = dot(c, C[i], HC[done], n);
        H[done + max_sub * i] = H[i + max_sub * done];
      }
    }
    solve(m);
    iters++;
    int unconv = 0;
    for (int k = 0; k < nroots; k++) {
      ritz(k, m);
      rn[k] = std::sqrt(dot(c, R, R, n));
      if (!(rn[k] < o->eps)) unconv++;
    }
    if (o->verbose) {
      std::cout << " Block Davidson iteration " << it << " (basis " << m << "):";
      for (int k = 0; k < nroots; k++) std::cout << " " << E[k] << " (" << rn[k] << ")";
      std::cout << std::endl;
    }
    if (unconv == 0) break;
    double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    if (elapsed > o->max_time || it + 1 == o->max_it) break;
    if (m + unconv > max_sub) {
      // small-space coefficients of the collapsed basis: the current Ritz
      // vectors, then the previous ones (zero on the vectors added since),
      // orthonormalised (two Gram-Schmidt passes; V is orthonormal)
      std::vector<std::vector<double>> Q;
      auto add_col = [&](std::vector<double> y) {
        for (int pass = 0; pass < 2; pass++)
          for (const auto& q : Q) {
            double d = 0.0;
            for (int i = 0; i < m; i++) d += q[i] * y[i];
            for (int i = 0; i < m; i++) y[i] -= d * q[i];
          }
        double nn = 0.0;
        for (int i = 0; i < m; i++) nn += y[i] * y[i];
        nn = std::sqrt(nn);
        if (nn > 1e-8) {
          for (int i = 0; i < m; i++) y[i] /= nn;
          Q.push_back(std::move(y));
        }
      };
      for (int k = 0; k < nroots; k++) {
        std::vector<double> y(m, 0.0);
        for (int i = 0; i < m; i++) y[i] = U[i + max_sub * k];
        add_col(std::move(y));
      }
      // at most max_nb - nroots vectors, so that every root can add a correction
      for (int k = 0; k < nroots && (int)Q.size() < max_sub - nroots; k++) {
        std::vector<double> y(m, 0.0);
        for (int i = 0; i < m_prev && i < m; i++) y[i] = Uprev[i + (size_t)max_sub * k];
        add_col(std::move(y));
      }
      const int kk = (int)Q.size();
      for (int j = 0; j < kk; j++) {
        // V q_j and -HV q_j: the Ritz update with E = 0
        ritz_update(C.data(), HC.data(), Q[j].data(), m, 0.0, T[j], TH[j], n, st);
        scale(TH[j], -1.0, n, st);
      }
      for (int j = 0; j < kk; j++) {
        std::swap(C[j], T[j]);
        std::swap(HC[j], TH[j]);
      }
      m = done = kk;
      for (int j = 0; j < m; j++)
        for (int i = 0; i <= j; i++) {
          H[i + max_sub * j] = dot(c, C[i], HC[j], n);
          H[j + max_sub * i] = H[i + max_sub * j];
        }
      solve(m);
    }
    // this cycle's Ritz coefficients, for the next collapse
    for (int k = 0; k < nroots; k++)
      for (int i = 0; i < m; i++) Uprev[i + (size_t)max_sub * k] = U[i + max_sub * k];
    m_prev = m;
    const int m_solved = m;  // U holds the eigenvectors of this basis only
    for (int k = 0; k < nroots && m < max_sub; k++) {
      if (rn[k] < o->eps) continue;
      ritz(k, m_solved);
      precondition(R, c->hii, E[k], eps_reg, C[m], n, st);
      if (orthonormalise(C[m], m)) m++;
    }
    if (m == done) break;  // no direction left to add
  }
  SBD_CUDA(cudaStreamSynchronize(st));
  for (int k = 0; k < nroots; k++) {
    ritz(k, m);
    double nx = std::sqrt(dot(c, X, X, n));
    scale(X, 1.0 / nx, n, st);
    apply_phase(c, X);
    SBD_CUDA(cudaMemcpyAsync(Wh + (size_t)k * n, X, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    energies[k] = E[k];
    if (resid) resid[k] = rn[k];
  }
  SBD_CUDA(cudaStreamSynchronize(st));
  if (n_iter) *n_iter = iters;
  if (n_sigma) *n_sigma = sigmas;
}

}  // namespace sbdgpu
