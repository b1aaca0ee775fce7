// Many independent problems at once.
//
// Each context owns its stream, tables and vectors, so the Davidson runs of
// different problems share nothing but the GPU.  Small problems are bound by
// launch latency and host round trips (a few microseconds of work per kernel,
// one host sync per dot product), so running them one after another leaves the
// GPU idle most of the time.  Here a pool of host threads takes problems from
// a shared counter and drives each one's Davidson (sbdgpu_davidson) on its own
// stream; the kernels of different problems overlap on the device.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "internal.cuh"

extern "C" int sbdgpu_davidson_batch(int nprob, sbdgpu_ctx* const* ctxs, const sbdgpu_opts* opts, double* const* W,
                                     double* energies, int* n_steps, int* status, int max_threads) {
  if (nprob < 0 || (nprob > 0 && (!ctxs || !opts || !W || !energies))) return SBDGPU_ERR_ARG;
  for (int i = 0; i < nprob; i++)
    if (!ctxs[i] || !W[i]) return SBDGPU_ERR_ARG;
  {
    // one thread per context at a time: the same context twice would race
    std::vector<sbdgpu_ctx*> seen(ctxs, ctxs + nprob);
    std::sort(seen.begin(), seen.end());
    if (std::adjacent_find(seen.begin(), seen.end()) != seen.end()) return SBDGPU_ERR_ARG;
  }
  // default pool: one thread per problem, at most one per host hardware
  // thread and at most 32 (each thread drives its own stream)
  const int hw = std::max(1, (int)std::thread::hardware_concurrency());
  int nt = max_threads > 0 ? std::min(max_threads, nprob) : std::min({nprob, hw, 32});
  std::atomic<int> next{0};
  std::vector<int> st(nprob, SBDGPU_OK);
  auto work = [&] {
    for (int i = next.fetch_add(1); i < nprob; i = next.fetch_add(1)) {
      int steps = 0;
      double e = 0.0;
      st[i] = sbdgpu_davidson(ctxs[i], opts, W[i], &e, nullptr, nullptr, 0, &steps);
      energies[i] = e;
      if (n_steps) n_steps[i] = steps;
    }
  };
  std::vector<std::thread> pool;
  try {
    pool.reserve(nt);
    for (int t = 0; t < nt; t++) pool.emplace_back(work);
  } catch (...) {
    // no exception crosses the C ABI: the threads started so far (or this
    // thread, if none started) finish the batch
  }
  if (pool.empty()) work();
  for (auto& t : pool) t.join();
  int first = SBDGPU_OK;
  for (int i = 0; i < nprob; i++) {
    if (status) status[i] = st[i];
    if (first == SBDGPU_OK && st[i] != SBDGPU_OK) first = st[i];
  }
  return first;
}
