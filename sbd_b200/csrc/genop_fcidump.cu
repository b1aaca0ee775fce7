// sbdgpu_genop_set_fcidump: the quantum-chemistry Hamiltonian of an FCIDUMP
// file as the operator of a generic-path object, built on the host with the
// operator algebra of sbd_gpu/generalop.h (GeneralOp_From_FCIDump,
// basic/out_of_place_func/stdmodel.h:13-98) and handed to
// sbdgpu_genop_set_terms.  Host code only.
#include <exception>
#include <string>

#include "internal.cuh"
#include "sbd_gpu/generalop.h"

extern "C" int sbdgpu_genop_set_fcidump(sbdgpu_genop* g, const char* path, int* norb, int* nelec) {
  if (!g || !path) return SBDGPU_ERR_ARG;
  sbd::GeneralOp<double> H;
  int L = 0, N = 0;
  try {
    sbd::GeneralOp_From_FCIDump<double>(std::string(path), MPI_COMM_WORLD, MPI_COMM_WORLD, L, N, H);
  } catch (const std::exception& e) {
    sbdgpu::genop_set_error(g, std::string("FCIDUMP: ") + e.what());
    return SBDGPU_ERR_ARG;
  }
  const int rc = sbd::gpu::set_terms(g, H);
  if (rc == SBDGPU_OK) {
    if (norb) *norb = L;
    if (nelec) *nelec = N;
  }
  return rc;
}
