// C-ABI shim around the UNMODIFIED reference headers' generic operator
// algebra (r-ccs-cms/sbd include/sbd/basic/): TEST INFRASTRUCTURE ONLY, built
// into oracle/_ref/libsbdref_generic.so by oracle/Makefile.
//
// It builds sbd::GeneralOp<double> objects with the reference's own
// operators (ElemT * FieldOp * FieldOp ..., as stdmodel.h:55-91 does), runs
// its NormalOrdering / Simplify (out_of_place_func/arithmetic.h:43-337) and
// GeneralOp_From_FCIDump (stdmodel.h:13-98), and exports the resulting term
// lists.  The generic mult itself is not exported: its basis search
// (Basis::IndexSearch, basis.h:317-322) bisects over the first nwords states
// only, and loops or reads past them for any other target.
#include <omp.h>
// the standard headers the reference sample driver includes before sbd.h
// (samples/selected_basis_diagonalization/main.cc:1-10)
#include <chrono>
#include <cmath>
#include <deque>
#include <fstream>
#include <iostream>
#include <random>
#include <unistd.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "mpi.h"
#include "sbd/sbd.h"

namespace {

using Op = sbd::GeneralOp<double>;

// (dag, site) of one field operator, read through the reference's own
// printing (arithmetic.h:445-454: "Adag(q)" or "A(q)")
void field(const sbd::ProductOp& p, int k, int* dag, int* q) {
  std::ostringstream s;
  s << p.extract(k, k + 1);
  const std::string t = s.str();
  *dag = t.rfind("Adag(", 0) == 0 ? 1 : 0;
  *q = std::stoi(t.substr(t.find('(') + 1));
}

}  // namespace

extern "C" {

void* sbdrefg_new() { return new Op(); }

void sbdrefg_free(void* h) { delete static_cast<Op*>(h); }

// H += coef * ops[0] * ops[1] * ... (each op = site | dag << 16); no
// operators: H += coef (a constant, filed as diagonal)
void sbdrefg_add_product(void* h, double coef, int nops, const int* ops) {
  Op& H = *static_cast<Op*>(h);
  if (nops == 0) {
    H += coef;
    return;
  }
  auto fop = [&](int k) { return sbd::FieldOp((ops[k] >> 16) & 1, ops[k] & 0xFFFF); };
  Op T = coef * fop(0);
  for (int k = 1; k < nops; k++) T = T * fop(k);
  H += T;
}

void sbdrefg_normal_order(void* h, int sign) { sbd::NormalOrdering(*static_cast<Op*>(h), sign != 0); }

void sbdrefg_simplify(void* h) { sbd::Simplify(*static_cast<Op*>(h)); }

void* sbdrefg_from_fcidump(const char* path, int* L, int* N) {
  Op* H = new Op();
  MPI_Comm comm = MPI_COMM_WORLD;
  sbd::GeneralOp_From_FCIDump(std::string(path), comm, comm, *L, *N, *H);
  return H;
}

// list 0: the diagonal terms (d_, e_); 1: the off-diagonal ones (o_, c_)
void sbdrefg_count(void* h, int list, size_t* nterms, size_t* nops) {
  const Op& H = *static_cast<Op*>(h);
  const size_t n = list == 0 ? H.NumNcTerms() : H.NumOpTerms();
  size_t ops = 0;
  for (size_t m = 0; m < n; m++) ops += (list == 0 ? H.NcTerm(m) : H.OpTerm(m)).size();
  *nterms = n;
  *nops = ops;
}

void sbdrefg_export(void* h, int list, double* coef, int* ndag, int64_t* off, int* ops) {
  const Op& H = *static_cast<Op*>(h);
  const size_t n = list == 0 ? H.NumNcTerms() : H.NumOpTerms();
  int64_t pos = 0;
  off[0] = 0;
  for (size_t m = 0; m < n; m++) {
    const sbd::ProductOp p = list == 0 ? H.NcTerm(m) : H.OpTerm(m);
    coef[m] = list == 0 ? H.NcCoef(m) : H.OpCoef(m);
    ndag[m] = p.n_dag();
    for (size_t k = 0; k < p.size(); k++) {
      int d = 0, q = 0;
      field(p, (int)k, &d, &q);
      ops[pos++] = q | (d << 16);
    }
    off[m + 1] = pos;
  }
}

}  // extern "C"
