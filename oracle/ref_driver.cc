/*
 * Reference harness: a C-ABI shim around the UNMODIFIED reference headers
 * (r-ccs-cms/sbd, include/sbd/...), compiled at MPI world size 1 against the
 * single-rank stub in oracle/mpi_stub.  Test infrastructure only: it is a
 * parity checker and the timed CPU baseline, never part of the product path.
 *
 * Every function below calls the reference's own code:
 *   sbdref_open        LoadFCIDump (framework/fcidump.h:27-139), LoadAlphaDets
 *                      (chemistry/basic/makedeterminants.h:160-185), ShuffleDet
 *                      (chemistry/basic/determinants.h:566-571), SetupIntegrals
 *                      (chemistry/basic/makeintegrals.h:10-55), TaskCommunicator /
 *                      MakeHelpers / RemakeHelpers (chemistry/tpb/helper.h:184-953)
 *                      exactly as sbd::tpb::diag does (chemistry/tpb/sbdiag.h:143-166)
 *   sbdref_tables      the helpers' flattened tables (helper.h:352-422)
 *   sbdref_hii         makeQChamDiagTerms (chemistry/tpb/qcham.h:314-366)
 *   sbdref_mult        direct mult (chemistry/tpb/mult.h:387-648), optionally on a
 *                      slice of bra alpha rows (rows are independent)
 *   sbdref_diag        sbd::tpb::diag (chemistry/tpb/sbdiag.h:102-456)
 *   sbdref_correlation Correlation (chemistry/tpb/correlation.h:194-443)
 *   sbdref_occupation  OccupationDensity (chemistry/tpb/occupation.h:10-95)
 *   sbdref_carryover   CarryOverAlphaDet (chemistry/tpb/rdmat.h:60-132)
 *   sbdref_save_wavefunction / sbdref_load_wavefunction
 *                      SaveWavefunction / LoadWavefunction (chemistry/tpb/restart.h:20-66,
 *                      414-658), the load mapping a saved basis onto this handle's
 */
#include <omp.h>
// the same standard headers the reference sample driver includes before sbd.h
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

struct RefHandle {
  sbd::FCIDump fcidump;
  std::vector<std::vector<size_t>> adet;
  std::vector<std::vector<size_t>> bdet;
  size_t bit_length = 20;
  int L = 0;
  int N = 0;
  double I0 = 0.0;
  sbd::oneInt<double> I1;
  sbd::twoInt<double> I2;
  std::vector<sbd::TaskHelpers> helper;
  std::vector<std::vector<size_t>> shared;
  std::vector<double> hii;
  bool have_hii = false;
  std::string last_output;
};

uint64_t pack_string(const std::vector<size_t>& s, size_t bit_length, int L) {
  uint64_t out = 0;
  for (int i = 0; i < L; i++) {
    size_t w = i / bit_length, b = i % bit_length;
    if ((s[w] >> b) & 1) out |= (uint64_t(1) << i);
  }
  return out;
}

void ensure_hii(RefHandle* h) {
  if (h->have_hii) return;
  sbd::makeQChamDiagTerms(h->adet, h->bdet, h->bit_length, (size_t)h->L, h->helper, h->I0, h->I1,
                          h->I2, h->hii, 0, 0, 0);
  h->have_hii = true;
}

}  // namespace

extern "C" {

int sbdref_max_threads() { return omp_get_max_threads(); }

void* sbdref_open(const char* fcidump_path, const char* adet_path, int bit_length, int shuffle) {
  try {
    RefHandle* h = new RefHandle();
    h->bit_length = (size_t)bit_length;
    h->fcidump = sbd::LoadFCIDump(fcidump_path);
    for (const auto& [key, value] : h->fcidump.header) {
      if (key == std::string("NORB")) h->L = std::atoi(value.c_str());
      if (key == std::string("NELEC")) h->N = std::atoi(value.c_str());
    }
    sbd::LoadAlphaDets(adet_path, h->adet, h->bit_length, (size_t)h->L);
    h->bdet = h->adet;
    if (shuffle != 0) {
      // sample driver main.cc:123-132
      sbd::ShuffleDet(h->adet, 1729u);
      sbd::ShuffleDet(h->bdet, 137u);
    }
    int L = 0, N = 0;
    sbd::SetupIntegrals(h->fcidump, L, N, h->I0, h->I1, h->I2);
    MPI_Comm hc, bc, tc;
    sbd::TaskCommunicator(0, 1, 1, 1, 1, hc, bc, tc);
    sbd::MakeHelpers(h->adet, h->bdet, h->bit_length, (size_t)h->L, h->helper, h->shared, hc, bc, tc,
                     1, 1);
    sbd::RemakeHelpers(h->adet, h->bdet, h->bit_length, (size_t)h->L, h->helper, h->shared, hc, bc,
                       tc, 1, 1);
    return h;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "sbdref_open: %s\n", e.what());
    return nullptr;
  }
}

void sbdref_close(void* hp) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  if (!h) return;
  sbd::FreeHelpers(h->helper);
  delete h;
}

int sbdref_norb(void* hp) { return static_cast<RefHandle*>(hp)->L; }
size_t sbdref_count(void* hp, int spin) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  return spin == 0 ? h->adet.size() : h->bdet.size();
}
double sbdref_ecore(void* hp) { return static_cast<RefHandle*>(hp)->I0; }

void sbdref_strings(void* hp, int spin, uint64_t* out) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  const auto& d = spin == 0 ? h->adet : h->bdet;
  for (size_t i = 0; i < d.size(); i++) out[i] = pack_string(d[i], h->bit_length, h->L);
}

/* kind 0 = singles, 1 = doubles.  Returns the total entry count; if offsets is
 * non-null fills offsets[n+1] and idx[total] (ascending ket index per bra). */
size_t sbdref_tables(void* hp, int spin, int kind, uint64_t* offsets, uint64_t* idx) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  const sbd::TaskHelpers& t = h->helper[0];
  size_t n = spin == 0 ? (t.braAlphaEnd - t.braAlphaStart) : (t.braBetaEnd - t.braBetaStart);
  size_t* len = spin == 0 ? (kind == 0 ? t.SinglesFromAlphaLen : t.DoublesFromAlphaLen)
                          : (kind == 0 ? t.SinglesFromBetaLen : t.DoublesFromBetaLen);
  const std::vector<size_t*>& sm = spin == 0 ? (kind == 0 ? t.SinglesFromAlphaSM : t.DoublesFromAlphaSM)
                                             : (kind == 0 ? t.SinglesFromBetaSM : t.DoublesFromBetaSM);
  size_t total = 0;
  for (size_t i = 0; i < n; i++) {
    if (offsets) offsets[i] = total;
    if (idx)
      for (size_t j = 0; j < len[i]; j++) idx[total + j] = sm[i][j];
    total += len[i];
  }
  if (offsets) offsets[n] = total;
  return total;
}

void sbdref_hii(void* hp, double* out) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  ensure_hii(h);
  std::memcpy(out, h->hii.data(), h->hii.size() * sizeof(double));
}

/* sigma rows [row_begin,row_end) of H*C, C full (na*nb), out (rows*nb). */
void sbdref_mult(void* hp, const double* C, double* out, size_t row_begin, size_t row_end) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  ensure_hii(h);
  size_t na = h->adet.size(), nb = h->bdet.size();
  std::vector<double> Wk(C, C + na * nb);
  std::vector<double> Wb(na * nb, 0.0);
  if (row_begin == 0 && row_end == na) {
    sbd::mult(h->hii, Wk, Wb, h->adet, h->bdet, h->bit_length, (size_t)h->L, 1, 1, h->helper, h->I0,
              h->I1, h->I2, 0, 0, 0);
    std::memcpy(out, Wb.data(), na * nb * sizeof(double));
    return;
  }
  // Row slice: same helpers with the bra-alpha window narrowed; the per-row
  // table pointers are shifted so each row still sees its own lists.
  std::vector<sbd::TaskHelpers> sl(h->helper.size());
  for (size_t k = 0; k < h->helper.size(); k++) {
    const sbd::TaskHelpers& f = h->helper[k];
    sbd::TaskHelpers& s = sl[k];
    s.braAlphaStart = row_begin;
    s.braAlphaEnd = row_end;
    s.ketAlphaStart = f.ketAlphaStart;
    s.ketAlphaEnd = f.ketAlphaEnd;
    s.braBetaStart = f.braBetaStart;
    s.braBetaEnd = f.braBetaEnd;
    s.ketBetaStart = f.ketBetaStart;
    s.ketBetaEnd = f.ketBetaEnd;
    s.taskType = f.taskType;
    s.adetShift = f.adetShift;
    s.bdetShift = f.bdetShift;
    s.SinglesFromAlphaLen = f.SinglesFromAlphaLen + row_begin;
    s.DoublesFromAlphaLen = f.DoublesFromAlphaLen + row_begin;
    s.SinglesFromBetaLen = f.SinglesFromBetaLen;
    s.DoublesFromBetaLen = f.DoublesFromBetaLen;
    s.SinglesFromAlphaSM.assign(f.SinglesFromAlphaSM.begin() + row_begin,
                                f.SinglesFromAlphaSM.begin() + row_end);
    s.DoublesFromAlphaSM.assign(f.DoublesFromAlphaSM.begin() + row_begin,
                                f.DoublesFromAlphaSM.begin() + row_end);
    s.SinglesFromBetaSM = f.SinglesFromBetaSM;
    s.DoublesFromBetaSM = f.DoublesFromBetaSM;
  }
  std::vector<double> zero(na * nb, 0.0);
  sbd::mult(zero, Wk, Wb, h->adet, h->bdet, h->bit_length, (size_t)h->L, 1, 1, sl, h->I0, h->I1,
            h->I2, 0, 0, 0);
  size_t rows = row_end - row_begin;
  for (size_t k = 0; k < rows * nb; k++) out[k] = Wb[k] + h->hii[row_begin * nb + k] * C[row_begin * nb + k];
}

/* Full sbd::tpb::diag.  Captures stdout (the reference's own log, which holds
 * the Davidson iteration trace).  The ground state W is written by the
 * reference itself when savename is given (SaveWavefunction, restart.h:20-66). */
double sbdref_diag(void* hp, int max_it, int max_nb, double eps, int do_rdm, double* density,
                   double* rdm1, double* rdm2, const char* savename) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  sbd::tpb::SBD d;
  d.max_it = max_it;
  d.max_nb = max_nb;
  d.eps = eps;
  d.do_rdm = do_rdm;
  d.bit_length = h->bit_length;
  double energy = 0.0;
  std::vector<double> dens;
  std::vector<std::vector<size_t>> co;
  std::vector<std::vector<double>> r1, r2;
  std::stringstream cap;
  std::streambuf* old = std::cout.rdbuf(cap.rdbuf());
  sbd::tpb::diag(0, d, h->fcidump, h->adet, h->bdet, std::string(""),
                 std::string(savename ? savename : ""), energy, dens, co, r1, r2);
  std::cout.rdbuf(old);
  h->last_output = cap.str();
  int L = h->L;
  if (density) for (int i = 0; i < 2 * L; i++) density[i] = dens[i];
  if (do_rdm && rdm1 && rdm2) {
    for (int s = 0; s < 2; s++) std::memcpy(rdm1 + s * L * L, r1[s].data(), sizeof(double) * L * L);
    size_t L4 = (size_t)L * L * L * L;
    for (int s = 0; s < 4; s++) std::memcpy(rdm2 + s * L4, r2[s].data(), sizeof(double) * L4);
  }
  return energy;
}

size_t sbdref_last_output(void* hp, char* buf, size_t cap) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  size_t n = h->last_output.size();
  if (buf && cap > 0) {
    size_t m = n < cap - 1 ? n : cap - 1;
    std::memcpy(buf, h->last_output.data(), m);
    buf[m] = 0;
  }
  return n;
}

void sbdref_correlation(void* hp, const double* W, double* rdm1, double* rdm2) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  size_t n = h->adet.size() * h->bdet.size();
  std::vector<double> w(W, W + n);
  std::vector<std::vector<double>> r1, r2;
  sbd::Correlation(w, h->adet, h->bdet, h->bit_length, (size_t)h->L, 1, 1, h->helper, 0, 0, 0, r1, r2);
  int L = h->L;
  size_t L4 = (size_t)L * L * L * L;
  for (int s = 0; s < 2; s++) std::memcpy(rdm1 + s * L * L, r1[s].data(), sizeof(double) * L * L);
  for (int s = 0; s < 4; s++) std::memcpy(rdm2 + s * L4, r2[s].data(), sizeof(double) * L4);
}

void sbdref_occupation(void* hp, const double* W, double* dens) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  size_t n = h->adet.size() * h->bdet.size();
  std::vector<double> w(W, W + n);
  std::vector<int> oidx(h->L);
  for (int i = 0; i < h->L; i++) oidx[i] = i;
  std::vector<double> res;
  sbd::OccupationDensity(oidx, w, h->adet, h->bdet, h->bit_length, 1, 1, 0, res);
  for (int i = 0; i < 2 * h->L; i++) dens[i] = res[i];
}

/* ratio == 0 uses the cumulative-weight threshold variant, else keeps ratio*Na
 * strings.  Writes the kept packed alpha strings to out (capacity na) and
 * returns the count; *weight receives the truncated weight (ratio variant). */
size_t sbdref_carryover(void* hp, const double* W, double ratio, double threshold, uint64_t* out,
                        double* weight) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  size_t n = h->adet.size() * h->bdet.size();
  std::vector<double> w(W, W + n);
  std::vector<std::vector<size_t>> rdet;
  double tw = 0.0;
  if (ratio == 0.0) {
    sbd::CarryOverAlphaDet(w, h->adet, h->bdet, 1, 1, 0, rdet, threshold);
  } else {
    size_t kept = static_cast<size_t>(ratio * h->adet.size());
    sbd::CarryOverAlphaDet(w, h->adet, h->bdet, 1, 1, 0, kept, rdet, tw);
  }
  if (weight) *weight = tw;
  for (size_t i = 0; i < rdet.size(); i++) out[i] = pack_string(rdet[i], h->bit_length, h->L);
  return rdet.size();
}

/* Writes W (this handle's basis) with the reference's SaveWavefunction. */
void sbdref_save_wavefunction(void* hp, const char* file, const double* W) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  std::vector<double> w(W, W + h->adet.size() * h->bdet.size());
  sbd::SaveWavefunction(std::string(file), h->adet, h->bdet, 1, 1, 0, 0, 0, w);
}

/* Reads a saved wavefunction onto this handle's basis (string lookup, then
 * normalisation) with the reference's LoadWavefunction. */
void sbdref_load_wavefunction(void* hp, const char* file, double* W) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  std::vector<double> w(h->adet.size() * h->bdet.size(), 0.0);
  sbd::LoadWavefunction(std::string(file), h->adet, h->bdet, 1, 1, 0, 0, 0, w);
  for (size_t i = 0; i < w.size(); i++) W[i] = w[i];
}

}  // extern "C"
