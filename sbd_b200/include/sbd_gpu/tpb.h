/*
 * sbd_gpu/tpb.h -- header-only C++ host library: the drop-in for the
 * reference's tensor-product-basis entry point sbd::tpb::diag
 * (r-ccs-cms/sbd include/sbd/chemistry/tpb/sbdiag.h:102-113 and 472-482),
 * running the Davidson hot path on one B200 through the C ABI in sbdgpu.h.
 *
 * Kept from the reference, with the same names, argument meaning and error
 * behaviour (C++ exceptions):
 *   sbd::FCIDump / LoadFCIDump           framework/fcidump.h:18-139
 *   sbd::LoadAlphaDets, from_string,     chemistry/basic/makedeterminants.h:160-185,
 *   makestring, sort_bitarray,           framework/bit_manipulation.h:135-172, 324-330
 *   DecodeAlphaDets, ShuffleDet          makedeterminants.h:63-108, determinants.h:566-571
 *   sbd::tpb::SBD, generate_sbd_data     chemistry/tpb/sbdiag.h:12-85
 *   SaveWavefunction, LoadWavefunction   chemistry/tpb/restart.h:20-66, 414-658
 *   CarryOverAlphaDet (both variants)    chemistry/tpb/rdmat.h:60-132
 *   sbd::tpb::diag (both overloads)      chemistry/tpb/sbdiag.h:102-565
 * The run is MPI world size 1 on one GPU: the communicator argument is
 * accepted for signature compatibility; with a real MPI build a communicator
 * of more than one rank is rejected.  Added options (not in the reference):
 * SBD::device (--device), SBD::precision (--precision), SBD::restart_keep
 * (--restart_keep) and SBD::restart_prev (--restart_prev).
 */
#ifndef SBD_GPU_TPB_H
#define SBD_GPU_TPB_H

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <numeric>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "sbdgpu.h"

#if defined(SBD_GPU_WITH_MPI) || __has_include(<mpi.h>)
#include <mpi.h>
#define SBD_GPU_HAVE_MPI 1
#else
typedef int MPI_Comm;
#ifndef MPI_COMM_WORLD
#define MPI_COMM_WORLD 0
#endif
#endif

namespace sbd {

struct FCIDump {
  std::map<std::string, std::string> header;
  std::vector<std::tuple<double, int, int, int, int>> integrals;
};

inline FCIDump LoadFCIDump(const std::string& filename) {
  FCIDump d;
  std::ifstream in(filename);
  if (!in.is_open()) throw std::runtime_error("Failed to open FCIDUMP file.");
  std::string line, head;
  bool in_header = true;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '!') continue;
    if (in_header) {
      if (line.find("&END") != std::string::npos) {
        in_header = false;
        continue;
      }
      size_t pos = line.find("&FCI");
      if (pos != std::string::npos) line.erase(pos, 4);
      head += line;
    } else {
      std::stringstream ss(line);
      double v = 0.0;
      int i = 0, j = 0, k = 0, l = 0;
      ss >> v >> i >> j >> k >> l;
      d.integrals.emplace_back(v, i, j, k, l);
    }
  }
  std::stringstream hs(head);
  std::string tok;
  while (std::getline(hs, tok, ',')) {
    size_t eq = tok.find('=');
    if (eq == std::string::npos) continue;
    std::string key = tok.substr(0, eq), val = tok.substr(eq + 1);
    auto trim = [](std::string& s) {
      s.erase(0, s.find_first_not_of(" \t"));
      s.erase(s.find_last_not_of(" \t") + 1);
    };
    trim(key);
    trim(val);
    d.header[key] = val;
  }
  return d;
}

inline std::string get_extension(const std::string& path) {
  size_t pos = path.rfind('.');
  if (pos == std::string::npos) return std::string();
  std::string ext = path.substr(pos + 1);
  for (auto& ch : ext) ch = (char)std::tolower((unsigned char)ch);
  while (!ext.empty() && (ext.back() == 0 || ext.back() == ' ')) ext.pop_back();
  return ext;
}

inline std::vector<size_t> from_string(const std::string& s, size_t bit_length, size_t L) {
  std::vector<size_t> r((L + bit_length - 1) / bit_length, 0);
  for (size_t i = 0; i < L; i++)
    if (s[L - 1 - i] == '1') r[i / bit_length] |= (size_t(1) << (i % bit_length));
  return r;
}

inline std::string makestring(const std::vector<size_t>& c, size_t bit_length, size_t L) {
  std::string s;
  for (size_t i = L; i > 0; i--) s += (c[(i - 1) / bit_length] >> ((i - 1) % bit_length)) & 1 ? '1' : '0';
  return s;
}

// numeric order, most significant word first (framework/bit_manipulation.h:26-43)
inline bool bitarray_less(const std::vector<size_t>& a, const std::vector<size_t>& b) {
  for (size_t n = a.size(); n > 0; n--) {
    if (a[n - 1] < b[n - 1]) return true;
    if (a[n - 1] > b[n - 1]) return false;
  }
  return false;
}

inline void sort_bitarray(std::vector<std::vector<size_t>>& a) {
  std::sort(a.begin(), a.end(), bitarray_less);
  a.erase(std::unique(a.begin(), a.end()), a.end());
}

inline std::vector<std::vector<size_t>> DecodeAlphaDets(const std::string& filename, size_t norb) {
  std::ifstream f(filename, std::ios::binary);
  if (!f) throw std::runtime_error("Failed to open file");
  size_t nbytes = (norb + 7) / 8;
  std::vector<std::vector<size_t>> out;
  std::vector<uint8_t> buf(nbytes);
  while (f.read(reinterpret_cast<char*>(buf.data()), nbytes)) {
    std::vector<size_t> bits;
    size_t idx = 0;
    for (size_t byte : buf)
      for (int i = 7; i >= 0; --i) {
        if (8 * nbytes - norb <= idx) bits.push_back((byte >> i) & 1);
        ++idx;
      }
    std::reverse(bits.begin(), bits.end());
    out.push_back(bits);
  }
  return out;
}

// change_bitlength from 1 bit per word to bit_length bits per word
inline std::vector<size_t> pack_bits(const std::vector<size_t>& one_bit_words, size_t bit_length) {
  size_t L = one_bit_words.size();
  std::vector<size_t> r((L + bit_length - 1) / bit_length, 0);
  for (size_t i = 0; i < L; i++)
    if (one_bit_words[i] & 1) r[i / bit_length] |= (size_t(1) << (i % bit_length));
  return r;
}

inline void LoadAlphaDets(const std::string& file, std::vector<std::vector<size_t>>& adet, size_t bit_length,
                          size_t total_bit_length) {
  std::string ext = get_extension(file);
  if (ext == "txt") {
    std::ifstream in(file);
    if (!in.is_open()) throw std::runtime_error("Failed to open alpha det file.");
    std::string line;
    adet.clear();
    while (std::getline(in, line)) adet.push_back(from_string(line, bit_length, total_bit_length));
  } else if (ext == "bin") {
    auto raw = DecodeAlphaDets(file, total_bit_length);
    adet.clear();
    for (auto& r : raw) adet.push_back(pack_bits(r, bit_length));
  }
  sort_bitarray(adet);
}

inline void ShuffleDet(std::vector<std::vector<size_t>>& det, unsigned int seed) {
  if (det.size() <= 1) return;
  std::mt19937 g(seed);
  std::shuffle(det.begin() + 1, det.end(), g);
}

namespace gpu_detail {

inline uint64_t to_u64(const std::vector<size_t>& s, size_t bit_length, int L) {
  uint64_t v = 0;
  for (int i = 0; i < L; i++)
    if ((s[i / bit_length] >> (i % bit_length)) & 1) v |= uint64_t(1) << i;
  return v;
}

struct Integrals {
  int L = 0, N = 0;
  double I0 = 0.0;
  std::vector<double> h1;   // [L*L]
  std::vector<double> eri;  // reference twoInt 8-fold store
};

// SetupIntegrals, chemistry/basic/makeintegrals.h:10-55
inline Integrals setup_integrals(const FCIDump& d) {
  Integrals x;
  for (const auto& [k, v] : d.header) {
    if (k == "NORB") x.L = std::atoi(v.c_str());
    if (k == "NELEC") x.N = std::atoi(v.c_str());
  }
  int L = x.L;
  if (L <= 0) throw std::invalid_argument("FCIDUMP header has no NORB");
  x.h1.assign((size_t)L * L, 0.0);
  size_t B = (size_t)L * (L + 1) / 2;
  x.eri.assign(B * (B + 1) / 2, 0.0);
  auto pair = [](int i, int j) { int a = std::max(i, j), b = std::min(i, j); return (size_t)a * (a + 1) / 2 + b; };
  for (const auto& [v, i, j, k, l] : d.integrals) {
    if (i == 0 && j == 0 && k == 0 && l == 0) {
      x.I0 = v;
    } else if (k == 0 && l == 0) {
      x.h1[(size_t)(i - 1) * L + (j - 1)] = v;
      x.h1[(size_t)(j - 1) * L + (i - 1)] = v;
    } else {
      size_t ij = pair(i - 1, j - 1), kl = pair(k - 1, l - 1);
      size_t a = std::max(ij, kl), b = std::min(ij, kl);
      x.eri[a * (a + 1) / 2 + b] = v;
    }
  }
  return x;
}

struct Ctx {
  sbdgpu_ctx* c = nullptr;
  ~Ctx() { sbdgpu_destroy(c); }
  void check(int rc, const char* what) {
    if (rc != SBDGPU_OK) throw std::runtime_error(std::string(what) + ": " + sbdgpu_last_error(c));
  }
};

inline void check_world_size(const MPI_Comm& comm) {
#ifdef SBD_GPU_HAVE_MPI
  int size = 1;
  MPI_Comm_size(comm, &size);
  if (size != 1) throw std::invalid_argument("sbd::tpb::diag on GPU runs at MPI world size 1");
#else
  (void)comm;
#endif
}

}  // namespace gpu_detail

inline std::string to_padded_string(size_t n, size_t d) {
  std::ostringstream oss;
  oss << std::setw(d) << std::setfill('0') << n;
  return oss.str();
}

// restart.h:20-66 at world size 1 (one file, rank tag 000000)
template <typename ElemT>
void SaveWavefunction(const std::string& file, const std::vector<std::vector<size_t>>& adet,
                      const std::vector<std::vector<size_t>>& bdet, const std::vector<ElemT>& W) {
  size_t det_length = adet[0].size(), ar = adet.size(), br = bdet.size();
  std::ofstream o(file + to_padded_string(0, 6), std::ios::binary);
  o.write(reinterpret_cast<const char*>(&ar), sizeof(size_t));
  o.write(reinterpret_cast<const char*>(&br), sizeof(size_t));
  o.write(reinterpret_cast<const char*>(&det_length), sizeof(size_t));
  for (const auto& s : adet) o.write(reinterpret_cast<const char*>(s.data()), sizeof(size_t) * det_length);
  for (const auto& s : bdet) o.write(reinterpret_cast<const char*>(s.data()), sizeof(size_t) * det_length);
  o.write(reinterpret_cast<const char*>(W.data()), sizeof(ElemT) * ar * br);
}

// restart.h:414-658 at world size 1: map a saved basis onto the current one by
// string lookup, then normalise.
template <typename ElemT>
void LoadWavefunction(const std::string& file, const std::vector<std::vector<size_t>>& adet,
                      const std::vector<std::vector<size_t>>& bdet, std::vector<ElemT>& W) {
  W.assign(adet.size() * bdet.size(), ElemT(0));
  std::ifstream in(file + to_padded_string(0, 6), std::ios::binary);
  if (!in.is_open()) throw std::runtime_error("Failed to open wavefunction file " + file + "000000");
  size_t la = 0, lb = 0, dl = 0;
  in.read(reinterpret_cast<char*>(&la), sizeof(size_t));
  in.read(reinterpret_cast<char*>(&lb), sizeof(size_t));
  in.read(reinterpret_cast<char*>(&dl), sizeof(size_t));
  std::vector<std::vector<size_t>> ld(la, std::vector<size_t>(dl)), lbd(lb, std::vector<size_t>(dl));
  for (auto& s : ld) in.read(reinterpret_cast<char*>(s.data()), sizeof(size_t) * dl);
  for (auto& s : lbd) in.read(reinterpret_cast<char*>(s.data()), sizeof(size_t) * dl);
  std::vector<ElemT> lw(la * lb);
  in.read(reinterpret_cast<char*>(lw.data()), sizeof(ElemT) * la * lb);
  std::map<std::vector<size_t>, size_t> amap, bmap;
  for (size_t i = 0; i < adet.size(); i++) amap.emplace(adet[i], i);
  for (size_t i = 0; i < bdet.size(); i++) bmap.emplace(bdet[i], i);
  std::vector<long long> ai(la, -1), bi(lb, -1);
  for (size_t i = 0; i < la; i++) {
    auto it = amap.find(ld[i]);
    if (it != amap.end()) ai[i] = (long long)it->second;
  }
  for (size_t i = 0; i < lb; i++) {
    auto it = bmap.find(lbd[i]);
    if (it != bmap.end()) bi[i] = (long long)it->second;
  }
  for (size_t i = 0; i < la; i++)
    if (ai[i] >= 0)
      for (size_t j = 0; j < lb; j++)
        if (bi[j] >= 0) W[(size_t)ai[i] * bdet.size() + (size_t)bi[j]] += lw[i * lb + j];
  double nrm = 0.0;
  for (auto x : W) nrm += x * x;
  nrm = std::sqrt(nrm);
  for (auto& x : W) x /= nrm;
}

// rdmat.h:60-97 (cumulative-weight threshold)
inline void CarryOverAlphaDet(const std::vector<double>& D, const std::vector<std::vector<size_t>>& adet,
                              std::vector<std::vector<size_t>>& rdet, double threshold) {
  size_t n = adet.size();
  std::vector<size_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](int i, int j) { return D[i] > D[j]; });
  std::vector<double> S(n);
  double sum = 0.0;
  for (size_t i = 0; i < n; i++) {
    sum += D[idx[i]];
    S[i] = sum;
  }
  size_t imax = (size_t)std::distance(S.begin(), std::upper_bound(S.begin(), S.end(), 1.0 - threshold)) + 1;
  imax = std::min(imax, n);
  rdet.assign(imax, std::vector<size_t>(adet[0].size()));
  for (size_t k = 0; k < imax; k++) rdet[k] = adet[idx[k]];
}

// rdmat.h:99-132 (keep a fixed count)
inline void CarryOverAlphaDet(const std::vector<double>& D, const std::vector<std::vector<size_t>>& adet,
                              size_t kept, std::vector<std::vector<size_t>>& rdet, double& discarded) {
  size_t n = adet.size();
  std::vector<size_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](int i, int j) { return D[i] > D[j]; });
  kept = std::min(kept, n);
  rdet.assign(kept, std::vector<size_t>(adet[0].size()));
  double sum = 0.0;
  for (size_t k = 0; k < kept; k++) {
    rdet[k] = adet[idx[k]];
    sum += D[idx[k]];
  }
  discarded = 1.0 - sum;
}

namespace tpb {

struct SBD {
  int task_comm_size = 1;
  int adet_comm_size = 1;
  int bdet_comm_size = 1;
  int h_comm_size = 1;
  int method = 0;
  int max_it = 1;
  int max_nb = 10;
  double eps = 1.0e-4;
  double max_time = 86400.0;
  int init = 0;
  int do_shuffle = 0;
  int do_rdm = 0;
  double ratio = 0.0;
  double threshold = 0.01;
  size_t bit_length = 20;
  int device = 0;     // added: CUDA device
  int precision = 0;  // added: SBDGPU_FP64
  int restart_keep = 0;  // added: mixed precisions, Ritz vectors kept at a restart (0/1: collapse)
  int restart_prev = 0;  // added: mixed precisions, also keep the previous Ritz vector
};

inline SBD generate_sbd_data(int argc, char* argv[]) {
  SBD d;
  for (int i = 0; i + 1 < argc; i++) {
    std::string a(argv[i]);
    const char* v = argv[i + 1];
    bool hit = true;
    if (a == "--adet_comm_size") d.adet_comm_size = std::atoi(v);
    else if (a == "--bdet_comm_size") d.bdet_comm_size = std::atoi(v);
    else if (a == "--task_comm_size") d.task_comm_size = std::atoi(v);
    else if (a == "--method") d.method = std::atoi(v);
    else if (a == "--iteration") d.max_it = std::atoi(v);
    else if (a == "--block") d.max_nb = std::atoi(v);
    else if (a == "--tolerance") d.eps = std::atof(v);
    else if (a == "--carryover_ratio") d.ratio = std::atof(v);
    else if (a == "--carryover_threshold") d.threshold = std::atof(v);
    else if (a == "--shuffle") d.do_shuffle = std::atoi(v);
    else if (a == "--rdm") d.do_rdm = std::atoi(v);
    else if (a == "--bit_length") d.bit_length = (size_t)std::atoi(v);
    else if (a == "--device") d.device = std::atoi(v);
    else if (a == "--precision") d.precision = std::atoi(v);
    else if (a == "--restart_keep") d.restart_keep = std::atoi(v);
    else if (a == "--restart_prev") d.restart_prev = std::atoi(v);
    else hit = false;
    if (hit) i++;
  }
  return d;
}

inline double elapsed_since(std::chrono::high_resolution_clock::time_point t0) {
  return 1.0e-6 * (double)std::chrono::duration_cast<std::chrono::microseconds>(
                      std::chrono::high_resolution_clock::now() - t0).count();
}

// sbdiag.h:102-456 on one GPU
inline void diag(const MPI_Comm& comm, const SBD& sbd_data, const FCIDump& fcidump,
                 const std::vector<std::vector<size_t>>& adet, const std::vector<std::vector<size_t>>& bdet,
                 const std::string& loadname, const std::string& savename, double& energy,
                 std::vector<double>& density, std::vector<std::vector<size_t>>& carryover_bitstrings,
                 std::vector<std::vector<double>>& one_p_rdm, std::vector<std::vector<double>>& two_p_rdm) {
  gpu_detail::check_world_size(comm);
  if (sbd_data.adet_comm_size * sbd_data.bdet_comm_size * sbd_data.task_comm_size != 1)
    throw std::invalid_argument("MPI Size of twister is not a square of a integer");
  if (adet.empty() || bdet.empty()) throw std::invalid_argument("empty determinant set");
  auto ints = gpu_detail::setup_integrals(fcidump);
  int L = ints.L;
  if (L > 64) throw std::invalid_argument("the GPU path supports norb <= 64");
  size_t bl = sbd_data.bit_length;
  std::vector<uint64_t> a(adet.size()), b(bdet.size());
  for (size_t i = 0; i < adet.size(); i++) a[i] = gpu_detail::to_u64(adet[i], bl, L);
  for (size_t i = 0; i < bdet.size(); i++) b[i] = gpu_detail::to_u64(bdet[i], bl, L);

  gpu_detail::Ctx g;
  auto t_help = std::chrono::high_resolution_clock::now();
  int rc = sbdgpu_create(&g.c, L, a.size(), b.size(), a.data(), b.data(), ints.I0, ints.h1.data(),
                         ints.eri.data(), sbd_data.device);
  if (rc != SBDGPU_OK) throw std::runtime_error("sbdgpu_create failed with status " + std::to_string(rc));
  g.check(sbdgpu_build_tables(g.c), "sbdgpu_build_tables");
  std::cout << " Elapsed time for helper construction " << elapsed_since(t_help) << " (sec) " << std::endl;

  auto t_init = std::chrono::high_resolution_clock::now();
  size_t n = a.size() * b.size();
  std::vector<double> W;
  if (loadname.empty()) {
    W.assign(n, 0.0);
    if (sbd_data.init == 1) {
      std::mt19937 gen((unsigned)std::chrono::high_resolution_clock::now().time_since_epoch().count());
      std::uniform_real_distribution<double> dist(-1, 1);
      double s = 0.0;
      for (auto& x : W) {
        x = dist(gen);
        s += x * x;
      }
      for (auto& x : W) x /= std::sqrt(s);
    } else {
      W[0] = 1.0;  // davidson.h:130-133
    }
  } else {
    LoadWavefunction(loadname, adet, bdet, W);
  }
  std::cout << " Elapsed time for init " << elapsed_since(t_init) << " (sec) " << std::endl;

  auto t_diag = std::chrono::high_resolution_clock::now();
  if (sbd_data.method == 1) {
    // method 1 (sbdiag.h:264-300): store the Hamiltonian, then Davidson on it
    auto t_mkham = std::chrono::high_resolution_clock::now();
    uint64_t nnz = 0;
    g.check(sbdgpu_store_hamiltonian(g.c, &nnz), "sbdgpu_store_hamiltonian");
    std::cout << " Elapsed time for make Hamiltonian " << elapsed_since(t_mkham) << " (sec) " << std::endl;
  } else if (sbd_data.method != 0) {
    std::cout << " method " << sbd_data.method
              << ": the GPU path builds H*C on the fly (method 0); results are the same" << std::endl;
  }
  sbdgpu_opts o{sbd_data.max_it,    sbd_data.max_nb, sbd_data.eps,          sbd_data.max_time,
                sbd_data.precision, 1,               sbd_data.restart_keep, sbd_data.restart_prev,
                SBDGPU_PRECOND_DIAGONAL};
  double e = 0.0;
  int steps = 0;
  auto t_dav = std::chrono::high_resolution_clock::now();
  g.check(sbdgpu_davidson(g.c, &o, W.data(), &e, nullptr, nullptr, 0, &steps), "sbdgpu_davidson");
  std::cout << " Elapsed time for davidson " << elapsed_since(t_dav) << " (sec) " << std::endl;
  std::cout << " Elapsed time for diagonalization " << elapsed_since(t_diag) << " (sec) " << std::endl;
  std::cout.precision(16);
  std::cout << " Energy = " << e << std::endl;
  energy = e;

  auto t_meas = std::chrono::high_resolution_clock::now();
  if (sbd_data.do_rdm == 0) {
    density.assign(2 * L, 0.0);
    g.check(sbdgpu_occupation(g.c, W.data(), density.data()), "sbdgpu_occupation");
  } else {
    size_t L2 = (size_t)L * L, L4 = L2 * L2;
    std::vector<double> one(2 * L2), two(4 * L4);
    g.check(sbdgpu_rdm(g.c, W.data(), one.data(), two.data()), "sbdgpu_rdm");
    one_p_rdm.assign(2, std::vector<double>(L2));
    two_p_rdm.assign(4, std::vector<double>(L4));
    for (int s = 0; s < 2; s++) std::copy(one.begin() + s * L2, one.begin() + (s + 1) * L2, one_p_rdm[s].begin());
    for (int s = 0; s < 4; s++) std::copy(two.begin() + s * L4, two.begin() + (s + 1) * L4, two_p_rdm[s].begin());
    density.assign(2 * L, 0.0);
    for (int io = 0; io < L; io++) {
      density[2 * io] = one_p_rdm[0][io + (size_t)L * io];
      density[2 * io + 1] = one_p_rdm[1][io + (size_t)L * io];
    }
  }
  std::cout << " Elapsed time for measurement " << elapsed_since(t_meas) << " (sec) " << std::endl;

  std::vector<double> D(adet.size());
  g.check(sbdgpu_alpha_weights(g.c, W.data(), D.data()), "sbdgpu_alpha_weights");
  if (sbd_data.ratio == 0.0) {
    CarryOverAlphaDet(D, adet, carryover_bitstrings, sbd_data.threshold);
  } else {
    size_t kept = static_cast<size_t>(sbd_data.ratio * adet.size());
    double tw = 0.0;
    CarryOverAlphaDet(D, adet, kept, carryover_bitstrings, tw);
    std::cout << " truncated weight in carry-over = " << tw << std::endl;
  }
  if (!savename.empty()) SaveWavefunction(savename, adet, bdet, W);
}

// sbdiag.h:472-565
inline void diag(const MPI_Comm& comm, const SBD& sbd_data, const std::string& fcidumpfile,
                 const std::string& adetfile, const std::string& loadname, const std::string& savename,
                 double& energy, std::vector<double>& density, std::vector<std::vector<size_t>>& carryover_bitstrings,
                 std::vector<std::vector<double>>& one_p_rdm, std::vector<std::vector<double>>& two_p_rdm) {
  FCIDump fcidump = LoadFCIDump(fcidumpfile);
  size_t L = 0;
  for (const auto& [k, v] : fcidump.header)
    if (k == "NORB") L = (size_t)std::atoi(v.c_str());
  std::vector<std::vector<size_t>> adet, bdet;
  LoadAlphaDets(adetfile, adet, sbd_data.bit_length, L);
  auto now_seed = [] { return (unsigned)std::chrono::high_resolution_clock::now().time_since_epoch().count(); };
  if (sbd_data.do_shuffle == 0) {
    bdet = adet;
  } else if (sbd_data.do_shuffle == 1) {
    ShuffleDet(adet, now_seed());
    bdet = adet;
  } else if (sbd_data.do_shuffle == 2) {
    bdet = adet;
    ShuffleDet(adet, now_seed());
    ShuffleDet(bdet, now_seed());
  } else if (sbd_data.do_shuffle == 3) {
    ShuffleDet(adet, 42u);
    bdet = adet;
  } else if (sbd_data.do_shuffle == 4) {
    bdet = adet;
    ShuffleDet(adet, 1729u);
    ShuffleDet(bdet, 137u);
  }
  diag(comm, sbd_data, fcidump, adet, bdet, loadname, savename, energy, density, carryover_bitstrings, one_p_rdm,
       two_p_rdm);
}

}  // namespace tpb
}  // namespace sbd

#endif  // SBD_GPU_TPB_H
