/*
 * sbd_gpu/generalop.h -- header-only C++ host library: the drop-in for the
 * reference's generic second-quantised path (r-ccs-cms/sbd include/sbd/basic/),
 * with the operator applied and the eigensolvers run on one B200 through the
 * C ABI in sbdgpu.h (sbdgpu_genop_*).
 *
 * Kept from the reference, with the same names and argument meaning:
 *   sbd::FieldOp, ProductOp, GeneralOp<double>   basic/generalop.h:17-826
 *   operator*, +, -, Cr, An, Sp, Sm, Sz, <<      out_of_place_func/arithmetic.h:10-42, 445-528
 *   NormalOrdering (product, operator), Simplify arithmetic.h:43-337
 *   sbd::Basis (one rank)                        basic/basis.h:15-400
 *   GeneralOp_From_FCIDump                       out_of_place_func/stdmodel.h:13-98
 *   mult (W += H C)                              out_of_place_func/mult.h:268-291
 *   Lanczos (operator overload)                  out_of_place_func/lanczos.h:176-310
 *   MeasHamSquare, ExpandBasis                   out_of_place_func/expand.h:10-366
 * and sbd::gpu::Davidson, a Davidson with on-the-fly sigma (an extension: the
 * reference's generic Davidson, out_of_place_func/davidson.h:19-196, runs on a
 * stored Hamiltonian).  One rank: communicators are accepted for signature
 * compatibility.  Element type double.
 *
 * Deliberate differences:
 *   - GeneralOp_From_FCIDump keeps the integrals at full precision.  The
 *     reference passes them through MpiBcast(FCIDump) (framework/fcidump.h:
 *     156-253), which re-reads them from text written at the stream's default
 *     six significant digits.
 *   - The basis search finds every state.  The reference's Basis::IndexSearch
 *     (basis.h:317-322) bisects over [0, target word count) only.
 *   - NormalOrdering reaches the same normal-ordered products and sums as the
 *     reference's by a rewrite of adjacent annihilator-creator pairs; terms may
 *     come out in another order.
 */
#ifndef SBD_GPU_GENERALOP_H
#define SBD_GPU_GENERALOP_H

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <deque>
#include <iostream>
#include <map>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "sbd_gpu/tpb.h"
#include "sbdgpu.h"

namespace sbd {

class FieldOp {
 public:
  FieldOp() : d_(false), q_(0) {}
  FieldOp(bool d, int q) : d_(d), q_(q) {}
  bool operator==(const FieldOp& o) const { return d_ == o.d_ && q_ == o.q_; }
  bool operator!=(const FieldOp& o) const { return !(*this == o); }
  bool operator<(const FieldOp& o) const { return q_ < o.q_; }
  bool operator>(const FieldOp& o) const { return q_ > o.q_; }
  void dagger() { d_ = !d_; }
  bool d() const { return d_; }
  int q() const { return q_; }

 private:
  bool d_;
  int q_;
};

class ProductOp {
 public:
  ProductOp() : n_dag_(0) {}
  ProductOp(const FieldOp& f) : n_dag_(f.d() ? 1 : 0), fops_(1, f) {}
  explicit ProductOp(int n) : n_dag_(0), fops_(n) {}
  bool operator==(const ProductOp& o) const { return fops_ == o.fops_; }
  ProductOp operator*(const ProductOp& o) const {
    ProductOp r(*this);
    r *= o;
    return r;
  }
  ProductOp operator*(const FieldOp& f) const {
    ProductOp r(*this);
    r *= f;
    return r;
  }
  ProductOp& operator*=(const ProductOp& o) {
    for (const auto& f : o.fops_) *this *= f;
    return *this;
  }
  ProductOp& operator*=(const FieldOp& f) {
    fops_.push_back(f);
    if (f.d()) n_dag_++;
    return *this;
  }
  ProductOp extract(int i1, int i2) const {
    ProductOp r;
    for (int i = i1; i < i2; i++) r *= fops_[i];
    return r;
  }
  // as many creators as annihilators, each creator's site also annihilated
  // (generalop.h:288-319)
  bool check_diagonal() const {
    int nc = 0;
    for (const auto& f : fops_) nc += f.d() ? 1 : 0;
    if (2 * nc != (int)fops_.size()) return false;
    for (size_t i = 0; i < fops_.size(); i++) {
      if (!fops_[i].d()) continue;
      bool found = false;
      for (size_t j = 0; j < fops_.size() && !found; j++)
        found = j != i && !fops_[j].d() && fops_[j].q() == fops_[i].q();
      if (!found) return false;
    }
    return true;
  }
  size_t size() const { return fops_.size(); }
  int n_dag() const { return n_dag_; }
  const FieldOp& op(size_t k) const { return fops_[k]; }
  void dagger() {
    std::reverse(fops_.begin(), fops_.end());
    for (auto& f : fops_) f.dagger();
  }
  int max_index() const {
    int m = 0;
    for (const auto& f : fops_) m = std::max(m, f.q());
    return m;
  }

 private:
  int n_dag_;
  std::vector<FieldOp> fops_;
};

inline ProductOp operator*(const FieldOp& a, const FieldOp& b) { return ProductOp(a) * b; }

template <typename ElemT>
class GeneralOp {
 public:
  GeneralOp() = default;
  GeneralOp(const ProductOp& p) : c_(1, ElemT(1.0)), o_(1, p) {}
  GeneralOp(ElemT c, const ProductOp& p) : c_(1, c), o_(1, p) {}

  GeneralOp& operator=(const ProductOp& p) {
    *this = GeneralOp();
    *this += p;
    return *this;
  }
  GeneralOp& operator=(const FieldOp& f) {
    *this = GeneralOp(ProductOp(f));
    return *this;
  }
  GeneralOp operator*(const GeneralOp& o) const {
    // products of the diagonal parts stay diagonal; every other product is
    // filed as off-diagonal (generalop.h:441-481)
    GeneralOp r;
    for (size_t i = 0; i < d_.size(); i++)
      for (size_t j = 0; j < o.d_.size(); j++) {
        r.e_.push_back(e_[i] * o.e_[j]);
        r.d_.push_back(d_[i] * o.d_[j]);
      }
    for (size_t i = 0; i < d_.size(); i++)
      for (size_t j = 0; j < o.o_.size(); j++) {
        r.c_.push_back(e_[i] * o.c_[j]);
        r.o_.push_back(d_[i] * o.o_[j]);
      }
    for (size_t i = 0; i < o_.size(); i++)
      for (size_t j = 0; j < o.d_.size(); j++) {
        r.c_.push_back(c_[i] * o.e_[j]);
        r.o_.push_back(o_[i] * o.d_[j]);
      }
    for (size_t i = 0; i < o_.size(); i++)
      for (size_t j = 0; j < o.o_.size(); j++) {
        r.c_.push_back(c_[i] * o.c_[j]);
        r.o_.push_back(o_[i] * o.o_[j]);
      }
    return r;
  }
  GeneralOp operator*(const ProductOp& p) const {
    GeneralOp r;
    const bool diag = p.check_diagonal();
    for (size_t i = 0; i < d_.size(); i++) {
      (diag ? r.d_ : r.o_).push_back(d_[i] * p);
      (diag ? r.e_ : r.c_).push_back(e_[i]);
    }
    for (size_t i = 0; i < o_.size(); i++) {
      r.o_.push_back(o_[i] * p);
      r.c_.push_back(c_[i]);
    }
    return r;
  }
  GeneralOp operator*(const FieldOp& f) const {
    GeneralOp r;
    for (size_t i = 0; i < d_.size(); i++) {
      r.o_.push_back(d_[i] * f);
      r.c_.push_back(e_[i]);
    }
    for (size_t i = 0; i < o_.size(); i++) {
      r.o_.push_back(o_[i] * f);
      r.c_.push_back(c_[i]);
    }
    return r;
  }
  GeneralOp& operator*=(const GeneralOp& o) { return *this = *this * o; }
  GeneralOp& operator*=(const ProductOp& p) { return *this = *this * p; }
  GeneralOp& operator*=(const FieldOp& f) { return *this = *this * f; }
  GeneralOp& operator*=(ElemT c) {
    for (auto& x : e_) x *= c;
    for (auto& x : c_) x *= c;
    return *this;
  }
  GeneralOp& operator+=(const GeneralOp& o) {
    d_.insert(d_.end(), o.d_.begin(), o.d_.end());
    e_.insert(e_.end(), o.e_.begin(), o.e_.end());
    o_.insert(o_.end(), o.o_.begin(), o.o_.end());
    c_.insert(c_.end(), o.c_.begin(), o.c_.end());
    return *this;
  }
  GeneralOp& operator+=(const ProductOp& p) { return add(p, ElemT(1.0)); }
  GeneralOp& operator+=(const FieldOp& f) { return add(ProductOp(f), ElemT(1.0)); }
  GeneralOp& operator+=(ElemT c) {
    d_.push_back(ProductOp());
    e_.push_back(c);
    return *this;
  }
  GeneralOp& operator-=(const GeneralOp& o) {
    GeneralOp m(o);
    m *= ElemT(-1.0);
    return *this += m;
  }
  GeneralOp& operator-=(const ProductOp& p) { return add(p, ElemT(-1.0)); }
  GeneralOp& operator-=(const FieldOp& f) { return add(ProductOp(f), ElemT(-1.0)); }
  GeneralOp& operator-=(ElemT c) { return *this += -c; }
  GeneralOp operator+(const GeneralOp& o) const {
    GeneralOp r(*this);
    return r += o;
  }
  GeneralOp operator+(const ProductOp& p) const {
    GeneralOp r(*this);
    return r += p;
  }
  GeneralOp operator+(const FieldOp& f) const {
    GeneralOp r(*this);
    return r += f;
  }
  GeneralOp operator+(ElemT c) const {
    GeneralOp r(*this);
    return r += c;
  }
  void dagger() {
    for (auto& p : o_) p.dagger();
  }
  size_t size() const { return d_.size() + o_.size(); }
  int num_terms() const { return (int)size(); }
  ProductOp& NcTerm(int i) { return d_[i]; }
  ProductOp NcTerm(int i) const { return d_[i]; }
  ElemT& NcCoef(int i) { return e_[i]; }
  ElemT NcCoef(int i) const { return e_[i]; }
  size_t NumNcTerms() const { return d_.size(); }
  ProductOp& OpTerm(int i) { return o_[i]; }
  ProductOp OpTerm(int i) const { return o_[i]; }
  ElemT& OpCoef(int i) { return c_[i]; }
  ElemT OpCoef(int i) const { return c_[i]; }
  size_t NumOpTerms() const { return o_.size(); }
  int max_index() const {
    int m = 0;
    for (const auto& p : d_) m = std::max(m, p.max_index());
    for (const auto& p : o_) m = std::max(m, p.max_index());
    return m;
  }
  // appends to the diagonal or the off-diagonal list
  void push_diag(const ProductOp& p, ElemT c) {
    d_.push_back(p);
    e_.push_back(c);
  }
  void push_off(const ProductOp& p, ElemT c) {
    o_.push_back(p);
    c_.push_back(c);
  }

 private:
  GeneralOp& add(const ProductOp& p, ElemT c) {
    if (p.check_diagonal())
      push_diag(p, c);
    else
      push_off(p, c);
    return *this;
  }
  std::vector<ElemT> e_, c_;
  std::vector<ProductOp> d_, o_;
};

template <typename ElemT>
GeneralOp<ElemT> operator*(ElemT c, const FieldOp& a) {
  return GeneralOp<ElemT>(c, ProductOp(a));
}
template <typename ElemT>
GeneralOp<ElemT> operator*(ElemT c, const GeneralOp<ElemT>& G) {
  GeneralOp<ElemT> r(G);
  return r *= c;
}
template <typename ElemT>
GeneralOp<ElemT> operator*(const ProductOp& P, ElemT c) {
  return GeneralOp<ElemT>(c, P);
}
template <typename ElemT>
GeneralOp<ElemT> operator+(const ProductOp& P, const GeneralOp<ElemT>& G) {
  GeneralOp<ElemT> r(P);
  return r += G;
}
template <typename ElemT>
GeneralOp<ElemT> operator-(const ProductOp& P, const GeneralOp<ElemT>& G) {
  GeneralOp<ElemT> r(P);
  return r -= G;
}

inline FieldOp Cr(int q) { return FieldOp(true, q); }
inline FieldOp An(int q) { return FieldOp(false, q); }
inline FieldOp Sp(int q) { return FieldOp(true, q); }
inline FieldOp Sm(int q) { return FieldOp(false, q); }
template <typename ElemT>
GeneralOp<ElemT> Sz(int q) {
  GeneralOp<ElemT> r;
  r += Sp(q) * Sm(q);
  r += ElemT(-0.5);
  return r;
}

// Normal order of one product: every annihilator directly followed by a
// creator is rewritten as c_x c+_y = delta_xy + s c+_y c_x (s = -1 with sign,
// +1 without) until none is left; the creators are then ordered by ascending
// site and the annihilators by descending site (s per transposition);
// products that repeat a site among their creators or among their
// annihilators vanish; equal products are summed and sums of magnitude
// <= 1e-8 dropped; each product is filed as diagonal or off-diagonal.
template <typename ElemT>
void NormalOrdering(const ProductOp& P, GeneralOp<ElemT>& G, bool sign) {
  const double s = sign ? -1.0 : 1.0;
  using Ops = std::vector<FieldOp>;
  std::deque<std::pair<double, Ops>> work;
  Ops first;
  for (size_t k = 0; k < P.size(); k++) first.push_back(P.op(k));
  work.emplace_back(1.0, first);
  std::vector<std::pair<double, Ops>> ordered;
  while (!work.empty()) {
    auto [c, o] = work.front();
    work.pop_front();
    size_t k = 0;
    while (k + 1 < o.size() && !(!o[k].d() && o[k + 1].d())) k++;
    if (k + 1 >= o.size()) {
      ordered.emplace_back(c, o);
      continue;
    }
    Ops sw(o);
    std::swap(sw[k], sw[k + 1]);
    work.emplace_back(c * s, sw);
    if (o[k].q() == o[k + 1].q()) {
      Ops con;
      for (size_t j = 0; j < o.size(); j++)
        if (j != k && j != k + 1) con.push_back(o[j]);
      work.emplace_back(c, con);
    }
  }
  std::vector<Ops> keys;
  std::vector<double> sums;
  for (auto& [c, o] : ordered) {
    Ops cr, an;
    for (const auto& f : o) (f.d() ? cr : an).push_back(f);
    double cc = c;
    // insertion sort counting transpositions: creators ascending, annihilators descending
    auto sort_count = [&](Ops& v, bool ascending) {
      int swaps = 0;
      for (size_t i = 1; i < v.size(); i++)
        for (size_t j = i; j > 0; j--) {
          const bool out = ascending ? v[j].q() < v[j - 1].q() : v[j].q() > v[j - 1].q();
          if (!out) break;
          std::swap(v[j], v[j - 1]);
          swaps++;
        }
      return swaps;
    };
    const int nsw = sort_count(cr, true) + sort_count(an, false);
    bool repeat = false;
    for (size_t i = 1; i < cr.size(); i++) repeat |= cr[i].q() == cr[i - 1].q();
    for (size_t i = 1; i < an.size(); i++) repeat |= an[i].q() == an[i - 1].q();
    if (repeat) continue;
    if (sign && (nsw & 1)) cc = -cc;
    Ops key(cr);
    key.insert(key.end(), an.begin(), an.end());
    auto it = std::find(keys.begin(), keys.end(), key);
    if (it == keys.end()) {
      keys.push_back(key);
      sums.push_back(cc);
    } else {
      sums[it - keys.begin()] += cc;
    }
  }
  GeneralOp<ElemT> r;
  for (size_t m = 0; m < keys.size(); m++) {
    if (std::abs(sums[m]) <= 1.0e-8) continue;
    ProductOp p;
    for (const auto& f : keys[m]) p *= f;
    if (p.check_diagonal())
      r.push_diag(p, ElemT(sums[m]));
    else
      r.push_off(p, ElemT(sums[m]));
  }
  G = r;
}

// every term of both lists normal-ordered in turn and scaled by its
// coefficient, with no summation across terms (arithmetic.h:247-287)
template <typename ElemT>
void NormalOrdering(GeneralOp<ElemT>& G, bool sign) {
  GeneralOp<ElemT> r;
  auto one = [&](const ProductOp& p, ElemT c) {
    GeneralOp<ElemT> g;
    NormalOrdering(p, g, sign);
    for (size_t k = 0; k < g.NumNcTerms(); k++) r.push_diag(g.NcTerm((int)k), c * g.NcCoef((int)k));
    for (size_t k = 0; k < g.NumOpTerms(); k++) r.push_off(g.OpTerm((int)k), c * g.OpCoef((int)k));
  };
  for (size_t m = 0; m < G.NumNcTerms(); m++) one(G.NcTerm((int)m), G.NcCoef((int)m));
  for (size_t m = 0; m < G.NumOpTerms(); m++) one(G.OpTerm((int)m), G.OpCoef((int)m));
  G = r;
}

// equal products summed within each list, sums of magnitude <= 1e-8 dropped
// (arithmetic.h:288-337)
template <typename ElemT>
void Simplify(GeneralOp<ElemT>& G) {
  GeneralOp<ElemT> r;
  for (int list = 0; list < 2; list++) {
    const size_t n = list == 0 ? G.NumNcTerms() : G.NumOpTerms();
    std::vector<ProductOp> keys;
    std::vector<ElemT> sums;
    for (size_t m = 0; m < n; m++) {
      const ProductOp p = list == 0 ? G.NcTerm((int)m) : G.OpTerm((int)m);
      const ElemT c = list == 0 ? G.NcCoef((int)m) : G.OpCoef((int)m);
      auto it = std::find(keys.begin(), keys.end(), p);
      if (it == keys.end()) {
        keys.push_back(p);
        sums.push_back(c);
      } else {
        sums[it - keys.begin()] += c;
      }
    }
    for (size_t m = 0; m < keys.size(); m++) {
      if (std::abs(sums[m]) <= 1.0e-8) continue;
      if (list == 0)
        r.push_diag(keys[m], sums[m]);
      else
        r.push_off(keys[m], sums[m]);
    }
  }
  G = r;
}

inline std::ostream& operator<<(std::ostream& s, const FieldOp& f) {
  return s << (f.d() ? "Adag(" : "A(") << f.q() << ")";
}
inline std::ostream& operator<<(std::ostream& s, const ProductOp& p) {
  for (size_t k = 0; k < p.size(); k++) s << p.op(k);
  return s;
}
template <typename ElemT>
std::ostream& operator<<(std::ostream& s, const GeneralOp<ElemT>& g) {
  bool first = true;
  auto line = [&](ElemT c, const ProductOp& p) {
    s << (first ? "   " : "\n + ") << c << p << " (# of creation " << p.n_dag() << ")";
    first = false;
  };
  for (size_t m = 0; m < g.NumNcTerms(); m++) line(g.NcCoef((int)m), g.NcTerm((int)m));
  for (size_t m = 0; m < g.NumOpTerms(); m++) line(g.OpCoef((int)m), g.OpTerm((int)m));
  if (!first)
    s << "\n # of diag. ops, # of off-diag. ops = " << g.NumNcTerms() << "(" << g.NumNcTerms() << "), "
      << g.NumOpTerms() << "(" << g.NumOpTerms() << ")" << std::endl;
  return s;
}

// The basis of one rank: configurations of bit_length-bit words, sorted and
// deduplicated by Init unless do_reordering is false.
class Basis {
 public:
  Basis() = default;
  Basis(const std::vector<std::vector<size_t>>& config, MPI_Comm comm, bool do_reordering = true) {
    Init(config, comm, do_reordering);
  }
  void Init(const std::vector<std::vector<size_t>>& config, MPI_Comm comm, bool do_reordering = true) {
    config_ = config;
    comm_ = comm;
    if (do_reordering) {
      std::sort(config_.begin(), config_.end());
      config_.erase(std::unique(config_.begin(), config_.end()), config_.end());
    }
  }
  MPI_Comm MpiComm() const { return comm_; }
  int MpiRank() const { return 0; }
  int MpiSize() const { return 1; }
  std::vector<std::vector<size_t>> Config() const { return config_; }
  std::vector<size_t> Config(size_t i) const { return config_[i]; }
  size_t Size() const { return config_.size(); }
  size_t BeginIndex() const { return 0; }
  size_t BeginIndex(int) const { return 0; }
  size_t EndIndex() const { return config_.size(); }
  size_t EndIndex(int) const { return config_.size(); }
  void IndexSearch(const std::vector<size_t>& v, size_t& index, bool& exist) const {
    auto it = std::lower_bound(config_.begin(), config_.end(), v);
    index = (size_t)(it - config_.begin());
    exist = it != config_.end() && *it == v;
  }

 private:
  std::vector<std::vector<size_t>> config_;
  MPI_Comm comm_ = MPI_COMM_WORLD;
};

// The quantum-chemistry Hamiltonian on 2L sites (alpha orbital p at site p,
// beta at site p + L), stdmodel.h:13-98
template <typename ElemT>
void GeneralOp_From_FCIDump(const std::string& filename, MPI_Comm, MPI_Comm, int& L, int& N, GeneralOp<ElemT>& H) {
  FCIDump fcidump = LoadFCIDump(filename);
  for (const auto& [key, value] : fcidump.header) {
    if (key == "NORB") L = std::atoi(value.c_str());
    if (key == "NELEC") N = std::atoi(value.c_str());
  }
  H = GeneralOp<ElemT>();
  for (const auto& [value, i, j, k, l] : fcidump.integrals) {
    if (i == 0 && j == 0 && k == 0 && l == 0) {
      H += ElemT(value);
    } else if (k == 0 && l == 0) {
      std::vector<std::vector<int>> index = {{i, j}, {j, i}};
      std::sort(index.begin(), index.end());
      index.erase(std::unique(index.begin(), index.end()), index.end());
      GeneralOp<ElemT> T;
      for (const auto& p : index) {
        T += ElemT(value) * Cr(p[0] - 1) * An(p[1] - 1);
        T += ElemT(value) * Cr(p[0] - 1 + L) * An(p[1] - 1 + L);
      }
      NormalOrdering(T, true);
      Simplify(T);
      H += T;
    } else {
      std::vector<std::vector<int>> index = {{i, j, k, l}, {j, i, k, l}, {i, j, l, k}, {j, i, l, k},
                                             {k, l, i, j}, {k, l, j, i}, {l, k, i, j}, {l, k, j, i}};
      std::sort(index.begin(), index.end());
      index.erase(std::unique(index.begin(), index.end()), index.end());
      GeneralOp<ElemT> V;
      const ElemT h = ElemT(0.5 * value);
      for (const auto& p : index) {
        V += h * Cr(p[0] - 1) * Cr(p[2] - 1) * An(p[3] - 1) * An(p[1] - 1);
        V += h * Cr(p[0] - 1) * Cr(p[2] - 1 + L) * An(p[3] - 1 + L) * An(p[1] - 1);
        V += h * Cr(p[0] - 1 + L) * Cr(p[2] - 1) * An(p[3] - 1) * An(p[1] - 1 + L);
        V += h * Cr(p[0] - 1 + L) * Cr(p[2] - 1 + L) * An(p[3] - 1 + L) * An(p[1] - 1 + L);
      }
      NormalOrdering(V, true);
      Simplify(V);
      H += V;
    }
  }
}

namespace gpu {

// Hand both lists of H to a device operator (sbdgpu_genop_set_terms): each
// field operator as site | dag << 16, in the order written.
inline int set_terms(sbdgpu_genop* g, const GeneralOp<double>& H) {
  std::vector<int64_t> doff{0}, ooff{0};
  std::vector<int32_t> dops, dnd, oops, ond;
  std::vector<double> dc, oc;
  auto flat = [](const ProductOp& p, std::vector<int64_t>& off, std::vector<int32_t>& ops, std::vector<int32_t>& nd) {
    for (size_t k = 0; k < p.size(); k++) ops.push_back(p.op(k).q() | (p.op(k).d() ? 0x10000 : 0));
    off.push_back((int64_t)ops.size());
    nd.push_back(p.n_dag());
  };
  for (size_t m = 0; m < H.NumNcTerms(); m++) {
    flat(H.NcTerm((int)m), doff, dops, dnd);
    dc.push_back(H.NcCoef((int)m));
  }
  for (size_t m = 0; m < H.NumOpTerms(); m++) {
    flat(H.OpTerm((int)m), ooff, oops, ond);
    oc.push_back(H.OpCoef((int)m));
  }
  return sbdgpu_genop_set_terms(g, dc.size(), doff.data(), dops.data(), dnd.data(), dc.data(), oc.size(), ooff.data(),
                                oops.data(), ond.data(), oc.data());
}

// The operator and basis on the GPU (sbdgpu_genop): build once, apply many times.
class DeviceOp {
 public:
  DeviceOp(const GeneralOp<double>& H, const Basis& B, size_t bit_length, bool sign, int device = 0) {
    if (B.Size() == 0) throw std::runtime_error("empty basis");
    const size_t words_in = B.Config(0).size();
    const size_t sites = words_in * bit_length;
    nw_ = sites <= 64 ? 1 : sites <= 128 ? 2 : sites <= 256 ? 4 : 0;
    if (nw_ == 0) throw std::runtime_error("more than 256 sites");
    std::vector<uint64_t> st(B.Size() * nw_, 0);
    for (size_t i = 0; i < B.Size(); i++) {
      const std::vector<size_t> c = B.Config(i);
      for (size_t r = 0; r < c.size(); r++)
        for (size_t x = 0; x < bit_length; x++)
          if ((c[r] >> x) & 1) {
            const size_t q = r * bit_length + x;
            st[i * nw_ + q / 64] |= 1ull << (q % 64);
          }
    }
    check(sbdgpu_genop_create(&g_, device, nw_, B.Size(), st.data(), sign ? 1 : 0), "sbdgpu_genop_create");
    check(set_terms(g_, H), "sbdgpu_genop_set_terms");
  }
  ~DeviceOp() { sbdgpu_genop_destroy(g_); }
  DeviceOp(const DeviceOp&) = delete;
  DeviceOp& operator=(const DeviceOp&) = delete;

  // W += H C
  void mult(const std::vector<double>& C, std::vector<double>& W) {
    check(sbdgpu_genop_mult(g_, C.data(), W.data()), "sbdgpu_genop_mult");
  }
  double lanczos(std::vector<double>& W, int max_it, double eps, int* n_iter = nullptr) {
    double e = 0.0;
    check(sbdgpu_genop_lanczos(g_, W.data(), max_it, eps, &e, n_iter), "sbdgpu_genop_lanczos");
    return e;
  }
  // <W|H^2|W> over the expanded space (MeasHamSquare)
  double ham_square(const std::vector<double>& W) {
    double r = 0.0;
    check(sbdgpu_genop_ham_square(g_, W.data(), &r), "sbdgpu_genop_ham_square");
    return r;
  }
  // the expanded basis (ExpandBasis) as configurations of bit_length-bit words
  std::vector<std::vector<size_t>> expand(const std::vector<double>& W, double eps_hb, size_t bit_length,
                                          size_t words_out) {
    size_t m = 0;
    check(sbdgpu_genop_expand(g_, W.data(), eps_hb, nullptr, 0, &m), "sbdgpu_genop_expand");
    std::vector<uint64_t> st(m * nw_);
    check(sbdgpu_genop_expand(g_, W.data(), eps_hb, st.data(), m, &m), "sbdgpu_genop_expand");
    std::vector<std::vector<size_t>> out(m, std::vector<size_t>(words_out, 0));
    for (size_t i = 0; i < m; i++)
      for (size_t q = 0; q < words_out * bit_length && q < 64 * (size_t)nw_; q++)
        if ((st[i * nw_ + q / 64] >> (q % 64)) & 1ull) out[i][q / bit_length] |= size_t(1) << (q % bit_length);
    return out;
  }
  double davidson(std::vector<double>& W, int max_it, int max_nb, double eps, bool verbose = false) {
    sbdgpu_opts o{};
    o.max_it = max_it;
    o.max_nb = max_nb;
    o.eps = eps;
    o.max_time = 1e30;
    o.verbose = verbose ? 1 : 0;
    double e = 0.0;
    check(sbdgpu_genop_davidson(g_, &o, W.data(), &e, nullptr, nullptr, 0, nullptr), "sbdgpu_genop_davidson");
    return e;
  }

 private:
  void check(int rc, const char* what) {
    if (rc != SBDGPU_OK)
      throw std::runtime_error(std::string(what) + ": " + (g_ ? sbdgpu_genop_last_error(g_) : "failed") +
                               " (status " + std::to_string(rc) + ")");
  }
  sbdgpu_genop* g_ = nullptr;
  int nw_ = 1;
};

// Davidson for the lowest eigenvalue with on-the-fly sigma (an extension)
template <typename ElemT, typename RealT>
ElemT Davidson(const GeneralOp<ElemT>& H, const Basis& B, std::vector<ElemT>& W, int max_iteration, int num_block,
               size_t bit_length, RealT eps, bool sign) {
  DeviceOp op(H, B, bit_length, sign);
  return op.davidson(W, max_iteration, num_block, eps);
}

}  // namespace gpu

// W += H C on one GPU (one rank: h_comm and data_width are not used)
template <typename ElemT>
void mult(const GeneralOp<ElemT>& H, const std::vector<ElemT>& C, const Basis& B, std::vector<ElemT>& W,
          size_t bit_length, int /*data_width*/, MPI_Comm /*h_comm*/, bool sign) {
  static_assert(std::is_same<ElemT, double>::value, "the B200 generic path runs in double");
  gpu::DeviceOp op(H, B, bit_length, sign);
  op.mult(C, W);
}

// <W|H^2|W> over every configuration H reaches from the basis
// (expand.h:10-215), on one GPU
template <typename ElemT>
void MeasHamSquare(const GeneralOp<ElemT>& H, const Basis& B, const std::vector<ElemT>& W, size_t bit_length,
                   MPI_Comm& /*comm*/, ElemT& res, bool sign) {
  static_assert(std::is_same<ElemT, double>::value, "the B200 generic path runs in double");
  gpu::DeviceOp op(H, B, bit_length, sign);
  res = op.ham_square(W);
}

// The basis plus every configuration an off-diagonal term reaches from basis
// state i with |coef * sign * W_i| > eps_hb (expand.h:217-366), on one GPU
template <typename ElemT, typename RealT>
void ExpandBasis(const GeneralOp<ElemT>& H, const Basis& B, const std::vector<ElemT>& W, Basis& Bnew, RealT eps_hb,
                 size_t bit_length, MPI_Comm& comm, bool sign) {
  static_assert(std::is_same<ElemT, double>::value, "the B200 generic path runs in double");
  gpu::DeviceOp op(H, B, bit_length, sign);
  Bnew.Init(op.expand(W, (double)eps_hb, bit_length, B.Config(0).size()), comm, true);
}

// Lanczos for the lowest eigenvalue (lanczos.h:176-310): W is the start
// vector on entry and the Ritz vector on return.
template <typename ElemT, typename RealT>
void Lanczos(const GeneralOp<ElemT>& H, const Basis& B, std::vector<ElemT>& W, MPI_Comm& /*h_comm*/,
             int max_iteration, size_t bit_length, int /*data_width*/, RealT eps, bool sign) {
  static_assert(std::is_same<ElemT, double>::value, "the B200 generic path runs in double");
  gpu::DeviceOp op(H, B, bit_length, sign);
  op.lanczos(W, max_iteration, (double)eps);
}

}  // namespace sbd

#endif  // SBD_GPU_GENERALOP_H
