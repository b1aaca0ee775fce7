"""The CPU restatement of the generic path (oracle/genop_oracle.py), pinned:

* its NormalOrdering equals the reference's own (the unmodified headers behind
  oracle/ref_generic.cc) on random products, with and without the fermionic
  sign;
* its mult sign rule reproduces an independent Jordan-Wigner construction of
  the same products on the full Fock space;
* its GeneralOp_From_FCIDump equals the reference's term for term, in order,
  when given the integrals the reference ends up with (six significant digits,
  after its text round trip in MpiBcast(FCIDump));
* on the full product basis that operator is the tensor-product-basis
  Hamiltonian of the same integrals (the tpb oracle), up to the diagonal phase
  between the site order alpha-then-beta and the reference's interleaved one;
* the header-only C++ algebra (sbd_b200/include/sbd_gpu/generalop.h) gives the
  oracle's products and coefficients."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from conftest import ROOT
from oracle import genop_oracle as G
from sbd_b200 import synth

needs_ref = pytest.mark.skipif(not os.path.exists(oracle.REF_GENERIC_SO), reason="reference shim not built")


def _canon(H, digits=12):
    return [sorted((tuple(o), round(c, digits)) for c, o in lst) for lst in H]


def _random_product(rng, nsites, max_ops=5):
    n = int(rng.integers(1, max_ops + 1))
    return [(bool(rng.integers(0, 2)), int(rng.integers(0, nsites))) for _ in range(n)]


@needs_ref
@pytest.mark.parametrize("sign", [True, False])
def test_normal_ordering_matches_reference(sign):
    rng = np.random.default_rng(11 if sign else 12)
    for _ in range(200):
        ops = _random_product(rng, 5)
        r = oracle.RefGeneric()
        r.add(1.25, ops)
        r.normal_order(sign)
        assert _canon(r.terms()) == _canon(G.normal_order(([], [(1.25, ops)]), sign)), ops


@needs_ref
def test_operator_sums_and_simplify_match_reference():
    rng = np.random.default_rng(5)
    r = oracle.RefGeneric()
    terms = []
    for _ in range(40):
        ops = _random_product(rng, 4, 4)
        c = float(rng.normal())
        r.add(c, ops)
        terms.append((c, ops))
    r.add(0.75, [])
    r.normal_order(True)
    r.simplify()
    mine = G.simplify(G.normal_order(([(0.75, [])], terms), True))
    got = r.terms()
    for a, b in zip(_canon(got, 10), _canon(mine, 10)):
        assert a == b


def test_sign_rule_matches_jordan_wigner():
    rng = np.random.default_rng(3)
    states = np.arange(32, dtype=np.uint64)  # the full Fock space of 5 sites
    for _ in range(120):
        ops = _random_product(rng, 5, 4)
        c = float(rng.normal())
        Hn = G.normal_order(([], [(c, ops)]), True)
        np.testing.assert_allclose(G.dense(states, Hn), G.jordan_wigner(states, [(c, ops)], 5), atol=1e-13)


def _fcidump(td, L, ne, seed):
    ints = synth.make_integrals(L, seed)
    p = os.path.join(td, "FCIDUMP")
    synth.write_fcidump(p, ints, 2 * ne)
    return ints, p


@needs_ref
def test_from_fcidump_matches_reference():
    with tempfile.TemporaryDirectory() as td:
        ints, p = _fcidump(td, 4, 2, 3)
        r, L, N = oracle.RefGeneric.from_fcidump(p)
        ref = r.terms()
        norb, nelec, il = G.read_fcidump(p)
    assert (L, N) == (norb, nelec) == (4, 4)
    # the reference's integrals after MpiBcast(FCIDump): written and re-read at
    # the stream's default six significant digits (framework/fcidump.h:156-253)
    mine = G.from_fcidump(norb, [(float(f"{v:.6g}"), i, j, k, l) for v, i, j, k, l in il])
    for a, b in zip(ref, mine):
        assert [o for _, o in a] == [o for _, o in b]
        assert max((abs(x - y) for (x, _), (y, _) in zip(a, b)), default=0.0) == 0.0


def test_fcidump_operator_is_the_product_basis_hamiltonian():
    L, ne = 4, 2
    with tempfile.TemporaryDirectory() as td:
        ints, p = _fcidump(td, L, ne, 7)
        norb, nelec, il = G.read_fcidump(p)
    H = G.from_fcidump(norb, il)
    strs = synth.full_strings(L, ne)
    states = np.array([int(a) | (int(b) << L) for a in strs for b in strs], dtype=np.uint64)
    Mg = G.dense(states, H)
    orc = oracle.Oracle(L, strs, strs, ints.ecore, ints.h, ints.eri)
    n = len(states)
    Mt = np.stack([orc.sigma(np.eye(n)[j]) for j in range(n)], axis=1)
    ph = oracle.phase(strs, strs).ravel()
    np.testing.assert_allclose(Mg, ph[:, None] * Mt * ph[None, :], atol=1e-12)


def test_lanczos_oracle_reaches_the_lowest_eigenvalue():
    L, ne = 4, 2
    with tempfile.TemporaryDirectory() as td:
        _, p = _fcidump(td, L, ne, 9)
        norb, _, il = G.read_fcidump(p)
    H = G.from_fcidump(norb, il)
    strs = synth.full_strings(L, ne)
    states = np.array([int(a) | (int(b) << L) for a in strs for b in strs], dtype=np.uint64)
    W0 = np.random.default_rng(1).normal(size=len(states))
    W0 /= np.linalg.norm(W0)
    e, W, steps = G.lanczos(states, H, W0, 60, 1e-12)
    ev = np.linalg.eigvalsh(G.dense(states, H))
    assert abs(e - ev[0]) < 1e-9
    r = G.mult(states, H, W) - e * W
    assert np.linalg.norm(r) < 1e-5 * np.linalg.norm(W)


CPP = r'''
#include <cstdio>
#include <sstream>
#include <string>
#include "sbd/sbd.h"
// stdin: lines "coef n dag site dag site ..."; argv[1] = sign; argv[2] = FCIDUMP (optional)
static void dump(const sbd::GeneralOp<double>& H) {
  for (size_t m = 0; m < H.NumNcTerms(); m++) {
    auto p = H.NcTerm((int)m);
    std::printf("D %.17g %zu", H.NcCoef((int)m), p.size());
    for (size_t k = 0; k < p.size(); k++) std::printf(" %d %d", (int)p.op(k).d(), p.op(k).q());
    std::printf("\n");
  }
  for (size_t m = 0; m < H.NumOpTerms(); m++) {
    auto p = H.OpTerm((int)m);
    std::printf("O %.17g %zu", H.OpCoef((int)m), p.size());
    for (size_t k = 0; k < p.size(); k++) std::printf(" %d %d", (int)p.op(k).d(), p.op(k).q());
    std::printf("\n");
  }
}
int main(int argc, char** argv) {
  if (argc > 2) {
    int L = 0, N = 0;
    sbd::GeneralOp<double> H;
    sbd::GeneralOp_From_FCIDump(argv[2], 0, 0, L, N, H);
    dump(H);
    return 0;
  }
  sbd::GeneralOp<double> H;
  std::string line;
  while (std::getline(std::cin, line)) {
    std::istringstream s(line);
    double c; int n;
    s >> c >> n;
    if (n == 0) { H += c; continue; }
    int d, q;
    s >> d >> q;
    sbd::GeneralOp<double> T = c * sbd::FieldOp(d != 0, q);
    for (int k = 1; k < n; k++) { s >> d >> q; T = T * sbd::FieldOp(d != 0, q); }
    H += T;
  }
  sbd::NormalOrdering(H, std::atoi(argv[1]) != 0);
  sbd::Simplify(H);
  dump(H);
  return 0;
}
'''


def _parse(text):
    H = ([], [])
    for line in text.splitlines():
        t = line.split()
        n = int(t[2])
        ops = [(t[3 + 2 * k] == "1", int(t[4 + 2 * k])) for k in range(n)]
        H[0 if t[0] == "D" else 1].append((float(t[1]), ops))
    return H


@pytest.fixture(scope="module")
def cpp_exe():
    td = tempfile.mkdtemp()
    src, exe = os.path.join(td, "g.cc"), os.path.join(td, "g")
    open(src, "w").write(CPP)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "sbd_b200", "include"), "-I",
                    os.path.join(ROOT, "include"), src, "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("sign", [True, False])
def test_cpp_algebra_matches_oracle(cpp_exe, sign):
    rng = np.random.default_rng(21 if sign else 22)
    terms = [(float(rng.normal()), _random_product(rng, 6, 5)) for _ in range(60)]
    lines = [f"{c!r} {len(o)} " + " ".join(f"{int(d)} {q}" for d, q in o) for c, o in terms] + ["-0.5 0"]
    out = subprocess.run([cpp_exe, "1" if sign else "0"], input="\n".join(lines) + "\n", capture_output=True,
                         text=True, check=True).stdout
    mine = G.simplify(G.normal_order(([(-0.5, [])], terms), sign))
    for a, b in zip(_canon(_parse(out), 10), _canon(mine, 10)):
        assert a == b


def test_cpp_from_fcidump_matches_oracle(cpp_exe):
    with tempfile.TemporaryDirectory() as td:
        _, p = _fcidump(td, 5, 2, 4)
        out = subprocess.run([cpp_exe, "1", p], capture_output=True, text=True, check=True).stdout
        norb, _, il = G.read_fcidump(p)
    got = _parse(out)
    mine = G.from_fcidump(norb, il)
    for a, b in zip(got, mine):
        assert [o for _, o in a] == [o for _, o in b]
        np.testing.assert_allclose([c for c, _ in a], [c for c, _ in b], rtol=0, atol=1e-15)
