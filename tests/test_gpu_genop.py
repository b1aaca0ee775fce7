"""The generic path on the GPU (sbdgpu_genop_*) against its CPU oracle
(oracle/genop_oracle.py) and against the tensor-product-basis path:

* mult (W += H C) and the diagonal on bases of 1, 2 and 4 words (sites across
  word boundaries), with and without the fermionic sign, with targets outside
  the basis, in the caller's (unsorted) state order;
* the quantum-chemistry operator of GeneralOp_From_FCIDump on the full
  alpha x beta product basis equals the tpb sigma up to the diagonal phase
  between the two site orders, and its Lanczos and Davidson energies equal the
  tpb Davidson energy;
* Lanczos takes the oracle's steps to the oracle's Ritz value and vector;
* bad input is refused."""
import itertools
import os
import tempfile

import numpy as np
import pytest

import sbd_b200
from oracle import genop_oracle as G
from oracle import phase
from sbd_b200 import synth

pytestmark = pytest.mark.gpu


def _words(x, nw):
    return [(x >> (64 * w)) & ((1 << 64) - 1) for w in range(nw)]


def _basis(sites, npart, drop, rng, nw):
    states = [sum(1 << s for s in c) for c in itertools.combinations(sites, npart)]
    keep = [s for s in states if rng.random() >= drop]
    rng.shuffle(keep)
    return keep, np.array([_words(x, nw) for x in keep], dtype=np.uint64)


def _operator(rng, sites, n1, n2, sign):
    terms = []
    for _ in range(n1):
        p, q = rng.choice(sites, 2)
        terms.append((float(rng.normal()), [(True, int(p)), (False, int(q))]))
    for _ in range(n2):
        p, q, r, s = rng.choice(sites, 4)
        terms.append((float(rng.normal()) * 0.3, [(True, int(p)), (True, int(q)), (False, int(r)), (False, int(s))]))
    terms.append((0.7, []))
    return G.simplify(G.normal_order(([], terms), sign))


@pytest.mark.parametrize("nw,sites", [
    (1, [0, 3, 5, 9, 12, 20, 33, 47, 50, 63]),
    (2, [1, 17, 40, 62, 63, 64, 65, 90, 101, 127]),
    (4, [2, 60, 63, 64, 127, 128, 150, 191, 192, 255]),
])
@pytest.mark.parametrize("sign", [True, False])
def test_mult_and_diagonal_match_oracle(nw, sites, sign):
    rng = np.random.default_rng(nw * 10 + int(sign))
    ints, states = _basis(sites, 4, 0.15, rng, nw)
    H = _operator(rng, sites, 30, 60, sign)
    C = rng.normal(size=len(ints))
    W0 = rng.normal(size=len(ints))
    g = sbd_b200.GenOp(states, sign=sign)
    g.set_terms(*H)
    got = g.mult(C, W0)
    ref = G.mult(_oracle_states(ints, nw), H, C, W0, sign)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-12 * scale
    dref = np.diag(G.dense(_oracle_states(ints, nw), H, sign))
    assert np.abs(g.diagonal() - dref).max() <= 1e-12 * np.abs(dref).max()
    g.close()


def _oracle_states(ints, nw):
    return np.array([_words(x, nw) for x in ints], dtype=np.uint64)


def _fcidump_op(L, ne, seed):
    ints = synth.make_integrals(L, seed)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "FCIDUMP")
        synth.write_fcidump(p, ints, 2 * ne)
        norb, _, il = G.read_fcidump(p)
    return ints, G.from_fcidump(norb, il)


def test_fcidump_operator_equals_tpb_path():
    import torch
    L, ne = 8, 3
    ints, H = _fcidump_op(L, ne, 5)
    strs = synth.full_strings(L, ne)
    states = np.array([int(a) | (int(b) << L) for a in strs for b in strs], dtype=np.uint64)
    g = sbd_b200.GenOp(states, sign=True)
    g.set_terms(*H)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs)
    C = np.random.default_rng(2).normal(size=len(states))
    ph = phase(strs, strs).ravel()
    s_gen = g.mult(C)
    s_tpb = ph * ctx.sigma(ph * C)
    assert np.abs(s_gen - s_tpb).max() <= 1e-11 * np.abs(s_tpb).max()
    # the device form on torch buffers
    dC = torch.from_numpy(C).cuda()
    dW = torch.zeros_like(dC)
    g.mult_device(dC.data_ptr(), dW.data_ptr())
    torch.cuda.synchronize()
    assert np.abs(dW.cpu().numpy() - s_gen).max() == 0.0
    hii = ph * ph * ctx.hii()
    assert np.abs(g.diagonal() - hii).max() <= 1e-11 * np.abs(hii).max()
    W0 = np.zeros(len(states))
    W0[0] = 1.0
    e_tpb, _, _, _ = ctx.davidson(W0, 200, 10, 1e-9)
    e_d, W_d, te, tt = g.davidson(W0, 200, 10, 1e-9)
    assert abs(e_d - e_tpb) < 1e-10 and tt[-1] < 1e-9
    e_l, W_l, it = g.lanczos(W0, 300, 1e-13)
    assert abs(e_l - e_tpb) < 1e-9
    assert abs(abs(W_l @ W_d) / np.linalg.norm(W_l) - 1.0) < 1e-6
    g.close()
    ctx.close()


def test_set_fcidump_equals_oracle_operator():
    """sbdgpu_genop_set_fcidump (the header's GeneralOp_From_FCIDump, in the
    library) gives the oracle's operator: the same mult and diagonal."""
    L, ne = 6, 2
    ints = synth.make_integrals(L, 13)
    strs = synth.full_strings(L, ne)
    states = np.array([int(a) | (int(b) << L) for a in strs for b in strs], dtype=np.uint64)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "FCIDUMP")
        synth.write_fcidump(p, ints, 2 * ne)
        norb, _, il = G.read_fcidump(p)
        g = sbd_b200.GenOp(states, sign=True)
        assert g.set_fcidump(p) == (L, 2 * ne)
    H = G.from_fcidump(norb, il)
    C = np.random.default_rng(3).normal(size=len(states))
    ref = G.mult(states, H, C)
    assert np.abs(g.mult(C) - ref).max() <= 1e-12 * np.abs(ref).max()
    with pytest.raises(sbd_b200.SbdGpuError):
        g.set_fcidump("/nonexistent/FCIDUMP")
    g.close()


@pytest.mark.parametrize("nw,sites", [(1, [0, 3, 5, 9, 12, 20, 33, 47, 50, 63]),
                                      (2, [1, 17, 40, 62, 63, 64, 65, 90, 101, 127])])
def test_ham_square_and_expand_match_oracle(nw, sites):
    rng = np.random.default_rng(40 + nw)
    ints, states = _basis(sites, 4, 0.6, rng, nw)  # many targets outside the basis
    H = _operator(rng, sites, 30, 60, True)
    W = rng.normal(size=len(ints))
    W /= np.linalg.norm(W)
    g = sbd_b200.GenOp(states, sign=True)
    g.set_terms(*H)
    ost = _oracle_states(ints, nw)
    ref = G.ham_square(ost, H, W)
    assert abs(g.ham_square(W) - ref) <= 1e-12 * ref
    for eps in (0.0, 0.02):
        got = g.expand(W, eps)
        want = G.expand(ost, H, W, eps)
        got_int = [sum(int(x) << (64 * k) for k, x in enumerate(row)) for row in got]
        assert got_int == want
    g.close()


def test_ham_square_on_a_closed_space_is_the_norm_of_hw():
    L, ne = 6, 2
    _, H = _fcidump_op(L, ne, 23)
    strs = synth.full_strings(L, ne)
    states = np.array([int(a) | (int(b) << L) for a in strs for b in strs], dtype=np.uint64)
    g = sbd_b200.GenOp(states, sign=True)
    g.set_terms(*H)
    W = np.random.default_rng(9).normal(size=len(states))
    hw = g.mult(W)
    # the full product space is closed under H: H^2 over the expanded space is |HW|^2
    assert abs(g.ham_square(W) - hw @ hw) <= 1e-11 * (hw @ hw)
    assert len(g.expand(W, 0.0)) == len(states)
    g.close()


def test_lanczos_matches_oracle():
    L, ne = 4, 2
    _, H = _fcidump_op(L, ne, 9)
    strs = synth.full_strings(L, ne)
    states = np.array([int(a) | (int(b) << L) for a in strs for b in strs], dtype=np.uint64)
    W0 = np.random.default_rng(4).normal(size=len(states))
    W0 /= np.linalg.norm(W0)
    g = sbd_b200.GenOp(states, sign=True)
    g.set_terms(*H)
    e, W, it = g.lanczos(W0, 40, 1e-10)
    e_ref, W_ref, it_ref = G.lanczos(states, H, W0, 40, 1e-10)
    assert it == it_ref
    assert abs(e - e_ref) < 1e-10
    assert abs(abs(W @ W_ref) / (np.linalg.norm(W) * np.linalg.norm(W_ref)) - 1.0) < 1e-9
    g.close()


def test_bad_input_is_refused():
    with pytest.raises(sbd_b200.SbdGpuError):
        sbd_b200.GenOp(np.array([3, 5, 3], dtype=np.uint64))  # repeated state
    with pytest.raises(sbd_b200.SbdGpuError):
        sbd_b200.GenOp(np.zeros((4, 3), dtype=np.uint64) + np.arange(4, dtype=np.uint64)[:, None])  # 3 words
    g = sbd_b200.GenOp(np.array([1, 2, 4], dtype=np.uint64))
    with pytest.raises(sbd_b200.SbdGpuError):
        g.mult(np.ones(3))  # no operator yet
    with pytest.raises(sbd_b200.SbdGpuError):
        g.set_terms([], [(1.0, [(True, 64), (False, 0)], 1)])  # site beyond one word
    g.close()


CPP = r"""
#include <cstdio>
#include "sbd/sbd.h"
// argv[1] FCIDUMP, argv[2] norb, argv[3] electrons per spin: full alpha x beta space,
// bit_length 20 (the reference's default word width)
int main(int argc, char** argv) {
  const int L = std::atoi(argv[2]), ne = std::atoi(argv[3]);
  const size_t bl = 20;
  MPI_Comm comm = MPI_COMM_WORLD;
  sbd::GeneralOp<double> H;
  int norb = 0, nelec = 0;
  sbd::GeneralOp_From_FCIDump(argv[1], comm, comm, norb, nelec, H);
  std::vector<std::vector<size_t>> cfg;
  for (uint64_t a = 0; a < (1ull << L); a++) {
    if (__builtin_popcountll(a) != ne) continue;
    for (uint64_t b = 0; b < (1ull << L); b++) {
      if (__builtin_popcountll(b) != ne) continue;
      const uint64_t x = a | (b << L);
      std::vector<size_t> w((2 * L + bl - 1) / bl, 0);
      for (int q = 0; q < 2 * L; q++)
        if ((x >> q) & 1) w[q / bl] |= size_t(1) << (q % bl);
      cfg.push_back(w);
    }
  }
  sbd::Basis B(cfg, comm);
  std::vector<double> W(B.Size(), 0.0);
  W[0] = 1.0;
  sbd::Lanczos(H, B, W, comm, 300, bl, 1, 1e-12, true);
  double nrm = 0;
  for (double x : W) nrm += x * x;
  for (double& x : W) x /= std::sqrt(nrm);
  std::vector<double> HW(B.Size(), 0.0);
  sbd::mult(H, W, B, HW, bl, 1, comm, true);
  double e = 0;
  for (size_t i = 0; i < W.size(); i++) e += W[i] * HW[i];
  double h2 = 0;
  sbd::MeasHamSquare(H, B, W, bl, comm, h2, true);
  sbd::Basis Bn;
  sbd::ExpandBasis(H, B, W, Bn, 0.0, bl, comm, true);
  std::printf("%zu %.15f %.15f %zu\n", B.Size(), e, h2, Bn.Size());
  return 0;
}
"""


def test_cpp_generic_path_on_the_gpu():
    """A program written against the reference's generic API (FCIDUMP ->
    GeneralOp, Basis of 20-bit words, Lanczos, mult, MeasHamSquare,
    ExpandBasis) runs on the GPU through the drop-in header: its energy equals
    the tpb Davidson energy, and at an eigenvector <H^2> = E^2 on the closed
    full space, whose expansion adds nothing."""
    import subprocess
    from conftest import ROOT
    L, ne = 5, 2
    ints = synth.make_integrals(L, 31)
    strs = synth.full_strings(L, ne)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs)
    W0 = np.zeros(ctx.n)
    W0[0] = 1.0
    e_tpb, _, _, _ = ctx.davidson(W0, 200, 10, 1e-10)
    ctx.close()
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "FCIDUMP")
        synth.write_fcidump(p, ints, 2 * ne)
        src, exe = os.path.join(td, "g.cc"), os.path.join(td, "g")
        open(src, "w").write(CPP)
        lib = os.path.join(ROOT, "sbd_b200")
        subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(lib, "include"), "-I",
                        os.path.join(ROOT, "include"), src, "-L", lib, "-lsbdgpu", f"-Wl,-rpath,{lib}", "-o", exe],
                       check=True)
        out = subprocess.run([exe, p, str(L), str(ne)], capture_output=True, text=True, check=True).stdout.split()
    n, e, h2, n_new = int(out[0]), float(out[1]), float(out[2]), int(out[3])
    assert n == len(strs) ** 2 and n_new == n
    assert abs(e - e_tpb) < 1e-9
    assert abs(h2 - e * e) < 1e-7 * e * e
