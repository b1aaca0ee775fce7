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
