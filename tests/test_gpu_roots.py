"""Block Davidson for several roots (sbdgpu_davidson_roots) on the GPU.

The reference follows the lowest root only, so the oracle for the higher
roots is the dense eigendecomposition of the C restatement's Hamiltonian
(bit-identical to the reference's sigma), built column by column on a basis
small enough for numpy; the lowest root is also checked against the
reference's own Davidson energy."""
import numpy as np
import pytest

import oracle
import sbd_b200
from conftest import load_golden
from test_gpu_parity import _seeded_system, gpu_ctx

pytestmark = pytest.mark.gpu


def _dense_oracle(norb, ints, a, b):
    orc = oracle.Oracle(norb, a, b, ints.ecore, ints.h, ints.eri)
    n = len(a) * len(b)
    H = np.zeros((n, n))
    e = np.zeros(n)
    for j in range(n):
        e[j] = 1.0
        H[:, j] = orc.sigma(e)
        e[j] = 0.0
    return orc, H


@pytest.mark.parametrize("norb,ne,count,seed,ragged", [(8, 3, 30, 21, False), (9, 3, 26, 22, True)])
def test_eight_roots_vs_dense_oracle(norb, ne, count, seed, ragged):
    ints, a, b = _seeded_system(norb, ne, count, seed, ragged)
    orc, H = _dense_oracle(norb, ints, a, b)
    lam = np.linalg.eigvalsh(H)
    ctx = sbd_b200.context_from_integrals(ints, a, b)
    E, W, r, it, ns = ctx.davidson_roots(8, 300, 24, 1e-6)
    assert np.all(r < 1e-6)
    assert np.abs(E - lam[:8]).max() < 1e-9
    # Ritz vectors in the reference convention: orthonormal eigenvectors of the oracle's H
    assert np.abs(W @ W.T - np.eye(8)).max() < 1e-9
    for k in range(8):
        assert np.linalg.norm(orc.sigma(W[k]) - E[k] * W[k]) < 2e-6
    assert ns >= 8 and it >= 1


def test_lowest_root_matches_reference():
    g = load_golden("g_L8_3e_full")
    ctx = gpu_ctx(g)
    E1, W1, r1, _, _ = ctx.davidson_roots(1, 300, 10, 1e-8)
    assert abs(E1[0] - float(g["energy"])) < 1e-10
    assert abs(abs(np.dot(W1[0], g["W"])) - 1.0) < 1e-10
    E4, W4, r4, _, _ = ctx.davidson_roots(4, 300, 16, 1e-7)
    assert abs(E4[0] - float(g["energy"])) < 1e-10
    assert np.all(np.diff(E4) > 0)
    # restart from converged vectors: done at once
    E5, _, r5, it5, ns5 = ctx.davidson_roots(4, 300, 16, 1e-6, W0=W4)
    assert it5 == 1 and ns5 == 4
    assert np.abs(E5 - E4).max() < 1e-10


def test_invalid_arguments():
    g = load_golden("g_L8_3e_full")
    ctx = gpu_ctx(g)
    with pytest.raises(sbd_b200.SbdGpuError, match="nroots"):
        ctx.davidson_roots(0, 10, 10, 1e-6)
    with pytest.raises(sbd_b200.SbdGpuError, match="max_nb"):
        ctx.davidson_roots(8, 10, 12, 1e-6)
    with pytest.raises(sbd_b200.SbdGpuError, match="max_nb"):
        ctx.davidson_roots(2, 10, 40, 1e-6)
