"""Many independent problems in one sbdgpu_davidson_batch call (the
device-resident Davidson with replayed step graphs): the same energies, ground
states and step counts as running each problem alone (and the reference's
energy on its own fixture); the mixed-precision form runs each problem in
turn.  The alpha-beta launch shapes (sbdgpu_set_tuning, sbdgpu_autotune) give
the default sigma."""
import numpy as np
import pytest

import sbd_b200
from conftest import load_golden
from test_gpu_parity import _seeded_system, gpu_ctx

pytestmark = pytest.mark.gpu

CASES = [(8, 3, None, 1, False), (9, 3, 40, 2, False), (10, 3, 50, 3, True), (10, 4, 60, 4, False),
         (11, 3, 70, 5, True), (12, 4, 80, 6, False)]


def _contexts():
    ctxs = []
    for norb, ne, count, seed, ragged in CASES:
        ints, a, b = _seeded_system(norb, ne, count, seed, ragged)
        ctxs.append(sbd_b200.context_from_integrals(ints, a, b))
    g = load_golden("g_L8_3e_full")
    ctxs.append(gpu_ctx(g))
    return ctxs, g


def _unit(n):
    w = np.zeros(n)
    w[0] = 1.0
    return w


@pytest.mark.parametrize("threads", [0, 2])
def test_batch_matches_single_runs(threads):
    ctxs, g = _contexts()
    E, Ws, steps = sbd_b200.davidson_batch(ctxs, [_unit(c.n) for c in ctxs], 300, 10, 1e-8, max_threads=threads)
    for c, e, w in zip(ctxs, E, Ws):
        e1, w1, te, tt = c.davidson(_unit(c.n), 300, 10, 1e-8)
        assert abs(e - e1) < 1e-10
        assert abs(abs(np.dot(w, w1)) - 1.0) < 1e-8
    assert abs(E[-1] - float(g["energy"])) < 1e-10
    assert all(s > 0 for s in steps)


def test_batch_rejects_a_context_given_twice():
    g = load_golden("g_L8_3e_full")
    c = gpu_ctx(g)
    with pytest.raises(sbd_b200.SbdGpuError, match="twice"):
        sbd_b200.davidson_batch([c, c], [_unit(c.n), _unit(c.n)], 10, 10, 1e-6)


def test_batch_step_counts_follow_single_runs():
    ctxs, g = _contexts()
    W0 = [_unit(c.n) for c in ctxs]
    E, Ws, steps = sbd_b200.davidson_batch(ctxs, W0, 300, 8, 1e-9)
    for c, e, s in zip(ctxs, E, steps):
        e1, _, te, _ = c.davidson(_unit(c.n), 300, 8, 1e-9)
        assert abs(e - e1) < 1e-10
        # the same algorithm: the FP64 atomics of sigma make both runs
        # reproducible only to rounding, which a slow residual tail amplifies
        assert abs(s - len(te)) <= max(5, 0.3 * len(te)), (s, len(te))


def _broken(n, seed):
    # the closed-shell determinant plus a 1 % seeded random part: FP64 runs from
    # the determinant alone stay in its spin-flip sector, FP32 rounding does not
    w = np.random.default_rng(seed).normal(size=n)
    w *= 0.01 / np.linalg.norm(w)
    w[0] += 1.0
    return w / np.linalg.norm(w)


def test_batch_mixed_precision_runs_each_problem():
    ctxs, g = _contexts()
    W0 = [_broken(c.n, i) for i, c in enumerate(ctxs[:3])]
    E, Ws, steps = sbd_b200.davidson_batch(ctxs[:3], W0, 300, 10, 1e-6, precision=sbd_b200.MIXED)
    for c, w0, e in zip(ctxs[:3], W0, E):
        e1, _, _, _ = c.davidson(w0, 300, 10, 1e-9)
        assert abs(e - e1) < 1e-8


def test_alpha_beta_shapes_give_the_default_sigma():
    ints, a, b = _seeded_system(14, 4, 300, 11, False)
    c = sbd_b200.context_from_integrals(ints, a, b)
    C = np.random.default_rng(7).normal(size=c.n)
    ref = c.sigma(C)
    for g, t in [(1, 128), (2, 256), (4, 512), (8, 1024), (16, 128)]:
        c.set_tuning(g, t)
        got = c.sigma(C)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), (g, t)
    with pytest.raises(sbd_b200.SbdGpuError):
        c.set_tuning(3, 256)
    with pytest.raises(sbd_b200.SbdGpuError):
        c.set_tuning(4, 200)
    g, t, ms = c.autotune(2)
    assert g in (1, 2, 4, 8, 16) and t in (128, 256, 512, 1024) and ms > 0
    np.testing.assert_allclose(c.sigma(C), ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    c.set_tuning(0, 0)
    c.close()
