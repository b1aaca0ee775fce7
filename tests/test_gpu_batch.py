"""Many independent problems in one sbdgpu_davidson_batch call: the same
energies and ground states as running each problem alone (and the
reference's energy on its own fixture), with one thread per problem or a
bounded pool."""
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
