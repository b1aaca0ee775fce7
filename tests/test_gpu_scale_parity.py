"""Parity at the benchmark sizes, against the reference itself.

The element-wise tests elsewhere run at up to 245,025 determinants.  Kernel
choices change with size: at 12,000 beta strings the FP64 alpha-beta kernel
runs as its 1024-thread variant (one CTA per SM: the source row and the
integral block take 188 KB of shared memory), and the tensor-core kernel
uses 6 M tiles (norb 36).  So here the GPU is compared, at the 16M- and
144M-determinant workloads (norb 26 / 36, 4,000 / 12,000 strings per spin)
and the 400M-determinant one (norb 48, 20,000 strings; tables only), with
the reference compiled from its own sources (oracle/_ref/libsbdref.so):

* excitation tables of both spins, bit-exact against the reference's helper
  lists (GenerateExcitation, chemistry/tpb/helper.h:132-182);
* FP64 sigma of a seeded normalised vector, element-wise within
  1e-12 * max|ref| on slices of alpha rows, against the reference's own mult
  (chemistry/tpb/mult.h:387-648) restricted to those bra rows (rows are
  independent, so a slice is exact);
* the FP32 sigma and the tensor-core sigma at 144M determinants against the
  FP64 sigma, within their precision's tolerance.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle
import sbd_b200
from sbd_b200 import synth

pytestmark = pytest.mark.gpu

SIGMA_TOL = 1e-12  # x max|ref|, the bar of every FP64 sigma test
FP32_TOL = 2e-5    # FP32 vectors and sums
TC_TOL = 5e-3      # BF16 operands in the alpha-beta term


def _host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


@pytest.fixture(scope="module")
def workloads():
    cache = {}

    def get(name):
        if name not in cache:
            if not oracle.reference_available():
                pytest.skip("the reference checker oracle/_ref/libsbdref.so is not built")
            ints, ne, strs = synth.make_workload(name, seed=0)
            td = tempfile.TemporaryDirectory()
            fp, dp = synth.write_workload(td.name, ints, ne, strs)
            ref = oracle.Reference(fp, dp)
            assert np.array_equal(ref.strings(0), np.asarray(strs, np.uint64))
            ctx = sbd_b200.context_from_integrals(ints, strs, strs)
            cache[name] = (ints, strs, ref, ctx, td)
        return cache[name]

    yield get
    for ints, strs, ref, ctx, td in cache.values():
        ctx.close()
        ref.close()
        td.cleanup()


@pytest.mark.parametrize("name", ["c1_L26_6e_4000", "c2_L36_8e_12000", "c4_L48_10e_20000"])
def test_tables_bit_exact_at_scale(workloads, name):
    ints, strs, ref, ctx, td = workloads(name)
    for spin in (0, 1):
        so, si, do, di = ctx.tables(spin)
        o1, i1 = ref.table(spin, 0)
        o2, i2 = ref.table(spin, 1)
        assert np.array_equal(so, o1) and np.array_equal(si, i1)
        assert np.array_equal(do, o2) and np.array_equal(di, i2)


def _row_slices(na, name):
    k = max(2, min(8, _host_cores()))
    if name.startswith("c1"):
        # the aufbau row (most singles and doubles), a middle slice, the last rows
        return [(0, 2), (na // 2, na // 2 + k), (na - 2, na)]
    # 144M: one slice of k rows in the middle and the last two rows
    return [(na // 2 + 17, na // 2 + 17 + k), (na - 2, na)]


@pytest.mark.parametrize("name", ["c1_L26_6e_4000", "c2_L36_8e_12000"])
def test_sigma_rows_vs_reference_at_scale(workloads, name):
    ints, strs, ref, ctx, td = workloads(name)
    C = np.random.default_rng(4242).normal(size=ctx.n)
    C /= np.linalg.norm(C)
    s = ctx.sigma(C)  # through the C ABI with host buffers
    assert np.all(np.isfinite(s))
    for r0, r1 in _row_slices(ctx.na, name):
        want = ref.sigma(C, (r0, r1))
        got = s[r0 * ctx.nb:r1 * ctx.nb]
        err = np.abs(got - want).max()
        assert err <= SIGMA_TOL * np.abs(want).max(), (name, r0, r1, err)


def test_mixed_and_tensor_core_sigma_at_144m(workloads):
    """norb 36 (666 folded pairs: 6 M tiles of the tensor-core kernel)."""
    ints, strs, ref, ctx, td = workloads("c2_L36_8e_12000")
    C = np.random.default_rng(77).normal(size=ctx.n)
    C /= np.linalg.norm(C)
    s64 = ctx.sigma(C)
    scale = np.abs(s64).max()
    s32 = ctx.sigma(C, precision=sbd_b200.MIXED)
    assert np.abs(s32 - s64).max() <= FP32_TOL * scale
    stc = ctx.sigma(C, precision=sbd_b200.MIXED_TC)
    assert np.abs(stc - s64).max() <= TC_TOL * scale
    # the tensor-core sigma differs from FP64 by BF16 rounding, not by missing
    # terms: its error is far below the alpha-beta term's own size
    rel = np.linalg.norm(stc - s64) / np.linalg.norm(s64)
    assert rel < 5e-3, rel
