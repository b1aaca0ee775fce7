"""The header-only C++ host library (sbd_b200/include/sbd_gpu/tpb.h): its
FCIDUMP / string-file readers and integral set-up agree with the reference
semantics (checked against the Python readers and the golden strings)."""
import os
import subprocess
import tempfile

import numpy as np

from conftest import ROOT, load_golden
from sbd_b200 import fcidump, synth

PROG = r'''
#include <cstdio>
#include "sbd/sbd.h"
int main(int argc, char** argv) {
  auto d = sbd::LoadFCIDump(argv[1]);
  auto x = sbd::gpu_detail::setup_integrals(d);
  std::vector<std::vector<size_t>> adet;
  sbd::LoadAlphaDets(argv[2], adet, 20, x.L);
  if (argc > 3) { sbd::ShuffleDet(adet, 1729u); }
  double s1 = 0, s2 = 0;
  for (size_t i = 0; i < x.h1.size(); i++) s1 += x.h1[i] * (i + 1);
  for (size_t i = 0; i < x.eri.size(); i++) s2 += x.eri[i] * ((i % 97) + 1);
  std::printf("%d %.17g %.17g %.17g %zu\n", x.L, x.I0, s1, s2, adet.size());
  for (auto& a : adet) std::printf("%llu\n", (unsigned long long)sbd::gpu_detail::to_u64(a, 20, x.L));
  return 0;
}
'''


def _compile(td):
    src = os.path.join(td, "t.cc")
    exe = os.path.join(td, "t")
    open(src, "w").write(PROG)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "sbd_b200", "include"), "-I",
                    os.path.join(ROOT, "include"), src, "-o", exe], check=True)
    return exe


def test_readers_match_reference_semantics():
    g = load_golden("g_L8_3e_shuffled")
    ints, ne, strs = synth.make_small(8, 3, None, int(g["seed"]))
    with tempfile.TemporaryDirectory() as td:
        fp, dp = synth.write_workload(td, ints, ne, strs[::-1])  # unsorted file: the loader sorts
        exe = _compile(td)
        out = subprocess.run([exe, fp, dp, "shuffle"], capture_output=True, text=True, check=True).stdout.split()
        L, I0, s1, s2, n = int(out[0]), float(out[1]), float(out[2]), float(out[3]), int(out[4])
        got = np.array([int(x) for x in out[5:5 + n]], dtype=np.uint64)
        fd = fcidump.read_fcidump(fp)
    assert L == 8 and I0 == fd.ecore
    h1 = fd.h.ravel()
    assert abs(s1 - (h1 * np.arange(1, h1.size + 1)).sum()) < 1e-12 * abs(s1)
    e = synth.pack_eri(fd.eri)
    assert abs(s2 - (e * ((np.arange(e.size) % 97) + 1)).sum()) < 1e-12 * abs(s2)
    # sorted, then the reference's seeded shuffle: identical to the reference's order
    assert np.array_equal(got, g["astr"])


WF_PROG = r'''
#include <cstdio>
#include <fstream>
#include "sbd/sbd.h"
// argv: adet file A, adet file B, W_A (binary FP64), save prefix, W_B out (binary FP64)
int main(int argc, char** argv) {
  std::vector<std::vector<size_t>> a, b;
  sbd::LoadAlphaDets(argv[1], a, 20, 8);
  sbd::LoadAlphaDets(argv[2], b, 20, 8);
  std::vector<double> wa(a.size() * a.size());
  std::ifstream(argv[3], std::ios::binary).read(reinterpret_cast<char*>(wa.data()), sizeof(double) * wa.size());
  sbd::SaveWavefunction(argv[4], a, a, wa);
  std::vector<double> wb;
  sbd::LoadWavefunction(argv[4], b, b, wb);
  std::ofstream(argv[5], std::ios::binary).write(reinterpret_cast<const char*>(wb.data()), sizeof(double) * wb.size());
  return 0;
}
'''


def test_wavefunction_save_load_remap_matches_reference():
    """SaveWavefunction / LoadWavefunction of the host header against the
    reference's (restart.h:20-66, 414-658) run here: the saved file is
    byte-identical, and loading it onto a different, partly overlapping
    basis maps and normalises W the same way."""
    import pytest
    import oracle
    if not oracle.reference_available():
        pytest.skip("compiled reference not available")
    ints = synth.make_integrals(8, 3)
    sa = synth.selected_strings(8, 3, 40, np.diag(ints.h), 11)
    rest = [int(x) for x in synth.full_strings(8, 3) if int(x) not in set(int(y) for y in sa)]
    sb = np.array(sorted(set(int(x) for x in sa[::2]) | set(rest[:6])), dtype=np.uint64)
    overlap = len(set(int(x) for x in sa) & set(int(x) for x in sb))
    assert 0 < overlap < min(len(sa), len(sb))
    with tempfile.TemporaryDirectory() as td:
        fp, dpa = synth.write_workload(os.path.join(td, "a"), ints, 3, sa)
        _, dpb = synth.write_workload(os.path.join(td, "b"), ints, 3, sb)
        ref_a = oracle.Reference(fp, dpa)
        ref_b = oracle.Reference(fp, dpb)
        wa = np.random.default_rng(5).normal(size=ref_a.na * ref_a.nb)
        wa /= np.linalg.norm(wa)
        ref_a.save_wavefunction(os.path.join(td, "wref"), wa)
        wb_ref = ref_b.load_wavefunction(os.path.join(td, "wref"))
        wa_path = os.path.join(td, "wa.bin")
        wa.tofile(wa_path)
        src = os.path.join(td, "wf.cc")
        exe = os.path.join(td, "wf")
        open(src, "w").write(WF_PROG)
        subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "sbd_b200", "include"), "-I",
                        os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        subprocess.run([exe, dpa, dpb, wa_path, os.path.join(td, "wours"), os.path.join(td, "wb.bin")], check=True)
        assert open(os.path.join(td, "wours000000"), "rb").read() == open(os.path.join(td, "wref000000"), "rb").read()
        wb = np.fromfile(os.path.join(td, "wb.bin"))
    assert wb.shape == wb_ref.shape
    assert np.abs(wb - wb_ref).max() < 1e-15
