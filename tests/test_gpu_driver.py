"""The sample driver (reference command line) and the C++ drop-in
sbd::tpb::diag, end to end on the GPU, against the reference's own outputs."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import load_golden
from sbd_b200 import build, synth

pytestmark = pytest.mark.gpu


def test_sample_driver_matches_reference():
    g = load_golden("g_L8_3e_full")
    exe = build.build_driver()
    ints, ne, strs = synth.make_small(8, 3, None, int(g["seed"]))
    with tempfile.TemporaryDirectory() as td:
        fp, dp = synth.write_workload(td, ints, ne, strs)
        r = subprocess.run([exe, "--fcidump", fp, "--adetfile", dp, "--method", "0", "--block", "10",
                            "--iteration", "1000", "--tolerance", "1e-8", "--rdm", "1", "--carryover_ratio", "0.5",
                            "--carryoverfile", os.path.join(td, "co.txt"), "--savename", os.path.join(td, "wf")],
                           cwd=td, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        out = r.stdout
        e = float(re.search(r"Sample-based diagonalization: Energy = (\S+)", out).group(1))
        assert abs(e - float(g["energy"])) < 1e-10
        ob = float(re.search(r"One-Body \+ Two-Body energy = (\S+)", out).group(1))
        assert abs(ob - float(g["energy"])) < 1e-9
        assert "Davidson iteration 0.0 (tol=" in out
        rdm1 = np.loadtxt(os.path.join(td, "1pRDM.txt"))
        L = 8
        ref1 = (g["rdm1"][:L * L] + g["rdm1"][L * L:]).reshape(L, L).T.ravel()
        assert np.abs(rdm1[:, 2] - ref1).max() < 1e-10
        co = [int(l.strip(), 2) for l in open(os.path.join(td, "co.txt")) if l.strip()]
        assert np.array_equal(np.array(co, dtype=np.uint64), g["carry_ratio_strings"])
        with open(os.path.join(td, "wf000000"), "rb") as f:
            hdr = np.frombuffer(f.read(24), dtype=np.uint64)
            assert list(hdr) == [len(strs), len(strs), 1]
            f.read(8 * 2 * len(strs))
            W = np.frombuffer(f.read(), dtype=np.float64)
        assert abs(abs(np.dot(W, g["W"])) - 1.0) < 1e-10
        # restart from the saved wavefunction: converges at once to the same energy
        r2 = subprocess.run([exe, "--fcidump", fp, "--adetfile", dp, "--iteration", "10", "--block", "10",
                             "--tolerance", "1e-6", "--loadname", os.path.join(td, "wf")],
                            cwd=td, capture_output=True, text=True)
        assert r2.returncode == 0, r2.stderr
        e2 = float(re.search(r"Sample-based diagonalization: Energy = (\S+)", r2.stdout).group(1))
        assert abs(e2 - float(g["energy"])) < 1e-10
        assert r2.stdout.count("Davidson iteration") == 1


def test_sample_driver_mixed_with_restarts():
    """The added options reach the solver: FP32 basis with thick restart and
    the previous Ritz vector gives the reference's energy to 1e-6 Eh."""
    g = load_golden("g_L8_3e_full")
    exe = build.build_driver()
    ints, ne, strs = synth.make_small(8, 3, None, int(g["seed"]))
    with tempfile.TemporaryDirectory() as td:
        fp, dp = synth.write_workload(td, ints, ne, strs)
        r = subprocess.run([exe, "--fcidump", fp, "--adetfile", dp, "--block", "10", "--iteration", "1000",
                            "--tolerance", "1e-5", "--rdm", "0", "--precision", "1", "--restart_keep", "3",
                            "--restart_prev", "1"], cwd=td, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        e = float(re.search(r"Sample-based diagonalization: Energy = (\S+)", r.stdout).group(1))
        assert abs(e - float(g["energy"])) < 1e-6
