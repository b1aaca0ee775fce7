"""Benchmark: sigma builds per second on the 144M-determinant workload.

Workload: norb 36, 8 alpha / 8 beta electrons, 12,000 x 12,000 selected
strings (144,000,000 determinants): every string of excitation rank <= 2 from
aufbau plus seeded higher-rank strings, seeded synthetic integrals (the
reference ships no usable input; see sbd_b200/synth.py).  A step is one full
sigma = H*C build on a normalised N(0,1) vector, in FP64.

  value   sigma/s with C and sigma resident in HBM (CUDA events on the
          library's stream around each build); the 1.15 GB vectors are far
          larger than the 126 MB L2, so no flush is needed between steps
  e2e     sigma/s through the C ABI call a user makes with host buffers
          (sbdgpu_sigma: pinned host C -> device, build, device -> host sigma)

--impl reference times the reference's own CPU mult (r-ccs-cms/sbd compiled at
MPI world size 1 into oracle/_ref/libsbdref.so) on a bounded slice of alpha
rows of the same workload with all host threads, extrapolated to a full build.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOAD = "c2_L36_8e_12000"
METRIC = "sigma builds/s at 144M determinants"
UNIT = "sigma/s"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
LAUNCHES_PER_SIGMA = 7  # phase, rows(alpha), transpose, rows(beta), transpose-add, alpha-beta, phase
# with the same-spin terms as INT8 products: phase, transpose, 2 row exponents,
# 2 residue passes, 2 singles-Coulomb kernels, 2 CRT reconstructions,
# transpose-add, alpha-beta, phase (the 30 INT8 GEMMs are cuBLAS's)
LAUNCHES_PER_SIGMA_INT8 = 13


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                           "--format=csv,noheader,nounits", "-lms", "200"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self._proc = None
            return
        threading.Thread(target=self._read, daemon=True).start()

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def stop(self):
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[4 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def max_over_ranks(values, dist, device):
    """Element-wise maximum of per-rank timings (ms) over all ranks of the
    process group: the job's time is its slowest rank's."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def measured_peaks():
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) of one launch,
# from single captures of smaller workloads of the same kernels:
#  - ab_kernel<double> at 16M determinants (norb 26, 6a/6b, 4000 strings):
#    1192.4 MB per launch, 74.5 bytes per determinant; the 144M line scales it
#    by the determinant count
#  - spmv_kernel (method 1) at 245,025 determinants: 4.236 GB per launch
AB_TRAFFIC_BYTES_PER_DET = 74.5
SPMV_TRAFFIC_BYTES_C0 = 4.236e9


def table_stats(ctx):
    st = {}
    for spin in (0, 1):
        so, si, do, di = ctx.tables(spin)
        st[spin] = (len(si), len(di))
        st[("singles", spin)] = np.diff(so.astype(np.int64))
    return st


def ab_smem_floor(st, group, sm_count, sm_mhz):
    """The shared-memory wavefront floor of the FP64 alpha-beta kernel
    (csrc/sigma.cu ab_kernel): every CTA (one source alpha string, `group` of
    its singles) walks every 32-string slice of beta strings for as many steps
    as the slice's longest singles list; a step is group/2 128-bit integral
    loads of 32 distinct rows (4 wavefronts each) and one 64-bit gather of C
    (2 wavefronts); an SM retires one wavefront per cycle.  Lanes of a warp
    that read the same integral row take fewer wavefronts, so the measured time
    can sit slightly below this figure."""
    na_s = st[("singles", 0)]
    nb_s = st[("singles", 1)]
    ctas = int(np.sum((na_s + group - 1) // group))
    pad = (-len(nb_s)) % 32
    widths = np.concatenate([nb_s, np.zeros(pad, np.int64)]).reshape(-1, 32).max(axis=1)
    warp_steps = ctas * int(widths.sum())
    per_step = 4 * (group // 2) + 2
    floor_ms = warp_steps * per_step / sm_count / (sm_mhz * 1e3)
    return {"group": group, "wavefronts_per_step": per_step, "ctas": ctas, "warp_steps": warp_steps,
            "sm_count": sm_count, "sm_mhz": sm_mhz, "floor_ms": floor_ms}


def ab_default_group(nb, P, smem_optin):
    """The FP64 alpha-beta group size the library picks without a tuning table:
    the largest of 16, 8, 4, 2 whose integral rows ([P][group + 2] doubles) fit
    in shared memory next to one row of C (csrc/sigma.cu alpha_beta)."""
    crow = (nb * 8 + 15) // 16 * 16
    for g in (16, 8, 4, 2):
        if crow + P * (g + 2) * 8 <= smem_optin - 1024:
            return g
    return None


def algorithmic(ctx, st):
    """Per-sigma flops 2*nnz(H) and compulsory bytes (vectors + tables)."""
    na, nb, n = ctx.na, ctx.nb, ctx.n
    nsa, nda = st[0]
    nsb, ndb = st[1]
    nnz = n + nb * (nsa + nda) + na * (nsb + ndb) + nsa * nsb
    table_bytes = (nsa + nsb) * (4 + 4 + 8) + (nda + ndb) * (4 + 8)
    sigma_bytes = 8 * n * 3 + table_bytes  # read C, read H_ii, write sigma
    # alpha-beta kernel alone: C read once, sigma read-modify-write, beta singles
    # (sliced ELL, 4 B) and alpha singles (16 B) read once
    ab_bytes = 8 * n * 3 + nsb * 4 + nsa * 16
    return {"flops": 2.0 * nnz, "nnz": nnz, "sigma_bytes": sigma_bytes, "ab_bytes": ab_bytes,
            "ab_flops": 2.0 * nsa * nsb}


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class RefSampler:
    """The reference's own CPU mult (chemistry/tpb/mult.h:387-648, compiled
    from the reference sources at MPI world size 1) on single alpha rows of the
    workload.  Rows are independent; a full sigma is extrapolated from the
    measured seconds per Hamiltonian element of the sampled rows, times the
    exact element count of the whole build (from the reference's own tables).
    The shim's fixed cost per call (copying the 144M-element vectors) is
    measured on an empty slice and subtracted."""

    def __init__(self, ints, ne, strs):
        import oracle
        from sbd_b200 import synth
        self._td = tempfile.TemporaryDirectory()
        fp, dp = synth.write_workload(self._td.name, ints, ne, strs)
        t0 = time.perf_counter()
        self.ref = oracle.Reference(fp, dp)
        self.t_setup = time.perf_counter() - t0
        self.na, self.nb = self.ref.na, self.ref.nb
        sa = np.diff(self.ref.table(0, 0)[0].astype(np.int64))
        da = np.diff(self.ref.table(0, 1)[0].astype(np.int64))
        nsb = int(self.ref.table(1, 0)[0][-1])
        ndb = int(self.ref.table(1, 1)[0][-1])
        # Hamiltonian elements of bra row ia (diagonal, alpha, beta, alpha-beta)
        self.row_nnz = self.nb * (1 + sa + da) + (nsb + ndb) + sa * nsb
        self.total_nnz = float(self.row_nnz.sum())
        C = np.random.default_rng(1234).normal(size=self.na * self.nb)
        self.C = C / np.linalg.norm(C)
        mid = self.na // 2
        t = time.perf_counter()
        self.ref.sigma(self.C, (mid, mid))
        self.overhead = time.perf_counter() - t
        self.calls = 0

    def sample(self) -> dict:
        # the reference's OpenMP loop deals bra rows to threads round-robin
        # (mult.h:490, 500), so a sample takes one row per host thread;
        # slices start at the middle, then step through the range
        k = min(self.na, host_cores())
        ia = (self.na // 2 + self.calls * 7919) % (self.na - k + 1)
        self.calls += 1
        t = time.perf_counter()
        self.ref.sigma(self.C, (ia, ia + k))
        dt = max(time.perf_counter() - t - self.overhead, 1e-9)
        nnz = float(self.row_nnz[ia:ia + k].sum())
        sec = dt / nnz * self.total_nnz
        return {"value": 1.0 / sec, "unit": UNIT, "cores": host_cores(), "kind": "reference",
                "seconds": dt,
                "sample": f"reference mult (r-ccs-cms/sbd, OpenMP x{host_cores()}, MPI world size 1) on alpha rows "
                          f"{ia}..{ia + k - 1} of {self.na}: {dt:.1f} s for {int(nnz)} Hamiltonian elements, "
                          f"extrapolated to the {self.total_nnz:.3e} elements of a full sigma "
                          f"(fixed per-call vector copies, {self.overhead:.1f} s, subtracted)"}

    def close(self):
        self.ref.close()
        self._td.cleanup()


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import oracle
    from sbd_b200 import synth
    if not oracle.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libsbdref.so was not built"}))
        return 0
    ints, ne, strs = synth.make_workload(args.workload, seed=0)
    rs = RefSampler(ints, ne, strs)
    # a CPU sample needs no warm-up beyond the set-up call above; each step is
    # one alpha row, and the run stops adding rows after --ref-budget seconds
    vals, base, spent = [], None, 0.0
    for i in range(args.steps):
        r = rs.sample()
        vals.append(r["value"])
        base = r
        spent += r["seconds"]
        if spent > args.ref_budget:
            break
    rs.close()
    v = len(vals) / sum(1.0 / x for x in vals)  # total elements / total time
    # steps = samples actually timed (the run stops adding samples after
    # --ref-budget seconds); no warm-up sample is taken
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": len(vals), "warmup": 0,
            "steps_requested": args.steps, "ref_budget_s": args.ref_budget, "sampled_seconds": spent,
            "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded integrals and strings)", "impl": "reference",
            "config": {"workload": args.workload, "determinants": int(len(strs)) ** 2, "norb": ints.norb,
                       "electrons": f"{ne}a/{ne}b", "strings_per_spin": int(len(strs)),
                       "parallelism": f"OpenMP x{host_cores()}, MPI world size 1"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": base["cores"], "kind": "reference",
                             "sample": base["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def learned_network(args, dev):
    """The learned preconditioner, trained on the 16M-determinant system
    (norb 26, 6a/6b, 4,000 strings) on the GPU: triples harvested at the ends
    of FP64 Davidson cycles, conjugate-gradient correction solves, Adam on the
    library's own training kernels.  Training time is reported, not counted
    in the time-to-E0 of the systems it is applied to."""
    import sbd_b200
    from sbd_b200 import synth
    ints, ne, strs = synth.make_workload("c1_L26_6e_4000", seed=0)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs, device=dev)
    trace, sec = ctx.precond_train(pairs=args.learn_pairs, cycle=10, cg_iters=args.learn_cg, samples=65536,
                                   steps=args.learn_steps, lr=1e-3, seed=0)
    w = ctx.precond_get()
    ctx.close()
    k = max(1, min(len(trace) // 10, args.learn_pairs))
    return w, {"trained_on": "c1_L26_6e_4000", "pairs": args.learn_pairs, "cg_iters": args.learn_cg,
               "steps": args.learn_steps, "harvest_s": float(sec[0]), "train_s": float(sec[1]),
               "loss_first": float(np.mean(trace[:k])), "loss_last": float(np.mean(trace[-k:]))}


def time_to_e0(ctx, args, learned=None):
    """Davidson from the aufbau determinant, plain FP64 against mixed precision.
    The FP64 run goes to a tight residual; its final <W|HW> is the reference
    energy.  Plain time-to-E0 = time of the first step whose Ritz value is
    within 1e-6 Eh of it (steps cost the same: one sigma each); mixed
    time-to-E0 = the whole mixed run including its FP64 refinement sigma, whose
    energy must land within 1e-6 Eh.  The plain run's first step within 1e-6 Eh
    is found in hindsight; the mixed runs stop on a residual norm they can check
    at run time (default 1e-3, where the energy error, about 0.16 r^2 on this
    system, is ~2e-7 Eh), and each one's error against the FP64 energy is
    reported with a flag for the 1e-6 Eh bound."""
    import sbd_b200
    W0 = np.zeros(ctx.n)
    W0[0] = 1.0
    t = time.perf_counter()
    e_ref, _, te, tt = ctx.davidson(W0, 100, 10, args.e0_tol, precision=sbd_b200.FP64)
    t_plain_all = time.perf_counter() - t
    hit = np.nonzero(te - e_ref < 1e-6)[0]
    k = int(hit[0]) + 1 if len(hit) else len(te)
    t_plain = t_plain_all * k / len(te)
    if not args.time_to_e0:
        # the default line: the plain run against the fastest mixed mode, with
        # the diagonal and with the learned correction
        t = time.perf_counter()
        e_mp, _, tmp_, ttmp = ctx.davidson(W0, 100, 10, args.mixed_tol, precision=sbd_b200.MIXED, restart_keep=3,
                                           restart_prev=1)
        t_mp = time.perf_counter() - t
        out = {"method": "mixed FP32 sigma + thick restart (3 Ritz vectors) + previous Ritz vector",
               "e_fp64": e_ref, "e_mixed": e_mp, "abs_err": abs(e_mp - e_ref), "within_1e-6": abs(e_mp - e_ref) < 1e-6,
               "plain_steps_total": len(te), "plain_steps_to_1e-6": k, "plain_s_to_1e-6": t_plain,
               "mixed_steps": len(tmp_), "mixed_s": t_mp, "mixed_final_residual": float(ttmp[-1]),
               "speedup": t_plain / t_mp, "mixed_tol": args.mixed_tol,
               "note": "wall-clock seconds (one sigma per step dominates); plain time prorated by steps; "
                       "--time-to-e0 adds the other mixed modes"}
        if learned is not None:
            w, info = learned
            ctx.precond_set(w)
            t = time.perf_counter()
            e_l, _, tl, ttl = ctx.davidson(W0, 100, 10, args.mixed_tol, precision=sbd_b200.MIXED, restart_keep=3,
                                           restart_prev=1, precond=sbd_b200.PRECOND_LEARNED)
            t_l = time.perf_counter() - t
            out["learned"] = {"steps": len(tl), "s": t_l, "e": e_l, "abs_err": abs(e_l - e_ref),
                              "within_1e-6": abs(e_l - e_ref) < 1e-6, "final_residual": float(ttl[-1]),
                              "speedup_vs_plain": t_plain / t_l, "speedup_vs_mixed_diagonal": t_mp / t_l,
                              "network": info}
        if args.olsen:
            t = time.perf_counter()
            e_o, _, to_, tto = ctx.davidson(W0, 100, 10, args.mixed_tol, precision=sbd_b200.MIXED, restart_keep=3,
                                            restart_prev=1, precond=sbd_b200.PRECOND_OLSEN)
            t_o = time.perf_counter() - t
            out["olsen"] = {"steps": len(to_), "s": t_o, "e": e_o, "abs_err": abs(e_o - e_ref),
                            "within_1e-6": abs(e_o - e_ref) < 1e-6, "final_residual": float(tto[-1]),
                            "speedup_vs_plain": t_plain / t_o, "speedup_vs_mixed_diagonal": t_mp / t_o}
        return out
    t = time.perf_counter()
    e_mix, _, tm, ttm = ctx.davidson(W0, 100, 10, args.mixed_tol, precision=sbd_b200.MIXED)
    t_mixed = time.perf_counter() - t
    t = time.perf_counter()
    e_mk, _, tmk, ttmk = ctx.davidson(W0, 100, 10, args.mixed_tol, precision=sbd_b200.MIXED, restart_keep=3)
    t_mk = time.perf_counter() - t
    t = time.perf_counter()
    e_mp, _, tmp_, _ = ctx.davidson(W0, 100, 10, args.mixed_tol, precision=sbd_b200.MIXED, restart_keep=3,
                                    restart_prev=1)
    t_mp = time.perf_counter() - t
    t = time.perf_counter()
    e_tc, _, ttc, tttc = ctx.davidson(W0, 100, 10, args.mixed_tol, precision=sbd_b200.MIXED_TC, restart_keep=3,
                                      restart_prev=1)
    t_tc = time.perf_counter() - t
    return {"e_mixed_thick3": e_mk, "abs_err_mixed_thick3": abs(e_mk - e_ref), "mixed_thick3_steps": len(tmk),
            "mixed_thick3_s": t_mk, "speedup_thick3": t_plain / t_mk,
            "e_mixed_thick3_prev": e_mp, "abs_err_mixed_thick3_prev": abs(e_mp - e_ref),
            "mixed_thick3_prev_steps": len(tmp_), "mixed_thick3_prev_s": t_mp, "speedup_thick3_prev": t_plain / t_mp,
            "e_mixed_tc": e_tc, "abs_err_mixed_tc": abs(e_tc - e_ref), "mixed_tc_steps": len(ttc),
            "mixed_tc_s": t_tc, "speedup_tc": t_plain / t_tc,"e_fp64": e_ref, "e_mixed": e_mix, "abs_err_mixed": abs(e_mix - e_ref),
            "plain_steps_total": len(te), "plain_steps_to_1e-6": k, "plain_s_to_1e-6": t_plain,
            "plain_final_residual": float(tt[-1]), "mixed_steps": len(tm), "mixed_s": t_mixed,
            "mixed_final_residual": float(ttm[-1]), "speedup": t_plain / t_mixed,
            "within_1e-6": {"mixed": abs(e_mix - e_ref) < 1e-6, "mixed_thick3": abs(e_mk - e_ref) < 1e-6,
                            "mixed_thick3_prev": abs(e_mp - e_ref) < 1e-6, "mixed_tc": abs(e_tc - e_ref) < 1e-6},
            "mixed_tol": args.mixed_tol,
            "note": "wall-clock seconds (one sigma per step dominates); plain time prorated by steps"}


def method1_block(args, dev, hbm_peak, peak_kind):
    """Method 1 (stored Hamiltonian, CSR SpMV) where it fits one GPU: the
    245,025-determinant full-space case (norb 12, 4a/4b; 349M stored elements,
    4.2 GB, larger than L2).  At 144M determinants the stored elements would
    take ~11 TB."""
    import torch
    import sbd_b200
    from sbd_b200 import synth
    ints, ne, strs = synth.make_workload("c0_L12_4e_full", seed=0)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs, device=dev)
    n = ctx.n
    C = torch.randn(n, dtype=torch.float64, device=f"cuda:{dev}",
                    generator=torch.Generator(device=f"cuda:{dev}").manual_seed(2))
    C /= torch.linalg.norm(C)
    S = torch.empty_like(C)
    fly = []
    for i in range(args.warmup + args.steps):
        ctx.sigma_device(C.data_ptr(), S.data_ptr())
        if i >= args.warmup:
            fly.append(ctx.last_sigma_ms()[3])
    nnz = ctx.store_hamiltonian()
    spmv, tot = [], []
    for i in range(args.warmup + args.steps):
        ctx.sigma_device(C.data_ptr(), S.data_ptr())
        if i >= args.warmup:
            ms = ctx.last_sigma_ms()
            spmv.append(ms[0])
            tot.append(ms[3])
    torch.cuda.synchronize()
    ctx.close()
    k_ms = sum(spmv) / len(spmv)
    bytes_per = 12.0 * nnz + 8.0 * (n + 1) + 24.0 * n
    achieved = bytes_per / (k_ms * 1e-3) / 1e9
    return {"workload": "c0_L12_4e_full", "determinants": n, "stored_elements": nnz,
            "sigma_per_s": 1000.0 * len(tot) / sum(tot), "on_the_fly_sigma_per_s": 1000.0 * len(fly) / sum(fly),
            "roofline": {"bound": "hbm", "kernel": "spmv_kernel (stored Hamiltonian)", "achieved": achieved,
                         "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak, "peak_source": peak_kind,
                         "algorithmic_bytes": bytes_per, "traffic": SPMV_TRAFFIC_BYTES_C0},
            "note": "12 bytes per stored element (uint32 ket, FP64 value) + row offsets + hii, C, sigma"}


def genop_block(args, dev):
    """The generic second-quantised path (sbdgpu_genop_*): the FCIDUMP
    Hamiltonian of the 245,025-determinant system (norb 12, 4a/4b, full
    space) as a GeneralOp on 24 sites, its on-the-fly mult per second, and its
    Davidson energy against the tensor-product-basis path's."""
    import os
    import tempfile
    import torch
    import sbd_b200
    from sbd_b200 import synth
    ints, ne, strs = synth.make_workload("c0_L12_4e_full", seed=0)
    L = ints.norb
    states = np.array([int(a) | (int(b) << L) for a in strs for b in strs], dtype=np.uint64)
    g = sbd_b200.GenOp(states, sign=True, device=dev)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "FCIDUMP")
        synth.write_fcidump(p, ints, 2 * ne)
        g.set_fcidump(p)
    n = len(states)
    C = torch.randn(n, dtype=torch.float64, device=f"cuda:{dev}")
    Wd = torch.zeros_like(C)
    for _ in range(3):
        g.mult_device(C.data_ptr(), Wd.data_ptr())
    # the object runs on its own stream: time over a device-wide synchronize
    torch.cuda.synchronize()
    reps = 20
    t = time.perf_counter()
    for _ in range(reps):
        g.mult_device(C.data_ptr(), Wd.data_ptr())
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t) * 1000.0 / reps
    ctx = sbd_b200.context_from_integrals(ints, strs, strs, device=dev)
    W0 = np.zeros(n)
    W0[0] = 1.0
    e_tpb, _, te_tpb, _ = ctx.davidson(W0, 200, 10, 1e-8)
    t = time.perf_counter()
    e_gen, _, te, tt = g.davidson(W0, 200, 10, 1e-8)
    t_gen = time.perf_counter() - t
    ctx.close()
    g.close()
    return {"workload": "c0_L12_4e_full as GeneralOp (24 sites)", "states": n, "mult_ms": ms, "mult_per_s": 1000.0 / ms, "davidson_steps": len(te),
            "davidson_s": t_gen, "e_generic": e_gen, "e_tpb": e_tpb, "abs_diff": abs(e_gen - e_tpb),
            "note": "mult timed over 20 launches between device synchronizations; no reference arm: the reference's generic mult cannot find most basis "
                    "states (Basis::IndexSearch bisects over the first nwords states only)"}


def config4_block(args, dev, learned):
    """The 400M-determinant workload (norb 48, 10a/10b, 20,000 x 20,000
    selected strings): FP64, FP32 and tensor-core sigma builds per second, and
    time-to-E0 within 1e-6 Eh for plain FP64, mixed precision with the
    diagonal correction and with the learned one (the network trained on the
    16M-determinant system).  FP64 vectors are 3.2 GB each."""
    import torch
    import sbd_b200
    from sbd_b200 import synth
    ints, ne, strs = synth.make_workload("c4_L48_10e_20000", seed=0)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs, device=dev)
    n = ctx.n
    C = torch.randn(n, dtype=torch.float64, device=f"cuda:{dev}",
                    generator=torch.Generator(device=f"cuda:{dev}").manual_seed(3))
    C /= torch.linalg.norm(C)
    S = torch.empty_like(C)
    out = {"workload": "c4_L48_10e_20000", "determinants": n}
    for name, prec in (("fp64", sbd_b200.FP64), ("mixed_fp32", sbd_b200.MIXED), ("mixed_tc", sbd_b200.MIXED_TC)):
        ms = []
        for i in range(2 + 3):
            ctx.sigma_device(C.data_ptr(), S.data_ptr(), precision=prec)
            if i >= 2:
                ms.append(ctx.last_sigma_ms())
        out[name] = {"sigma_per_s": 1000.0 * len(ms) / sum(m[3] for m in ms),
                     "phases_ms": [sum(m[k] for m in ms) / len(ms) for k in range(3)]}
    del C, S
    torch.cuda.empty_cache()
    W0 = np.zeros(n)
    W0[0] = 1.0
    t = time.perf_counter()
    e_ref, _, te, tt = ctx.davidson(W0, 100, 10, args.e0_tol, precision=sbd_b200.FP64)
    t_all = time.perf_counter() - t
    hit = np.nonzero(te - e_ref < 1e-6)[0]
    k = int(hit[0]) + 1 if len(hit) else len(te)
    t_plain = t_all * k / len(te)
    out["plain"] = {"steps_total": len(te), "steps_to_1e-6": k, "s_to_1e-6": t_plain, "e": e_ref,
                    "final_residual": float(tt[-1])}
    t = time.perf_counter()
    e_m, _, tm, ttm = ctx.davidson(W0, 100, 10, args.mixed_tol, precision=sbd_b200.MIXED, restart_keep=3,
                                   restart_prev=1)
    t_m = time.perf_counter() - t
    out["mixed"] = {"steps": len(tm), "s": t_m, "abs_err": abs(e_m - e_ref), "within_1e-6": abs(e_m - e_ref) < 1e-6,
                    "speedup": t_plain / t_m}
    if learned is not None:
        ctx.precond_set(learned[0])
        t = time.perf_counter()
        e_l, _, tl, ttl = ctx.davidson(W0, 100, 10, args.mixed_tol, precision=sbd_b200.MIXED, restart_keep=3,
                                       restart_prev=1, precond=sbd_b200.PRECOND_LEARNED)
        t_l = time.perf_counter() - t
        out["learned"] = {"steps": len(tl), "s": t_l, "abs_err": abs(e_l - e_ref),
                          "within_1e-6": abs(e_l - e_ref) < 1e-6, "speedup": t_plain / t_l,
                          "speedup_vs_mixed_diagonal": t_m / t_l, "network": learned[1]}
    ctx.close()
    return out


def rdm_block(args, dev):
    """1/2-RDMs (sbdgpu_rdm) of a seeded normalised vector on args.rdm_workload,
    wall-clock including the host copies of the 4 L^4 two-body array."""
    import sbd_b200
    from sbd_b200 import synth
    ints, ne, strs = synth.make_workload(args.rdm_workload, seed=0)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs, device=dev)
    W = np.random.default_rng(5).normal(size=ctx.n)
    W /= np.linalg.norm(W)
    ctx.hii()  # tables and diagonal outside the timing
    t = time.perf_counter()
    one, two = ctx.rdm(W)
    sec = time.perf_counter() - t
    ctx.close()
    return {"workload": args.rdm_workload, "determinants": int(len(strs)) ** 2, "seconds": sec,
            "trace_alpha": float(np.trace(one[:ints.norb ** 2].reshape(ints.norb, ints.norb)))}


def roots_block(args, dev):
    """Block Davidson for the lowest args.roots roots (FP64) on the
    16M-determinant system (norb 26, 6a/6b, 4000 x 4000 strings): wall time,
    cycles, sigma builds, residual norms, and root 0 against the single-root
    FP64 Davidson of the same system."""
    import sbd_b200
    from sbd_b200 import synth
    ints, ne, strs = synth.make_workload(args.roots_workload, seed=0)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs, device=dev)
    k = args.roots
    nb = min(32, max(2 * k, 3 * k))
    W0 = np.zeros(ctx.n)
    W0[0] = 1.0
    t = time.perf_counter()
    e1, w1, te, _ = ctx.davidson(W0, 200, 10, args.roots_tol)
    t_one = time.perf_counter() - t
    # the block run starts from the single-root ground state and the
    # lowest-H_ii determinants: from determinants alone its first collapse can
    # drop the ground state's symmetry sector (see DESIGN)
    Wb = np.zeros((k, ctx.n))
    Wb[0] = w1
    t = time.perf_counter()
    E, W, r, it, ns = ctx.davidson_roots(k, 400, nb, args.roots_tol, W0=Wb)
    t_block = time.perf_counter() - t
    ctx.close()
    return {"workload": args.roots_workload, "roots": k, "max_nb": nb, "eps": args.roots_tol, "seconds": t_block,
            "cycles": it, "sigma_builds": ns, "energies": [float(x) for x in E],
            "residuals": [float(x) for x in r],
            "note": "each Ritz value lies within its residual norm of an eigenvalue (symmetric H); block run started "
                    "from the single-root ground state and the lowest-H_ii determinants",
            "root0_minus_single_root": float(E[0] - e1),
            "single_root_seconds": t_one, "single_root_steps": len(te)}


def batch_block(args, dev):
    """args.batch independent problems drawn as the batching workload
    describes (norb uniform in 10-20, electrons per spin in 3-6, 200-2000
    selected strings per spin capped at C(norb, ne), seeded integrals per
    problem): lowest-root FP64 Davidson one problem after another against one
    sbdgpu_davidson_batch call on the same contexts (set-up done before
    either), as problems/s, with the largest energy difference."""
    import math
    import sbd_b200
    from sbd_b200 import synth
    rng = np.random.default_rng(2024)
    ctxs, sizes = [], []
    for i in range(args.batch):
        L = int(rng.integers(10, 21))
        ne = int(rng.integers(3, 7))
        cnt = min(int(rng.integers(200, 2001)), math.comb(L, ne))
        ints, ne, strs = synth.make_small(L, ne, cnt, 1000 + i)
        c = sbd_b200.context_from_integrals(ints, strs, strs, device=dev)
        c.hii()  # tables and diagonal, outside both timings
        ctxs.append(c)
        sizes.append(c.n)
    # the same seeded start for both arms: the aufbau determinant plus a 1 %
    # random part, so that every run reaches the lowest state whatever its
    # spin-flip symmetry (from the closed-shell determinant alone, rounding
    # decides whether a run leaves the spin-flip-even sector)
    W0s = []
    for i, c in enumerate(ctxs):
        w = np.random.default_rng(5000 + i).normal(size=c.n)
        w *= 0.01 / np.linalg.norm(w)
        w[0] += 1.0
        W0s.append(w / np.linalg.norm(w))
    # the committed launch shapes of the alpha-beta kernel, in both arms
    from sbd_b200 import autotune
    table = autotune.load()
    tuned = sum(1 for c in ctxs if autotune.apply(c, table))
    max_it = 300
    t = time.perf_counter()
    e_seq, s_seq = [], []
    for c, w in zip(ctxs, W0s):
        e1, _, te, _ = c.davidson(w, max_it, 10, args.batch_tol)
        e_seq.append(e1)
        s_seq.append(len(te))
    t_seq = time.perf_counter() - t
    t = time.perf_counter()
    e_bat, _, steps = sbd_b200.davidson_batch(ctxs, W0s, max_it, 10, args.batch_tol)
    t_bat = time.perf_counter() - t
    for c in ctxs:
        c.close()
    diff = np.abs(np.array(e_bat) - np.array(e_seq))
    return {"problems": args.batch, "determinants_min": int(min(sizes)), "determinants_max": int(max(sizes)),
            "determinants_total": int(sum(sizes)), "eps": args.batch_tol,
            "sequential_problems_per_s": args.batch / t_seq, "batch_problems_per_s": args.batch / t_bat,
            "speedup": t_seq / t_bat, "max_abs_energy_diff": float(diff.max()),
            "problems_differing_by_more_than_1e-6": int((diff > 1e-6).sum()),
            "steps_total": int(sum(steps)), "steps_max": int(max(steps)),
            "sequential_steps_total": int(sum(s_seq)),
            "problems_at_step_cap": int(sum(1 for x in steps if x >= max_it * 10)),
            "tuned_contexts": tuned, "tuning_classes": len(table),
            "note": "batch: device-resident Davidson, one replayed CUDA graph per problem step, one host wait per "
                    "round; sequential: sbdgpu_davidson per problem (one host round trip per dot product)"}


def run_gpu(args):
    import torch
    import sbd_b200
    from sbd_b200 import synth

    rank, world, local = dist_env()
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    ints, ne, strs = synth.make_workload(args.workload, seed=0)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs, device=dev)
    ctx.set_fp64_same_spin(args.fp64_same_spin)
    st = table_stats(ctx)
    alg = algorithmic(ctx, st)
    n = ctx.n
    C = torch.randn(n, dtype=torch.float64, device=f"cuda:{dev}", generator=torch.Generator(device=f"cuda:{dev}").manual_seed(1))
    C /= torch.linalg.norm(C)
    S = torch.empty_like(C)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        ctx.sigma_device(C.data_ptr(), S.data_ptr())
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(dev)
    sampler.start()
    tot, ab, parts = 0.0, 0.0, [0.0, 0.0, 0.0]
    for _ in range(args.steps):
        ctx.sigma_device(C.data_ptr(), S.data_ptr())
        ms = ctx.last_sigma_ms()
        tot += ms[3]
        for k in range(3):
            parts[k] += ms[k]
    torch.cuda.synchronize()
    # the mixed-precision sigma (FP32 vectors) on the same resident vector
    mixed_ms = []
    for i in range(args.warmup + args.steps):
        ctx.sigma_device(C.data_ptr(), S.data_ptr(), precision=sbd_b200.MIXED)
        if i >= args.warmup:
            mixed_ms.append(ctx.last_sigma_ms())
    tc_ms = []
    for i in range(args.warmup + args.steps):
        ctx.sigma_device(C.data_ptr(), S.data_ptr(), precision=sbd_b200.MIXED_TC)
        if i >= args.warmup:
            tc_ms.append(ctx.last_sigma_ms())
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    # end to end: pinned host buffers through the C ABI
    Ch = torch.empty(n, dtype=torch.float64, pin_memory=True)
    Ch.copy_(C.cpu())
    Sh = torch.empty(n, dtype=torch.float64, pin_memory=True)
    e2e_ms = 0.0
    Cnp = Ch.numpy()
    Snp = Sh.numpy()
    import ctypes
    for _ in range(args.steps):
        rc = sbd_b200.lib().sbdgpu_sigma(ctx._h, Cnp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         Snp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0)
        ctx._check(rc)
        e2e_ms += ctx.last_sigma_ms()[4]
    torch.cuda.synchronize()
    sampler.stop()
    if pg:
        pg.barrier()
    t_step = tot / args.steps
    t_e2e = e2e_ms / args.steps
    if pg:
        t_step, t_e2e = max_over_ranks([t_step, t_e2e], pg, f"cuda:{dev}")
    if rank != 0:
        ctx.close()
        if pg:
            pg.destroy_process_group()
        return 0
    hbm_peak, peak_kind = measured_peaks()
    ab_ms = parts[2] / args.steps
    kernel_names = ["rows_kernel<true> (diag + alpha same-spin)", "beta same-spin (transpose, rows_kernel<false>, transpose-add)",
                    "ab_kernel (alpha-beta)"]
    dom = int(np.argmax(parts))
    dom_ms = parts[dom] / args.steps
    dom_bytes = [8.0 * n * 3 + st[0][0] * 16 + st[0][1] * 12, 8.0 * n * 6 + st[1][0] * 16 + st[1][1] * 12,
                 alg["ab_bytes"]][dom]
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    traffic = args.traffic
    if traffic is None and dom == 2:
        traffic = AB_TRAFFIC_BYTES_PER_DET * n
    smem_floor = None
    if dom == 2:
        props = torch.cuda.get_device_properties(dev)
        group = ab_default_group(ctx.nb, ctx.norb * (ctx.norb + 1) // 2,
                                 getattr(props, "shared_memory_per_block_optin", 232448))
        clk = sampler.summary().get("sm_mhz") or 1965.0
        if group:
            smem_floor = ab_smem_floor(st, group, props.multi_processor_count, clk)
            smem_floor["measured_ms"] = ab_ms
            smem_floor["frac"] = smem_floor["floor_ms"] / ab_ms
    line = {
        "metric": METRIC, "value": world * 1000.0 / t_step, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded integrals and strings)",
        "config": {"workload": args.workload, "determinants": n, "norb": ints.norb, "electrons": f"{ne}a/{ne}b",
                   "strings_per_spin": ctx.na, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs (1.15 GB per vector) larger than L2; no flush"},
        "e2e": {"value": world * 1000.0 / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 8 * n},
        "gpu_launches": (LAUNCHES_PER_SIGMA_INT8 if args.fp64_same_spin == 0 and min(ctx.na, ctx.nb) >= 1024
                         and ctx.na % 4 == 0 and ctx.nb % 4 == 0 else LAUNCHES_PER_SIGMA) * args.steps * 2,
        "roofline": {"bound": "hbm", "kernel": kernel_names[dom], "achieved": achieved, "peak": hbm_peak,
                     "unit": "GB/s", "frac": achieved / hbm_peak, "peak_source": peak_kind,
                     "traffic": traffic,
                     "limiter": ("shared-memory pipe: one gathered 8-byte integral per FP64 FMA (ncu at 16M "
                                 "dets: l1tex 90.8 %, FP64 pipe 24.7 %, profiles/ab_kernel_c1_L26_6e_4000.md)")
                     if dom == 2 else "L1/L2 streaming of C rows (profiles/rows_kernel_c1_L26_6e_4000.md)",
                     "smem_floor": smem_floor},
        "phases_ms": {"alpha_same_spin_with_diag": parts[0] / args.steps,
                      "beta_same_spin": parts[1] / args.steps, "alpha_beta": ab_ms},
        "flops_per_sigma": alg["flops"], "fp64_tflops": alg["flops"] / (t_step * 1e-3) / 1e12,
        "mixed_fp32": {"sigma_per_s": 1000.0 * len(mixed_ms) / sum(m[3] for m in mixed_ms),
                       "phases_ms": [sum(m[k] for m in mixed_ms) / len(mixed_ms) for k in range(3)],
                       "note": "FP32 vectors and sigma incl. FP64<->FP32 conversion at the ABI"},
        "mixed_tc": {"sigma_per_s": 1000.0 * len(tc_ms) / sum(m[3] for m in tc_ms),
                     "phases_ms": [sum(m[k] for m in tc_ms) / len(tc_ms) for k in range(3)],
                     "note": "FP32 vectors; alpha-beta term on tcgen05 tensor cores (BF16 operands, FP32 accumulation)"},
        "clocks": sampler.summary(),
    }
    learned = None
    if world == 1 and not args.no_learned and (not args.no_time_to_e0 or args.config4):
        learned = learned_network(args, dev)
    if world == 1 and not args.no_time_to_e0:
        line["time_to_e0"] = time_to_e0(ctx, args, learned)
    if not args.no_method1:
        line["method1_stored"] = method1_block(args, dev, hbm_peak, peak_kind)
    if args.roots > 0:
        line["block_roots"] = roots_block(args, dev)
    if args.genop and world == 1:
        line["genop"] = genop_block(args, dev)
    if args.rdm:
        line["rdm"] = rdm_block(args, dev)
    if args.config4 and world == 1:
        ctx.close()
        line["config4"] = config4_block(args, dev, learned)
    if args.batch > 0:
        line["batch"] = batch_block(args, dev)
    if not args.no_cpu_baseline:
        try:
            rs = RefSampler(ints, ne, strs)
            line["cpu_baseline"] = rs.sample()
            line["cpu_baseline"].pop("seconds", None)
            rs.close()
        except Exception as e:  # the reference checker may be absent on a fresh box
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    print(json.dumps(line))
    ctx.close()
    if pg:
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-budget", type=float, default=120.0, help="seconds of reference CPU work in --impl reference")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--traffic", type=float, default=None, help="ncu DRAM bytes per launch of the dominant kernel")
    ap.add_argument("--workload", default=WORKLOAD, help="named workload (smaller ones for profiling captures)")
    ap.add_argument("--time-to-e0", action="store_true",
                    help="time-to-E0 with every mixed mode (by default: plain FP64 against the fastest one)")
    ap.add_argument("--no-time-to-e0", action="store_true", help="skip the time-to-E0 runs")
    ap.add_argument("--no-method1", action="store_true", help="skip the stored-Hamiltonian (method 1) block")
    ap.add_argument("--roots", type=int, default=0, help="also time block Davidson for this many roots")
    ap.add_argument("--roots-workload", default="c1_L26_6e_4000", help="workload of the block Davidson block")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-preconditioner run")
    ap.add_argument("--olsen", action="store_true", help="also time the mixed run with Olsen's correction")
    ap.add_argument("--learn-pairs", type=int, default=12, help="harvested triples for the learned preconditioner")
    ap.add_argument("--learn-cg", type=int, default=40, help="MINRES steps per harvested correction")
    ap.add_argument("--learn-steps", type=int, default=600, help="Adam steps of the learned preconditioner")
    ap.add_argument("--rdm", action="store_true", help="also time the 1/2-RDMs")
    ap.add_argument("--genop", action="store_true", help="also time the generic second-quantised path")
    ap.add_argument("--fp64-same-spin", type=int, default=0,
                    help="FP64 same-spin terms: 0 = exact INT8 tensor-core products, 1 = rows kernels")
    ap.add_argument("--rdm-workload", default="c1_L26_6e_4000", help="workload of the RDM block")
    ap.add_argument("--config4", action="store_true",
                    help="also run the 400M-determinant workload (norb 48, 10a/10b, 20,000 strings)")
    ap.add_argument("--batch", type=int, default=0, help="also time this many independent small problems at once")
    ap.add_argument("--batch-tol", type=float, default=1e-6, help="residual target of the batched problems")
    ap.add_argument("--roots-tol", type=float, default=1e-5, help="residual target of the block Davidson block")
    ap.add_argument("--e0-tol", type=float, default=1e-7, help="residual target of the FP64 reference run")
    ap.add_argument("--mixed-tol", type=float, default=1e-3, help="residual target of the mixed runs")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
