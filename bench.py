#!/usr/bin/env python
"""Groth16 prover benchmark on B200: proofs/s and p50/p99 latency at 2^20
constraints, plus the G1 MSM at 2^20 in ms.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one Groth16 proof of the synthetic 2^20-constraint circuit (a
fresh witness per step, alternating among pre-solved witnesses), through
lzk_groth16_prove.  `value` is whole-job proofs/s with the witness already
in HBM; `e2e` adds, every step, the host->device copy of that step's witness
from pinned memory and the device->host read of the proof.  With N > 1 each
rank is an independent replica (proofs do not shard) and the slowest rank's
time is used.  `--impl reference` times the reference's own CPU path (the
libff-derived host arithmetic built into oracle/_ref) on a bounded sample
and extrapolates to one proof.
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Groth16 proofs/s & p50/p99 latency at 2^20 constraints; G1 MSM 2^20 ms"
IMAD_PER_FP_MUL = 264          # 8x8 lo + 8x8 hi products, 8 x (1 + 8 + 8) reduction
FP_MUL_PER_G1_MADD = 10        # XYZZ mixed addition: 8M + 2S


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--log-m", type=int, default=20)
    ap.add_argument("--mode", choices=["standard", "reference"], default="standard")
    ap.add_argument("--circuit", choices=["synthetic", "matmul"], default="synthetic",
                    help="synthetic = the benchmark circuit (--log-m); matmul = the reference's own MatMul "
                         "circuit (--matmul-p; p = 100 gives 2^20 constraints)")
    ap.add_argument("--matmul-p", type=int, default=100)
    ap.add_argument("--window", type=int, default=17)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--case", choices=["prove", "msm-g1", "msm-g2", "ntt", "spmv", "batch", "serve", "reference-gpu",
                                       "tune"],
                    default="prove",
                    help="prove = the benchmark; msm-g1/msm-g2/ntt run one operator at --log-n for profiling; "
                         "reference-gpu times the reference's own GPU programs (built by make -C oracle refgpu)")
    ap.add_argument("--log-n", type=int, default=20)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--plain", action="store_true", help="msm cases: plain affine bases instead of a shifted table")
    ap.add_argument("--inflight", type=int, default=4)
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--tune-out", default=None, help="tune case: write the measured tuning table (JSON) here")
    ap.add_argument("--retune", action="store_true", help="batch case: measure the tuning table instead of loading "
                                                          "the packaged one")
    ap.add_argument("--no-tuning-table", action="store_true", help="do not load the packaged tuning table")
    return ap.parse_args()


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region"""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def mark(self, which):
        """wall-clock bounds of the timed region ("begin" / "end")"""
        setattr(self, which, datetime.datetime.now())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f")
            except ValueError:
                continue
            rows.append((ts, f[1:]))
        os.unlink(self.path)
        lo, hi = getattr(self, "begin", None), getattr(self, "end", None)
        inside = [f for ts, f in rows if lo and hi and lo <= ts <= hi]
        window = "timed region" if inside else "whole run (no sample fell inside the timed region)"
        rows = inside or [f for _, f in rows]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows), "window": window}


# --------------------------------------------------------------- CPU side
def cpu_reference_sample(log_m, n_vars, n_l, seed=3):
    """Time the reference's own CPU path (oracle/_ref: libff-derived host
    arithmetic) on a bounded sample and extrapolate to one 2^log_m proof:
    the naive MSM of test/msm-check.cu:45-55 (OpenMP over all cores) per G1
    and G2 point, the reference's radix-2 NTT (poly.cuh:32-73 restated on
    libff Fr) per butterfly, and the CSR SpMV per row.  Returns a dict."""
    from oracle import FR, Oracle, Ref, have_ref
    orc = Oracle()
    lib = Ref() if have_ref() else None
    kind = "reference" if lib else "port"
    L = lib if lib else orc
    st = np.array([seed], np.uint64)
    M = 1 << log_m
    n1, n2, nt = 1 << 13, 1 << 11, 1 << 16
    k = orc.rand_field(FR, n1, st)
    jac1 = orc.aff_to_jac(1, orc.fixed_base(1, k))
    jac2 = orc.aff_to_jac(2, orc.fixed_base(2, k[:n2]))
    s = orc.rand_field(FR, n1, st)
    t0 = time.perf_counter()
    if lib:
        lib.g1_msm_naive_jac(s, jac1)
    else:
        orc.msm(1, s, orc.jac_to_aff(1, jac1), naive=True)
    t_g1 = (time.perf_counter() - t0) / n1
    t0 = time.perf_counter()
    if lib:
        lib.g2_msm_naive_jac(s[:n2], jac2)
    else:
        orc.msm(2, s[:n2], orc.jac_to_aff(2, jac2), naive=True)
    t_g2 = (time.perf_counter() - t0) / n2
    tab = L.ntt_setup(nt)
    c = orc.rand_field(FR, nt, st)
    t0 = time.perf_counter()
    L.ntt_ref(c, tab[nt:2 * nt], tab[2 * nt])
    t_bfly = (time.perf_counter() - t0) / ((nt // 2) * 16)
    # reference chain: 3 iNTT_M + 3 NTT_2M + 1 iNTT_2M (groth16.cuh:166-185)
    bfly = 3 * (M // 2) * log_m + 4 * M * (log_m + 1)
    rows = 1 << 14
    per = np.full(rows, 2, np.int64)
    rp = np.concatenate([[0], np.cumsum(per)[:-1]]).astype(np.uint64)
    col = np.random.default_rng(1).integers(0, rows, 2 * rows).astype(np.uint64)
    val = orc.rand_field(FR, 2 * rows, st)
    z = orc.rand_field(FR, rows, st)
    t0 = time.perf_counter()
    L.spmv(val, col, rp, z) if lib else orc.spmv(val, col, rp, z)
    t_row = (time.perf_counter() - t0) / rows
    t_proof = (2 * n_vars + n_l + (M - 1)) * t_g1 + n_vars * t_g2 + bfly * t_bfly + 3 * M * t_row
    return {"value": 1.0 / t_proof, "unit": "proofs/s", "cores": os.cpu_count(), "kind": kind,
            "sample": (f"naive MSM (test/msm-check.cu:45-55, OpenMP) on {n1} G1 and {n2} G2 points, "
                       f"radix-2 NTT of 2^16 and SpMV of {rows} rows, extrapolated to one 2^{log_m} proof "
                       f"(4 G1 MSMs + 1 G2 MSM over {n_vars} variables, 7 NTTs, 3 SpMVs)"),
            "seconds_per_proof": t_proof, "per_point_us": {"g1": t_g1 * 1e6, "g2": t_g2 * 1e6}}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    M = 1 << args.log_m
    n_vars = M + 4096 + 2
    vals = []
    for _ in range(args.warmup):
        cpu_reference_sample(min(args.log_m, 12), n_vars, n_vars - 2)
    t_start = time.perf_counter()
    for i in range(args.steps):
        vals.append(cpu_reference_sample(args.log_m, n_vars, n_vars - 2, seed=3 + i))
    wall = time.perf_counter() - t_start
    v = float(np.mean([x["value"] for x in vals]))
    cb = dict(vals[-1])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "proofs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 limbs (Fr/Fq mod p)",
            "data": "synthetic", "config": {"workload": f"groth16_prove_2^{args.log_m}", "constraints": M,
                                            "variables": n_vars, "sample": "bounded CPU sample per step"},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "proofs/s", "h2d_bytes_per_step": 0,
                                         "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU side
def hbm_peak_gbs():
    """the measured copy bandwidth of this pool's B200s (MEASURED_PEAKS.json),
    else the profiling recipe's fallback"""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def spmv_bytes(circ):
    """algorithmic bytes of A.z, B.z, C.z: per matrix nnz (32 B value +
    index + 32 B z gather) + rows (row offset + 32 B output)"""
    tot = 0
    for m in circ.mats:
        ib = m.col.element_size()
        tot += m.nnz * (32 + ib + 32) + m.rows * (ib + 32)
    return tot


def ntt_algorithmic(log_n, coset=True):
    """IMAD-class operations and bytes of one transform of 2^log_n: (n/2) log n
    butterfly products (+ n for the coset scaling) at 264 each; two passes
    reading and writing 32 B per element"""
    n = 1 << log_n
    return ((n // 2) * log_n + (n if coset else 0)) * IMAD_PER_FP_MUL, 2 * 2 * 32 * n


def run_reference_gpu_case(args):
    """The reference's own GPU path on this GPU, as its test programs run it:
    oracle/_ref/groth16_gpu is test/groth16.cu (Groth16_BN254 with
    MatMul_p_100: 2^20 constraints, Setup(12) then one Prove, whose phase
    timers groth16.cuh:157-217 print wall times around synchronised
    launches) and oracle/_ref/msm_check_gpu is test/msm-check.cu (G1 MSM
    2^20, c = 12, timer msm-check.cu:38-41).  Both are the unmodified
    reference sources compiled for sm_100a by oracle/Makefile.  Prints one
    JSON line; the reference's inputs are its own unseeded random ones."""
    import re
    import subprocess
    exe = {k: os.path.join(ROOT, "oracle", "_ref", k) for k in ("groth16_gpu", "msm_check_gpu")}
    missing = [k for k, v in exe.items() if not os.path.exists(v)]
    if missing:
        print(json.dumps({"case": "reference-gpu", "unavailable": f"not built: {', '.join(missing)} "
                          "(make -C oracle refgpu needs the reference tree)"}), flush=True)
        return
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    timing = re.compile(r"\[Timing\]\S*\s+(.*?) in: ([0-9.]+) seconds")

    def run(path, timeout):
        p = subprocess.run([path], env=env, capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"{os.path.basename(path)} exited {p.returncode}: {p.stdout[-400:]}{p.stderr[-400:]}")
        return [(m.group(1), float(m.group(2)) * 1e3) for m in timing.finditer(p.stdout)], p.stdout

    msm_t, msm_out = run(exe["msm_check_gpu"], 900)
    # timers in order: key generation, the MSM, the CPU check (msm-check.cu:31,41,55)
    g1_ms = msm_t[1][1] if len(msm_t) >= 2 else None
    g16_t, _ = run(exe["groth16_gpu"], 1500)
    phases = {k: v for k, v in g16_t if k.startswith("Phase")}
    prove_ms = sum(phases.values())
    print(json.dumps({"case": "reference-gpu", "impl": "reference (its own GPU code on this GPU)",
                      "workload": "groth16_prove_2^20 (MatMul_p_100: M = 2^20, N = 1030000)",
                      "prove_ms": prove_ms, "proofs_per_s": 1e3 / prove_ms if prove_ms else None,
                      "phases_ms": phases, "setup_ms": {k: v for k, v in g16_t if not k.startswith("Phase")},
                      "g1_msm_2e20_ms": g1_ms, "g1_msm_window_bits": 12,
                      "msm_check_ok": "Everything is OK!" in msm_out}), flush=True)


def run_batch_case(args):
    """the batched-operator workload (64 G1 MSMs of 2^10..2^20 points and 32
    NTTs of 2^12..2^22 elements): one batch plan replayed as a CUDA graph,
    against the same operators called one at a time"""
    import torch

    from liblightzk_b200 import autotune, batch, msm, ntt
    # the tuning table (window width, reduction run, accumulation chunk, NTT
    # pass block): the packaged table measured on this GPU model, or measured
    # here for this workload's size classes with --retune
    table_src = None if args.retune else autotune.load_default()
    if table_src is None:
        autotune.tune_msm(1, log_ns=range(10, 21), spread=2, reps=2)
        autotune.tune_msm_table(1, log_ns=range(10, 21), reps=2)
        autotune.tune_ntt(range(12, 23), reps=2)
        table_src = "measured in this run"
    msms, ntts, _pool = batch.workload_config3()
    plan = batch.BatchPlan(1, msms, ntts)
    plan_fx = batch.BatchPlan(1, msms, ntts, fixed_bases=True)
    plan_px = batch.BatchPlan(1, msms, ntts, fixed_bases=True, persistent=True)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()

    def timed(fn, reps):
        out = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            out.append(a.elapsed_time(b))
        return out

    plan.run(use_graph=True, stream=stream)
    plan_fx.run(use_graph=True, stream=stream)
    torch.cuda.synchronize()
    plan_ms = timed(lambda: plan.run(use_graph=True, stream=stream), args.reps)
    plan_fx_ms = timed(lambda: plan_fx.run(use_graph=True, stream=stream), args.reps)
    # the MSM phases after the sort as one persistent launch (eager, synchronous runs)
    plan_px.run(stream=stream)
    plan_px_ms = timed(lambda: plan_px.run(stream=stream), args.reps)

    def one_by_one():
        for s, b, o in msms:
            msm.msm(1, s, b, out=o, stream=stream)
        for d, k, di in ntts:
            ntt.ntt(d, k, di, stream=stream)

    one_by_one()
    seq_ms = timed(one_by_one, args.reps)
    # one at a time over shifted-copy tables too (built outside the timing,
    # at the width the tuning table gives tables)
    tabs = []
    for s, b, o in msms:
        n = int(s.shape[0])
        c = msm.autotune_window(1, n, precomputed=True)
        w = msm.windows_for(c)
        tabs.append((s, msm.precompute(1, b, c, w, n), c, w, n, o))

    def one_by_one_tables():
        for s, t, c, w, n, o in tabs:
            msm.msm_precomputed(1, s, t, c, w, n, out=o, stream=stream)
        for d, k, di in ntts:
            ntt.ntt(d, k, di, stream=stream)

    one_by_one_tables()
    seq_tab_ms = timed(one_by_one_tables, args.reps)
    del tabs
    # per-phase device times of one eager (uncaptured) run of each plan
    from liblightzk_b200 import _capi

    def phases_of(pl):
        _capi.trace_reset()
        _capi.trace_enable(True)
        pl.run(use_graph=False, stream=stream)
        torch.cuda.synchronize()
        _capi.trace_enable(False)
        return {ph: _capi.trace_get(f"batch_{ph}")[0] for ph in ("msm_sort", "msm_accumulate", "msm_fixup",
                                                                  "msm_reduce", "msm_finish", "msm_persistent",
                                                                  "ntt")}

    phases, phases_fx, phases_px = phases_of(plan), phases_of(plan_fx), phases_of(plan_px)
    pts = sum(int(m[0].shape[0]) for m in msms)
    elems = sum(1 << k for _, k, _ in ntts)
    med = lambda x: float(np.median(x))  # noqa: E731
    print(json.dumps({"case": "batch", "msms": len(msms), "ntts": len(ntts), "msm_points": pts,
                      "ntt_elements": elems,
                      "plan_fixed_bases_graph_ms": plan_fx_ms, "plan_graph_ms": plan_ms,
                      "plan_fixed_bases_persistent_ms": plan_px_ms,
                      "speedup_persistent": med(seq_ms) / med(plan_px_ms),
                      "one_by_one_ms": seq_ms, "one_by_one_tables_ms": seq_tab_ms,
                      "speedup": med(seq_ms) / med(plan_fx_ms),
                      "speedup_vs_one_by_one_tables": med(seq_tab_ms) / med(plan_fx_ms),
                      "speedup_plain_plan": med(seq_ms) / med(plan_ms),
                      "plan_device_bytes": plan.device_bytes(), "plan_fixed_bases_device_bytes": plan_fx.device_bytes(),
                      "phases_ms_eager": phases, "phases_ms_eager_fixed_bases": phases_fx,
                      "phases_ms_persistent": phases_px,
                      "tuning_table": table_src,
                      "tuned": {"msm_g1": {lg: {k: autotune.get_value(k, 1, lg)
                                                for k in ("window", "run", "chunk", "table_window", "table_run",
                                                          "table_chunk")}
                                           for lg in range(10, 21)},
                                "ntt_block": {lg: autotune.get_value("ntt", 0, lg) for lg in range(12, 23)}}}),
          flush=True)


def run_serve_case(args):
    """the serving workload: three resident circuits (2^16, 2^18, 2^20
    constraints, built like the benchmark circuit), requests with witnesses
    from pools of pre-solved witnesses (pinned host memory) and fresh (r, s);
    capacity under a burst, latency under Poisson arrivals, and the plain
    one-proof-at-a-time path on the same requests"""
    import torch

    from liblightzk_b200 import device, groth16, serve, synth
    logs = [16, 18, 20]
    provers, pools, circs = [], [], []
    for lg in logs:
        c = synth.Circuit(lg, seed=lg)
        pk = synth.ProvingKey(c, seed=lg + 1)
        provers.append(groth16.Prover(c, pk, mode=groth16.STANDARD, window_bits=args.window))
        pools.append([torch.from_numpy(device.to_host(c.witness(1000 + i)).view(np.int64)).pin_memory()
                      for i in range(4)])
        circs.append(c)
        del pk
    torch.cuda.synchronize()
    budget = 60 << 30
    srv = serve.Server(budget, max_inflight=args.inflight)
    cids = [srv.add(p) for p in provers]
    rs = device.to_host(synth.random_fr(2 * args.requests, 9, 55)).reshape(args.requests, 2, 4)

    def burst(which):
        srv.reset_stats()
        ids = [srv.submit(cids[w], pools[w][i % 4], rs[i, 0], rs[i, 1], pinned=True) for i, w in enumerate(which)]
        srv.wait_idle()
        for rid in ids:
            srv.poll(rid)
        return srv.stats()

    def plain(which):
        stream = torch.cuda.Stream()
        zdev = [torch.empty((c.n_vars, 4), dtype=torch.int64, device="cuda") for c in circs]
        proof = torch.empty(groth16.PROOF_WORDS, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        lat = []
        t0 = time.perf_counter()
        for i, w in enumerate(which):
            t1 = time.perf_counter()
            with torch.cuda.stream(stream):
                zdev[w].copy_(pools[w][i % 4], non_blocking=True)
            provers[w].prove(zdev[w], rs[i, 0], rs[i, 1], proof=proof, stream=stream)
            stream.synchronize()
            proof.cpu()
            lat.append((time.perf_counter() - t1) * 1e3)
        return len(which) / (time.perf_counter() - t0), lat

    rng = np.random.default_rng(4)
    mix = rng.integers(0, 3, args.requests)
    for w in range(3):                     # warm-up: one context per slot and circuit
        burst(np.full(args.inflight, w))
    cap = burst(mix)
    plain(mix[:6])
    plain_pps, plain_lat = plain(mix)
    only20 = np.full(min(args.requests, 24), 2)
    cap20 = burst(only20)
    plain20_pps, _ = plain(only20)
    sweep = {}
    for inflight in (1, 2, 3):
        s2 = serve.Server(budget, max_inflight=inflight)
        ids2 = [s2.add(p) for p in provers]
        # contexts are created on first admission: one warm-up request per
        # in-flight slot keeps their allocation out of the measured window
        warm = [s2.submit(ids2[2], pools[2][i % 4], rs[i, 0], rs[i, 1], pinned=True) for i in range(inflight)]
        s2.wait_idle()
        for rid in warm:
            s2.poll(rid)
        s2.reset_stats()
        rids = [s2.submit(ids2[2], pools[2][i % 4], rs[i, 0], rs[i, 1], pinned=True) for i in range(12)]
        s2.wait_idle()
        for rid in rids:
            s2.poll(rid)
        sweep[inflight] = s2.stats()["proofs_per_s"]
        s2.close()
    poisson = []
    for frac in (0.5, 0.85):
        rate = frac * cap["proofs_per_s"]
        st = serve.poisson_run(srv, cids, pools, rate, args.requests, seed=int(frac * 100))
        poisson.append({"offered_per_s": rate, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                        "proofs_per_s": st["proofs_per_s"], "completed": st["completed"]})
    out = {"case": "serve", "circuits": [f"2^{lg}" for lg in logs], "max_inflight": args.inflight,
           "requests": args.requests, "burst_mix": {"proofs_per_s": cap["proofs_per_s"], "p50_ms": cap["p50_ms"],
                                                   "p99_ms": cap["p99_ms"]},
           "plain_mix": {"proofs_per_s": plain_pps, "p50_ms": float(np.percentile(plain_lat, 50)),
                         "p99_ms": float(np.percentile(plain_lat, 99))},
           "served_over_plain_mix": cap["proofs_per_s"] / plain_pps,
           "burst_2e20": {"proofs_per_s": cap20["proofs_per_s"], "p50_ms": cap20["p50_ms"], "p99_ms": cap20["p99_ms"]},
           "plain_2e20_proofs_per_s": plain20_pps, "served_over_plain_2e20": cap20["proofs_per_s"] / plain20_pps,
           "poisson": poisson, "device_bytes": srv.stats()["device_bytes"],
           "inflight_sweep_2e20_proofs_per_s": sweep}
    srv.close()
    print(json.dumps(out), flush=True)


def run_tune_case(args):
    """measure the whole tuning table on this GPU and write it (--tune-out):
    plain-base MSM window, reduction run and chunk per size class (G1 and
    G2), NTT pass block per transform size, and the chunk and run of the
    benchmark prover's own MSMs, chosen by timing whole proofs"""
    from liblightzk_b200 import autotune, groth16, synth
    t0 = time.time()
    t1 = autotune.tune_msm(1, log_ns=range(10, 22), spread=2, reps=2)
    t2 = autotune.tune_msm(2, log_ns=range(10, 21), spread=1, reps=2)
    tt = autotune.tune_msm_table(1, log_ns=range(10, 21), reps=2)
    tt2 = autotune.tune_msm_table(2, log_ns=range(10, 21), spread=(4, 1), reps=2)
    tn = autotune.tune_ntt(range(10, 25), reps=2)
    circ = synth.Circuit(args.log_m, seed=1)
    pk = synth.ProvingKey(circ, seed=7)
    tp = autotune.tune_prover(circ, pk, window_bits=args.window)
    if args.tune_out:
        autotune.save(args.tune_out)
    print(json.dumps({"case": "tune", "seconds": time.time() - t0,
                      "msm_g1": {lg: {k: v[k] for k in ("window", "run", "chunk")} for lg, v in t1.items()},
                      "msm_g2": {lg: {k: v[k] for k in ("window", "run", "chunk")} for lg, v in t2.items()},
                      "msm_g1_table": {lg: {k: v[k] for k in ("window", "run", "chunk", "ms", "chunk_ms")}
                                       for lg, v in tt.items()},
                      "msm_g2_table": {lg: {k: v[k] for k in ("window", "run", "chunk", "ms", "chunk_ms")}
                                       for lg, v in tt2.items()},
                      "ntt_block": {lg: {"best": v[0], "ms": v[1]} for lg, v in tn.items()},
                      "prover_ms_per_proof": {f"chunk {c}, run {r}": ms for (c, r), ms in tp.items()}}), flush=True)


def run_case(args):
    """one operator at 2^log_n, `reps` times, for profiling (prints ms)"""
    import torch

    from liblightzk_b200 import _capi, autotune, msm, ntt, synth
    if args.case == "tune":
        return run_tune_case(args)
    if not args.no_tuning_table:
        autotune.load_default()
    if args.case == "batch":
        return run_batch_case(args)
    if args.case == "serve":
        return run_serve_case(args)
    if args.case == "reference-gpu":
        return run_reference_gpu_case(args)
    if args.case == "spmv":
        circ = synth.Circuit(args.log_n, seed=1)
        z = circ.witness(5)
        outs = [torch.zeros((circ.M, 4), dtype=torch.int64, device="cuda") for _ in range(3)]
        fn = lambda: ntt.spmv3(circ.A.desc(), circ.B.desc(), circ.C.desc(), z, *outs)  # noqa: E731
        times = []
        for _ in range(args.reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        print(json.dumps({"case": "spmv", "log_n": args.log_n, "ms": times, "bytes": spmv_bytes(circ)}), flush=True)
        return
    n = 1 << args.log_n
    sc = synth.random_fr(n, 5, 77)
    out = []
    if args.case in ("msm-g1", "msm-g2"):
        g = 1 if args.case == "msm-g1" else 2
        bases = synth.fixed_base(g, synth.random_fr(n, 5, 78))
        if args.plain:
            fn = lambda: msm.msm(g, sc, bases)  # noqa: E731   (autotuned window)
        else:
            c = args.window
            W = msm.windows_for(c)
            table = msm.precompute(g, bases, c, W, n)
            ws = torch.empty(msm.workspace_bytes(g, n, c, True, n), dtype=torch.uint8, device="cuda")
            fn = lambda: msm.msm_precomputed(g, sc, table, c, W, n, workspace=ws)  # noqa: E731
    else:
        ntt.prepare(args.log_n)
        fn = lambda: ntt.ntt(sc, args.log_n, ntt.COSET_FORWARD)  # noqa: E731
    stages = {}
    for r in range(args.reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        last = r == args.reps - 1
        if last:     # per-stage device times of the last repetition
            _capi.trace_reset()
            _capi.trace_enable(True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
        if last:
            _capi.trace_enable(False)
            if args.case in ("msm-g1", "msm-g2"):
                for st in ("sort", "accumulate", "fixup", "reduce", "finish"):
                    stages[st] = _capi.trace_get(f"msm_g{g}_{st}")[0]
    print(json.dumps({"case": args.case, "log_n": args.log_n, "window": args.window, "ms": out,
                      "stages_ms": stages}), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.case != "prove":
        run_case(args)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from liblightzk_b200 import _capi, autotune, device, groth16, msm, synth
    dev = f"cuda:{local}"
    tuning = None if args.no_tuning_table else autotune.load_default()
    # ---------------- setup (untimed) ----------------
    if args.circuit == "matmul":
        circ = synth.MatMulCircuit(args.matmul_p, device=dev)
        workload = f"groth16_prove_matmul_p{args.matmul_p}"
    else:
        circ = synth.Circuit(args.log_m, seed=1, device=dev)
        workload = f"groth16_prove_2^{args.log_m}"
    log_m = circ.log_m
    M = circ.M
    pk = synth.ProvingKey(circ, seed=7)
    mode = groth16.STANDARD if args.mode == "standard" else groth16.REFERENCE
    prover = groth16.Prover(circ, pk, mode=mode, window_bits=args.window)
    nw = 2
    wits = [circ.witness(100 + rank * 10 + i) for i in range(nw)]
    host_wits = [device.to_host(w) for w in wits]
    pinned = [torch.from_numpy(h.view(np.int64)).pin_memory() for h in host_wits]
    nsteps = args.warmup + args.steps
    rs = device.to_host(synth.random_fr(2 * nsteps, 9 + rank, 99, device=dev)).reshape(nsteps, 2, 4)
    proofs = torch.empty((nsteps, groth16.PROOF_WORDS), dtype=torch.int64, device=dev)
    torch.cuda.synchronize()

    def step(i, z):
        prover.prove(z, rs[i, 0], rs[i, 1], proof=proofs[i])

    clocks = Clocks(local)
    clocks.start()          # sampling starts during the warm-up
    for i in range(args.warmup):
        step(i, wits[i % nw])
    torch.cuda.synchronize()

    # ---------------- timed: device-resident inputs ----------------
    # only the G1 accumulation launches are traced here (for the roofline):
    # every traced region adds two timing events to its stream, and all of
    # them together cost about 1 % of a proof
    _capi.trace_reset()
    _capi.trace_only(["msm_g1_accumulate"])
    _capi.trace_enable(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = _capi.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.mark("begin")
    e0.record()
    for k in range(args.steps):
        ev[k][0].record()
        step(args.warmup + k, wits[k % nw])
        ev[k][1].record()
    e1.record()
    torch.cuda.synchronize()
    clocks.mark("end")
    launches = _capi.launch_count() - launches0
    _capi.trace_enable(False)
    ms_total = e0.elapsed_time(e1)
    lat = sorted(a.elapsed_time(b) for a, b in ev)
    acc_ms, acc_n = _capi.trace_get("msm_g1_accumulate")
    _capi.trace_only(None)
    clk = clocks.stop()

    # per-stage breakdown from a separate, untimed pass with every region traced
    nbd = 3
    _capi.trace_reset()
    _capi.trace_enable(True)
    for k in range(nbd):
        step(k % nsteps, wits[k % nw])
    torch.cuda.synchronize()
    _capi.trace_enable(False)
    bd = {name: _capi.trace_get(name)[0] / nbd
          for name in ("msm_g1", "msm_g2", "msm_g1_accumulate", "msm_g2_accumulate")}

    # ---------------- timed: end to end through host memory ----------------
    # Each step copies its witness from pinned host memory and reads its proof
    # back; the witness of step k + 1 is copied on a second stream into the
    # other of two device buffers while proof k runs (double buffering, as a
    # serving loop would), and every copy lies inside the timed region.
    zbuf = [torch.empty_like(wits[0]) for _ in range(2)]
    host_proofs = torch.empty((args.steps, groth16.PROOF_WORDS), dtype=torch.int64).pin_memory()
    main = torch.cuda.current_stream()
    cs = torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_free = [torch.cuda.Event() for _ in range(2)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(main)
    cs.wait_event(f0)
    with torch.cuda.stream(cs):
        zbuf[0].copy_(pinned[0], non_blocking=True)
        ev_in[0].record(cs)
    for k in range(args.steps):
        cur, nxt = k & 1, (k + 1) & 1
        if k + 1 < args.steps:
            with torch.cuda.stream(cs):
                if k >= 1:
                    cs.wait_event(ev_free[nxt])      # proof k - 1 has finished with that buffer
                zbuf[nxt].copy_(pinned[(k + 1) % nw], non_blocking=True)
                ev_in[nxt].record(cs)
        main.wait_event(ev_in[cur])
        p = prover.prove(zbuf[cur], rs[args.warmup + k, 0], rs[args.warmup + k, 1], proof=proofs[args.warmup + k])
        ev_free[cur].record(main)
        host_proofs[k].copy_(p, non_blocking=True)
    f1.record(main)
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1)

    # max over ranks
    if dist:
        t = torch.tensor([ms_total, e2e_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total, e2e_ms = float(t[0]), float(t[1])

    # ---------------- G1 MSM at 2^20 (precomputed table, as msm-check.cu) ----------------
    g1_ms = g1_plain_ms = g1_window = None
    iso_ms = iso_n = iso_pts = 0
    other = {}
    if rank == 0:
        n = 1 << 20
        sc = synth.random_fr(n, 5, 77, device=dev)
        bases = pk.a[:n] if pk.a.shape[0] >= n else synth.fixed_base(1, synth.random_fr(n, 5, 78, device=dev))
        # the width the tuning table gives a 2^20-point table MSM, else the prover's
        c = autotune.get_value("table_window", 1, 20) or args.window
        g1_window = c
        W = msm.windows_for(c)
        table = msm.precompute(1, bases, c, W, n)
        ws = torch.empty(msm.workspace_bytes(1, n, c, True, n), dtype=torch.uint8, device=dev)
        times = []
        for it in range(8):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            if it == 3:     # accumulation-kernel times of the measured repetitions, alone on the GPU
                _capi.trace_reset()
                _capi.trace_enable(True)
            a.record()
            msm.msm_precomputed(1, sc, table, c, W, n, workspace=ws)
            b.record()
            torch.cuda.synchronize()
            if it >= 3:
                times.append(a.elapsed_time(b))
        _capi.trace_enable(False)
        iso_ms, iso_n = _capi.trace_get("msm_g1_accumulate")
        iso_pts = n
        g1_ms = float(np.median(times))
        del table
        times = []
        for it in range(5):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            msm.msm(1, sc, bases)
            b.record()
            torch.cuda.synchronize()
            if it >= 2:
                times.append(a.elapsed_time(b))
        g1_plain_ms = float(np.median(times))

        # ---------------- the other configurations of the benchmark set ----------------
        def timed(fn, reps=5, warm=3):
            out = []
            for it in range(warm + reps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                fn()
                b.record()
                torch.cuda.synchronize()
                if it >= warm:
                    out.append(a.elapsed_time(b))
            return float(np.median(out))
        from liblightzk_b200 import ntt
        n16 = 1 << 16
        s16, b16 = sc[:n16], bases[:n16]
        other["g1_msm_2e16_plain_ms"] = timed(lambda: msm.msm(1, s16, b16))
        if pk.b2.shape[0] >= n:
            c2 = autotune.get_value("table_window", 2, 20) or args.window
            W2 = msm.windows_for(c2)
            t2 = msm.precompute(2, pk.b2[:n], c2, W2, n)
            ws2 = torch.empty(msm.workspace_bytes(2, n, c2, True, n), dtype=torch.uint8, device=dev)
            other["g2_msm_2e20_ms"] = timed(lambda: msm.msm_precomputed(2, sc, t2, c2, W2, n, workspace=ws2))
            other["g2_msm_2e20_window_bits"] = c2
            del t2, ws2
        big = synth.random_fr(1 << 24, 6, 80, device=dev)
        ntt.prepare(24)
        other["ntt_coset_fwd_2e24_ms"] = timed(lambda: ntt.ntt(big, 24, ntt.COSET_FORWARD), reps=3, warm=1)
        other["ntt_coset_inv_2e24_ms"] = timed(lambda: ntt.ntt(big, 24, ntt.COSET_INVERSE), reps=3, warm=1)
        del big
        outs = [torch.zeros((circ.M, 4), dtype=torch.int64, device=dev) for _ in range(3)]
        other["spmv3_ms"] = timed(lambda: ntt.spmv3(circ.A.desc(), circ.B.desc(), circ.C.desc(), wits[0], *outs))
        del outs

    if dist:
        dist.barrier()
    if rank != 0:
        dist.destroy_process_group()
        return

    # ---------------- roofline of the dominant kernel ----------------
    mad_chain_rate = _capi.probe_imad_rate()
    mont_rate = _capi.probe_mont_rate()
    mont_rate_int = _capi.probe_mont_rate_int()
    # the roofline's denominator: Montgomery products per second in the
    # fastest product form measured on this GPU (the FP64-pipe product with
    # operands kept as limbs), counted in the IMAD-class unit of the
    # algorithmic work (264 per product)
    imad_peak = max(mont_rate, mont_rate_int) * IMAD_PER_FP_MUL
    W = msm.windows_for(args.window)
    nl = circ.n_vars - circ.n_public - 1
    # G1 accumulation launches per proof: A, B1, and L + H as one MSM
    g1_points_per_proof = 2 * circ.n_vars + nl + (M - 1)
    g1_launches_per_proof = 3
    avg_pts = g1_points_per_proof / g1_launches_per_proof
    alg_imad = avg_pts * W * FP_MUL_PER_G1_MADD * IMAD_PER_FP_MUL
    acc_avg_ms = acc_ms / max(acc_n, 1)
    achieved = alg_imad / (acc_avg_ms * 1e-3) if acc_n else None
    traffic = pipe_util = pipe_util_probe = pipe_name = None
    prof = os.path.join(ROOT, "profiles", "msm_g1_accumulate_traffic.json")
    if os.path.exists(prof):
        try:
            tj = json.load(open(prof))
            # per average launch of this proof, scaled by its points from the
            # captured launch (traffic grows with the entries)
            traffic = tj["bytes_per_launch_at_2e20"] * avg_pts / tj["points_at_2e20"]
            # ncu's activity of the pipe that binds the products (FP64) in
            # that launch and in the product probe that sets `peak`
            if tj.get("pipe_active_pct") is not None:
                pipe_name = tj["pipe"]
                pipe_util = tj["pipe_active_pct"] / 100.0
                pipe_util_probe = tj["pipe_active_pct_probe"] / 100.0
        except Exception:
            traffic = pipe_util = pipe_util_probe = pipe_name = None

    iso_line = None
    if iso_n:
        iso_alg = iso_pts * msm.windows_for(g1_window) * FP_MUL_PER_G1_MADD * IMAD_PER_FP_MUL
        iso_avg = iso_ms / iso_n
        iso_line = {"workload": f"G1 MSM 2^{int(np.log2(iso_pts))} alone", "avg_launch_ms": iso_avg,
                    "launches": iso_n, "achieved": iso_alg / (iso_avg * 1e-3) / 1e12,
                    "frac": iso_alg / (iso_avg * 1e-3) / imad_peak,
                    "traffic_bytes": traffic * iso_pts / (avg_pts if avg_pts else 1) if traffic else None,
                    "algorithmic_imad_per_launch": iso_alg}

    rooflines_other = {}
    hbm, hbm_src = hbm_peak_gbs()
    if "ntt_coset_fwd_2e24_ms" in other:
        imad, nbytes = ntt_algorithmic(24)
        t = other["ntt_coset_fwd_2e24_ms"] * 1e-3
        rooflines_other["ntt_coset_fwd_2e24"] = {
            "ms": other["ntt_coset_fwd_2e24_ms"], "imad_achieved_T": imad / t / 1e12,
            "imad_frac": imad / t / imad_peak, "hbm_gbs": nbytes / t / 1e9, "hbm_frac": nbytes / t / 1e9 / hbm,
            "bound": "int"}
    if "spmv3_ms" in other:
        nbytes = spmv_bytes(circ)
        t = other["spmv3_ms"] * 1e-3
        rooflines_other["spmv3_2e20"] = {"ms": other["spmv3_ms"], "bytes": nbytes, "hbm_gbs": nbytes / t / 1e9,
                                         "hbm_frac": nbytes / t / 1e9 / hbm, "bound": "hbm"}
    if rooflines_other:
        rooflines_other["hbm_peak_gbs"] = hbm
        rooflines_other["hbm_peak_source"] = hbm_src

    proofs_s = world * args.steps / (ms_total * 1e-3)
    line = {
        "metric": METRIC, "value": proofs_s, "unit": "proofs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 limbs (Fr/Fq mod p, Montgomery)",
        "data": "synthetic (seeded R1CS, witness and proving key generated on the device)",
        "config": {"workload": workload, "constraints": M, "variables": circ.n_vars,
                   "public_inputs": circ.n_public, "prove_mode": args.mode, "msm_window_bits": args.window,
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (GB-scale key tables)",
                   "tuning_table": os.path.relpath(tuning, ROOT) if tuning else "built-in defaults"},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "mean": float(np.mean(lat))},
        "g1_msm_2e20_ms": g1_ms, "g1_msm_2e20_window_bits": g1_window, "g1_msm_2e20_plain_ms": g1_plain_ms,
        "other_configs_ms": other,
        "rooflines_other": rooflines_other,
        "e2e": {"value": world * args.steps / (e2e_ms * 1e-3), "unit": "proofs/s",
                "h2d_bytes_per_step": int(wits[0].numel() * 8), "d2h_bytes_per_step": groth16.PROOF_WORDS * 8},
        "gpu_launches": launches,
        # the dominant kernel timed alone, on the metric's own G1 MSM 2^20
        # (CUDA events around each accumulation launch, nothing else on the
        # GPU); inside a proof the same kernel shares the GPU with three other
        # streams, so its event time there measures the interleaving as much
        # as the kernel (reported as in_proof)
        "roofline": {"kernel": "k_accumulate<Fq> (G1 bucket accumulation)", "bound": "int",
                     "workload": iso_line["workload"] if iso_line else None,
                     "achieved": iso_line["achieved"] if iso_line else None, "peak": imad_peak / 1e12,
                     "unit": "T IMAD/s", "frac": iso_line["frac"] if iso_line else None,
                     "traffic": iso_line["traffic_bytes"] if iso_line else None,
                     "peak_source": "measured: lzk_probe_mont_rate (independent Fq Montgomery products on the "
                                    "FP64 pipe, operands kept as radix-2^52 limbs, full occupancy; the faster of "
                                    "it and the 32-bit-limb integer form) x 264 IMAD-class per product",
                     "mont_products_per_s": mont_rate, "mont_products_per_s_int_form": mont_rate_int,
                     "pipe": pipe_name, "pipe_util": pipe_util, "pipe_util_probe": pipe_util_probe,
                     "pipe_util_source": "ncu sm__pipe_fp64_cycles_active of one G1 accumulation launch at 2^20 "
                                         "and of the probe (profiles/k_accumulate_2e20.md)",
                     "peak_mad_chains_T": mad_chain_rate / 1e12,
                     "algorithmic_imad_per_launch": iso_line["algorithmic_imad_per_launch"] if iso_line else None,
                     "avg_launch_ms": iso_line["avg_launch_ms"] if iso_line else None,
                     "launches": iso_line["launches"] if iso_line else None,
                     "in_proof": {"achieved": achieved / 1e12 if achieved else None,
                                  "frac": (achieved / imad_peak) if achieved else None,
                                  "algorithmic_imad_per_launch": alg_imad, "avg_launch_ms": acc_avg_ms,
                                  "launches": acc_n, "traffic": traffic,
                                  "timing": "CUDA events around each launch inside the timed proofs; the three "
                                            "G1 MSMs of a proof (A, B1, and L + H as one) overlap each other and "
                                            "the G2 MSM on four streams, so a launch shares the GPU"}},
        # sums of per-call device times (a separate traced pass of 3 proofs);
        # calls on different streams overlap
        "breakdown_ms_per_proof": bd,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_reference_sample(log_m, circ.n_vars, nl)
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
