#!/usr/bin/env python
"""Benchmark of the ADMIXTURE hot path on B200: one step = one quasi-Newton iteration of
admixture_qn! (2 Q + 2 P SQP updates, 2 log-likelihood passes, ZAL extrapolation,
accept/reject) over a seeded synthetic cohort.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c5] [--impl ours|reference]

Metric: genotype*K^2/s per iteration (I*J*K^2 / seconds per iteration), whole job, of the chosen
(mixed-precision) form, with the plain FP64 form's iteration timed beside it.  Also reported:
time to converge (rtol 1e-7) of the chosen form from the learned warm start and from the random
start + 5 EM, and of the plain FP64 form from the random start + 5 EM (1 GPU), scored against
the plain solve's log-likelihood; per-pass device times, the roofline of the dominant kernel,
an end-to-end number through the C ABI with host buffers, and the oracle (CPU restatement)
timed on the host cores.  Default workload: I=200000, J=500000, K=8 (25 GB packed genotypes).

Multi-GPU (torchrun): every rank solves its own cohort (seed = rank) -- independent problems,
no collective on the data path; timing is the max over ranks (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "oracle"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

METRIC = "genotype*K^2/s per iteration (chosen form; plain FP64 form timed beside it), 1 B200"
UNIT = "genotype*K^2/s"


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c5")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="mixed", choices=["plain", "mixed"],
                    help="plain: FP64 sweeps; mixed: tensor-core BF16 Hessian, FP32 gradient")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ttc", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain FP64 form beside the chosen one")
    ap.add_argument("--stream-block", type=int, default=None,
                    help="keep the genotypes in host memory and stream SNP blocks of this size (out-of-core "
                         "handle); times the iteration only")
    ap.add_argument("--I", type=int, default=None, help="override the configuration's I (--pass-only runs)")
    ap.add_argument("--J", type=int, default=None, help="override the configuration's J (--pass-only runs)")
    ap.add_argument("--precision", action="store_true",
                    help="report the mixed form's errors against the FP64 form (default for c3)")
    ap.add_argument("--cpu-ttc", action="store_true",
                    help="also time the oracle to convergence on the whole cohort (default for c1)")
    ap.add_argument("--skfr", type=int, default=None, metavar="SPARSITY",
                    help="time the SKFR AIM pre-selection (admix_skfr) with this sparsity on the cohort instead")
    ap.add_argument("--skfr-mode", default="global", choices=["global", "local"])
    ap.add_argument("--skfr-cpu", action="store_true",
                    help="also time the SKFR oracle on the same cohort and check the result (default for c1)")
    ap.add_argument("--pass-only", default=None,
                    choices=["loglik", "q_sweep", "p_sweep", "q_qp", "p_qp", "em"],
                    help="set up the cohort and launch one pass warmup+steps times (for profilers)")
    return ap.parse_args()


def run_pass_only(args):
    """One pass of the hot path launched 1 + steps times on the cohort (no EM, no QN loop):
    the command the per-kernel ncu captures run."""
    import torch
    import openadmixture_b200 as oa
    from openadmixture_b200 import _native as N
    torch.cuda.set_device(0)
    spec = oa.COHORTS[args.config].scaled(I=args.I, J=args.J)
    if spec.I * spec.J > 2_000_000_000:
        qt, pt = oa.truth(spec)
        g = oa.genotypes_device(spec, qt, pt)
    else:
        g, _, _ = oa.make_cohort(spec)
    d = oa.AdmixData(spec.I, spec.J, spec.K, 3, rng=100)
    flags = oa.ADMIX_FLAG_MIXED if args.form == "mixed" else 0
    with oa.CuAdmixData(d, g, flags=flags) as d_cu:
        pid = {"loglik": N.ADMIX_PASS_LOGLIK, "q_sweep": N.ADMIX_PASS_QSWEEP, "p_sweep": N.ADMIX_PASS_PSWEEP,
               "q_qp": N.ADMIX_PASS_QQP, "p_qp": N.ADMIX_PASS_PQP, "em": N.ADMIX_PASS_EM}[args.pass_only]
        if pid in (N.ADMIX_PASS_QQP, N.ADMIX_PASS_PQP):   # give the QPs real sweep outputs
            d_cu.time_pass(N.ADMIX_PASS_QSWEEP if pid == N.ADMIX_PASS_QQP else N.ADMIX_PASS_PSWEEP, 1)
        ms = d_cu.time_pass(pid, max(1, args.steps))
    print(json.dumps({"pass": args.pass_only, "config": spec.name, "I": spec.I, "J": spec.J, "K": spec.K,
                      "form": args.form, "ms_per_launch": ms}), flush=True)
    return 0


def run_skfr(args):
    """SKFR AIM pre-selection on the cohort (the step run_admixture runs when `sparsity` is given):
    warmup + steps calls of admix_skfr on one handle, each timed on the host clock around the call
    (the call is host-orchestrated: k-means++ draws and one convergence count per iteration cross to
    the host), the median reported.  With --skfr-cpu (default for c1) the oracle runs the same
    selection on the host and the device result is checked against it."""
    import ctypes as C
    import torch
    import numpy as np
    import openadmixture_b200 as oa
    from openadmixture_b200 import _native as N
    torch.cuda.set_device(0)
    spec = oa.COHORTS[args.config].scaled(I=args.I, J=args.J)
    qt, pt = oa.truth(spec)
    g = oa.genotypes_device(spec, qt, pt)
    K, s, local = spec.K, int(args.skfr), args.skfr_mode == "local"
    cap = min(spec.J, s * (K if local else 1))
    seed = 7
    d = oa.AdmixData(spec.I, spec.J, K, 1, rng=0)
    times = []
    with oa.CuAdmixData(d, g) as h:
        for rep in range(max(0, args.warmup) + max(1, args.steps)):
            cl = np.empty(spec.I, np.int32)
            aims = np.empty(max(cap, 1), np.int32)
            n, obj, it = C.c_int64(0), C.c_double(0.0), C.c_int32(0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            h._chk(N.admix_lib().admix_skfr(h.handle, K, s, N.ADMIX_SKFR_LOCAL if local else N.ADMIX_SKFR_GLOBAL, 50, 1,
                                            seed, N.i32ptr(cl), N.i32ptr(aims), cap, C.byref(n), C.byref(obj),
                                            C.byref(it)))
            torch.cuda.synchronize()
            if rep >= args.warmup:
                times.append(time.perf_counter() - t0)
    true = np.argmax(qt, axis=1)
    purity = float(sum(np.bincount(true[cl == k], minlength=K).max() for k in range(K) if (cl == k).any()) / spec.I)
    sec = float(np.median(times))
    out = {"skfr": args.skfr_mode, "config": spec.name, "I": spec.I, "J": spec.J, "K": K, "sparsity": s,
           "s_per_run": sec, "runs": len(times), "s_runs": [round(t, 4) for t in times], "iterations": it.value, "ms_per_iteration": 1e3 * sec / it.value,
           "n_aims": n.value, "objective": obj.value, "purity_vs_truth": purity, "seed": seed}
    if args.skfr_cpu or args.config == "c1":
        import skfr_oracle as S
        host = g.to_host()
        t0 = time.perf_counter()
        c_o, a_o, obj_o, it_o = S.skfr(np.asarray(host.data), spec.I, K, s, mode=args.skfr_mode, seed=seed)
        cpu = time.perf_counter() - t0
        out["cpu_oracle"] = {"s_per_run": cpu, "cores": 1, "kind": "port",
                             "identical": bool(np.array_equal(c_o, cl) and np.array_equal(a_o, aims[: n.value])
                                               and it_o == it.value and abs(obj_o - obj.value) <= 1e-12 * abs(obj_o))}
    print(json.dumps(out), flush=True)
    return 0


def max_over_ranks(value: float, world: int, device: str) -> float:
    """The largest value over all ranks (device-timed milliseconds: the job's time is its
    slowest rank's).  One collective on every rank when world > 1."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _peaks():
    """(HBM GB/s, burst bf16 TFLOP/s, sustained bf16 TFLOP/s, 'measured' | 'fallback')"""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        burst = float(d["bf16_tflops"])
        return float(d["hbm_gbs"]), burst, float(d.get("bf16_tflops_sustained", burst)), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def _traffic(kernel: str, config: str):
    """DRAM bytes per launch from a committed ncu summary (profiles/traffic.txt), if any."""
    f = ROOT / "profiles" / "traffic.txt"
    if not f.exists():
        return None
    for ln in f.read_text().splitlines():
        if ln.startswith("#") or "=" not in ln:
            continue
        kv = dict(x.split("=", 1) for x in ln.split())
        if kv.get("kernel") == kernel and kv.get("config") == config:
            return float(kv["dram_bytes_per_launch"])
    return None


def _cpu_sample_J(spec, cells=2e8):
    """SNP subset for the CPU runs: about `cells` genotype cells per pass."""
    return int(max(200, min(spec.J, cells / spec.I)))


def cpu_baseline(oa, spec, steps=5):
    """The oracle (C restatement, OpenMP on all host cores) on a bounded SNP sample of the
    same cohort: QN iterations from an EM-primed start, metric scaled by the sample."""
    import oracle
    J_s = _cpu_sample_J(spec)
    s = spec.scaled(J=J_s)
    g, _, _ = oa.make_cohort(s)
    x0 = oa.init_x(s.I, s.J, s.K, 5)
    r = oracle.OracleRun(g.data, s.I, s.J, s.K, 3, x0)
    r.init_em(1)
    times = []
    for it in range(1, steps + 1):
        t0 = time.perf_counter()
        r.qn_iteration(it)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return {"value": s.I * s.J * s.K ** 2 / t, "unit": UNIT, "cores": oracle.num_threads(), "kind": "port",
            "sample": f"oracle admixture_qn iteration on I={s.I}, J={s.J} (SNP subset), K={s.K}; "
                      f"median of {steps} iterations, {t:.2f} s each"}


def cpu_ttc(oa, g, spec, seed):
    """Time to converge of the oracle on the whole cohort from the random start the GPU legs use
    (init_x(seed), 5 EM iterations, then admixture_qn! to reldiff < 1e-7): the reference's CPU
    path restated, on all host cores."""
    import oracle
    x0 = oa.init_x(spec.I, spec.J, spec.K, seed)
    host = g.to_host() if hasattr(g, "to_host") else g
    t0 = time.perf_counter()
    r = oracle.OracleRun(host.data, spec.I, spec.J, spec.K, 3, x0)
    r.init_em(5)
    hist, conv = r.admixture_qn(1000, 1e-7)
    secs = time.perf_counter() - t0
    return {"seconds": secs, "iterations": int(len(hist)), "converged": bool(conv), "final_ll": float(r.ll_new),
            "cores": oracle.num_threads(), "kind": "port",
            "start": f"init_x(seed={seed}) + 5 EM, rtol 1e-7 (the GPU legs' start)"}


def _row_rel(a, b):
    import numpy as np
    a = a.reshape(a.shape[0], -1); b = b.reshape(b.shape[0], -1)
    scale = np.abs(b).max(axis=1, keepdims=True)
    return np.max(np.abs(a - b) / np.maximum(scale, 1e-300), axis=1)


def precision_report(oa, g, spec, x, ll):
    """Error of the mixed form against the FP64 form at one point (x, an EM-primed start):
    Q- and P-side gradients and Hessians (relative to the largest entry of each problem's row;
    max and median over problems), the signed relative bias of the Hessian diagonals, and the
    mixed form's in-iteration log-likelihoods against the FP64 pass at the points they were taken."""
    import numpy as np
    out = {}
    d = oa.AdmixData(spec.I, spec.J, spec.K, 3, rng=0)
    with oa.CuAdmixData(d, g) as h64, oa.CuAdmixData(d, g, flags=oa.ADMIX_FLAG_MIXED) as hmx:
        for h in (h64, hmx):
            h.upload(oa.X, x)
        for side in ("q", "p"):
            H0, z0 = getattr(h64, f"grad_hess_{side}")(oa.X, oa.X)
            H1, z1 = getattr(hmx, f"grad_hess_{side}")(oa.X, oa.X)
            gz, gh = _row_rel(z1, z0), _row_rel(H1, H0)
            dg0 = np.diagonal(H0, axis1=1, axis2=2)
            dg1 = np.diagonal(H1, axis1=1, axis2=2)
            bias = (dg1 - dg0) / dg0
            out[f"grad_{side}"] = {"max": float(gz.max()), "median": float(np.median(gz))}
            out[f"hess_{side}"] = {"max": float(gh.max()), "median": float(np.median(gh))}
            out[f"hess_{side}_diag_bias"] = {"mean": float(bias.mean()), "max_abs": float(np.abs(bias).max())}
            del H0, H1
        d.x[:] = x
        d.ll_new = ll
        recs = oa.admixture_qn(d, g, 1, 0.0, d_cu=hmx, quiet=True)
        ll_b, ll_q = hmx.loglik(oa.X_NEXT2), hmx.loglik(oa.X_TMP)     # admix_loglik: the FP64 pass
        out["loglik_basic_rel"] = float((recs[-1]["ll_basic"] - ll_b) / abs(ll_b))
        out["loglik_qn_rel"] = float((recs[-1]["ll_qn"] - ll_q) / abs(ll_q))
    out["note"] = ("mixed vs FP64 form at the EM-primed start; loglik_*_rel: signed relative error of the "
                   "mixed in-iteration log-likelihood against the FP64 pass at the same point")
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import oracle
    import openadmixture_b200 as oa
    spec = oa.COHORTS[args.config]
    J_s = _cpu_sample_J(spec)
    s = spec.scaled(J=J_s)
    g, _, _ = oa.make_cohort(s)
    r = oracle.OracleRun(g.data, s.I, s.J, s.K, 3, oa.init_x(s.I, s.J, s.K, 5))
    r.init_em(1)
    it = 0
    for _ in range(args.warmup):
        it += 1
        r.qn_iteration(it)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        it += 1
        r.qn_iteration(it)
    dt = (time.perf_counter() - t0) / args.steps
    value = s.I * s.J * s.K ** 2 / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{spec.name}: I={spec.I} J={spec.J} K={spec.K} (timed on a SNP subset J={J_s})",
                   "I": spec.I, "J": spec.J, "K": spec.K},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": oracle.num_threads(), "kind": "port",
                         "sample": f"oracle (C restatement of the Julia loops; Julia is not installed) "
                                   f"QN iterations on I={s.I}, J={J_s}, K={s.K}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _leg(r: dict, extra: dict | None = None) -> dict:
    out = {k: r[k] for k in ("iterations", "seconds", "iterations_to_target", "seconds_to_target")}
    out["final_ll_fp64"] = r["ll"]
    out.update(extra or {})
    return out


def _hit(r: dict, target: float):
    """first (iteration, seconds) of a run's trace at or above target"""
    return next(((it, t) for it, ll, t in r["trace"] if ll >= target), (None, None))


def ttc_legs(oa, g, spec, rank, world, mixed: bool, plain: bool) -> dict:
    """Time to converge (reldiff < 1e-7, admixture_qn's test) from the start of initialisation:
    the chosen form from the learned warm start (sketch + MLP + closed-form P step + LEARNED_EM EM; when a
    model for K applies) and from the random start + 5 EM iterations; with plain=True also the
    plain FP64 form from the random start + 5 EM, whose final log-likelihood sets the target
    (within 1e-6 relative) that every leg is scored against.  Wall-clock seconds with the device
    synchronised at both ends: the runs include the host-side control of every iteration."""
    import torch
    from openadmixture_b200 import warmstart as ws
    K, seed = spec.K, 100 + rank
    flags = oa.ADMIX_FLAG_MIXED if mixed else 0
    legs = {}
    model = ws.load_default(K) if mixed else None
    ws_info = {}
    if model is not None:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        start = ws.learned_start(g, K, model, info=ws_info)
        t_pred = time.perf_counter() - t0
        if start is not None:
            r = ws.run_to_target(g, K, flags=flags, start=start, rng=seed)
            r["seconds"] += t_pred
            r["trace"] = [(it, ll, t + t_pred) for it, ll, t in r["trace"]]
            r["predict_seconds"] = t_pred
            legs["chosen_learned"] = r
    legs["chosen_random_em5"] = ws.run_to_target(g, K, flags=flags, rng=seed)
    if plain:
        legs["plain_fp64_random_em5"] = ws.run_to_target(g, K, flags=0, rng=seed)
    chosen = "chosen_learned" if "chosen_learned" in legs else "chosen_random_em5"
    out = {"criterion": "reldiff < 1e-7; seconds from the start of initialisation (wall clock, device "
                        "synchronised at both ends)",
           "warm_start_check": ws_info,
           "chosen": chosen, "form": ("mixed" if mixed else "plain-fp64")
           + (" + learned warm start" if chosen == "chosen_learned" else " + random start, 5 EM")}
    ref = legs.get("plain_fp64_random_em5")
    for name, r in legs.items():
        extra = {"predict_seconds": r["predict_seconds"]} if "predict_seconds" in r else {}
        if ref is not None:
            target = ref["ll"] - 1e-6 * abs(ref["ll"])
            r["iterations_to_target"], r["seconds_to_target"] = _hit(r, target)
            extra["final_ll_rel_vs_plain"] = abs(r["ll"] - ref["ll"]) / abs(ref["ll"])
            # the converged Q and P against the plain FP64 solve (same start for the random legs;
            # population labels can differ for the learned start, so only the random legs compare)
            if name != "chosen_learned":
                extra["final_q_maxabs_vs_plain"] = float(abs(r["x"][: g.I] - ref["x"][: g.I]).max())
                extra["final_p_maxabs_vs_plain"] = float(abs(r["x"][g.I:] - ref["x"][g.I:]).max())
        else:
            r["iterations_to_target"] = r["seconds_to_target"] = None
        out[name] = _leg(r, extra)
    if ref is not None:
        c = legs[chosen]
        out["target_rel"] = 1e-6
        out["chosen_within_target"] = abs(c["ll"] - ref["ll"]) <= 1e-6 * abs(ref["ll"])
        out["speedup_vs_plain"] = ref["seconds"] / c["seconds"]
        if c["seconds_to_target"] and ref["seconds_to_target"]:
            out["speedup_vs_plain_to_target"] = ref["seconds_to_target"] / c["seconds_to_target"]
    if chosen == "chosen_learned":
        out["learned_vs_random_start"] = legs["chosen_random_em5"]["seconds"] / legs[chosen]["seconds"]
    return out


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist
    import openadmixture_b200 as oa
    from openadmixture_b200 import _native as N

    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    spec = oa.COHORTS[args.config].scaled(seed=rank)
    t0 = time.perf_counter()
    if spec.I * spec.J > 2_000_000_000:          # large cohorts: draw the genotypes on the GPU
        qt, pt = oa.truth(spec)
        g = oa.genotypes_device(spec, qt, pt)
    else:
        g, _, _ = oa.make_cohort(spec)
    if args.stream_block:                        # out-of-core: the genotypes live in host memory
        gd = g
        g = oa.Genotypes(gd.data.cpu().numpy() if hasattr(gd.data, "cpu") else gd.data, spec.I, spec.J)
        del gd
        torch.cuda.empty_cache()
        args.no_ttc = args.no_plain = args.no_cpu_baseline = True
    t_gen = time.perf_counter() - t0
    d = oa.AdmixData(spec.I, spec.J, spec.K, 3, rng=100 + rank)
    x_init = d.x.copy()
    t0 = time.perf_counter()
    flags = oa.ADMIX_FLAG_MIXED if args.form == "mixed" else 0
    d_cu = oa.CuAdmixData(d, g, flags=flags, stream_block=args.stream_block)
    t_upload = time.perf_counter() - t0
    oa.init_em(d, g, 5, d_cu=d_cu, quiet=True)
    x_em, ll_em = d.x.copy(), d.ll_new
    precision = None
    if (args.precision or args.config == "c3") and args.form == "mixed" and not args.stream_block:
        precision = precision_report(oa, g, spec, x_em, ll_em)
    d_cu.upload(oa.X, x_em)
    d_cu.set_ll(ll_em)
    lib = N.admix_lib()
    stream = torch.cuda.ExternalStream(d_cu.stream())
    info = N.IterInfo()
    it = 0
    for _ in range(args.warmup):
        it += 1
        d_cu._chk(lib.admix_qn_iteration(d_cu.handle, it, C_byref(info)))
    n_kern = d_cu.iteration_kernels()

    clocks = ClockSampler(local_rank)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        it += 1
        d_cu._chk(lib.admix_qn_iteration(d_cu.handle, it, C_byref(info)))
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms_max = max_over_ranks(ms, world, "cuda")
    work = spec.I * spec.J * spec.K ** 2
    value = world * work * args.steps / (ms_max / 1e3)

    # per-pass device times (live, CUDA events on the engine's stream)
    passes = {}
    for name, pid in (("loglik", N.ADMIX_PASS_LOGLIK), ("q_sweep", N.ADMIX_PASS_QSWEEP),
                      ("p_sweep", N.ADMIX_PASS_PSWEEP), ("q_qp", N.ADMIX_PASS_QQP), ("p_qp", N.ADMIX_PASS_PQP)):
        passes[name] = d_cu.time_pass(pid, 5)
    per_iter = {k: 2 * v for k, v in passes.items()}
    dom = max(per_iter, key=per_iter.get)
    mx = args.form == "mixed"
    kern_name = {"loglik": "k_loglik_mixed" if mx else "k_loglik_f64",
                 "q_sweep": "k_sweep_q_mixed" if mx else "k_sweep_q_f64",
                 "p_sweep": "k_sweep_p_mixed" if mx else "k_sweep_p_f64",
                 "q_qp": "k_qp", "p_qp": "k_qp"}[dom]
    Ib = (spec.I + 3) // 4
    K = spec.K
    bytes_bed = Ib * spec.J
    # algorithmic bytes per launch: the packed genotypes + the Q/P inputs + outputs
    alg_bytes = {
        "loglik": bytes_bed + 8 * K * (spec.I + spec.J),
        "q_sweep": bytes_bed + 8 * K * (spec.I + spec.J) + 8 * (K * (K + 1) // 2 + K) * spec.I,
        "p_sweep": bytes_bed + 8 * K * (spec.I + spec.J) + 8 * (K * (K + 1) // 2 + K) * spec.J,
        "q_qp": 8 * (K * (K + 1) // 2 + 2 * K) * spec.I + 8 * K * spec.I,
        "p_qp": 8 * (K * (K + 1) // 2 + 2 * K) * spec.J + 8 * K * spec.J,
    }
    flops = {   # reference full-K^2 form (cell counts x ops), for context
        "q_sweep": 2 * spec.I * spec.J * (2 * K * K + 2 * K) + 2 * spec.I * spec.J * K,
        "p_sweep": 2 * spec.I * spec.J * (K * K + K) + 2 * spec.I * spec.J * K,
        "loglik": 2 * spec.I * spec.J * K,
    }
    hbm, bf16, bf16_sus, peak_kind = _peaks()
    achieved = alg_bytes[dom] / (passes[dom] / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": kern_name, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_kind": peak_kind,
            "traffic": _traffic(kern_name, spec.name),
            "alg_bytes_per_launch": alg_bytes[dom], "launch_ms": passes[dom]}
    T = K * (K + 1) // 2
    if mx and dom in ("q_sweep", "p_sweep"):
        terms = 2 if dom == "q_sweep" else 1          # [W1 | W2] x [PP ; PbPb]  or  C x QQ
        roof["tensor_tflops"] = 2 * spec.I * spec.J * terms * T / (passes[dom] / 1e3) / 1e12
        roof["tensor_peak_tflops"] = bf16_sus
        roof["tensor_frac"] = roof["tensor_tflops"] / bf16_sus
        roof["note"] = ("mixed form: the Hessian contraction runs on tcgen05 (tensor_tflops against the "
                        "sustained bf16 peak: tensor_frac); the sweep is bound by the per-chunk hand-offs "
                        "between the producer warps' FP32 cell work, the controller's MMA issue and the "
                        "tensor core (issue activity about 55 %), not by HBM or the tensor pipe; frac is the "
                        "HBM fraction of its packed-genotype stream")
    if args.stream_block:
        # 6 genotype passes per iteration, each streamed host -> device once
        roof["stream_h2d_gbs"] = 6 * bytes_bed / (ms_max / args.steps / 1e3) / 1e9
        roof["note"] = ("out-of-core handle: every pass streams the packed genotypes from page-locked host "
                        "memory; stream_h2d_gbs is the host-to-device rate the iteration sustained")
    elif not mx and dom in flops:
        roof["fp64_tflops"] = flops[dom] / (passes[dom] / 1e3) / 1e12
        roof["note"] = ("FP64 plain form: the sweep is bound by the FP64 pipe, not HBM; frac is the HBM "
                        "fraction of its packed-genotype stream")

    # end-to-end through the C ABI with host buffers (pinned), H2D + D2H inside the timed region
    qh = torch.from_numpy(np.ascontiguousarray(x_em[: spec.I])).pin_memory()
    ph = torch.from_numpy(np.ascontiguousarray(x_em[spec.I:])).pin_memory()
    qo = torch.empty_like(qh).pin_memory(); po = torch.empty_like(ph).pin_memory()
    import ctypes as C
    dp = lambda t_: C.cast(C.c_void_p(t_.data_ptr()), C.POINTER(C.c_double))
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True); f1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(3, args.steps // 2)
    f0.record(stream)
    for _ in range(e2e_steps):
        it += 1
        d_cu._chk(lib.admix_set_x(d_cu.handle, oa.X, dp(qh), dp(ph)))
        d_cu._chk(lib.admix_qn_iteration(d_cu.handle, it, C_byref(info)))
        d_cu._chk(lib.admix_get_x(d_cu.handle, oa.X, dp(qo), dp(po)))
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1) / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, world, "cuda")
    xbytes = 8 * K * (spec.I + spec.J)

    d_cu.close()          # frees its copy of the genotypes before the time-to-converge legs

    # time to converge (rtol 1e-7): the chosen form from its own start, the plain FP64 form from
    # the random start + 5 EM iterations
    ttc = None
    if not args.no_ttc:
        ttc = ttc_legs(oa, g, spec, rank, world, mx, plain=mx and not args.no_plain and world == 1)

    # the plain FP64 form's iteration on the same cohort and start, for the per-iteration ratio
    vs_plain = None
    if mx and not args.no_plain:
        with oa.CuAdmixData(d, g, flags=0) as hp:
            hp.upload(oa.X, x_em)
            hp.set_ll(ll_em)
            sp_ = torch.cuda.ExternalStream(hp.stream())
            ps = 3
            hp._chk(lib.admix_qn_iteration(hp.handle, 1, C_byref(info)))
            torch.cuda.synchronize()
            h0 = torch.cuda.Event(enable_timing=True); h1 = torch.cuda.Event(enable_timing=True)
            h0.record(sp_)
            for w in range(2, 2 + ps):
                hp._chk(lib.admix_qn_iteration(hp.handle, w, C_byref(info)))
            h1.record(sp_)
            torch.cuda.synchronize()
            plain_ms = h0.elapsed_time(h1) / ps
            vs_plain = {"plain_ms_per_step": plain_ms, "plain_value": world * work / (plain_ms / 1e3),
                        "speedup_per_iteration": plain_ms / (ms_max / args.steps)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(oa, spec)
        if args.cpu_ttc or args.config == "c1":
            cpu["ttc"] = cpu_ttc(oa, g, spec, 100 + rank)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32+f64" if mx else "f64", "data": "synthetic",
        "config": {"workload": f"{spec.name}: admixture_qn iteration, I={spec.I} J={spec.J} K={spec.K}, "
                               f"{spec.miss:.1%} missing, "
                               + ("mixed form: tcgen05 BF16 Hessians, FP32 gradients and loglik cells, FP64 "
                                  "reductions / QPs / QN" if mx else "plain FP64 form"),
                   "I": spec.I, "J": spec.J, "K": spec.K, "Q": 3, "form": "mixed" if mx else "plain-fp64",
                   "l2": f"inputs larger than L2: {bytes_bed / 1e6:.0f} MB packed genotypes streamed per pass",
                   "per_rank": "independent cohort per rank (seed = rank)",
                   "genotypes": (f"host memory, streamed in blocks of {args.stream_block} SNPs" if args.stream_block
                                 else "device-resident")},
        "e2e": {"value": world * work / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": xbytes,
                "d2h_bytes_per_step": xbytes + 0, "ms_per_step": e2e_ms,
                "path": "admix_set_x(host q,p) + admix_qn_iteration + admix_get_x(host q,p)"},
        "gpu_launches": n_kern * args.steps,
        "roofline": roof,
        "passes_ms": passes,
        "ttc": ttc,
        "precision": precision,
        "vs_plain": vs_plain,
        "setup_s": {"generate": t_gen, "create_upload": t_upload},
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def C_byref(x):
    import ctypes
    return ctypes.byref(x)


BATCH_RESTARTS, BATCH_KS = 64, tuple(range(2, 13))


def run_batch(args, rank, world, local_rank):
    """The batching configuration: one batch of 64 random restarts at K=6 plus a K sweep
    K=2..12 over one cohort (I=20000, J=50000), advanced together -- one graph launch per batch
    iteration, work split chosen by the autotuner.  A step is one batch iteration (every member
    one admixture_qn! iteration); value = sum over members of I*J*K^2 per second.  Beside it:
    the same members' solo iterations one after another (the reference's one-run-per-call
    usage), and time to converge of the whole batch from the random starts + 5 EM."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import openadmixture_b200 as oa

    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    spec = oa.COHORTS[args.config].scaled(seed=rank)
    qt, pt = oa.truth(spec)
    g = oa.genotypes_device(spec, qt, pt)
    Ks = [spec.K] * BATCH_RESTARTS + list(BATCH_KS)
    seeds = list(range(BATCH_RESTARTS)) + [0] * len(BATCH_KS)
    flags = oa.ADMIX_FLAG_MIXED if args.form == "mixed" else 0
    work = sum(spec.I * spec.J * K * K for K in Ks)
    b = oa.AdmixBatch(g, Ks, flags=flags, seeds=seeds)
    t0 = time.perf_counter()
    divisor, probe_ms = b.autotune()
    t_tune = time.perf_counter() - t0
    b.init_em(5)
    b.run_qn(args.warmup, 0.0)                         # rtol 0: no member leaves
    clocks = ClockSampler(local_rank)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    rec = b.run_qn(args.steps, 0.0)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(rec["ms_device"], world, "cuda")
    value = world * work * args.steps / (ms / 1e3)

    # end to end through the public API: every member's q, p from pinned host memory, one batch
    # iteration, every member's q, p back (all calls synchronous; wall clock)
    hx = [torch.from_numpy(np.ascontiguousarray(b.x(m))).pin_memory() for m in range(len(Ks))]
    ho = [torch.empty_like(x).pin_memory() for x in hx]
    e2e_steps = max(2, args.steps // 3)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    for _ in range(e2e_steps):
        for m, mem in enumerate(b.members):
            mem.upload(oa.X, hx[m].numpy())
        b.run_qn(1, 0.0)
        for m, mem in enumerate(b.members):
            mem.download(oa.X, ho[m].numpy())
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - w0) * 1e3 / e2e_steps
    xbytes = sum(8 * K * (spec.I + spec.J) for K in Ks)

    # solo iterations of each distinct K, one problem at a time
    solo_ms = {}
    for K in sorted(set(Ks)):
        d = oa.AdmixData(spec.I, spec.J, K, 3, rng=0)
        with oa.CuAdmixData(d, g, flags=flags) as h:
            oa.init_em(d, g, 2, d_cu=h, quiet=True)
            h.set_ll(d.ll_new)
            from openadmixture_b200 import _native as N
            info = N.IterInfo()
            h._chk(N.admix_lib().admix_qn_iteration(h.handle, 1, C_byref(info)))
            st = torch.cuda.ExternalStream(h.stream())
            torch.cuda.synchronize()
            a0 = torch.cuda.Event(enable_timing=True); a1 = torch.cuda.Event(enable_timing=True)
            a0.record(st)
            for it in range(2, 5):
                h._chk(N.admix_lib().admix_qn_iteration(h.handle, it, C_byref(info)))
            a1.record(st)
            torch.cuda.synchronize()
            solo_ms[K] = a0.elapsed_time(a1) / 3
    seq_ms = sum(solo_ms[K] for K in Ks)

    # time to converge of the whole batch from the random starts + 5 EM
    ttc = None
    if not args.no_ttc:
        for m, mem in enumerate(b.members):
            mem.upload(oa.X, oa.init_x(spec.I, spec.J, Ks[m], seeds[m]))
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        b.init_em(5)
        r = b.run_qn(1000, 1e-7)
        torch.cuda.synchronize()
        lls = np.array([mem.loglik(oa.X) for mem in b.members])
        best = int(np.argmax(lls[:BATCH_RESTARTS]))
        ttc = {"seconds": time.perf_counter() - w0, "members": len(Ks), "all_converged": bool(r["converged"].all()),
               "iterations_max": int(r["iterations"].max()), "iterations_mean": float(r["iterations"].mean()),
               "qn_device_ms": r["ms_device"], "best_restart": best, "best_restart_ll_fp64": float(lls[best]),
               "k_sweep_ll_fp64": {int(K): float(lls[BATCH_RESTARTS + t]) for t, K in enumerate(BATCH_KS)}}
    n_kern = sum(mem.iteration_kernels() for mem in b.members)
    b.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(oa, spec)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    hbm, _, _, peak_kind = _peaks()
    Ib = (spec.I + 3) // 4
    alg = len(Ks) * 6 * Ib * spec.J                  # 6 genotype passes per member iteration
    achieved = alg / (ms / args.steps / 1e3) / 1e9
    line = {
        "metric": "genotype*K^2/s per batch iteration (64 restarts at K=6 + K sweep 2..12, one launch), 1 B200",
        "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16+f32+f64" if flags else "f64", "data": "synthetic",
        "config": {"workload": f"{spec.name}: batch of {len(Ks)} problems on I={spec.I} J={spec.J}: "
                               f"{BATCH_RESTARTS} restarts at K={spec.K} and K={BATCH_KS[0]}..{BATCH_KS[-1]}",
                   "I": spec.I, "J": spec.J, "members": len(Ks), "form": args.form,
                   "l2": f"inputs larger than L2: {Ib * spec.J / 1e6:.0f} MB packed genotypes, "
                         f"{len(Ks)} members' iterates",
                   "autotune": {"divisor": divisor, "probe_ms": probe_ms, "seconds": t_tune}},
        "e2e": {"value": world * work / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": xbytes,
                "d2h_bytes_per_step": xbytes, "ms_per_step": e2e_ms,
                "path": "admix_set_x per member + admix_batch_run_qn(1) + admix_get_x per member"},
        "gpu_launches": n_kern * args.steps,
        "roofline": {"bound": "hbm", "kernel": "batch iteration (all members)", "achieved": achieved,
                     "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": None,
                     "alg_bytes_per_launch": alg,
                     "note": "packed-genotype bytes the members' passes stream per batch iteration"},
        "vs_sequential": {"solo_ms_per_iteration": solo_ms, "sequential_ms_per_step": seq_ms,
                          "speedup_per_iteration": seq_ms / (ms / args.steps)},
        "ttc": ttc,
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = _args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if args.gpus == 1 else 1)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.pass_only:
        return run_pass_only(args)
    if args.skfr is not None:
        return run_skfr(args)
    if args.config == "c4":
        return run_batch(args, rank, world, local_rank)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
