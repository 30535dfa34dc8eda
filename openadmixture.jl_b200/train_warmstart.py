"""Train the warm-start encoder on cohorts solved by this engine, then compare it with the random
start on a held-out cohort of the same ancestral populations.

    python openadmixture.jl_b200/train_warmstart.py [--cohorts 50] [--I 20000] [--J 100000] [--K 8]
        [--alpha 0.2] [--world 777] [--eval c5|held-out|other-world] [--out models/warmstart_k8.npz]
    python openadmixture.jl_b200/train_warmstart.py --add-freq models/warmstart_k8.npz   (CPU only)

Training cohorts and the evaluation cohort share their ancestral allele frequencies SNP by SNP
(CohortSpec.p_seed = --world); individuals and admixture proportions differ.  Each training
cohort is solved by the plain FP64 engine (5 EM iterations + quasi-Newton to rtol 1e-7); its
converged Q, relabelled to the populations' order, is the target.  The model file also records the
training cohorts' allele frequencies at the sketch SNPs; a cohort whose frequencies do not
correlate with them (other ancestral populations) gets the random start instead
(warmstart.learned_start).  --add-freq computes that record for an existing model file from the
training cohorts' genotypes, drawn on the host.  The evaluation reports, for
the random start (+ 5 EM iterations) and for the learned start, the iterations and seconds the
chosen (mixed) form needs to reach a log-likelihood within 1e-6 relative of the plain FP64
solution.  One JSON line is printed at the end.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

import numpy as np  # noqa: E402


def log(msg):
    print(msg, flush=True)


def host_sketch_freq(g, snps: np.ndarray) -> np.ndarray:
    """Allele frequency of each sketch SNP from host genotypes, as the sketch kernel computes it:
    sum of dosages over non-missing individuals / (2 x their count)."""
    cols = g.data[snps]                                       # (S, ceil(I/4)) bytes
    codes = np.stack([(cols >> (2 * s)) & 3 for s in range(4)], axis=2).reshape(len(snps), -1)[:, : g.I]
    dose = np.where(codes == 3, 2, np.where(codes == 2, 1, 0)).astype(np.float64)
    nm = (codes != 1)
    n = 2.0 * nm.sum(1)
    return np.where(n > 0, (dose * nm).sum(1) / np.maximum(n, 1), 0.5).astype(np.float32)


def add_freq(path: str, cohorts: int, I: int, J: int, K: int, alpha: float, world: int) -> None:
    """Record the training world's sketch-SNP allele frequencies (mean over `cohorts` training
    cohorts, drawn on the host) in an existing model file."""
    import openadmixture_b200 as oa
    z = dict(np.load(path))
    snps = z["snps"]
    acc = np.zeros(len(snps))
    for c in range(cohorts):
        spec = oa.CohortSpec(f"train{c}", I, J, K, alpha=alpha, miss=0.01, seed=1000 + c, p_seed=world)
        g, _, _ = oa.make_cohort(spec)
        acc += host_sketch_freq(g, snps)
        log(f"cohort {c}: sketch frequencies")
    z["freq"] = (acc / cohorts).astype(np.float32)
    np.savez_compressed(path, **z)
    log(f"wrote freq ({len(snps)} SNPs) into {path}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cohorts", type=int, default=50)
    ap.add_argument("--I", type=int, default=20_000)
    ap.add_argument("--J", type=int, default=100_000)
    ap.add_argument("--K", type=int, default=8)
    ap.add_argument("--alpha", type=float, default=0.2)
    ap.add_argument("--world", type=int, default=None, help="p_seed of the world (default: warmstart.WORLD_SEED)")
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--eval", default="c5", help="'c5' or 'held-out' (one more training-size cohort)")
    ap.add_argument("--out", default=str(HERE / "models" / "warmstart_k8.npz"))
    ap.add_argument("--max-iter", type=int, default=100, help="QN iteration cap of each evaluation run")
    ap.add_argument("--model", default=None, help="skip training and evaluate this model file")
    ap.add_argument("--add-freq", default=None, metavar="MODEL",
                    help="record the training world's sketch-SNP frequencies in MODEL (host only) and exit")
    ap.add_argument("--freq-cohorts", type=int, default=4)
    args = ap.parse_args()
    if args.add_freq:
        from openadmixture_b200.synth import WARMSTART_WORLD
        add_freq(args.add_freq, args.freq_cohorts, args.I, args.J, args.K, args.alpha,
                 WARMSTART_WORLD if args.world is None else args.world)
        return

    import torch
    import openadmixture_b200 as oa
    from openadmixture_b200 import warmstart as ws
    torch.cuda.set_device(0)
    if args.world is None:
        args.world = ws.WORLD_SEED
    snps = ws.sketch_snps(args.J)
    report = {"cohorts": args.cohorts, "I": args.I, "J": args.J, "K": args.K, "alpha": args.alpha}

    if args.model:
        model = ws.WarmStartMLP.load(args.model)
        if model.snps is None:
            model.snps = snps
    else:
        data, t_solve = [], time.perf_counter()
        for c in range(args.cohorts):
            spec = oa.CohortSpec(f"train{c}", args.I, args.J, args.K, alpha=args.alpha, miss=0.01,
                                 seed=1000 + c, p_seed=args.world)
            qt, pt = oa.truth(spec)
            g = oa.genotypes_device(spec, qt, pt)
            r = ws.run_to_target(g, args.K, flags=0, rng=c, max_iter=300)
            q_conv, p_conv = r["x"][: g.I], r["x"][g.I:]
            tgt = ws.align_to_populations(q_conv, p_conv, pt)
            sk = ws.sketch(g, snps)
            data.append((sk, torch.tensor(tgt.astype(np.float32), device="cuda")))
            log(f"cohort {c}: plain solve {r['iterations']} iterations, {r['seconds']:.1f} s, ll {r['ll']:.6e}")
            del g
        report["solve_seconds"] = time.perf_counter() - t_solve
        freq = np.mean([sk.freq.detach().cpu().numpy() for sk, _ in data], axis=0)
        model = ws.WarmStartMLP(len(snps), 32, args.K, seed=0, snps=snps, freq=freq)
        t_train = time.perf_counter()
        hist = ws.train(model, data, epochs=args.epochs, log=log)
        report["train_seconds"] = time.perf_counter() - t_train
        report["train_loss"] = hist
        Path(args.out).parent.mkdir(parents=True, exist_ok=True)
        model.save(args.out)
        model = ws.WarmStartMLP.load(args.out)          # evaluate the stored FP16 weights
        del data

    if args.eval == "c5":
        spec = oa.COHORTS["c5"].scaled(p_seed=args.world, seed=5)
    elif args.eval == "other-world":     # populations the model was not trained on
        spec = oa.COHORTS["c5"].scaled(p_seed=args.world + 1, seed=5)
    else:
        spec = oa.CohortSpec("held-out", args.I, args.J, args.K, alpha=args.alpha, miss=0.01, seed=999,
                             p_seed=args.world)
    qt, pt = oa.truth(spec)
    g = oa.genotypes_device(spec, qt, pt)
    log(f"evaluation cohort {spec.name}: I={spec.I} J={spec.J} K={spec.K}")
    # the reference optimum: plain FP64 form from the random start + EM
    plain = ws.run_to_target(g, spec.K, flags=0, rng=1, max_iter=args.max_iter)
    target = plain["ll"] - 1e-6 * abs(plain["ll"])
    hit = next((t for t in plain["trace"] if t[1] >= target), None)
    plain["iterations_to_target"], plain["seconds_to_target"] = (hit[0], hit[2]) if hit else (None, None)
    log(f"plain FP64 solve: {plain['iterations']} iterations, {plain['seconds']:.1f} s, ll {plain['ll']:.10e}")
    rand = ws.run_to_target(g, spec.K, flags=oa.ADMIX_FLAG_MIXED, rng=1, target=target, max_iter=args.max_iter)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    check = {}
    start = ws.predict_start(model, g, info=check, check=True)
    report["warm_start_check"] = dict(check)
    if start is None:     # the run_admixture path falls back; time the refused start anyway
        start = ws.predict_start(model, g)
    t_pred = time.perf_counter() - t0
    learned = ws.run_to_target(g, spec.K, flags=oa.ADMIX_FLAG_MIXED, rng=1, start=start, target=target,
                               max_iter=args.max_iter)
    for r in (plain, rand, learned):
        del r["x"]
    learned["predict_seconds"] = t_pred
    learned["seconds"] += t_pred
    if learned["seconds_to_target"] is not None:
        learned["seconds_to_target"] += t_pred
    report.update({"eval": {"workload": f"{spec.name}: I={spec.I} J={spec.J} K={spec.K}", "target_rel": 1e-6},
                   "plain_fp64_random_start_em5": plain, "mixed_random_start_em5": rand, "mixed_learned_start": learned})
    if plain["seconds_to_target"] and learned["seconds_to_target"]:
        report["speedup_vs_plain_to_target"] = plain["seconds_to_target"] / learned["seconds_to_target"]
    if rand["seconds_to_target"] and learned["seconds_to_target"]:
        report["speedup_vs_mixed_random_to_target"] = rand["seconds_to_target"] / learned["seconds_to_target"]
    print(json.dumps(report), flush=True)


if __name__ == "__main__":
    main()
