"""Training data, training loop and evaluation of the learned audit surrogate.

Labels come from the library's own exact audit: at a sequence of states
along a batched LOD walk of each training mesh, every legal midpoint collapse
is audited through the four gates, giving (accepted, error / limit of the
worst evaluated gate) per candidate. The surrogate is then fitted with the
tensor-core train step and judged on held-out meshes by what it prunes:
the false-reject rate (exact-accepted candidates outside the kept share),
and, for whole LOD steps, the triangle-count gap and the time against the
walk without it.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

import blitzremesher_b200 as br
from blitzremesher_b200 import synthetic as syn

ERROR_CAP = 4.0  # error ratios above this (and infinite errors) are clipped


def c1_gates(screen: float = 24.0, views: int = 32, supersample: int = 8, lod0: float = 2.0,
             transition: float = 1.0, max_changed_area: float = 1.0):
    """The four gates of the 20,480-face icosphere workload: LOD0 bound 2 px,
    transition bound 1 px, `views` orthographic views, screen x supersample."""
    v = (views, 0, 0xB1172026)
    return [br.eval_settings(screen, lod0, v, supersample, supersample, max_changed_area),
            br.eval_settings(screen, transition, v, supersample, supersample, max_changed_area),
            br.eval_settings(screen, lod0, v, supersample, supersample, max_changed_area),
            br.eval_settings(screen, transition, v, supersample, supersample, max_changed_area)]


def labels_of(verdicts: np.ndarray, meas: np.ndarray, gates) -> np.ndarray:
    """(accepted, worst error / limit over the evaluated gates) per candidate."""
    n = verdicts.size
    out = np.zeros((n, 2), np.float32)
    out[:, 0] = verdicts["accepted"]
    limits = np.array([g.limit for g in gates], np.float64)
    ratio = meas["error"] / limits[None, :]
    evaluated = np.arange(4)[None, :] < np.where(verdicts["accepted"] == 1, 4, verdicts["failed_gate"])[:, None]
    ratio = np.where(evaluated, ratio, 0.0)
    ratio = np.where(np.isfinite(ratio), ratio, ERROR_CAP)
    out[:, 1] = np.minimum(ratio.max(1), ERROR_CAP)
    return out


@dataclass
class LabelSet:
    features: object          # torch CUDA tensor n x 48
    labels: object            # torch CUDA tensor n x 2
    state_of: np.ndarray      # state index of each row
    states: List[dict] = field(default_factory=list)


def generate(seeds: Sequence[int], fractions: Sequence[float], gates, level: int = 5, batch: int = 64,
             amplitude: float = 0.02, trial_budget: int = 1 << 30, log=None) -> LabelSet:
    """Exact-audit labels of every legal edit at the states reached by a
    batched walk of each mesh through the face fractions `fractions`
    (descending)."""
    import torch
    feats, labs, owner, states = [], [], [], []
    screen, screen2 = gates[0].screen_size, gates[2].screen_size
    for seed in seeds:
        mesh = syn.noisy_icosphere(level, seed, amplitude)
        with br.AuditSession(mesh) as s:
            for frac in fractions:
                t0 = time.perf_counter()
                target = max(1, int(round(mesh.face_count * frac)))
                faces = mesh.face_count
                if frac < 1:
                    faces = s.execute(target, trial_budget, gates, batch=batch)["final_faces"]
                t1 = time.perf_counter()
                f, cols = s.surrogate_features(screen, screen2)
                if not len(cols):
                    break
                v, m = s.candidates(cols, gates, measurements=True)
                lab = labels_of(v, m, gates)
                state = {"seed": seed, "fraction": frac, "faces": int(faces), "candidates": int(len(cols)),
                         "accepted": float(lab[:, 0].mean()), "exact_path": float(v["exact_path"].mean()),
                         "walk_s": t1 - t0, "label_s": time.perf_counter() - t1}
                states.append(state)
                if log:
                    log(state)
                feats.append(f.clone())
                labs.append(torch.from_numpy(lab).cuda())
                owner.append(np.full(len(cols), len(states) - 1, np.int32))
    return LabelSet(torch.cat(feats), torch.cat(labs), np.concatenate(owner), states)


def normalisation(features):
    """Per-feature mean and 1/std (std floored) of a feature tensor."""
    x = features.double()
    mean = x.mean(0)
    std = x.std(0).clamp_min(1e-3)
    return mean.float().cpu().numpy(), (1.0 / std).float().cpu().numpy()


def fit(model: br.Surrogate, data: LabelSet, epochs: int = 4, batch_size: int = 8192, lr: float = 1e-3,
        seed: int = 0) -> List[float]:
    """Adam on shuffled minibatches, halving the rate each epoch; returns the
    mean loss of each epoch."""
    import torch
    mean, inv = normalisation(data.features)
    params, _, _ = model.parameters()
    model.load(params, mean, inv)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    n = data.features.shape[0]
    batch_size = min(batch_size, n)
    history = []
    for epoch in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        total, steps = 0.0, 0
        step_lr = lr * (0.5 ** epoch)
        for i in range(0, n - batch_size + 1, batch_size):
            idx = perm[i:i + batch_size]
            total += model.train_step(data.features[idx].contiguous(), data.labels[idx].contiguous(), step_lr)
            steps += 1
        history.append(total / max(1, steps))
    return history


def pruning_stats(model: br.Surrogate, data: LabelSet, keep: float = 0.25) -> dict:
    """Per state, keep the `keep` share of edits with the highest predicted
    acceptance; report the false-reject rate (exact-accepted edits outside
    the kept share, over all exact-accepted edits) and the acceptance rate
    inside the kept share against the base rate."""
    out = model.score(data.features).cpu().numpy()
    lab = data.labels.cpu().numpy()
    accepted_total = rejected_kept = 0
    false_reject = kept_total = kept_accepted = 0
    for k in range(len(data.states)):
        rows = np.nonzero(data.state_of == k)[0]
        n_keep = max(1, int(np.ceil(len(rows) * keep)))
        order = np.argsort(-out[rows, 0], kind="stable")
        kept = np.zeros(len(rows), bool)
        kept[order[:n_keep]] = True
        acc = lab[rows, 0] > 0.5
        accepted_total += acc.sum()
        false_reject += (acc & ~kept).sum()
        kept_total += kept.sum()
        kept_accepted += (acc & kept).sum()
        rejected_kept += (~acc & kept).sum()
    return {"false_reject_rate": float(false_reject / max(1, accepted_total)),
            "kept_acceptance": float(kept_accepted / max(1, kept_total)),
            "base_acceptance": float(accepted_total / max(1, len(data.state_of))),
            "kept_rejections": int(rejected_kept)}


def chain_compare(model: br.Surrogate, seeds: Sequence[int], fraction: float, gates, level: int = 5,
                  batch: int = 64, keep_permille: int = 250, sequential: bool = False,
                  trial_budget: int = 1 << 30) -> dict:
    """One LOD step of each held-out mesh to `fraction` of its faces: the plain
    batched walk, the surrogate-pruned walk and (optionally) the sequential
    walk. Returns per-mesh faces, trials and wall times, and the totals."""
    import torch
    rows = []
    for seed in seeds:
        mesh = syn.noisy_icosphere(level, seed)
        target = max(1, int(round(mesh.face_count * fraction)))
        row = {"seed": seed, "faces": mesh.face_count, "target": target}
        with br.AuditSession(mesh) as s:
            s.attach_surrogate(model)
            runs = [("plain", batch, 0), ("surrogate", batch, keep_permille)]
            if sequential:
                runs.append(("sequential", 1, 0))
            for name, b, keep in runs:
                s.reset()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                r = s.execute(target, trial_budget, gates, batch=b, keep_permille=keep)
                torch.cuda.synchronize()
                row[name] = {"seconds": time.perf_counter() - t0, "final_faces": int(r["final_faces"]),
                             "trials": int(r["trials"]), "commits": int(len(r["commits"])),
                             "stop": int(r["stop"]), "fallbacks": int(r["fallbacks"])}
        rows.append(row)
    names = [k for k, v in rows[0].items() if isinstance(v, dict)]
    total = {name: {"seconds": sum(r[name]["seconds"] for r in rows),
                    "final_faces": sum(r[name]["final_faces"] for r in rows),
                    "trials": sum(r[name]["trials"] for r in rows)} for name in names}
    gap = (total["surrogate"]["final_faces"] - total["plain"]["final_faces"]) / max(1, total["plain"]["final_faces"])
    return {"meshes": rows, "total": total, "triangle_gap": gap,
            "speedup_vs_plain_batched": total["plain"]["seconds"] / max(1e-9, total["surrogate"]["seconds"])}


def mlp_timing(model: br.Surrogate, features, labels, repeats: int = 5) -> dict:
    """Device time of the tensor-core forward over all rows and of one fused
    train step over the first 8192 rows (CUDA events on the current stream)."""
    import torch
    n = features.shape[0]
    m = min(8192, n)
    f8, l8 = features[:m].contiguous(), labels[:m].contiguous()
    model.score(features)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(repeats):
        model.score(features)
    b.record()
    torch.cuda.synchronize()
    fwd_ms = a.elapsed_time(b) / repeats
    params, mean, inv = model.parameters()
    a.record()
    for _ in range(repeats):
        model.gradients(f8, l8)
    b.record()
    torch.cuda.synchronize()
    train_ms = a.elapsed_time(b) / repeats
    model.load(params, mean, inv)
    flops_row = 2 * (48 * 128 + 128 * 128 + 128 * 2)
    return {"forward_rows": int(n), "forward_ms": fwd_ms, "forward_rows_per_s": n / (fwd_ms * 1e-3),
            "forward_tflops": flops_row * n / (fwd_ms * 1e-3) / 1e12, "train_rows": int(m),
            "train_ms_incl_host": train_ms, "train_tflops": 3 * flops_row * m / (train_ms * 1e-3) / 1e12,
            "flops_per_row_forward": flops_row}


def main(argv=None) -> None:
    """Trains a surrogate on exact-audit labels of the 20,480-face icosphere
    family and reports pruning and LOD-step statistics on held-out meshes."""
    import argparse
    import json
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--train-seeds", type=int, default=8)
    ap.add_argument("--held-seeds", type=int, default=4)
    ap.add_argument("--screen", type=float, default=24.0)
    ap.add_argument("--views", type=int, default=32)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--fraction", type=float, default=0.5)
    ap.add_argument("--keep-permille", type=int, default=250)
    ap.add_argument("--fractions", default="1,0.7,0.5,0.35,0.25", help="label states (face fractions)")
    ap.add_argument("--out", default=None, help="write the trained parameters (.npz)")
    a = ap.parse_args(argv)
    gates = c1_gates(screen=a.screen, views=a.views)
    fractions = [float(x) for x in a.fractions.split(",")]
    t0 = time.perf_counter()
    train = generate(range(2, 2 + a.train_seeds), fractions, gates)
    gen_s = time.perf_counter() - t0
    model = br.Surrogate(seed=1)
    t0 = time.perf_counter()
    history = fit(model, train, epochs=a.epochs)
    fit_s = time.perf_counter() - t0
    held_seeds = list(range(1001, 1001 + a.held_seeds))
    held = generate(held_seeds, fractions, gates)
    untrained = br.Surrogate(seed=1)
    untrained.load(untrained.parameters()[0], *normalisation(train.features))
    report = {"screen": a.screen, "train_rows": int(train.features.shape[0]), "label_s": gen_s, "fit_s": fit_s,
              "loss": history, "held_rows": int(held.features.shape[0]),
              "pruning": pruning_stats(model, held, a.keep_permille / 1000),
              "pruning_untrained": pruning_stats(untrained, held, a.keep_permille / 1000),
              "chain": chain_compare(model, held_seeds, a.fraction, gates, keep_permille=a.keep_permille)["total"],
              "mlp": mlp_timing(model, held.features, held.labels)}
    if a.out:
        p, mean, inv = model.parameters()
        np.savez(a.out, params=p, mean=mean, inv_std=inv)
    print(json.dumps(report), flush=True)


if __name__ == "__main__":
    main()
