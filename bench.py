"""Audited-collapse throughput of the B200 candidate-audit engine.

Workload ("plain audit, icosphere 20,480 triangles"): a seeded icosphere
subdivided to 20,480 faces with +-2% radial noise, 32 orthographic views at a
256x256 coverage raster (screen 24 px x supersample 8), every topologically
legal directed edge collapse with midpoint placement, audited through the
four gates (source@search, previous@search, source@audit, previous@audit) with
a 2 px LOD0 bound and a 1 px transition bound. For the first LOD step the
previous LOD is the source.

One step = the batched four-gate audit of every candidate. `value` is device
time with inputs resident in HBM (CUDA events around K steps); `e2e` goes
through the host C ABI (blitz_audit_candidates) with pinned host buffers,
copies included. Under torchrun each rank audits its own seeded mesh (weak
scaling, no data-path collective).

`--impl reference` times the reference's own CPU audit (oracle/_ref, the
reference sources compiled unmodified) on the host cores for the same
workload, on a bounded sample of candidates per step.
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

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "plain-audit icosphere-20480 32 ortho views 256x256 (24px x ss8), all legal midpoint collapses, 4 gates"
METRIC = "audited collapses/s"
VIEWS = (32, 0, 0xB1172026)
SCREEN, SS = 24.0, 8
SOURCE_LIMIT, TRANSITION_LIMIT = 2.0, 1.0
GATE_ARGS = [(SCREEN, SOURCE_LIMIT, VIEWS, SS, SS, 1.0), (SCREEN, TRANSITION_LIMIT, VIEWS, SS, SS, 1.0),
             (SCREEN, SOURCE_LIMIT, VIEWS, SS, SS, 1.0), (SCREEN, TRANSITION_LIMIT, VIEWS, SS, SS, 1.0)]


# DRAM bytes (read + write) of one k_audit launch of this workload and its
# issue-slot utilisation, from one ncu --set full capture on a B200: the
# working set is L2-resident, the kernel is issue-bound.
K_AUDIT_TRAFFIC = 45_381_120
K_AUDIT_ISSUE_PCT = 65.6
# DRAM bytes (read + write) of the batched workload's audit kernels per
# batch, from one ncu capture of each tier on the 2-mesh case (huge tier
# 22.6 KB a unit, warp tier 1.0 KB a unit) scaled to the 64-mesh batch's
# units (126,277 huge-tier, 262,144 warp-tier).
K_BATCH_TRAFFIC = 3_120_000_000
K_BATCH_TRAFFIC_NOTE = ("ncu dram__bytes_read + dram__bytes_write on the 2-mesh case per tier, scaled by units "
                        "to the full batch")


BATCH_WORKLOAD = ("batched plain audit: 64 meshes (noisy spheres, R/r=3 tori, value-noise heightfields; "
                  "2k-200k faces log-uniform; FP32 UVs with 4-16 chart seams), 64 ortho views at 512 px x ss8, "
                  "64 legal midpoint collapses per mesh = 4,096 per launch, 4 gates")
BATCH_MESHES, BATCH_PER_MESH = 64, 64
BATCH_VIEWS = (64, 0, 0xB1172026)
BATCH_SCREEN = 512.0
BATCH_GATE_ARGS = [(BATCH_SCREEN, SOURCE_LIMIT, BATCH_VIEWS, SS, SS, 1.0),
                   (BATCH_SCREEN, TRANSITION_LIMIT, BATCH_VIEWS, SS, SS, 1.0),
                   (BATCH_SCREEN, SOURCE_LIMIT, BATCH_VIEWS, SS, SS, 1.0),
                   (BATCH_SCREEN, TRANSITION_LIMIT, BATCH_VIEWS, SS, SS, 1.0)]


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.stop = threading.Event()
        self.thread = threading.Thread(target=self.run, daemon=True)

    def run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                parts = [x.strip() for x in out.stdout.strip().split(",")]
                if len(parts) >= 9:
                    self.samples.append(parts)
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.thread.start()
        return self

    def __exit__(self, *exc):
        self.stop.set()
        self.thread.join(timeout=10)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_reference_sample(n_candidates: int, seed: int = 1, threads: int = 1) -> dict:
    """Times the reference CPU audit (oracle/_ref) on a bounded candidate sample."""
    from concurrent.futures import ProcessPoolExecutor
    import multiprocessing as mp

    from blitzremesher_b200 import synthetic as syn
    from oracle.oracle import Oracle, Reference

    mesh = syn.config1_mesh(seed)
    O = Oracle()
    edits = O.actions(mesh, placement=True)
    picks = np.linspace(0, len(edits) - 1, n_candidates).astype(int)
    jobs = [(int(edits[p].from_), int(edits[p].to), seed) for p in picks]
    t0 = time.perf_counter()
    if threads <= 1:
        results = [_reference_audit(j) for j in jobs]
    else:
        with ProcessPoolExecutor(max_workers=threads, mp_context=mp.get_context("spawn")) as ex:
            results = list(ex.map(_reference_audit, jobs))
    wall = time.perf_counter() - t0
    busy = sum(r[0] for r in results)
    return {"candidates": len(jobs), "wall_s": wall, "busy_s": busy, "accepted": sum(r[1] for r in results)}


def _reference_audit(job):
    """One four-gate audit with the reference's evaluate (evaluate.cpp:353);
    the midpoint trial mesh is built by the oracle (the reference has midpoint
    placement only in CUDA), outside the timed part."""
    frm, to, seed = job
    sys.path.insert(0, str(ROOT))
    from blitzremesher_b200 import synthetic as syn
    from oracle.oracle import BoEdit, Oracle, Reference, settings

    mesh = syn.config1_mesh(seed)
    O, R = Oracle(), Reference()
    e = BoEdit()
    e.from_, e.to = frm, to
    idx, pos, _, valid = O.trial_midpoint(mesh, e)
    b = R.bounds(mesh)
    cand = syn.Mesh(pos, idx)
    t0 = time.perf_counter()
    ok = valid
    if valid:
        for a in GATE_ARGS:
            m = R.evaluate(mesh, cand, b, settings(*a))
            if not (m.complete and m.passed and not m.resource_limited):
                ok = False
                break
    return time.perf_counter() - t0, int(ok)


def host_cpu() -> dict:
    """The host's CPU model and the threads this process may use."""
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count() or 1
    return {"model": model, "nproc": usable}


def _reference_gate(job):
    """One gate of the reference's four-gate audit: blitz::evaluate
    (evaluate.cpp:353) of a midpoint trial against the source on all 64 views
    at 512 px x ss 8. Returns (busy seconds, passed)."""
    pos, idx, trial_idx, trial_pos, gate = job
    sys.path.insert(0, str(ROOT))
    from blitzremesher_b200 import synthetic as syn
    from oracle.oracle import Reference, settings

    R = Reference()
    src, cand = syn.Mesh(pos, idx), syn.Mesh(trial_pos, trial_idx)
    a = BATCH_GATE_ARGS[gate]
    t0 = time.perf_counter()
    m = R.evaluate(src, cand, R.bounds(src), settings(*a))
    return time.perf_counter() - t0, bool(m.complete and m.passed and not m.resource_limited)


def _noop(_):
    return 0


class ReferenceSampler:
    """The reference CPU audit on a bounded sample of the batched workload.

    Sample: one mesh from each face-count quartile of the 64 (the quartile's
    median), several of the benchmark's own candidates per mesh, every
    candidate audited in full: the four gates (blitz::evaluate each, all 64
    views at 512 px x ss 8, no scaling) as independent jobs on a pool of
    host processes. A step audits `per_step` candidates (four gate jobs each)
    round-robin over the quartiles; its wall time is the step time. The
    midpoint trials come from the oracle, outside the timed part (the
    reference has midpoint placement only in CUDA)."""

    def __init__(self, meshes, picks_of, threads: int):
        from concurrent.futures import ProcessPoolExecutor
        import multiprocessing as mp

        from oracle.oracle import BoEdit, Oracle

        order = np.argsort([m.face_count for m in meshes], kind="stable")
        q = len(order) // 4
        self.quartile_meshes = [int(order[min(len(order) - 1, k * q + q // 2)]) for k in range(4)]
        self.threads = max(1, threads)
        self.per_step = max(1, self.threads // 4)
        O = Oracle()
        self.meshes = meshes
        self.items = []  # (mesh index, pick position, trial job payload, placement valid)
        for slot in range(16):
            mi = self.quartile_meshes[slot % 4]
            picks = picks_of(mi)
            pick = (slot // 4 * 21) % len(picks)
            e = BoEdit()
            e.from_, e.to = int(picks[pick]["from"]), int(picks[pick]["to"])
            tidx, tpos, _, valid = O.trial_midpoint(meshes[mi], e, preserve_uv=False)
            self.items.append((mi, pick, (meshes[mi].positions, meshes[mi].indices, tidx, tpos), bool(valid)))
        self.pool = ProcessPoolExecutor(max_workers=self.threads, mp_context=mp.get_context("spawn"))
        list(self.pool.map(_noop, range(self.threads)))
        self.cursor = 0
        self.results = []  # (mesh index, pick, faces, sequential seconds, accepted)

    def step(self) -> float:
        chosen = [self.items[(self.cursor + k) % len(self.items)] for k in range(self.per_step)]
        self.cursor += self.per_step
        jobs, owners = [], []
        for n, (mi, pick, payload, valid) in enumerate(chosen):
            if not valid:
                continue
            for g in range(4):
                jobs.append((*payload, g))
                owners.append(n)
        t0 = time.perf_counter()
        out = list(self.pool.map(_reference_gate, jobs))
        wall = time.perf_counter() - t0
        for n, (mi, pick, _, valid) in enumerate(chosen):
            gates = [r for r, o in zip(out, owners) if o == n]
            seq, ok = 0.0, valid
            for busy, passed in gates:  # the reference's sequential audit stops at the first failing gate
                seq += busy
                if not passed:
                    ok = False
                    break
            self.results.append((mi, pick, self.meshes[mi].face_count, seq, ok))
        return wall

    def close(self):
        self.pool.shutdown()

    def summary(self, wall_s: float, steps: int) -> dict:
        per_mesh = {}
        for mi, pick, faces, seq, ok in self.results:
            d = per_mesh.setdefault(mi, {"faces": faces, "candidates": 0, "seconds": 0.0, "accepted": 0})
            d["candidates"] += 1
            d["seconds"] += seq
            d["accepted"] += int(ok)
        for d in per_mesh.values():
            d["collapses_per_s_1thread"] = d["candidates"] / d["seconds"] if d["seconds"] else None
        total_faces = sum(d["faces"] * d["candidates"] for d in per_mesh.values())
        weighted = sum(d["faces"] * d["candidates"] / d["seconds"] for d in per_mesh.values() if d["seconds"])
        n = len(self.results)
        return {"value": n / wall_s if wall_s else 0.0, "candidates": n, "wall_s": wall_s,
                "ms_per_step": 1e3 * wall_s / max(1, steps),
                "collapses_per_s_1thread_face_weighted": weighted / total_faces if total_faces else None,
                "per_mesh": {self.meshes[k].name: v for k, v in per_mesh.items()},
                "sample": f"{n} of the benchmark's midpoint collapses, {self.per_step} per step, on 4 meshes "
                          f"(one per face-count quartile: {[self.meshes[k].face_count for k in self.quartile_meshes]} "
                          f"faces), each audited in full by the reference's blitz::evaluate: four gates, all 64 "
                          f"views at 512 px x ss8, no scaling; the four gate evaluations of a candidate run as "
                          f"parallel jobs on {self.threads} host processes"}


def run_reference(args) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if args.config == "batched":
        from blitzremesher_b200 import synthetic as syn
        from oracle.oracle import Oracle

        meshes = syn.batched_set(BATCH_MESHES, seed=2)
        cpu = host_cpu()
        threads = min(cpu["nproc"], 64)
        oracle = Oracle()

        def picks_of(mi):
            acts = oracle.actions(meshes[mi], placement=True, preserve_uv=False)
            idx = np.linspace(0, len(acts) - 1, min(BATCH_PER_MESH, len(acts))).astype(np.int64)
            return [{"from": acts[i].from_, "to": acts[i].to} for i in idx]

        sampler = ReferenceSampler(meshes, picks_of, threads)
        for _ in range(args.warmup):  # warm-up: pool round trips (the trials are prepared untimed above)
            list(sampler.pool.map(_noop, range(sampler.threads)))
        wall = sum(sampler.step() for _ in range(args.steps))
        r = sampler.summary(wall, args.steps)
        sampler.close()
        value = r["value"]
        line = {"metric": METRIC, "value": value, "unit": "collapses/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": BATCH_WORKLOAD, "threads": threads, "cpu": cpu,
                           "step": f"{sampler.per_step} candidate audits (4 gate jobs each) on {threads} processes"},
                "cpu_baseline": {"value": value, "unit": "collapses/s", "cores": threads, "kind": "reference",
                                 "sample": r["sample"], "cpu_model": cpu["model"], "nproc": cpu["nproc"],
                                 "collapses_per_s_1thread_face_weighted": r["collapses_per_s_1thread_face_weighted"],
                                 "per_mesh": r["per_mesh"]},
                "e2e": {"value": value, "unit": "collapses/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    per_step = max(threads, 8)
    times = []
    for _ in range(args.steps):
        r = cpu_reference_sample(per_step, 1, threads)
        times.append(r["wall_s"] / r["candidates"])
    per_cand = sum(times) / len(times)
    value = 1.0 / per_cand
    line = {"metric": METRIC, "value": value, "unit": "collapses/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_cand * 1e3 * per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "sample_candidates_per_step": per_step, "threads": threads},
            "cpu_baseline": {"value": value, "unit": "collapses/s", "cores": threads, "kind": "reference",
                             "sample": f"{per_step} evenly spaced legal midpoint collapses per step, reference "
                                       f"blitz::evaluate over the four gates with early exit"},
            "e2e": {"value": value, "unit": "collapses/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_icosphere(args, rank: int, world: int, local: int) -> dict:
    """The 20,480-face icosphere workload: audit throughput, LOD-chain steps,
    the learned surrogate and the reference CPU audit. Returns its line."""
    import torch

    import blitzremesher_b200 as br
    from blitzremesher_b200 import synthetic as syn

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    mesh = syn.config1_mesh(seed=1 + rank)
    session = br.AuditSession(mesh, br.neural_options(device=local))
    gates = [br.eval_settings(*a) for a in GATE_ARGS]
    acts = session.actions()
    cands = br.midpoint_collapses(acts)
    n = cands.size
    # Device-resident inputs and outputs.
    cand_dev = torch.from_numpy(cands.view(np.uint8).copy()).to(device)
    verdict_dev = torch.empty(n * br.VERDICT_DTYPE.itemsize, dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream(device)

    def step():
        session.candidates_device(cand_dev.data_ptr(), n, gates, verdict_dev.data_ptr(), 0, stream.cuda_stream)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize(device)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    # Device-timed region (inputs resident; the 256x256 masks and counts of all
    # 32 views, 2.5 MB, are L2-resident by design — reported in config).
    barrier()
    torch.cuda.synchronize(device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        torch.cuda.synchronize(device)
    barrier()
    elapsed_ms = start.elapsed_time(end)
    t = torch.tensor([elapsed_ms], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    verdicts = verdict_dev.cpu().numpy().view(br.VERDICT_DTYPE)
    accepted = int(verdicts["accepted"].sum())

    # Kernel profile: the samples the audit kernel touched (counting replay),
    # and its device time from a replay whose kernels run without counters.
    session.profile(1)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize(device)
    prof = session.profile()
    session.profile(2)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize(device)
    timing = session.profile()
    session.profile(0)
    audit_ms = timing["audit_ms"] / max(1, timing["audit_launches"])
    # Algorithmic bytes per audit launch: candidate records, per sample one
    # state-count byte plus one reference-mask bit, one 16-byte view record out.
    launches = max(1, prof["audit_launches"])
    alg_bytes = (prof["record_bytes"] + prof["region_samples"] * (1 + 1 / 8) + prof["units"] * 16) / launches
    achieved_gbs = alg_bytes / (audit_ms * 1e-3) / 1e9
    pk = peaks()

    # End to end through the host C ABI with pinned buffers.
    pinned = torch.empty(n * br.COLLAPSE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = cands.view(np.uint8)
    host_cands = pinned.numpy().view(br.COLLAPSE_DTYPE)
    out_pinned = torch.empty(n * br.VERDICT_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    host_out = out_pinned.numpy().view(br.VERDICT_DTYPE)
    import ctypes as C

    g4 = (br.EvalSettings * 4)(*gates)
    err = C.create_string_buffer(256)

    def e2e_step():
        st = session.lib.blitz_audit_candidates(session.handle, host_cands.ctypes.data, n, g4,
                                                host_out.ctypes.data, None, err, 256)
        assert st == 0, err.value

    for _ in range(2):
        e2e_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_s = float(te.item())
    assert np.array_equal(host_out, verdicts), "host and device entry points disagree"

    value = n * world * args.steps / (max_ms * 1e-3)
    e2e_value = n * world * args.steps / e2e_s
    line = {"metric": METRIC, "value": value, "unit": "collapses/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": max_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "mesh": "icosphere level 5, +-2% radial noise, seed 1+rank",
                       "faces": int(mesh.face_count), "candidates_per_step": int(n), "views": 32,
                       "raster": "256x256", "gates": 4, "distinct_plans": 1, "accepted": accepted,
                       "l2": "resident working set 2.5 MB < L2 (no flush); per step all candidates re-audited",
                       "parallelism": f"dp{world} (one mesh per rank)"},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved_gbs / pk["hbm_gbs"], "traffic": K_AUDIT_TRAFFIC,
                         "issue_active_pct_ncu": K_AUDIT_ISSUE_PCT,
                         "kernel": "k_audit", "kernel_ms": audit_ms, "algorithmic_bytes": alg_bytes,
                         "peak_source": pk["source"] + " hbm_gbs (burst)",
                         "units_per_launch": prof["units"] / launches,
                         "samples_per_launch": prof["region_samples"] / launches},
            "clocks": clocks.summary(),
            "e2e": {"value": e2e_value, "unit": "collapses/s",
                    "h2d_bytes_per_step": int(n * br.COLLAPSE_DTYPE.itemsize + 4 * 64),
                    "d2h_bytes_per_step": int(n * br.VERDICT_DTYPE.itemsize + 4)},
            "gpu_launches": int(prof["launches"] // max(1, args.steps) * args.steps),
            "kernel_ms": {"prepare": timing["prepare_ms"] / args.steps, "audit": timing["audit_ms"] / args.steps,
                          "verdicts": timing["verdict_ms"] / args.steps,
                          "note": "CUDA events around each launch of a replay without counters"}}
    # Learned surrogate: trained on exact-audit labels of the icosphere family
    # (seeds 2..9, states at 100/70/50/35/25% faces), judged on 16 held-out
    # seeds (1001..1016): pruning to the top 25% and whole LOD steps.
    model = None
    if not args.no_surrogate:
        from blitzremesher_b200 import surrogate_train as st
        t0 = time.perf_counter()
        train = st.generate(range(2, 10), [1.0, 0.7, 0.5, 0.35, 0.25], gates)
        label_s = time.perf_counter() - t0
        model = br.Surrogate(seed=1, device=local)
        t0 = time.perf_counter()
        history = st.fit(model, train)
        fit_s = time.perf_counter() - t0
        held_seeds = list(range(1001, 1017))
        held = st.generate(held_seeds, [1.0, 0.5], gates)
        cmp = st.chain_compare(model, held_seeds, 0.5, gates)
        mlp = st.mlp_timing(model, held.features, held.labels)
        line["surrogate"] = {
            "model": "MLP 48-128-128-2, BF16 weights, FP32 accumulate (tcgen05)", "train_rows": int(
                train.features.shape[0]), "label_s": label_s, "fit_s": fit_s, "loss": history,
            "held_out_meshes": len(held_seeds), "held_rows": int(held.features.shape[0]),
            "keep": 0.25, "pruning": st.pruning_stats(model, held), "lod_step_50pct": cmp["total"],
            "triangle_gap": cmp["triangle_gap"], "speedup_vs_plain_batched": cmp["speedup_vs_plain_batched"],
            "mlp": mlp,
            "roofline": {"bound": "tensor", "kernel": "k_mlp<false>", "achieved": mlp["forward_tflops"],
                         "peak": pk["bf16_tflops"], "unit": "TFLOP/s",
                         "frac": mlp["forward_tflops"] / pk["bf16_tflops"],
                         "peak_source": pk["source"] + " bf16_tflops (burst)"}}
    # LOD-chain step: the greedy executor from the source to 50% of its faces,
    # with batches of one (the reference's sequential walk), of 64, and of 64
    # pruned by the surrogate.
    if not args.no_chain:
        line["chain"] = {"metric": "LOD-chain s/mesh", "unit": "s/mesh", "step": "one LOD step to 50% faces",
                         "timing": "wall clock around the host-orchestrated executor"}
        if model is not None:
            session.attach_surrogate(model)
        for batch, keep in ((1, 0), (64, 0), (64, 250)):
            if keep and model is None:
                continue
            session.reset()
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            chain = session.execute(mesh.face_count // 2, 1 << 30, gates, batch=batch, keep_permille=keep)
            torch.cuda.synchronize(device)
            chain_s = time.perf_counter() - t0
            line["chain"][f"batch{batch}" + ("_surrogate" if keep else "")] = {
                "seconds": chain_s, "commits": int(len(chain["commits"])), "trials": int(chain["trials"]),
                "audited": int(chain["audited"]), "final_faces": int(chain["final_faces"]),
                "stop": int(chain["stop"])}
        line["chain"]["seconds"] = line["chain"]["batch1"]["seconds"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference_sample(args.cpu_sample, 1, 1)
        line["cpu_baseline"] = {"value": r["candidates"] / r["busy_s"], "unit": "collapses/s", "cores": 1,
                                "kind": "reference",
                                "sample": f"{r['candidates']} evenly spaced legal midpoint collapses of the same "
                                          f"mesh, reference blitz::evaluate over the four gates with early exit, "
                                          f"{r['busy_s']:.1f} s"}
    session.close()
    return line


def _shares(values) -> list:
    total = float(sum(values))
    return [round(v / total, 4) if total else 0.0 for v in values]


def _region_split(r) -> dict:
    """Region-phase sub-phases of a profiled batch (SM cycles, per unit)."""
    zero, dcyc, dunits, scyc, sunits, sev, spc, srows, wcyc, wunits, wiv, wmask, wwords, wlost, wrows = \
        [float(x) for x in r]
    units = dunits + sunits + wunits

    def per(x, n):
        return x / n if n else 0.0

    return {"zeroing_cycles_per_unit": per(zero, units),
            "direct": {"units": int(dunits), "cycles_per_unit": per(dcyc, dunits)},
            "sweep": {"units": int(sunits), "cycles_per_unit": per(scyc, sunits),
                      "event_cycles_per_unit": per(sev, sunits), "piece_cycles_per_unit": per(spc, sunits),
                      "rows_per_unit": per(srows, sunits)},
            "word_rows": {"units": int(wunits), "cycles_per_unit": per(wcyc, wunits),
                          "interval_cycles_per_unit": per(wiv, wunits), "mask_cycles_per_unit": per(wmask, wunits),
                          "word_cycles_per_unit": per(wwords, wunits), "lost_cycles_per_unit": per(wlost, wunits),
                          "rows_per_unit": per(wrows, wunits)}}


def _barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _max_over_ranks(x: float, world: int, device) -> float:
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def batched_picks(session, per_mesh: int):
    """`per_mesh` evenly spaced legal midpoint collapses of a session's LOD0."""
    import blitzremesher_b200 as br
    c = br.midpoint_collapses(session.actions())
    idx = np.linspace(0, c.size - 1, min(per_mesh, c.size)).astype(np.int64)
    return c[idx]


def run_batched(args, rank: int, world: int, local: int) -> dict:
    """Batched plain audit: one graph-replayed batch of 4,096 candidates (64
    per mesh) over 64 meshes per rank, 64 views at 512 px x ss 8."""
    import torch

    import blitzremesher_b200 as br
    from blitzremesher_b200 import synthetic as syn

    device = torch.device("cuda", local)
    stream = torch.cuda.current_stream(device)
    t0 = time.perf_counter()
    meshes = syn.batched_set(args.meshes, seed=2 + 1000 * rank)
    opts = br.neural_options(device=local, preserve_uv=0)
    sessions = [br.AuditSession(m, opts) for m in meshes]
    gates = [br.eval_settings(*a) for a in BATCH_GATE_ARGS]
    picks = [batched_picks(s, BATCH_PER_MESH) for s in sessions]
    counts = [int(p.size) for p in picks]
    cat = np.concatenate(picks)
    n = int(cat.size)
    cand_dev = torch.from_numpy(cat.view(np.uint8).copy()).to(device)
    verdict_dev = torch.zeros(n * br.VERDICT_DTYPE.itemsize, dtype=torch.uint8, device=device)
    batch = br.AuditBatch(sessions)

    def step(flags=br.BATCH_GRAPH):
        batch.candidates_device(cand_dev.data_ptr(), counts, gates, verdict_dev.data_ptr(), flags, stream.cuda_stream)

    step(br.BATCH_AUTOTUNE)  # builds every plan (reference rasters, state counts) and picks the warp tier
    setup_s = time.perf_counter() - t0
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize(device)
    _barrier(world)
    torch.cuda.synchronize(device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        torch.cuda.synchronize(device)
    _barrier(world)
    max_ms = _max_over_ranks(start.elapsed_time(end), world, device)
    verdicts = verdict_dev.cpu().numpy().view(br.VERDICT_DTYPE).copy()
    # Audit kernels: work counters of one counting batch, device time of one
    # batch whose kernels run without counters (as in the graph replays).
    step(br.BATCH_PROFILE)
    torch.cuda.synchronize(device)
    info = batch.info()
    assert np.array_equal(verdict_dev.cpu().numpy().view(br.VERDICT_DTYPE), verdicts)
    step(br.BATCH_TIMING)
    torch.cuda.synchronize(device)
    audit_ms = batch.info()["audit_ms"]
    alg_bytes = n * 624 * 1 + info["region_samples"] * (1 + 1 / 8) + info["units"] * 16
    achieved_gbs = alg_bytes / (audit_ms * 1e-3) / 1e9
    pk = peaks()
    # The integer-pipe bound of the audit: per launch, 2 ops for each of the 3
    # edge tests of every (face, bbox sample) pair a per-sample raster makes,
    # plus 2 ops per region sample (XOR / OR popcounts), over the SMs' INT32
    # lanes (128 per SM) at the SM clock sampled during the timed steps.
    int_ops = 2 * 3 * info["face_samples"] + 2 * info["region_samples"]
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    sm_mhz = clocks.summary().get("sm_mhz") or 1965.0
    int_peak = sms * 128 * sm_mhz * 1e6 / 1e12
    int_achieved = int_ops / (audit_ms * 1e-3) / 1e12
    # End to end through the host C ABI (blitz_audit_batch_candidates_host):
    # pinned host candidates in, host verdicts out, copies inside every step.
    pinned = torch.empty(n * br.COLLAPSE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = cat.view(np.uint8)
    host_cands = pinned.numpy().view(br.COLLAPSE_DTYPE)
    out_pinned = torch.empty(n * br.VERDICT_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    host_out = out_pinned.numpy().view(br.VERDICT_DTYPE)

    def e2e_step():
        batch.candidates_host(host_cands, counts, gates, host_out, br.BATCH_GRAPH)

    for _ in range(2):
        e2e_step()
    _barrier(world)
    t1 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = _max_over_ranks(time.perf_counter() - t1, world, device)
    assert np.array_equal(host_out, verdicts)
    faces = [m.face_count for m in meshes]
    line = {"metric": METRIC, "value": n * world * args.steps / (max_ms * 1e-3), "unit": "collapses/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": BATCH_WORKLOAD, "meshes": len(meshes), "faces_min": min(faces),
                       "faces_max": max(faces), "faces_total": int(sum(faces)),
                       "kinds": "sphere/torus/heightfield cycling, seeded 2+1000*rank", "uv_charts": "4-16, seams",
                       "candidates_note": "first of the set if --meshes < 64 (then not the workload)",
                       "views": 64, "raster": "4160x4160 (512 px x ss8)", "gates": 4,
                       "candidates_per_step": n, "candidates_per_mesh": BATCH_PER_MESH,
                       "accepted": int(verdicts["accepted"].sum()), "setup_s": setup_s,
                       "warp_tier": ["small 128x64", "medium 256x128"][info["tier"] & 1]
                                    + (", heavy units to the huge tier" if info["tier"] & 2 else ""),
                       "autotune_ms": info["tune_ms"], "graph": "captured once, replayed every step",
                       "exact_path_candidates": int(verdicts["exact_path"].sum()),
                       "l2": "inputs larger than L2 (about 1.2 GB of state counts and masks per mesh)",
                       "parallelism": f"dp{world} (64 meshes per rank)"},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved_gbs / pk["hbm_gbs"], "traffic": K_BATCH_TRAFFIC,
                         "traffic_note": K_BATCH_TRAFFIC_NOTE,
                         "int32": {"achieved": int_achieved, "peak": int_peak, "unit": "Tops/s",
                                   "frac": int_achieved / int_peak, "ops_per_launch": int_ops,
                                   "face_bbox_samples": info["face_samples"],
                                   "peak_source": f"{sms} SMs x 128 INT32 lanes x {sm_mhz:.0f} MHz (sampled)"},
                         "kernel": "k_audit (+ large and huge tiers)", "kernel_ms": audit_ms,
                         "kernel_ms_counting": info["audit_ms"],
                         "tier_ms": dict(zip(("warp", "huge", "giant"), batch.info()["tier_ms"])),
                         "algorithmic_bytes": alg_bytes, "units_per_launch": info["units"],
                         "samples_per_launch": info["region_samples"],
                         "peak_source": pk["source"] + " hbm_gbs (burst)",
                         "tiers": {"units": dict(zip(("warp", "large", "huge", "giant"), info["tier_units"])),
                                   "warp_busy_share": dict(zip(("warp", "large", "huge", "giant"),
                                                               _shares(info["tier_cycles"]))),
                                   "cycles_per_unit": dict(zip(("warp", "large", "huge", "giant"),
                                                               [c / u if u else 0.0 for c, u in
                                                                zip(info["tier_cycles"], info["tier_units"])])),
                                   "max_cycles_per_unit": dict(zip(("warp", "large", "huge", "giant"),
                                                                   info["tier_max_cycles"])),
                                   "phase_share": dict(zip(("setup", "region", "distance"),
                                                           _shares(info["phase_cycles"]))),
                                   "flipped_samples": info["flipped_samples"],
                                   "region_split": _region_split(info["region_split"]),
                                   "note": "SM cycles of each unit's warp, summed per tier and per phase"}},
            "clocks": clocks.summary(),
            "e2e": {"value": n * world * args.steps / e2e_s, "unit": "collapses/s",
                    "h2d_bytes_per_step": int(n * br.COLLAPSE_DTYPE.itemsize),
                    "d2h_bytes_per_step": int(n * br.VERDICT_DTYPE.itemsize)},
            "gpu_launches": int((2 * len(meshes) + 3 + 3) * args.steps)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and len(meshes) == BATCH_MESHES:
        # The reference CPU audit of some of the same candidates, on all host
        # cores for one bounded step; its verdicts must equal the GPU's.
        cpu = host_cpu()
        sampler = ReferenceSampler(meshes, lambda mi: picks[mi], min(cpu["nproc"], 64))
        wall = sampler.step()
        r = sampler.summary(wall, 1)
        sampler.close()
        offsets = np.concatenate([[0], np.cumsum(counts)])
        checked = [(mi, pick, ok) for mi, pick, _, _, ok in sampler.results]
        mismatches = [(mi, pick) for mi, pick, ok in checked if bool(verdicts[offsets[mi] + pick]["accepted"]) != ok]
        assert not mismatches, f"reference and GPU verdicts differ: {mismatches}"
        line["parity_checked"] = len(checked)
        line["cpu_baseline"] = {"value": r["value"], "unit": "collapses/s", "cores": sampler.threads,
                                "kind": "reference", "sample": r["sample"], "cpu_model": cpu["model"],
                                "nproc": cpu["nproc"], "wall_s": wall,
                                "collapses_per_s_1thread_face_weighted": r["collapses_per_s_1thread_face_weighted"],
                                "per_mesh": r["per_mesh"],
                                "parity": f"{len(checked)} reference verdicts equal the GPU's"}
    batch.close()
    for s_ in sessions:
        s_.close()
    return line


ROCK_CHAIN = {"levels": 6, "base": 240.0, "last": 7.5, "curve": ((0.0, 1.0), (1.0, 3.0)), "lod0": 2.0,
              "views": 32, "ss": 8, "batch": 64, "budget": 300}
# The 1M-face rock of the full LOD-chain workload: 6 levels scheduled 1024 ->
# 32 px (audits at 512 ... 32 px x ss 8), transition 1 px at LOD1 rising to
# 3 px, LOD0 bound 2 px, 128 search and 128 audit views, uv preserved.
ROCK_1M_CHAIN = {"levels": 6, "base": 1024.0, "last": 32.0, "curve": ((0.0, 1.0), (1.0, 3.0)), "lod0": 2.0,
                 "views": 128, "ss": 8, "batch": 64, "budget": 40, "memory_mib": 160_000}
# The thin-structure workload: 2,000 ribbon cards (400k faces), 256 views at
# 512 px, 6-level chain (512 -> 16 px, the same 32:1 ratio).
RIBBON_CHAIN = {"levels": 6, "base": 512.0, "last": 16.0, "curve": ((0.0, 1.0), (1.0, 3.0)), "lod0": 2.0,
                "views": 256, "ss": 8, "batch": 64, "budget": 40, "memory_mib": 160_000}


def run_chain(args, local: int, mesh, c: dict, preserve_uv: int = 0, label: str = "", model=None,
              keep_permille: int = 0) -> dict:
    """One LOD chain (blitz_audit_chain: schedule, four gates per level,
    previous-level binding, batched executor, confirmation of every emitted
    level) of `mesh` under the chain settings `c`; wall clock around it."""
    import torch

    import blitzremesher_b200 as br

    # the plans of 128-256 views at 4160 x 4160 samples need more than the
    # default 6 GiB workspace
    session = br.AuditSession(mesh, br.neural_options(device=local, preserve_uv=preserve_uv,
                                                      memory_mib=c.get("memory_mib", 6144)))
    if model is not None:
        session.attach_surrogate(model)
    settings = br.chain_settings(c["levels"], c["base"], c["last"], c["curve"], c["lod0"], (c["views"], 0, 0xB1172024),
                                 (c["views"], 0, 0xB1172026), c["ss"], c["ss"], c["ss"], 1.0, c["batch"],
                                 keep_permille, c["budget"], 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    levels, _ = session.chain(settings, meshes=False)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    info = session.info()
    session.close()
    return {"metric": "LOD-chain s/mesh", "seconds": seconds, "unit": "s/mesh", "mesh": label,
            "faces": int(mesh.face_count), "schedule": c,
            "levels": [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in l.items()
                        if k not in ("source_audit", "transition_audit")}
                       | {"source_error": l["source_audit"].error, "transition_error": l["transition_audit"].error}
                       for l in levels],
            "all_confirmed": all(l["confirmed"] for l in levels),
            "audited_collapses": int(info["decoded"]),
            "timing": "wall clock around blitz_audit_chain (executor, previous-level binding, confirmation)"}


def run_rock_chain(args, local: int, preserve_uv: int = 0) -> dict:
    """Multi-level LOD chain of a ridged-noise rock (81,920 faces, 8 UV charts):
    6 levels scheduled 240 -> 7.5 px (the 1024 -> 32 px ratio of the 1M-face
    configuration), transition 1 -> 3 px, LOD0 bound 2 px, 32 ortho views at
    ss 8, batches of 64, 300 trials per level, each level confirmed. With
    preserve_uv the collapses carry the transported uv and placements that
    fold a uv triangle are rejected."""
    from blitzremesher_b200 import synthetic as syn

    mesh = syn.rock(6, 3)
    label = (f"rock: icosphere level 6 ({mesh.face_count} faces), 6-octave ridged noise, 8 UV charts "
             + ("(preserve_uv: uv transported, uv flips rejected)" if preserve_uv else "(uv not preserved)"))
    return run_chain(args, local, mesh, ROCK_CHAIN, preserve_uv, label)


def run_rock_1m(args, local: int) -> dict:
    """The full LOD-chain workload: the 1,310,720-face rock (icosphere level 8,
    6-octave ridged noise, 8 UV charts, uv preserved), 128 views, 1024 -> 32 px."""
    from blitzremesher_b200 import synthetic as syn

    level = args.rock_level
    mesh = syn.rock(level, 3)
    c = dict(ROCK_1M_CHAIN)
    if args.chain_budget:
        c["budget"] = args.chain_budget
    label = (f"rock: icosphere level {level} ({mesh.face_count} faces), 6-octave ridged noise, 8 UV charts, "
             f"preserve_uv" + ("" if level == 8 and not args.chain_budget else " (not the workload: smaller case)"))
    out = run_chain(args, local, mesh, c, 1, label)
    out["note"] = f"trial budget {c['budget']} batches of up to 64 collapses per level"
    return out


def ribbon_first_level_gates(c: dict):
    """The four gates of the chain's first level: its screen (the schedule's
    second size), 1 px LOD0 and transition bounds, the chain's search and
    audit views."""
    import blitzremesher_b200 as br

    px = c["base"] * (c["last"] / c["base"]) ** (1.0 / (c["levels"] - 1))
    search, audit = (c["views"], 0, 0xB1172024), (c["views"], 0, 0xB1172026)
    return px, [br.eval_settings(px, 1.0, search, c["ss"], c["ss"], 1.0),
                br.eval_settings(px, 1.0, search, c["ss"], c["ss"], 1.0),
                br.eval_settings(px, 1.0, audit, c["ss"], c["ss"], 1.0),
                br.eval_settings(px, 1.0, audit, c["ss"], c["ss"], 1.0)]


def ribbon_surrogate(args, local: int, mesh, c: dict, sample: int = 8192):
    """The thin-structure figures beyond the plain chain: the share of the
    source's legal collapses that the exact audit rejects at the first
    level's gates (an evenly spaced sample), and a surrogate trained on exact
    verdicts of four smaller ribbon meshes (250 cards each, other seeds) at
    the same gates: its false-reject rate when it keeps the top 25% of the
    sample. Returns (figures, model)."""
    import torch

    import blitzremesher_b200 as br
    from blitzremesher_b200 import surrogate_train as st
    from blitzremesher_b200 import synthetic as syn

    px, gates = ribbon_first_level_gates(c)
    opts = br.neural_options(device=local, preserve_uv=0, memory_mib=c.get("memory_mib", 6144))

    def labelled(m):
        with br.AuditSession(m, opts) as s:
            feats, cols = s.surrogate_features(px, px)
            v = s.candidates(cols, gates)
        lab = np.zeros((cols.size, 2), np.float32)
        lab[:, 0] = v["accepted"]
        lab[:, 1] = np.where(v["accepted"] == 1, 0.0, st.ERROR_CAP)  # verdict-only labels
        return feats, torch.from_numpy(lab).cuda(), v

    t0 = time.perf_counter()
    parts = [labelled(syn.ribbons(250, seed=100 + k)) for k in range(4)]
    label_s = time.perf_counter() - t0
    train = st.LabelSet(torch.cat([p[0] for p in parts]), torch.cat([p[1] for p in parts]),
                        np.concatenate([np.full(p[1].shape[0], k, np.int32) for k, p in enumerate(parts)]),
                        [{} for _ in parts])
    model = br.Surrogate(seed=1, device=local)
    t0 = time.perf_counter()
    history = st.fit(model, train)
    fit_s = time.perf_counter() - t0
    # the workload mesh: an evenly spaced sample of its legal collapses
    with br.AuditSession(mesh, opts) as s:
        f_all, cols = s.surrogate_features(px, px)
        pick = np.linspace(0, cols.size - 1, min(sample, cols.size)).astype(np.int64)
        t0 = time.perf_counter()
        v = s.candidates(cols[pick], gates)
        audit_s = time.perf_counter() - t0
        feats = f_all[torch.from_numpy(pick).cuda()].contiguous()
    lab = np.zeros((pick.size, 2), np.float32)
    lab[:, 0] = v["accepted"]
    held = st.LabelSet(feats, torch.from_numpy(lab).cuda(), np.zeros(pick.size, np.int32), [{}])
    return {"level_gates": f"{px:g} px, LOD0 and transition bounds 1 px, {c['views']} search and {c['views']} audit "
                           f"views, ss {c['ss']}",
            "legal_collapses": int(cols.size), "sample": int(pick.size),
            "exact_reject_share": float(1.0 - v["accepted"].mean()), "sample_audit_s": audit_s,
            "surrogate": {"train": "exact verdicts of every legal collapse of 4 ribbon meshes of 250 cards "
                                   "(seeds 100-103) at the same gates",
                          "train_rows": int(train.features.shape[0]), "label_s": label_s, "fit_s": fit_s,
                          "loss": history, "keep": 0.25, "pruning": st.pruning_stats(model, held)}}, model


def run_ribbons(args, local: int) -> dict:
    """The thin-structure workload: 2,000 two-sided ribbon cards (400k faces),
    256 views at 512 px, 6-level chain; with the share of collapses the exact
    audit rejects, the surrogate's false-reject rate, and the chain with the
    surrogate keeping the top 25% of each ranking (its triangle-count gap to
    the plain chain)."""
    from blitzremesher_b200 import synthetic as syn

    cards = args.ribbon_cards
    mesh = syn.ribbons(cards, seed=5)
    label = f"{cards:,} ribbon cards ({mesh.face_count} faces), two-sided" + (
        "" if cards == 2000 else " (not the workload: smaller case)")
    out = run_chain(args, local, mesh, RIBBON_CHAIN, 0, label)
    out["note"] = f"trial budget {RIBBON_CHAIN['budget']} batches of up to 64 collapses per level"
    if not args.no_surrogate:
        stress, model = ribbon_surrogate(args, local, mesh, RIBBON_CHAIN)
        pruned = run_chain(args, local, mesh, RIBBON_CHAIN, 0, label, model=model, keep_permille=250)
        plain_faces, pruned_faces = out["levels"][-1]["faces"], pruned["levels"][-1]["faces"]
        stress["chain_with_surrogate"] = {"seconds": pruned["seconds"], "all_confirmed": pruned["all_confirmed"],
                                          "faces_per_level": [l["faces"] for l in pruned["levels"]],
                                          "triangle_gap": (pruned_faces - plain_faces) / plain_faces,
                                          "speedup_vs_plain": out["seconds"] / pruned["seconds"]}
        out["stress"] = stress
    return out


def run_gpu(args) -> None:
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    if args.config == "batched":
        line = run_batched(args, rank, world, local)
        if not args.no_rock:
            line["lod_chain_rock"] = run_rock_chain(args, local)
            try:
                line["lod_chain_rock_preserve_uv"] = run_rock_chain(args, local, preserve_uv=1)
            except Exception as e:  # recorded in the line; the headline stands
                line["lod_chain_rock_preserve_uv"] = {"error": f"{type(e).__name__}: {e}"}
        if not args.no_icosphere:
            ico = run_icosphere(args, rank, world, local)
            for k in ("metric", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "vs_baseline", "data"):
                ico.pop(k, None)
            line["icosphere_20480"] = ico
    elif args.config == "rock1m":
        line = run_rock_1m(args, local)
    elif args.config == "ribbons":
        line = run_ribbons(args, local)
    else:
        line = run_icosphere(args, rank, world, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=32)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-chain", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--config", default="batched", choices=["batched", "icosphere", "rock1m", "ribbons"])
    ap.add_argument("--no-icosphere", action="store_true")
    ap.add_argument("--no-rock", action="store_true")
    ap.add_argument("--meshes", type=int, default=BATCH_MESHES, help="meshes of the batched set (64 = the workload)")
    ap.add_argument("--rock-level", type=int, default=8,
                    help="icosphere level of the rock1m chain's mesh (8 = the workload, 1.31 M faces)")
    ap.add_argument("--ribbon-cards", type=int, default=2000,
                    help="cards of the ribbons chain's mesh (2000 = the workload, 400k faces)")
    ap.add_argument("--chain-budget", type=int, default=0,
                    help="trials per level of the rock1m chain (0 = the workload's 40)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
