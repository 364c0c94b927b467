#!/usr/bin/env python
"""Benchmark of the Tsetlin-machine hot path on B200.

Metric: "TM train+predict samples/s" -- one step is one training epoch of a
machine from its initial state (`train{iterations = 1}`, capi.c:1484) plus
predict over the held-out set (capi.c:1088), the unit of work the
reference's search driver repeats per trial epoch (optimize.lua:586-653).

Default workload (N = 1): the large sparse classifier -- 20 classes, 16,384
features (flip-packed to 32,768 literal bits, 4 KB per sample), 2,048
clauses per class, specificity 25, target 200, clause_tolerance 64,
clause_maximum 64, 8-bit state; 100,000 train and 20,000 test samples of
Zipf(1.1) features at ~1.5 % density with per-class boosted subsets
(synthetic, seeded; datagen.sparse_classifier).

Arms:
  default           the CUDA library through the C ABI (santoku_tsetlin)
  --impl reference  the reference's CPU implementation of the same step on
                    this host's cores: the reference's own capi.c/automata.h
                    (oracle/_ref) where it was built, else the C restatement
                    (oracle/), on a bounded sample of units, scaled.

Under torchrun each rank trains its own replica of the machine (independent
units, no data-path collective): weak scaling; `value` = all ranks' samples
over the max-over-ranks device time.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "lua-santoku-tsetlin_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "TM train+predict samples/s"
UNIT = "samples/s"

WORKLOADS = {
    "c1": dict(
        name="large-sparse-classifier", kind="classifier", classes=20, features=16384,
        clauses=2048, clause_tolerance=64, clause_maximum=64, specificity=25.0, target=200,
        n_train=100000, n_test=20000),
    # the large sparse classifier's rows and data with 112 clauses per class
    # (280 units: one wave at two CTAs per SM), for profiler captures
    "c1_small": dict(
        name="large-sparse-classifier", kind="classifier", classes=20, features=16384,
        clauses=112, clause_tolerance=64, clause_maximum=64, specificity=25.0, target=200,
        n_train=40000, n_test=4000),
    "c0": dict(
        name="plain-classifier", kind="classifier", classes=10, features=784, clauses=256,
        clause_tolerance=64, clause_maximum=64, specificity=10.0, target=50,
        n_train=8000, n_test=2000),
    "c2_small": dict(
        name="encoder", kind="encoder", classes=256, features=4096, clauses=1024,
        clause_tolerance=64, clause_maximum=64, specificity=15.0, target=100,
        n_train=2000, n_test=2000),
    "c2": dict(
        name="encoder", kind="encoder", classes=256, features=4096, clauses=1024,
        clause_tolerance=64, clause_maximum=64, specificity=15.0, target=100,
        n_train=200000, n_test=20000),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_data(w, rank=0):
    from santoku_tsetlin import datagen
    n = w["n_train"] + w["n_test"]
    cache = "/tmp/tsetlin_b200_%s_%d_r%d.npz" % (w["name"], n, rank)
    if os.path.exists(cache):
        z = np.load(cache)
        return {k: z[k] for k in z.files}
    t = time.time()
    if w["name"] == "large-sparse-classifier":
        x, y = datagen.sparse_classifier(n, classes=w["classes"], features=w["features"],
                                         seed=1 + 1000 * rank)
        d = dict(x=x, y=y)
    elif w["name"] == "plain-classifier":
        x, y, _ = datagen.prototype_classifier(n, classes=w["classes"], features=w["features"],
                                               seed=1 + 1000 * rank)
        d = dict(x=x, y=y)
    else:
        x, c = datagen.latent_encoder(n, visible=w["features"], hidden=w["classes"],
                                      seed=2 + 1000 * rank)
        d = dict(x=x, codes=c)
    log("data %s generated in %.1fs" % (w["name"], time.time() - t))
    try:
        np.savez(cache, **d)
    except OSError:
        pass
    return d


def create_table(w, seed):
    t = dict(clauses=w["clauses"], clause_tolerance=w["clause_tolerance"],
             clause_maximum=w["clause_maximum"], specificity=w["specificity"],
             target=w["target"], seed=seed, reusable=True, device=0)
    if w["kind"] == "classifier":
        t.update(classes=w["classes"], features=w["features"])
    else:
        t.update(hidden=w["classes"], visible=w["features"])
    return t


def train_table(w, x, lab):
    t = {"samples": w["n_train"], "iterations": 1}
    if w["kind"] == "classifier":
        t.update(problems=x, solutions=lab)
    else:
        t.update(sentences=x, codes=lab)
    return t


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = "/tmp/tsetlin_b200_clocks_%d.csv" % os.getpid()

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [q.strip() for q in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# ---------------------------------------------------------------------------
# CPU baseline: the reference's path on a bounded sample of units
# ---------------------------------------------------------------------------
def cpu_step(w, d, threads, budget_units=None):
    """One step of the workload on the CPU, on a machine with the same rows
    but fewer clauses per class (units are independent 8-clause chunks, so
    per-unit work is unchanged), scaled to the full clause count.  Predict is
    timed on a slice of the test set and scaled likewise."""
    import oracle as O
    which = "ref" if O.ref_available() else "oracle"
    threads = threads or os.cpu_count()
    units_per_class = max(1, min(w["clauses"] // 8, (2 * threads + w["classes"] - 1) // w["classes"]))
    if budget_units:
        units_per_class = max(1, min(units_per_class, budget_units // w["classes"]))
    clauses = 8 * units_per_class
    cfg = dict(type=w["kind"], classes=w["classes"], features=w["features"], clauses=clauses,
               clause_tolerance=w["clause_tolerance"], clause_maximum=w["clause_maximum"],
               specificity=w["specificity"], target=w["target"])
    m = O.Machine(which=which, **cfg)
    n = w["n_train"]
    x = d["x"][:n]
    kw = dict(labels=d["y"][:n]) if w["kind"] == "classifier" else dict(codes=d["codes"][:n])
    t0 = time.perf_counter()
    m.train(x.ravel(), n, 1, seed=0, mode=O.REFSTRUCT if which == "ref" else O.PHILOX,
            threads=threads, **kw)
    t_train = time.perf_counter() - t0
    nt = min(w["n_test"], 2000)
    xt = d["x"][n:n + nt]
    t0 = time.perf_counter()
    m.predict(xt.ravel(), nt, threads=threads)
    t_pred = time.perf_counter() - t0
    scale_units = (w["clauses"] // 8) / units_per_class
    step_s = t_train * scale_units + t_pred * scale_units * (w["n_test"] / nt)
    samples = w["n_train"] + w["n_test"]
    sample = ("1 train epoch of %d of %d clauses per class (%d of %d units) over all %d "
              "samples + predict of %d of %d test samples; times scaled by units and samples"
              % (clauses, w["clauses"], units_per_class * w["classes"],
                 (w["clauses"] // 8) * w["classes"], n, nt, w["n_test"]))
    return dict(value=samples / step_s, step_s=step_s, kind="reference" if which == "ref" else "port",
                cores=threads, sample=sample, measured_s=t_train + t_pred)


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def run_reference(args, w):
    ws, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    d = make_data(w)
    threads = os.cpu_count()
    for _ in range(args.warmup if args.warmup < 1 else 1):
        pass
    vals = []
    for _ in range(max(1, min(args.steps, 3))):
        r = cpu_step(w, d, threads)
        vals.append(r)
    v = float(np.median([r["value"] for r in vals]))
    step_s = float(np.median([r["step_s"] for r in vals]))
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
        "steps": len(vals), "warmup": 0, "ms_per_step": step_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": config_of(w, ws),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": vals[0]["cores"],
                         "kind": vals[0]["kind"], "sample": vals[0]["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def config_of(w, ws):
    return {
        "workload": w["name"], "type": w["kind"], "classes": w["classes"],
        "features": w["features"], "literal_bits": 2 * w["features"], "clauses": w["clauses"],
        "clause_tolerance": w["clause_tolerance"], "clause_maximum": w["clause_maximum"],
        "specificity": w["specificity"], "target": w["target"], "state_bits": 8,
        "n_train": w["n_train"], "n_test": w["n_test"],
        "step": "train{iterations=1} from the initial state + predict(test)",
        "parallelism": "replicas" if ws > 1 else "single",
        "l2": "inputs larger than L2 (train set and automata exceed 126 MB)",
    }


def train_algorithmic_bytes(w, resident_units):
    """Minimum DRAM bytes of one train launch: the automata read and written
    once, plus each wave of resident units streaming the train set."""
    rows = w["classes"] * w["clauses"]
    wp = ((2 * w["features"] + 31) // 32 + 3) // 4 * 4
    state = rows * 8 * wp * 4
    units = rows // 8
    waves = max(1, -(-units // max(1, resident_units)))
    return 2 * state + waves * w["n_train"] * wp * 4


def run_ours(args, w):
    import torch
    import santoku_tsetlin as tm
    ws, rank, local = dist_init()
    dev = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(dev)
    d = make_data(w, rank)
    n, nt = w["n_train"], w["n_test"]
    lab_key = "y" if w["kind"] == "classifier" else "codes"
    # device-resident inputs (value) and pinned host inputs (e2e)
    x_dev = torch.from_numpy(np.ascontiguousarray(d["x"][:n])).to(dev)
    lab_dev = torch.from_numpy(np.ascontiguousarray(d[lab_key][:n])).to(dev)
    xt_dev = torch.from_numpy(np.ascontiguousarray(d["x"][n:n + nt])).to(dev)
    x_host = torch.from_numpy(np.ascontiguousarray(d["x"][:n])).pin_memory()
    lab_host = torch.from_numpy(np.ascontiguousarray(d[lab_key][:n])).pin_memory()
    xt_host = torch.from_numpy(np.ascontiguousarray(d["x"][n:n + nt])).pin_memory()
    t = tm.create(w["kind"], create_table(w, seed=rank))
    t.stats_enable(True)

    def step_dev():
        t.train(train_table(w, x_dev, lab_dev))
        return t.predict(xt_dev, nt)

    def step_host():
        t.train(train_table(w, x_host.numpy(), lab_host.numpy()))
        return t.predict(xt_host.numpy(), nt)

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def timed(fn, k):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            fn()
        e1.record()
        torch.cuda.synchronize()
        barrier()
        from santoku_tsetlin import multi
        return multi.max_over_ranks(e0.elapsed_time(e1), device=dev)

    for _ in range(args.warmup):
        step_dev()
    t.reset_stats()
    clocks = ClockSampler(dev.index)
    clocks.start()
    ms = timed(step_dev, args.steps)
    ck = clocks.stop()
    st = t.stats()
    # end to end through the public API from pinned host buffers
    step_host()
    ms_e2e = timed(step_host, max(1, min(args.steps, 3)))
    k_e2e = max(1, min(args.steps, 3))
    samples = (n + nt) * ws
    value = samples * args.steps / (ms / 1e3)
    e2e_value = samples * k_e2e / (ms_e2e / 1e3)
    peaks, peak_kind = measured_peaks()
    # roofline of the dominant kernel (the fused train kernel), timed with CUDA
    # events on the library's stream
    occ_units = 2 * 148
    alg = train_algorithmic_bytes(w, occ_units)
    # DRAM bytes of one k_train launch from an ncu capture of the same kernel
    # on the large sparse classifier's rows with 280 units and 40,000 samples
    # (profiles/k_train_c1_small_ncu.md: 1.856 GB read + 8.695 GB written),
    # scaled by units x samples to this launch.
    traffic = None
    if w["name"] == "large-sparse-classifier":
        per_unit_sample = (1.855563e9 + 8.695468e9) / (280 * 40000)
        traffic = per_unit_sample * (w["classes"] * w["clauses"] // 8) * w["n_train"]
    avg_ms = st["train_kernel_ms"] / max(1, st["train_launches"])
    achieved = alg / (avg_ms / 1e3) / 1e9
    wp = ((2 * w["features"] + 31) // 32 + 3) // 4 * 4
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": config_of(w, ws),
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int(n * d["x"].shape[1] + d[lab_key][:n].nbytes +
                                          nt * d["x"].shape[1]),
                "d2h_bytes_per_step": int(nt * (8 if w["kind"] == "classifier"
                                                else (w["classes"] + 7) // 8))},
        "gpu_launches": int(st["kernel_launches"]),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "kernel": "k_train", "peak_source": peak_kind,
                     "frac_of_nominal": achieved / 8000.0, "nominal_peak": 8000.0,
                     "algorithmic_bytes_per_launch": alg, "avg_launch_ms": avg_ms},
        "kernels": {
            "train_ms_per_step": st["train_kernel_ms"] / args.steps,
            "predict_ms_per_step": st["predict_kernel_ms"] / args.steps,
            "train_unit_steps": st["train_unit_steps"],
            "literal_evals_per_s_train_upper": st["train_unit_steps"] * 8 * 32 * wp /
                                               (st["train_kernel_ms"] / 1e3 + 1e-12),
            "predict_literal_evals_per_s": nt * w["classes"] * w["clauses"] * 2 * w["features"] /
                                           (st["predict_kernel_ms"] / max(1, st["predict_launches"]) / 1e3 + 1e-12),
        },
    }
    if rank == 0:
        # integer-pipe roofline of clause evaluation (after the timed region):
        # per 32 words k_predict's inner loop issues 62 logic ops (5 carry-save
        # steps of 4 AND-NOT + 6 LOP3, 3 direct steps of 4 AND-NOT) and 17
        # POPC (5 + 12); POPC and the logic ops issue on separate pipes
        pk = tm.int_peaks(dev.index if dev.index is not None else 0)
        wops = out["kernels"]["predict_literal_evals_per_s"] / 32
        bound = min(32 * pk["lop3"] / 62, 32 * pk["popc"] / 17)
        out["kernels"].update({"int_peaks_ops_per_s": pk, "predict_word_ops_per_s": wops,
                               "predict_int_bound_word_ops_per_s": bound,
                               "predict_frac_of_int_bound": wops / bound})
    if ck:
        out["clocks"] = ck
    if rank == 0 and ws == 1 and not args.no_cpu:
        cb = cpu_step(w, d, os.cpu_count())
        out["cpu_baseline"] = {"value": cb["value"], "unit": UNIT, "cores": cb["cores"],
                               "kind": cb["kind"], "sample": cb["sample"]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    t.destroy()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# batched hyper-parameter search: 64 machines, batched vs one per launch
# ---------------------------------------------------------------------------
def run_search(args):
    import torch
    import santoku_tsetlin as tm
    from santoku_tsetlin import datagen, multi
    ws, rank, local = dist_init()
    count, n_train, n_test = args.machines, 60000, 6000
    epochs = args.epochs or 2
    all_params = datagen.search_machines(count)
    # machines are independent: LPT partition by units across ranks (strong
    # scaling: the 64-machine round is fixed)
    parts = multi.partition_lpt([p["clauses"] * (p["features"] + 31) // 32 for p in all_params], ws)
    params = [all_params[i] for i in parts[rank]]
    count_local = len(params)
    protos = np.random.default_rng(7919 + 1).random((10, 784)) < 0.2
    xs = {}
    for negated in (True, False):
        x, y, _ = datagen.prototype_classifier(n_train + n_test, classes=10, features=784,
                                               seed=1, negated=negated, prototypes=protos)
        xs[negated] = (np.ascontiguousarray(x[:n_train]), np.ascontiguousarray(x[n_train:]))
    yv = y
    y_tr, y_te = np.ascontiguousarray(yv[:n_train]), yv[n_train:]
    dev = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(dev)
    xd = {k: (torch.from_numpy(v[0]).to(dev), torch.from_numpy(v[1]).to(dev)) for k, v in xs.items()}
    yd = torch.from_numpy(y_tr).to(dev)

    def make():
        out = []
        for p in params:
            out.append(tm.create("classifier", dict(
                classes=10, features=p["features"], clauses=p["clauses"],
                clause_tolerance=p["clause_tolerance"], clause_maximum=p["clause_maximum"],
                specificity=p["specificity"], target=p["target"], seed=p["seed"],
                reusable=True)))
        return out

    def tables():
        return [{"samples": n_train, "problems": xd[p["negated"]][0], "solutions": yd,
                 "iterations": epochs} for p in params]

    def timed(fn):
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return multi.max_over_ranks(e0.elapsed_time(e1), device=dev)

    warm = make()
    tm.train_batch(warm[:4], tables()[:4])
    for m in warm:
        m.destroy()
    batched = make()
    clocks = ClockSampler(0)
    clocks.start()
    ms_b = timed(lambda: tm.train_batch(batched, tables()) if batched else None)
    ck = clocks.stop()
    plain = make()
    tabs = tables()
    ms_p = timed(lambda: [m.train(t) for m, t in zip(plain, tabs)])
    same = all(np.array_equal(a.export_state()[0], b.export_state()[0])
               for a, b in zip(batched[:8], plain[:8]))
    acc_b = [float((m.predict(xd[p["negated"]][1], n_test).cpu().numpy() == y_te).mean())
             for m, p in zip(batched, params)]
    acc_p = [float((m.predict(xd[p["negated"]][1], n_test).cpu().numpy() == y_te).mean())
             for m, p in zip(plain, params)]
    samples = count * n_train * epochs
    units = sum(10 * p["clauses"] // 8 for p in all_params)
    out = {
        "metric": "TM batched search train samples/s", "value": samples / (ms_b / 1e3),
        "unit": "samples/s", "n_gpus": ws, "steps": 1, "warmup": 1, "ms_per_step": ms_b,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": "batched-search", "machines": count, "units": units,
                   "n_train": n_train, "epochs": epochs,
                   "clauses_per_class": [p["clauses"] for p in all_params],
                   "parallelism": "machines partitioned across ranks (LPT)" if ws > 1 else "single",
                   "step": "%d machines x %d epochs in one tm_train_batch" % (count, epochs)},
        "plain": {"value": samples / (ms_p / 1e3), "ms": ms_p,
                  "form": "one tm_train call (one launch group) per machine, in sequence"},
        "batched_over_plain": ms_p / ms_b,
        "bit_identical_first_8": bool(same),
        "accuracy": {"batched_mean": float(np.mean(acc_b)), "plain_mean": float(np.mean(acc_p))},
    }
    if ck:
        out["clocks"] = ck
    if rank == 0:
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# predict serving: 16 resident machines, Poisson arrivals
# ---------------------------------------------------------------------------
def run_serve(args):
    import ctypes
    import threading
    import santoku_tsetlin as tm
    L = tm.lib()
    rng = np.random.default_rng(11)
    shapes = ([("classifier", 10, 784, 256)] * 6 + [("classifier", 20, 16384, 2048)] * 5 +
              [("encoder", 256, 4096, 1024)] * 5)
    machines, pools = [], []
    for i, (kind, classes, feats, clauses) in enumerate(shapes):
        tbl = dict(clauses=clauses, clause_tolerance=64, clause_maximum=64, specificity=10.0,
                   seed=i)
        tbl.update(dict(classes=classes, features=feats) if kind == "classifier"
                   else dict(hidden=classes, visible=feats))
        t = tm.create(kind, tbl)
        info = t.info()
        acts = np.packbits(rng.random(info["action_chunks"] * 8) < 0.01, bitorder="little")
        t.import_state(actions=acts)
        blob = t.persist()
        t.destroy()
        machines.append(tm.load(blob, True))
        dens = 0.015 if feats == 16384 else 0.2
        pools.append(np.packbits(np.concatenate([(b := rng.random((4096, feats)) < dens), ~b],
                                                axis=1), axis=1, bitorder="little"))
    out = serve_at(args, L, tm, machines, pools, rng, args.rate)
    out["at_sustainable_rate"] = serve_at(args, L, tm, machines, pools, rng, args.sustainable_rate,
                                          requests=max(200, args.requests // 4))
    print(json.dumps(out), flush=True)


def serve_at(args, L, tm, machines, pools, rng, rate, requests=None):
    import ctypes
    import threading
    nreq = requests or args.requests
    gaps = rng.exponential(1.0 / rate, size=nreq)
    arrive = np.cumsum(gaps)
    sizes = np.exp(rng.uniform(0, np.log(4096), size=nreq)).astype(np.int64)
    which = rng.integers(0, len(machines), size=nreq)
    starts = [int(rng.integers(0, 4096 - s + 1)) for s in sizes]
    inputs = [np.ascontiguousarray(pools[w][st:st + s]).ravel()
              for w, st, s in zip(which, starts, sizes)]
    cfg = tm._ServerConfig(args.hbm_budget << 20, 8, 4096, 0)
    hs = (ctypes.c_void_p * len(machines))(*[m.handle.value for m in machines])
    srv = ctypes.c_void_p()
    assert L.tm_serve_open(ctypes.byref(cfg), hs, len(machines), ctypes.byref(srv)) == 0, \
        L.tm_last_error()
    ids = [0] * nreq
    t0 = time.perf_counter()

    def submit():
        for i in range(nreq):
            d = t0 + arrive[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            rid = ctypes.c_uint64()
            L.tm_serve_submit(srv, int(which[i]), inputs[i].ctypes.data, int(sizes[i]),
                              ctypes.byref(rid))
            ids[i] = rid.value

    th = threading.Thread(target=submit)
    th.start()
    th.join()
    lat = []
    for i in range(nreq):
        info_t = machines[which[i]]
        out = np.zeros(int(sizes[i]) * 32, dtype=np.int64)
        assert L.tm_serve_poll(srv, ids[i], out.ctypes.data, out.ctypes.data, 60_000_000) == 1
        us = ctypes.c_double()
        L.tm_serve_latency_us(srv, ids[i], ctypes.byref(us))
        lat.append(us.value / 1e3)
    makespan = float(np.max(arrive + np.array(lat) / 1e3))
    L.tm_serve_close(srv)
    # serial per-request predict under the same arrivals
    lat_s = []
    t0 = time.perf_counter()
    for i in range(nreq):
        d = t0 + arrive[i] - time.perf_counter()
        if d > 0:
            time.sleep(d)
        machines[which[i]].predict(inputs[i], int(sizes[i]))
        lat_s.append((time.perf_counter() - (t0 + arrive[i])) * 1e3)
    t_end_s = time.perf_counter()
    total = int(sizes.sum())
    out = {
        "metric": "serve p99 ms", "value": float(np.percentile(lat, 99)), "unit": "ms",
        "n_gpus": 1, "steps": nreq, "warmup": 0, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": "predict-serving", "machines": len(machines),
                   "shapes": "6 plain classifiers, 5 large sparse classifiers, 5 encoders",
                   "requests": nreq, "rate_per_s": rate, "batch": "log-uniform [1, 4096]",
                   "hbm_budget_mb": args.hbm_budget},
        "p50_ms": float(np.percentile(lat, 50)),
        "offered_samples_per_s": float(sizes.sum() / arrive[-1]),
        "samples_per_s": total / makespan,
        "serial": {"p50_ms": float(np.percentile(lat_s, 50)),
                   "p99_ms": float(np.percentile(lat_s, 99)),
                   "samples_per_s": total / (t_end_s - t0),
                   "form": "one tm_predict call per request, in arrival order"},
    }
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c1", choices=sorted(WORKLOADS) + ["search", "serve"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--machines", type=int, default=64, help="search: machines")
    ap.add_argument("--epochs", type=int, default=0, help="search: epochs (default 2)")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests")
    ap.add_argument("--rate", type=float, default=5000.0, help="serve: arrivals per second")
    ap.add_argument("--hbm-budget", type=int, default=2048, help="serve: staging MB")
    ap.add_argument("--sustainable-rate", type=float, default=150.0,
                    help="serve: second, sustainable arrival rate")
    args = ap.parse_args()
    if args.workload == "search":
        run_search(args)
        return
    if args.workload == "serve":
        run_serve(args)
        return
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, w)
    else:
        run_ours(args, w)


if __name__ == "__main__":
    main()
