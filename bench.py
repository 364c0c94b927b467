#!/usr/bin/env python
"""Benchmark of the Tsetlin-machine hot path on B200.

Metric: "TM train+predict samples/s (batched vs plain, equal accuracy)".

Default workload (N = 1): the batched hyper-parameter search -- 64
classifiers of uneven size (clauses per class log-uniform over 64..4,096,
specificity U[2, 40], target U[20, 400], negated literals on or off) on
plain-classifier data (10 classes, 784 features, class prototypes with 40 %
bit flips: a trained machine scores about 98 % macro F1) scaled to 60,000
train and 15,000 holdout samples.  A search
round trains all 64 for 10 epochs and scores each on the holdout after
every epoch (the reference's search loop, optimize.lua:424-471, with
train_tm's epoch logic, :586-653; search metric = macro F1 of
evaluator.class_accuracy).  One step is one epoch of the round: all 64
machines train one epoch over the 60,000 samples, then predict and score
the 15,000 holdout samples -- `tm_train_batch_search`, one CUDA graph
replay per epoch (the train kernels of the two row widths on two streams,
the holdout predict of the large machines as 8-bit GEMM nodes).  `value` counts machine-samples (train + holdout) per
second over K consecutive epochs; rounds restart after 10 epochs and their
set-up (machine creation, staging, graph capture) is inside the timed
region.  `plain` is the same round run the reference's way: one machine at
a time, one launch per epoch, the metric on the host between epochs.
`accuracy` checks that both forms end every machine with the same score
(they are bit-identical).

Other workloads (--workload): c1 / c0 / c2 -- one machine, one step = one
training epoch from the initial state + predict of the test set (large
predicts as the 8-bit GEMM); serve -- resident machines under Poisson
requests.

Arms:
  default           the CUDA library through the C ABI (santoku_tsetlin)
  --impl reference  the reference's CPU implementation of the same step on
                    this host's cores: the reference's own capi.c/automata.h
                    (oracle/_ref) where it was built, else the C restatement
                    (oracle/), on a bounded sample of units and samples,
                    scaled.

Under torchrun the search's machines are partitioned across ranks by cost
(LPT; no data-path collective) -- the 64-machine round is fixed work
(strong scaling); the single-machine workloads train one machine split by
class ranges (multi.train_sharded: every rank trains its classes, then one
all-gather of their automata, device to device over NCCL) and each rank
predicts its share of the test set.  `value` = the job's samples over the
max-over-ranks time.
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
# common
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
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def balanced_chunks(classes, threads, at_most):
    """8-clause chunks per class for a CPU sample whose unit count
    (classes x chunks) is a multiple of the thread count when possible, so
    that OpenMP's static schedule gives every thread the same units."""
    k = max(1, -(-threads // classes))
    while (classes * k) % threads and k < at_most:
        k += 1
    return max(1, min(k, at_most))


# Warp-instructions the fused train kernels issue per active (unit, sample)
# step -- a sample the unit trains on after negative sampling -- counted by
# ncu (smsp__inst_executed.sum of one launch divided by the launch's active
# steps, which the library counts itself), per (workload, mode, clauses per
# warp).  The int_issue roofline below is that count x the live active steps
# / the train kernel's live time, against 4 warp-instructions per clock per
# SM.  Capture commands:
#   TSETLIN_B200_AUTOTUNE=0 TSETLIN_B200_VARIANT=<mode>:<cpw> ncu --clock-control none \
#       -k regex:k_train -c 1 --metrics smsp__inst_executed.sum \
#       python bench.py --profile-launch search --search-train 6000
#   ncu --clock-control none -k regex:k_train -c 1 --metrics smsp__inst_executed.sum \
#       python bench.py --profile-launch c1_small
INSTR_PER_PAIR = {
    # batched search rows (784 / 392 features, 40 % flipped bits), 64
    # machines, one epoch over 6,000 samples: 87.03e9, 87.91e9 and 90.86e9
    # / 105.91e6
    ("search", 3, 1): 821.7,     # one warp per unit, four units per CTA
    ("search", 3, 2): 830.0,     # one warp per unit, one unit per CTA
    ("search", 4, 7): 857.9,     # one warp per unit, 2 words per lane in registers
    # large sparse classifier rows (16,384 features), c1_small (1.091e6 active
    # steps): 13.54e9 global planes; 11.66e9 word-per-thread (512 x 2 words)
    ("c1", 1, 1): 12410.0,
    ("c1_small", 1, 1): 12410.0,
    ("c1", 4, 1): 10681.0,
    ("c1_small", 4, 1): 10681.0,
}


def issue_roofline(key, pairs, kernel_ms, sm_mhz, extra=None):
    peak = 148 * 4 * sm_mhz * 1e6
    ipp = INSTR_PER_PAIR.get(key)
    r = {"bound": "int_issue", "unit": "warp-instr/s", "peak": peak,
         "peak_source": "148 SMs x 4 warp-instructions per clock x median SM clock under load",
         "variant": list(key[1:]), "active_pairs": int(pairs), "train_kernel_ms": kernel_ms,
         "instr_per_active_pair": ipp}
    if ipp and kernel_ms > 0:
        r["achieved"] = ipp * pairs / (kernel_ms / 1e3)
        r["frac"] = r["achieved"] / peak
    else:
        r["achieved"] = r["frac"] = None
    if extra:
        r.update(extra)
    return r


# ---------------------------------------------------------------------------
# single-machine workloads (c1 / c0 / c2)
# ---------------------------------------------------------------------------
def cpu_step(w, d, threads):
    """One step of the workload on the CPU, on a machine with the same rows
    but fewer clauses per class (units are independent 8-clause chunks, so
    per-unit work is unchanged), scaled to the full clause count.  Predict is
    timed on a slice of the test set and scaled likewise."""
    import oracle as O
    which = "ref" if O.ref_available() else "oracle"
    threads = threads or os.cpu_count()
    chunks = balanced_chunks(w["classes"], threads, w["clauses"] // 8)
    clauses = 8 * chunks
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
    scale_units = (w["clauses"] // 8) / chunks
    step_s = t_train * scale_units + t_pred * scale_units * (w["n_test"] / nt)
    samples = w["n_train"] + w["n_test"]
    sample = ("1 train epoch of %d of %d clauses per class (%d of %d units, a multiple of the "
              "%d threads) over all %d samples + predict of %d of %d test samples; times "
              "scaled by units and samples"
              % (clauses, w["clauses"], chunks * w["classes"],
                 (w["clauses"] // 8) * w["classes"], threads, n, nt, w["n_test"]))
    return dict(value=samples / step_s, step_s=step_s, kind="reference" if which == "ref" else "port",
                cores=threads, sample=sample, measured_s=t_train + t_pred)


def config_of(w, ws):
    return {
        "workload": w["name"], "type": w["kind"], "classes": w["classes"],
        "features": w["features"], "literal_bits": 2 * w["features"], "clauses": w["clauses"],
        "clause_tolerance": w["clause_tolerance"], "clause_maximum": w["clause_maximum"],
        "specificity": w["specificity"], "target": w["target"], "state_bits": 8,
        "n_train": w["n_train"], "n_test": w["n_test"],
        "step": "train{iterations=1} from the initial state + predict(test)",
        "parallelism": "class-sharded" if ws > 1 else "single",
        "l2": "inputs larger than L2 (train set and automata exceed 126 MB)",
    }


def run_reference(args, w):
    ws, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    d = make_data(w)
    threads = os.cpu_count()
    vals = []
    for _ in range(max(1, min(args.steps, 3))):
        vals.append(cpu_step(w, d, threads))
    v = float(np.median([r["value"] for r in vals]))
    step_s = float(np.median([r["step_s"] for r in vals]))
    # a step is the bounded sample: ms_per_step is its measured time (so
    # steps x ms_per_step is the arm's own wall time); the full workload's
    # equivalent step, from which `value` is computed, is reported beside it
    meas = float(sum(r["measured_s"] for r in vals))
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
        "steps": len(vals), "warmup": 0, "ms_per_step": meas / len(vals) * 1e3,
        "scaled_ms_per_step": step_s * 1e3, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": config_of(w, ws),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": vals[0]["cores"],
                         "kind": vals[0]["kind"], "sample": vals[0]["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "measured_s": float(sum(r["measured_s"] for r in vals)),
    }
    print(json.dumps(out), flush=True)


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
    from santoku_tsetlin import multi
    ws, rank, local = dist_init()
    dev = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(dev)
    d = make_data(w, 0)
    n, nt = w["n_train"], w["n_test"]
    # one machine trained class-sharded; every rank (holding the whole
    # trained machine after the exchange) predicts its share of the test set
    lo_s, hi_s = multi.class_range(nt, ws, rank)
    lab_key = "y" if w["kind"] == "classifier" else "codes"
    # device-resident inputs (value) and pinned host inputs (e2e)
    x_dev = torch.from_numpy(np.ascontiguousarray(d["x"][:n])).to(dev)
    lab_dev = torch.from_numpy(np.ascontiguousarray(d[lab_key][:n])).to(dev)
    xt_dev = torch.from_numpy(np.ascontiguousarray(d["x"][n + lo_s:n + hi_s])).to(dev)
    x_host = torch.from_numpy(np.ascontiguousarray(d["x"][:n])).pin_memory()
    lab_host = torch.from_numpy(np.ascontiguousarray(d[lab_key][:n])).pin_memory()
    xt_host = torch.from_numpy(np.ascontiguousarray(d["x"][n + lo_s:n + hi_s])).pin_memory()
    t = tm.create(w["kind"], create_table(w, seed=0))
    t.stats_enable(True)

    def train(tbl):
        if ws > 1:
            multi.train_sharded(t, tbl, device=dev)
        else:
            t.train(tbl)

    def step_dev():
        train(train_table(w, x_dev, lab_dev))
        return t.predict(xt_dev, hi_s - lo_s)

    def step_host():
        train(train_table(w, x_host.numpy(), lab_host.numpy()))
        return t.predict(xt_host.numpy(), hi_s - lo_s)

    def timed(fn, k):
        barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            fn()
        e1.record()
        torch.cuda.synchronize()
        barrier(ws)
        return multi.max_over_ranks(e0.elapsed_time(e1), device=dev)

    for _ in range(args.warmup):
        step_dev()
    t.reset_stats()
    clocks = ClockSampler(dev.index)
    clocks.start()
    ms = timed(step_dev, args.steps)
    ck = clocks.stop()
    st = t.stats()
    step_host()
    k_e2e = max(1, min(args.steps, 3))
    ms_e2e = timed(step_host, k_e2e)
    samples = n + nt
    value = samples * args.steps / (ms / 1e3)
    e2e_value = samples * k_e2e / (ms_e2e / 1e3)
    peaks, peak_kind = measured_peaks()
    avg_ms = st["train_kernel_ms"] / max(1, st["train_launches"])
    alg = train_algorithmic_bytes(w, max(1, st["train_resident"]))
    wp = ((2 * w["features"] + 31) // 32 + 3) // 4 * 4
    sm_mhz = (ck or {}).get("sm_mhz") or 1965.0
    key = (args.workload, st["train_mode"], st["train_cpw"])
    roof = issue_roofline(key, st["train_active_pairs"] / max(1, st["train_launches"]), avg_ms,
                          sm_mhz, extra={
                              "kernel": "k_train_warp" if st["train_mode"] == 3 else "k_train",
                              "hbm": {"algorithmic_bytes_per_launch": alg,
                                      "achieved_gbs": alg / (avg_ms / 1e3) / 1e9,
                                      "peak_gbs": peaks["hbm_gbs"], "peak_source": peak_kind,
                                      "resident_units": st["train_resident"]},
                              "avg_launch_ms": avg_ms, "traffic": None})
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": config_of(w, ws),
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int(n * d["x"].shape[1] + d[lab_key][:n].nbytes +
                                          (hi_s - lo_s) * d["x"].shape[1]),
                "d2h_bytes_per_step": int((hi_s - lo_s) * (8 if w["kind"] == "classifier"
                                                           else (w["classes"] + 7) // 8))},
        "gpu_launches": int(st["kernel_launches"]),
        "roofline": roof,
        "kernels": {
            "train_ms_per_step": st["train_kernel_ms"] / args.steps,
            "predict_ms_per_step": st["predict_kernel_ms"] / args.steps,
            "train_unit_steps": st["train_unit_steps"],
            "train_active_pairs": st["train_active_pairs"],
            "literal_evals_per_s_train_upper": st["train_unit_steps"] * 8 * 32 * wp /
                                               (st["train_kernel_ms"] / 1e3 + 1e-12),
            "predict_literal_evals_per_s": (hi_s - lo_s) * w["classes"] * w["clauses"] * 2 *
                                           w["features"] /
                                           (st["predict_kernel_ms"] / max(1, st["predict_launches"])
                                            / 1e3 + 1e-12),
        },
    }
    if rank == 0 and st["predict_gemm"]:
        # the predict ran as an 8-bit GEMM: clauses x samples x literal
        # bytes (32 per row word), two operations per product
        words = (((2 * w["features"] + 7) // 8 + 3) // 4)
        ops = 2.0 * w["classes"] * w["clauses"] * (hi_s - lo_s) * 32 * words
        t_s = st["predict_kernel_ms"] / max(1, st["predict_launches"]) / 1e3 + 1e-12
        out["kernels"].update({
            "predict_path": "int8 GEMM" if st["predict_gemm"] == 1 else "e4m3 GEMM",
            "predict_tensor_ops_per_s": ops / t_s,
            "predict_tensor_peak_ops_per_s": 4.5e15,
            "predict_tensor_peak_source": "nominal dense 8-bit rate of a B200 (no measured "
                                          "8-bit peak here); the predict time includes the "
                                          "byte expansions and the vote epilogue",
            "predict_frac_of_tensor_peak": ops / t_s / 4.5e15})
    elif rank == 0:
        pk = tm.int_peaks(dev.index if dev.index is not None else 0)
        wops = out["kernels"]["predict_literal_evals_per_s"] / 32
        bound = min(32 * pk["lop3"] / 62, 32 * pk["popc"] / 17)
        out["kernels"].update({"predict_path": "bitwise", "int_peaks_ops_per_s": pk,
                               "predict_word_ops_per_s": wops,
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
# batched hyper-parameter search (default): 64 machines, device-resident
# rounds vs the plain one-machine-per-launch form
# ---------------------------------------------------------------------------
# flip: each bit of a sample differs from its class prototype with this
# probability; at 0.4 a trained machine scores about 98 % on the holdout
# (MNIST-like), so the search metric is not saturated
SEARCH = dict(machines=64, n_train=60000, n_test=15000, epochs=10, classes=10, features=784,
              flip=0.4)


def search_data():
    from santoku_tsetlin import datagen
    n = SEARCH["n_train"] + SEARCH["n_test"]
    cache = "/tmp/tsetlin_b200_search_%d_f%g.npz" % (n, SEARCH["flip"])
    if os.path.exists(cache):
        z = np.load(cache)
        return {True: (z["x1"], z["xt1"]), False: (z["x0"], z["xt0"]), "y": z["y"], "yt": z["yt"]}
    protos = np.random.default_rng(7919 + 1).random((SEARCH["classes"], SEARCH["features"])) < 0.2
    out = {}
    for negated in (True, False):
        x, y, _ = datagen.prototype_classifier(n, classes=SEARCH["classes"],
                                               features=SEARCH["features"], seed=1,
                                               flip=SEARCH["flip"], negated=negated,
                                               prototypes=protos)
        out[negated] = (np.ascontiguousarray(x[:SEARCH["n_train"]]),
                        np.ascontiguousarray(x[SEARCH["n_train"]:]))
    out["y"] = np.ascontiguousarray(y[:SEARCH["n_train"]])
    out["yt"] = np.ascontiguousarray(y[SEARCH["n_train"]:])
    try:
        np.savez(cache, x1=out[True][0], xt1=out[True][1], x0=out[False][0],
                 xt0=out[False][1], y=out["y"], yt=out["yt"])
    except OSError:
        pass
    return out


def search_params(ws=1, rank=0):
    from santoku_tsetlin import datagen, multi
    allp = datagen.search_machines(SEARCH["machines"])
    parts = multi.partition_lpt([p["clauses"] * (p["features"] + 31) // 32 for p in allp], ws)
    return allp, [allp[i] for i in parts[rank]]


def search_config(ws, allp, n_train):
    return {
        "workload": "batched-search", "machines": len(allp), "classes": SEARCH["classes"],
        "features": SEARCH["features"],
        "clauses_per_class": [p["clauses"] for p in allp],
        "units": sum(SEARCH["classes"] * p["clauses"] // 8 for p in allp),
        "negated": [p["negated"] for p in allp],
        "specificity_range": [2, 40], "target_range": [20, 400], "clause_tolerance": 64,
        "clause_maximum": 64, "state_bits": 8, "n_train": n_train, "n_test": SEARCH["n_test"],
        "epochs_per_round": SEARCH["epochs"], "search_metric": "macro F1 (class_accuracy)",
        "step": "one epoch of the device-resident round: every machine trains one epoch over "
                "the train set, then predicts and scores the holdout (one CUDA graph replay)",
        "parallelism": "machines partitioned across ranks (LPT)" if ws > 1 else "single",
        "l2": "inputs larger than L2 (the 64 machines' automata, 1.2 GB, exceed 126 MB)",
    }


def make_search_machines(tm, params):
    return [tm.create("classifier", dict(
        classes=SEARCH["classes"], features=p["features"], clauses=p["clauses"],
        clause_tolerance=p["clause_tolerance"], clause_maximum=p["clause_maximum"],
        specificity=p["specificity"], target=p["target"], seed=p["seed"], reusable=True))
        for p in params]


def run_search_bench(args):
    import torch
    import santoku_tsetlin as tm
    from santoku_tsetlin import multi
    ws, rank, local = dist_init()
    dev = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(dev)
    n_train = args.search_train or SEARCH["n_train"]
    allp, params = search_params(ws, rank)
    d = search_data()
    nt, E = SEARCH["n_test"], SEARCH["epochs"]
    xd = {k: (torch.from_numpy(d[k][0][:n_train]).to(dev), torch.from_numpy(d[k][1]).to(dev))
          for k in (True, False)}
    yd = torch.from_numpy(d["y"][:n_train]).to(dev)
    ytd = torch.from_numpy(d["yt"]).to(dev)

    def round_(iters, host=False, stats=None):
        """One device-resident round of `iters` epochs of every local
        machine (fresh machines, as the search creates them per trial)."""
        ms = make_search_machines(tm, params)
        if stats is not None and ms:
            ms[0].stats_enable(True)  # the round's statistics gather on its first machine
        tabs = [{"samples": n_train,
                 "problems": d[p["negated"]][0][:n_train] if host else xd[p["negated"]][0],
                 "solutions": d["y"][:n_train] if host else yd, "iterations": iters}
                for p in params]
        test = {"samples": nt, "solutions": d["yt"] if host else ytd,
                "problems_each": [d[p["negated"]][1] if host else xd[p["negated"]][1]
                                  for p in params]}
        r = tm.train_batch_search(ms, tabs, test, patience=0, metric="f1") if ms else None
        if stats is not None and ms:
            stats.append(ms[0].stats())
        for m in ms:
            m.destroy()
        return r

    if args.profile_launch:
        # one round of one epoch: the launch an ncu capture profiles
        st = []
        round_(1, stats=st)
        print(json.dumps({"profile_launch": "search", "mode": st[0]["train_mode"],
                          "cpw": st[0]["train_cpw"],
                          "active_pairs": st[0]["train_active_pairs"],
                          "train_kernel_ms": st[0]["search_train_ms"],
                          "resident_units": st[0]["train_resident"]}), flush=True)
        return
    # ---- warm-up: W epochs (tuning, first-touch allocations) ---------------
    round_(max(1, args.warmup))
    torch.cuda.synchronize()
    # ---- timed: K epochs of device-resident rounds ---------------------------
    K = args.steps
    stats = []
    clocks = ClockSampler(dev.index if dev.index is not None else 0)
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.start()
    e0.record()
    done = 0
    while done < K:
        it = min(E, K - done)
        round_(it, stats=stats)
        done += it
    e1.record()
    torch.cuda.synchronize()
    ck = clocks.stop()
    barrier(ws)
    ms_b = multi.max_over_ranks(e0.elapsed_time(e1), device=dev)
    train_ms = sum(x["search_train_ms"] for x in stats)
    graph_ms = sum(x["search_epoch_ms"] for x in stats)
    pairs = sum(x["train_active_pairs"] for x in stats)
    launches = sum(x["kernel_launches"] for x in stats)
    modes = sorted({(x["train_mode"], x["train_cpw"]) for x in stats})
    value = len(allp) * (n_train + nt) * K / (ms_b / 1e3)

    # ---- plain: one machine at a time, one launch per epoch, host metric ---
    pe = min(args.plain_epochs, E)
    plain_final = {}
    # untimed: one short train call per machine, so that the variant choice
    # of every machine's launch shape is tuned and cached before the timing
    # (the batched form's was, in its warm-up round)
    for p in params:
        m = make_search_machines(tm, [p])[0]
        k = min(2048, n_train)
        m.train({"samples": k, "problems": xd[p["negated"]][0][:k], "solutions": yd[:k],
                 "iterations": 1})
        m.destroy()
    barrier(ws)
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    for i, p in enumerate(params):
        m = make_search_machines(tm, [p])[0]
        scores = []

        def each(epoch, m=m, xt=xd[p["negated"]][1], scores=scores):
            scores.append(tm.class_accuracy(m.predict(xt, nt), ytd, nt, SEARCH["classes"])["f1"])
            return True
        m.train({"samples": n_train, "problems": xd[p["negated"]][0], "solutions": yd,
                 "iterations": pe, "each": each})
        plain_final[i] = scores[-1]
        m.destroy()
    p1.record()
    torch.cuda.synchronize()
    barrier(ws)
    ms_p = multi.max_over_ranks(p0.elapsed_time(p1), device=dev)
    plain_value = len(allp) * (n_train + nt) * pe / (ms_p / 1e3)

    # ---- end to end from host buffers: one round of the plain form's epochs
    # (so the two forms' final scores must agree machine by machine) ---------
    barrier(ws)
    torch.cuda.synchronize()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record()
    r = round_(pe, host=True)
    q1.record()
    torch.cuda.synchronize()
    barrier(ws)
    ms_e = multi.max_over_ranks(q0.elapsed_time(q1), device=dev)
    e2e_value = len(allp) * (n_train + nt) * pe / (ms_e / 1e3)
    batched_final = {i: float(r["final"][i]) for i in range(len(params))} if r else {}
    same = all(batched_final[i] == plain_final[i] for i in range(len(params)))
    # bytes copied per round: each machine's train rows and holdout (the
    # library stages identical inputs once: one copy per literal layout)
    # and the labels; back: the per-machine states once per epoch
    h2d = sum(d[neg][0][:n_train].nbytes + d[neg][1].nbytes
              for neg in {p["negated"] for p in params}) + d["y"][:n_train].nbytes + \
        d["yt"].nbytes
    sm_mhz = (ck or {}).get("sm_mhz") or 1965.0
    key = ("search",) + (modes[-1] if len(modes) == 1 else (-1, -1))
    # HBM view of one epoch's train launch: the automata read and written
    # once, the rows once per wave of resident units
    wp = {p["negated"]: ((2 * p["features"] + 31) // 32 + 3) // 4 * 4 for p in params}
    state = sum(SEARCH["classes"] * p["clauses"] * 8 * wp[p["negated"]] * 4 for p in params)
    resident = stats[0]["train_resident"] if stats else 1
    units = sum(SEARCH["classes"] * p["clauses"] // 8 for p in params)
    waves = -(-units // max(1, resident))
    alg = 2 * state + waves * n_train * max(wp.values()) * 4
    per_launch_ms = train_ms / max(1, K)
    roof = issue_roofline(key, pairs, train_ms, sm_mhz, extra={
        "kernel": "k_train_warp" if key[1] == 3 else ("k_train_wpt" if key[1] == 4 else "k_train"),
        "epoch_graph_ms": graph_ms, "train_share_of_graph": train_ms / graph_ms if graph_ms else None,
        "resident_units": resident,
        "hbm": {"algorithmic_bytes_per_launch": alg,
                "achieved_gbs": alg / (per_launch_ms / 1e3) / 1e9 if per_launch_ms else None,
                "peak_gbs": measured_peaks()[0]["hbm_gbs"]},
        # DRAM bytes of the one-warp kernel's launch in an ncu capture of
        # one epoch over 6,000 samples (0.967 GB read + 0.890 GB written):
        # the automata once each way; the rows of both literal layouts stay
        # in L2 between waves, so only their first read grows with samples
        "traffic": (1.857e9 + (n_train - 6000) * sum(wp.values()) * 4)
        if key[1] == 3 else None,
        "traffic_source": "ncu capture at 6,000 samples, rows' first read scaled to the "
                          "launch's samples"})
    peaks, peak_kind = measured_peaks()
    out = {
        "metric": METRIC + " (batched vs plain, equal accuracy)", "value": value, "unit": UNIT,
        "n_gpus": ws, "steps": K, "warmup": args.warmup, "ms_per_step": ms_b / K,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic", "config": search_config(ws, allp, n_train),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d / pe),
                "d2h_bytes_per_step": int(len(params) * 64),
                "form": "train_batch_search from host numpy buffers, one round of %d epochs; "
                        "the round's copies spread over its epochs" % pe},
        "gpu_launches": int(launches),
        "plain": {"value": plain_value, "ms": ms_p, "epochs": pe,
                  "form": "one tm_train per machine in turn with an `each` callback that "
                          "predicts and scores the holdout (one launch per epoch per machine: "
                          "the reference's train_tm flow)"},
        "batched_over_plain": value / plain_value,
        "accuracy": {"equal": bool(same), "epochs": pe,
                     "batched_mean_f1": float(np.mean(list(batched_final.values()))),
                     "plain_mean_f1": float(np.mean(list(plain_final.values())))},
        "roofline": roof,
        "hbm_peak": {"value": peaks["hbm_gbs"], "unit": "GB/s", "source": peak_kind},
    }
    if ck:
        out["clocks"] = ck
    if rank == 0 and ws == 1 and not args.no_cpu:
        cb = cpu_search_step(allp, d, os.cpu_count(), n_sample=args.cpu_samples)
        out["cpu_baseline"] = {"value": cb["value"], "unit": UNIT, "cores": cb["cores"],
                               "kind": cb["kind"], "sample": cb["sample"]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def cpu_search_step(allp, d, threads, n_sample=6000):
    """One epoch of the 64-machine round on the CPU: each machine, with
    enough 8-clause chunks per class for its units to be a multiple of the
    thread count (units are independent, so per-unit work is the full
    machine's), trains one epoch over `n_sample` of the train samples and
    predicts `n_sample` / 4 holdout samples; times scaled by the machine's
    units and by samples."""
    import oracle as O
    which = "ref" if O.ref_available() else "oracle"
    total_s, measured = 0.0, 0.0
    n_pred = max(1, n_sample // 4)
    n_train, nt = SEARCH["n_train"], SEARCH["n_test"]
    for p in allp:
        chunks = balanced_chunks(SEARCH["classes"], threads, p["clauses"] // 8)
        cfg = dict(type="classifier", classes=SEARCH["classes"], features=p["features"],
                   clauses=8 * chunks, clause_tolerance=p["clause_tolerance"],
                   clause_maximum=p["clause_maximum"], specificity=p["specificity"],
                   target=p["target"])
        m = O.Machine(which=which, **cfg)
        x, xt = d[p["negated"]]
        t0 = time.perf_counter()
        m.train(x[:n_sample].ravel(), n_sample, 1, labels=d["y"][:n_sample], seed=p["seed"],
                mode=O.REFSTRUCT if which == "ref" else O.PHILOX, threads=threads)
        t1 = time.perf_counter()
        m.predict(xt[:n_pred].ravel(), n_pred, threads=threads)
        t2 = time.perf_counter()
        scale = (p["clauses"] // 8) / chunks
        total_s += (t1 - t0) * scale * (n_train / n_sample) + (t2 - t1) * scale * (nt / n_pred)
        measured += t2 - t0
    samples = len(allp) * (n_train + nt)
    sample = ("one epoch of each of the %d machines with a thread-balanced %d-%d units each "
              "over %d of %d train samples, predict of %d of %d holdout samples; scaled by "
              "units and samples" % (len(allp), SEARCH["classes"],
                                     SEARCH["classes"] * balanced_chunks(SEARCH["classes"], threads, 512),
                                     n_sample, n_train, n_pred, nt))
    return dict(value=samples / total_s, step_s=total_s, measured_s=measured,
                kind="reference" if which == "ref" else "port", cores=threads, sample=sample)


def run_search_reference(args):
    ws, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    allp, _ = search_params(1, 0)
    d = search_data()
    threads = os.cpu_count()
    vals = []
    for _ in range(max(1, args.steps)):
        vals.append(cpu_search_step(allp, d, threads, n_sample=args.cpu_samples))
        if sum(v["measured_s"] for v in vals) > args.cpu_budget:
            break
    v = float(np.median([r["value"] for r in vals]))
    step_s = float(np.median([r["step_s"] for r in vals]))
    meas = float(sum(r["measured_s"] for r in vals))
    out = {
        "impl": "reference", "metric": METRIC + " (batched vs plain, equal accuracy)",
        "value": v, "unit": UNIT, "n_gpus": ws, "steps": len(vals), "warmup": 0,
        # the bounded sample's measured time per step; the full epoch's
        # equivalent (from which `value` is computed) beside it
        "ms_per_step": meas / len(vals) * 1e3, "scaled_ms_per_step": step_s * 1e3,
        "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": search_config(ws, allp, SEARCH["n_train"]),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": vals[0]["cores"],
                         "kind": vals[0]["kind"], "sample": vals[0]["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "measured_s": float(sum(r["measured_s"] for r in vals)),
    }
    print(json.dumps(out), flush=True)


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


class Heartbeat:
    """A host thread that sleeps 1 ms at a time and records every wake-up
    that came more than 10 ms late: times when this process did not run (or
    its interpreter lock was held) for that long.  Beside the requests'
    latencies it tells a pause of the whole process from one of the GPU."""

    def __init__(self, t0):
        import threading
        self.t0, self.gaps, self.stop = t0, [], False
        self.th = threading.Thread(target=self.run, daemon=True)
        self.th.start()

    def run(self):
        last = time.perf_counter()
        while not self.stop:
            time.sleep(0.001)
            now = time.perf_counter()
            if now - last > 0.010:
                self.gaps.append((last - self.t0, (now - last) * 1e3))
            last = now

    def finish(self, k=5):
        self.stop = True
        self.th.join()
        return {"late_wakeups_over_10ms": len(self.gaps),
                "largest": [{"at_s": float(a), "gap_ms": float(g)}
                            for a, g in sorted(self.gaps, key=lambda v: -v[1])[:k]]}


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
    cfg = tm._ServerConfig(args.hbm_budget << 20, 8, 4096, 0, 0, 0)
    hs = (ctypes.c_void_p * len(machines))(*[m.handle.value for m in machines])
    srv = ctypes.c_void_p()
    assert L.tm_serve_open(ctypes.byref(cfg), hs, len(machines), ctypes.byref(srv)) == 0, \
        L.tm_last_error()
    # warm-up, untimed: a request of each size class for every machine, so
    # that first-use costs (kernel loading, library set-up) stay out of the
    # measured latencies, as they do for the serial form, which runs later
    nwarm = 0
    for k in range(len(machines)):
        for s_ in (1, 40, 300, 4096):
            x = np.ascontiguousarray(pools[k][:s_]).ravel()
            rid = ctypes.c_uint64()
            assert L.tm_serve_submit(srv, k, x.ctypes.data, s_, ctypes.byref(rid)) == 0
            out = np.zeros(s_ * 32, dtype=np.int64)
            assert L.tm_serve_poll(srv, rid.value, out.ctypes.data, out.ctypes.data,
                                   60_000_000) == 1
            nwarm += 1
    ids = [0] * nreq
    t0 = time.perf_counter()
    hb = Heartbeat(t0)

    def submit():
        for i in range(nreq):
            d = t0 + arrive[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            rid = ctypes.c_uint64()
            rc = L.tm_serve_submit(srv, int(which[i]), inputs[i].ctypes.data, int(sizes[i]),
                                   ctypes.byref(rid))
            ids[i] = rid.value if rc == 0 else None  # refused: the queue was full

    th = threading.Thread(target=submit)
    th.start()
    th.join()
    lat, acc_sizes, acc_arrive, acc_which, phases = [], [], [], [], []
    for i in range(nreq):
        if ids[i] is None:
            continue
        acc_which.append(int(which[i]))
        out = np.zeros(int(sizes[i]) * 32, dtype=np.int64)
        assert L.tm_serve_poll(srv, ids[i], out.ctypes.data, out.ctypes.data, 60_000_000) == 1
        us = ctypes.c_double()
        L.tm_serve_latency_us(srv, ids[i], ctypes.byref(us))
        lat.append(us.value / 1e3)
        ph = (ctypes.c_double * 4)()
        L.tm_serve_phases_us(srv, ids[i], ph)
        phases.append([v / 1e3 for v in ph])
        acc_sizes.append(int(sizes[i]))
        acc_arrive.append(arrive[i])
    makespan = float(np.max(np.array(acc_arrive) + np.array(lat) / 1e3))
    host_server = hb.finish()
    L.tm_serve_close(srv)
    # serial per-request predict under the same arrivals
    lat_s = []
    t0 = time.perf_counter()
    hb = Heartbeat(t0)
    for i in range(nreq):
        d = t0 + arrive[i] - time.perf_counter()
        if d > 0:
            time.sleep(d)
        machines[which[i]].predict(inputs[i], int(sizes[i]))
        lat_s.append((time.perf_counter() - (t0 + arrive[i])) * 1e3)
    t_end_s = time.perf_counter()
    host_serial = hb.finish()
    total = int(sizes.sum())
    out = {
        "metric": "serve p99 ms", "value": float(np.percentile(lat, 99)), "unit": "ms",
        "n_gpus": 1, "steps": nreq, "warmup": nwarm, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": "predict-serving", "machines": len(machines),
                   "shapes": "6 plain classifiers, 5 large sparse classifiers, 5 encoders",
                   "requests": nreq, "rate_per_s": rate, "batch": "log-uniform [1, 4096]",
                   "hbm_budget_mb": args.hbm_budget,
                   "queue_bound_samples": 64 * 4096},
        "p50_ms": float(np.percentile(lat, 50)),
        "small_requests": {"max_samples": 256,
                           "p50_ms": float(np.percentile([v for v, z in zip(lat, acc_sizes)
                                                          if z <= 256] or [0], 50)),
                           "p99_ms": float(np.percentile([v for v, z in zip(lat, acc_sizes)
                                                          if z <= 256] or [0], 99))},
        "accepted": len(lat), "refused_queue_full": nreq - len(lat),
        "slowest": [{"machine": acc_which[j], "samples": acc_sizes[j],
                     "latency_ms": lat[j], "arrival_s": float(acc_arrive[j]),
                     "queue_ms": phases[j][0], "host_launch_ms": phases[j][1],
                     "device_ms": phases[j][2], "launch_gpu_span_ms": phases[j][3]}
                    for j in np.argsort(lat)[::-1][:6]],
        # each phase's own p99 over the accepted requests: the wait in the
        # queue, the worker's staging and launch calls, the device work and
        # the completion; and of the launches' device spans (CUDA events
        # around each launch)
        "phase_p99_ms": {k: float(np.percentile([p[i] for p in phases], 99))
                         for i, k in enumerate(("queue", "host_launch", "device",
                                                "launch_gpu_span"))},
        # late wake-ups of a 1 ms host heartbeat while the server ran and
        # while the serial form ran (seconds from each form's start)
        "host_heartbeat": {"server": host_server, "serial": host_serial},
        "offered_samples_per_s": float(sizes.sum() / arrive[-1]),
        "samples_per_s": float(sum(acc_sizes)) / makespan,
        "serial": {"p50_ms": float(np.percentile(lat_s, 50)),
                   "p99_ms": float(np.percentile(lat_s, 99)),
                   "small_p99_ms": float(np.percentile([v for v, z in zip(lat_s, sizes)
                                                        if z <= 256] or [0], 99)),
                   "samples_per_s": total / (t_end_s - t0),
                   "form": "one tm_predict call per request, in arrival order"},
    }
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="search", choices=sorted(WORKLOADS) + ["search", "serve"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--plain-epochs", type=int, default=10,
                    help="search: epochs of the plain form and of the e2e round")
    ap.add_argument("--search-train", type=int, default=0,
                    help="search: train samples (default 60,000; fewer for profiler captures)")
    ap.add_argument("--cpu-samples", type=int, default=6000,
                    help="search: train samples of the CPU reference's sampled epoch")
    ap.add_argument("--cpu-budget", type=float, default=150.0,
                    help="search --impl reference: stop after this many measured CPU seconds")
    ap.add_argument("--profile-launch", default="", choices=["", "search"] + sorted(WORKLOADS),
                    help="run only the train launch a profiler capture looks at")
    ap.add_argument("--epoch-times", type=int, default=0,
                    help="c1/c0/c2: train this many epochs and print each epoch's kernel time")
    ap.add_argument("--predict-sizes", default="",
                    help="c1/c0/c2: comma-separated batch sizes; print each predict's kernel time")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests")
    ap.add_argument("--rate", type=float, default=5000.0, help="serve: arrivals per second")
    ap.add_argument("--hbm-budget", type=int, default=4096, help="serve: launch-slot memory, MB")
    ap.add_argument("--sustainable-rate", type=float, default=150.0,
                    help="serve: second, sustainable arrival rate")
    args = ap.parse_args()
    if args.profile_launch and args.profile_launch != "search":
        run_profile_launch(args, WORKLOADS[args.profile_launch])
        return
    if args.epoch_times:
        run_epoch_times(args, WORKLOADS[args.workload])
        return
    if args.predict_sizes:
        run_predict_sizes(args, WORKLOADS[args.workload])
        return
    if args.workload == "search" or args.profile_launch == "search":
        if args.impl == "reference":
            run_search_reference(args)
        else:
            run_search_bench(args)
        return
    if args.workload == "serve":
        run_serve(args)
        return
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, w)
    else:
        run_ours(args, w)


def run_epoch_times(args, w):
    """Device time of the train kernel in each of `--epoch-times` epochs of
    one training (one launch per epoch: an `each` callback between epochs
    that predicts 2,000 held-out samples)."""
    import torch
    import santoku_tsetlin as tm
    d = make_data(w, 0)
    n = w["n_train"]
    nt = min(2000, w["n_test"])
    lab_key = "y" if w["kind"] == "classifier" else "codes"
    x = torch.from_numpy(np.ascontiguousarray(d["x"][:n])).cuda()
    lab = torch.from_numpy(np.ascontiguousarray(d[lab_key][:n])).cuda()
    xt = torch.from_numpy(np.ascontiguousarray(d["x"][n:n + nt])).cuda()
    t = tm.create(w["kind"], create_table(w, seed=0))
    t.stats_enable(True)
    per, acc, last = [], [], [0.0]

    def each(epoch):
        st = t.stats()
        per.append(st["train_kernel_ms"] - last[0])
        last[0] = st["train_kernel_ms"]
        if w["kind"] == "classifier":
            acc.append(float((t.predict(xt, nt).cpu().numpy() == d["y"][n:n + nt]).mean()))
        return True
    tbl = train_table(w, x, lab)
    tbl.update(iterations=args.epoch_times, each=each)
    t.train(tbl)
    st = t.stats()
    print(json.dumps({"epoch_times": w["name"], "train_kernel_ms": per, "holdout_accuracy": acc,
                      "mode": st["train_mode"], "cpw": st["train_cpw"],
                      "mean_ms": float(np.mean(per))}), flush=True)
    t.destroy()


def run_predict_sizes(args, w):
    """Predict on a trained-state-sized machine with random actions (1 % of
    the automata included) for each batch size of `--predict-sizes`, across
    the small-batch (warp per clause row) and tiled kernels' switch:
    kernel_ms = the predict kernel's CUDA-event time; call_us = wall time of
    one tm_predict call through the C ABI from host buffers (copies in and
    out, launches, the wait for the result), the latency a caller sees."""
    import ctypes
    import torch
    import santoku_tsetlin as tm
    d = make_data(w, 0)
    t = tm.create(w["kind"], create_table(w, seed=0))
    info = t.info()
    rng = np.random.default_rng(5)
    t.import_state(actions=np.packbits(rng.random(info["action_chunks"] * 8) < 0.01,
                                       bitorder="little"))
    t.stats_enable(True)
    lib = tm.lib()
    out, call = {}, {}
    for k in [int(v) for v in args.predict_sizes.split(",")]:
        xs = torch.from_numpy(np.ascontiguousarray(d["x"][:k])).cuda()
        for _ in range(3):
            t.predict(xs, k)
        torch.cuda.synchronize()
        t.reset_stats()
        for _ in range(20):
            t.predict(xs, k)
        st = t.stats()
        out[k] = st["predict_kernel_ms"] / max(1, st["predict_launches"])
        xh = np.ascontiguousarray(d["x"][:k])
        yh = np.zeros(max(1, k * (1 if info["type"] == tm.CLASSIFIER else info["class_chunks"])),
                      dtype=np.int64 if info["type"] == tm.CLASSIFIER else np.uint8)
        args_c = (t.handle, xh.ctypes.data_as(ctypes.c_void_p), None, k) + (
            (yh.ctypes.data_as(ctypes.c_void_p), None) if info["type"] == tm.CLASSIFIER
            else (None, yh.ctypes.data_as(ctypes.c_void_p))) + (0,)
        t.stats_enable(False)  # no timing events on the measured calls
        for _ in range(20):
            lib.tm_predict(*args_c)
        reps = 200 if k <= 64 else 20
        t0 = time.perf_counter()
        for _ in range(reps):
            rc = lib.tm_predict(*args_c)
        call[k] = (time.perf_counter() - t0) / reps * 1e6
        assert rc == 0
        t.stats_enable(True)
    a_bytes = info["action_chunks"]
    print(json.dumps({"predict_sizes": w["name"], "kernel_ms": out, "call_us": call,
                      "action_bytes": a_bytes,
                      "hbm_floor_ms": a_bytes / (measured_peaks()[0]["hbm_gbs"] * 1e9) * 1e3}),
          flush=True)
    t.destroy()


def run_profile_launch(args, w):
    """One train launch of a single-machine workload (1 epoch), printing
    the library's count of its active steps: the launch a profiler capture
    looks at."""
    import torch
    import santoku_tsetlin as tm
    d = make_data(w, 0)
    n = w["n_train"]
    lab_key = "y" if w["kind"] == "classifier" else "codes"
    x = torch.from_numpy(np.ascontiguousarray(d["x"][:n])).cuda()
    lab = torch.from_numpy(np.ascontiguousarray(d[lab_key][:n])).cuda()
    t = tm.create(w["kind"], create_table(w, seed=0))
    t.set_autotune(0)
    t.stats_enable(True)
    t.train(train_table(w, x, lab))
    st = t.stats()
    print(json.dumps({"profile_launch": w["name"], "mode": st["train_mode"], "cpw": st["train_cpw"],
                      "active_pairs": st["train_active_pairs"],
                      "train_kernel_ms": st["train_kernel_ms"]}), flush=True)
    t.destroy()


if __name__ == "__main__":
    main()
