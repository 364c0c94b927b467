"""santoku.tsetlin.optimize on B200: the hyper-parameter search driver of
the reference (lib/santoku/tsetlin/optimize.lua, TM part :182-844),
restated in Python over this package's machines.

Same structure as the reference:
  * samplers (`build_sampler`, optimize.lua:187-258): fixed values, ranges
    (log / int / pow2 / round, Gaussian jitter around a centre), lists;
  * `search` (:391-516): rounds of trials; the best parameters recentre the
    samplers after each round and the 1/5 success rule adapts the jitter;
  * `train_tm` (:586-653): a trial trains with a per-epoch metric, patience
    early stop, a checkpoint of the best epoch, and a restore at the end;
  * `classifier` / `encoder` (:657-844): search, then a final training of a
    fresh machine with the best parameters.

Added here: `batched=True` runs all trials of a round -- independent until
the samplers are recentred -- in one `train_batch(..., each=...)` call.
Each trial's machine trains exactly as it would alone (the keyed draws make
machines independent), so the per-trial epochs, scores and chosen
parameters are the same as the sequential form.

`search_metric` may also name a metric the GPU computes itself -- a table
{"metric": "f1" | "accuracy" | "mean_hamming", "samples": n, "problems" /
"sentences": holdout, "solutions" / "codes": truth} standing for the
reference's usual `function (t) ... class_accuracy(t:predict(...)).f1`.
A batched round then runs device-resident (`train_batch_search`): each
epoch of all trials -- training, holdout predict, scores, patience,
checkpoints -- is one CUDA graph replay, and no per-trial data leaves the
GPU until the round ends.  Scores and chosen parameters are the same as
with the equivalent callable.

The reference's generator for sampling (santoku's num.random /
rand.fast_normal) is not available; a seeded numpy Generator stands in.
The landmark-encoding options of the encoder search (HLTH) are out of
scope.
"""
import math

import numpy as np

from . import class_accuracy, create, encoding_accuracy, train_batch, train_batch_search

PARAM_NAMES = ("clauses", "clause_tolerance", "clause_maximum", "target", "specificity",
               "include_bits")


def _round_to_pow2(x):
    return 2.0 ** math.floor(math.log(x) / math.log(2) + 0.5)


class Sampler:
    """optimize.lua:187-258"""

    def __init__(self, spec, global_dev, rng):
        self.rng = rng
        self.jitter = None
        if isinstance(spec, (int, float, bool, str)):
            self.type, self.center, self.spec = "fixed", spec, spec
            return
        if isinstance(spec, dict) and ("def" in spec or ("min" in spec and "max" in spec)):
            self.type = "range"
            self.spec = spec
            self.center = spec.get("def")
            minv, maxv = spec["min"], spec["max"]
            self.is_log = bool(spec.get("log"))
            shift = (1 - minv) if (self.is_log and minv <= 0) else 0
            self.shift = shift
            smin, smax = minv + shift, maxv + shift
            self.span = (math.log(smax) - math.log(smin)) if self.is_log else (maxv - minv)
            self.smin = smin
            self.jitter = (spec.get("dev") or global_dev or 1.0) * self.span
            return
        if isinstance(spec, (list, tuple)) and len(spec) > 0:
            self.type, self.spec, self.center = "list", list(spec), spec[0]
            return
        raise ValueError("Bad hyper-parameter specification: %r" % (spec,))

    def sample(self, center=None):
        if self.type == "fixed":
            return self.spec
        if self.type == "list":
            return self.spec[int(self.rng.integers(0, len(self.spec)))]
        s = self.spec
        minv, maxv = s["min"], s["max"]
        if center is not None:
            c = math.log(center + self.shift) if self.is_log else center
            x = self.rng.normal(c, self.jitter)
            if self.is_log:
                x = math.exp(x) - self.shift
        elif self.is_log:
            x = math.exp(self.rng.random() * self.span + math.log(self.smin)) - self.shift
        else:
            x = self.rng.random() * self.span + minv
        if x > maxv:
            x = 2 * maxv - x
        if x < minv:
            x = 2 * minv - x
        x = min(max(x, minv), maxv)
        if s.get("pow2"):
            x = _round_to_pow2(x)
        elif s.get("round"):
            x = math.floor(x / s["round"] + 0.5) * s["round"]
        elif s.get("int"):
            x = math.floor(x + 0.5)
        return min(max(x, minv), maxv)

    def adapt(self, factor):
        if self.jitter is not None:
            self.jitter *= factor


def build_samplers(args, param_names, global_dev, rng):
    """optimize.lua:260-266"""
    return {n: Sampler(args[n], global_dev, rng) for n in param_names if args.get(n) is not None}


def sample_params(samplers, param_names, base=None, exact_defaults=False):
    """optimize.lua:268-288"""
    p = dict(base or {})
    for n in param_names:
        s = samplers.get(n)
        if s is None:
            continue
        if exact_defaults and s.center is not None:
            p[n] = s.center
        elif s.type == "range":
            p[n] = s.sample(s.center)
        else:
            p[n] = s.sample()
    return p


def all_fixed(samplers):
    return all(s.type == "fixed" for s in samplers.values())


def recenter(samplers, param_names, best):
    """optimize.lua:362-370"""
    for n in param_names:
        s = samplers.get(n)
        if s is not None and s.type == "range" and best.get(n) is not None:
            s.center = best[n]


def adapt_jitter(samplers, factor):
    for s in samplers.values():
        s.adapt(factor)


def success_factor(rate):
    """optimize.lua:379-389: the 1/5 success rule"""
    if rate > 0.2:
        return 1.0
    if rate > 0.05:
        return 0.8
    return 0.5


def search(param_names, samplers, trial_fn, rounds=3, trials=10, tolerance=1e-8, make_key=None,
           each=None, skip_final=False, round_fn=None):
    """optimize.lua:391-516.  `round_fn(list of params, infos)` runs a whole
    round at once (returning (score, metrics, result) per trial in order);
    otherwise trials run one by one through `trial_fn`."""
    best_score, best_params, best_result, best_metrics = -math.inf, None, None, None
    if all_fixed(samplers) or rounds <= 0 or trials <= 0:
        best_params = sample_params(samplers, param_names, None, True)
        if skip_final:
            return None, best_params, None
        _, metrics, result = trial_fn(best_params, {"is_final": True})
        return result, best_params, metrics
    for r in range(1, rounds + 1):
        seen = set()
        plist, infos = [], []
        for t in range(1, trials + 1):
            params = sample_params(samplers, param_names)
            if make_key is not None:
                key = make_key(params)
                if key in seen:
                    continue
                seen.add(key)
            plist.append(params)
            infos.append({"round": r, "trial": t, "is_final": False})
        if round_fn is not None:
            outcomes = round_fn(plist, infos)
        else:
            outcomes = [trial_fn(p, i) for p, i in zip(plist, infos)]
        round_best_score, round_best_params, improvements = -math.inf, None, 0
        for params, info, (score, metrics, result) in zip(plist, infos, outcomes):
            if each:
                each({"event": "trial", "round": r, "trial": info["trial"], "params": params,
                      "score": score, "metrics": metrics})
            if score > round_best_score:
                round_best_score, round_best_params = score, params
            if score > best_score + tolerance:
                improvements += 1
                best_score, best_params, best_result, best_metrics = score, params, result, metrics
        if best_params is not None:
            recenter(samplers, param_names, best_params)
        rate = improvements / len(plist) if plist else 0
        factor = success_factor(rate)
        adapt_jitter(samplers, factor)
        if each:
            each({"event": "round", "round": r, "round_best_score": round_best_score,
                  "round_best_params": round_best_params, "global_best_score": best_score,
                  "global_best_params": best_params, "success_rate": rate,
                  "adapt_factor": factor})
    if not skip_final and best_params is not None:
        score, metrics, result = trial_fn(best_params, {"is_final": True})
        best_result, best_metrics = result, metrics
    return best_result, best_params, best_metrics


class _Tracker:
    """The per-trial epoch logic of train_tm (optimize.lua:599-625): metric,
    each callback, patience, checkpoint of the best epoch."""

    def __init__(self, machine, params, info, metric_fn, each_cb, patience, tolerance):
        self.m, self.params, self.info = machine, params, info
        self.metric_fn, self.each_cb = metric_fn, each_cb
        self.patience, self.tolerance = patience, tolerance
        self.best = -math.inf
        self.since = 0
        self.last = (-math.inf, None)
        self.checkpoint = bytearray() if (patience and patience > 0) else None
        self.has_checkpoint = False

    def epoch(self, e):
        score, metrics = self.metric_fn(self.m)
        self.last = (score, metrics)
        if self.each_cb:
            r = self.each_cb(self.m, self.info.get("is_final", False), metrics, self.params, e,
                             self.info.get("round"), self.info.get("trial"))
            if r is False:
                return False
        if score > self.best + self.tolerance:
            self.best = score
            self.since = 0
            if self.checkpoint is not None:
                self.m.checkpoint(self.checkpoint)
                self.has_checkpoint = True
        else:
            self.since += 1
        if self.patience and self.patience > 0 and self.since >= self.patience:
            return False
        return True

    def finish(self):
        if self.checkpoint is not None and self.has_checkpoint:
            self.m.restore(self.checkpoint)
            self.last = self.metric_fn(self.m)
        return self.last


def _train_table(typ, args, iterations):
    t = {"samples": args["samples"], "iterations": iterations}
    if typ == "classifier":
        t.update(problems=args["problems"], solutions=args["solutions"])
    else:
        t.update(sentences=args["sentences"], codes=args["codes"])
    if args.get("dim_offsets") is not None:
        t["dim_offsets"] = args["dim_offsets"]
    return t


def train_tm(typ, machine, args, params, iterations, patience, tolerance, metric_fn, each_cb,
             info):
    """optimize.lua:586-653"""
    tr = _Tracker(machine, params, info, metric_fn, each_cb, patience, tolerance)
    machine.train(dict(_train_table(typ, args, iterations), each=tr.epoch))
    return tr.finish()


def train_tm_batch(typ, machines, args, plist, iterations, patience, tolerance, metric_fn,
                   each_cb, infos):
    """train_tm for a whole round of machines in one batched training."""
    trs = [_Tracker(m, p, i, metric_fn, each_cb, patience, tolerance)
           for m, p, i in zip(machines, plist, infos)]
    live = [True] * len(machines)

    def each(e):
        for k, tr in enumerate(trs):
            if live[k] and not tr.epoch(e):
                live[k] = False
        return [not v for v in live]

    train_batch(machines, [_train_table(typ, args, iterations)] * len(machines), each=each)
    return [tr.finish() for tr in trs]


def device_metric_fn(typ, spec):
    """The host form of a device metric table: predict the holdout and score
    it with the GPU evaluator (used for single trials and the final
    training; equal to what the device-resident round computes)."""
    n = int(spec["samples"])
    name = spec.get("metric", "mean_hamming" if typ == "encoder" else "f1")
    dof = spec.get("dim_offsets")
    rest = [dof, n] if dof is not None else [n]

    def fn(t, _enc_info=None):
        if typ == "encoder":
            acc = encoding_accuracy(t.predict(spec["sentences"], *rest), spec["codes"], n,
                                    t.info()["classes"])
            return acc["mean_hamming"], acc
        pred = t.predict(spec["problems"], *rest)
        if name == "accuracy":
            pv = pred.cpu().numpy() if hasattr(pred, "cpu") else pred
            yv = spec["solutions"]
            yv = yv.cpu().numpy() if hasattr(yv, "cpu") else np.asarray(yv)
            acc = float((pv == yv).sum()) / n
            return acc, {"accuracy": acc}
        acc = class_accuracy(pred, spec["solutions"], n, t.info()["classes"])
        return acc["f1"], acc
    return fn


def _machine_table(typ, args, params, reusable):
    t = {"clauses": params["clauses"], "clause_tolerance": params["clause_tolerance"],
         "clause_maximum": params["clause_maximum"], "target": params["target"],
         "specificity": params["specificity"], "include_bits": params.get("include_bits", 1),
         "reusable": reusable, "seed": args.get("seed", 0), "device": args.get("device", 0)}
    if typ == "classifier":
        t.update(classes=args["classes"], features=args["features"],
                 negative=args.get("negative"))
    else:
        t.update(hidden=args["hidden"], visible=args["visible"])
    if args.get("individualized"):
        t.update(individualized=True, feat_offsets=args["feat_offsets"])
    return t


def _optimize_tm(args, typ):
    """optimize.lua:657-836 (without landmark encodings)"""
    rng = np.random.default_rng(args.get("search_seed", 0))
    patience = args.get("search_patience", 10)
    final_patience = args.get("final_patience", 40)
    tolerance = args.get("search_tolerance", 1e-8)
    iters = args.get("search_iterations", 10)
    final_iters = args.get("final_iterations", iters * 10)
    metric_spec = args["search_metric"] if isinstance(args["search_metric"], dict) else None
    metric_fn = device_metric_fn(typ, metric_spec) if metric_spec else args["search_metric"]
    each_cb = args.get("each")
    samplers = build_samplers(args, PARAM_NAMES, args.get("search_dev", 0.2), rng)

    def fix(params):
        # optimize.lua:731-733: keep clause_tolerance <= clause_maximum
        if params["clause_tolerance"] > params["clause_maximum"]:
            params["clause_tolerance"], params["clause_maximum"] = (
                params["clause_maximum"], params["clause_tolerance"])
        return params

    def trial_fn(params, info):
        params = fix(params)
        m = create(typ, _machine_table(typ, args, params, True))
        score, metrics = train_tm(typ, m, args, params, iters, patience if patience > 0 else None,
                                  tolerance, metric_fn, each_cb, info)
        m.destroy()
        return score, metrics, None

    def round_fn(plist, infos):
        plist = [fix(p) for p in plist]
        ms = [create(typ, _machine_table(typ, args, p, True)) for p in plist]
        if metric_spec is not None and each_cb is None:
            # device-resident round: per-epoch scores never leave the GPU
            test = {k: v for k, v in metric_spec.items() if k != "metric"}
            r = train_batch_search(ms, [_train_table(typ, args, iters)] * len(ms), test,
                                   patience=patience if patience > 0 else 0,
                                   tolerance=tolerance, metric=metric_spec.get("metric"))
            res = [(float(r["final"][k]), {"score": float(r["final"][k]),
                                           "epochs": int(r["epochs"][k])})
                   for k in range(len(ms))]
        else:
            res = train_tm_batch(typ, ms, args, plist, iters,
                                 patience if patience > 0 else None, tolerance, metric_fn,
                                 each_cb, infos)
        for m in ms:
            m.destroy()
        return [(score, metrics, None) for score, metrics in res]

    def make_key(p):
        return "%d|%d|%d|%d|%d|%d" % (p["clauses"], p["clause_tolerance"], p["clause_maximum"],
                                      math.floor(p["target"] * 1e6 + 0.5),
                                      math.floor(p["specificity"] * 1e6 + 0.5),
                                      p.get("include_bits") or 1)

    _, best, _ = search(PARAM_NAMES, samplers, trial_fn, rounds=args.get("search_rounds", 3),
                        trials=args.get("search_trials", 10), tolerance=tolerance,
                        make_key=make_key, skip_final=True,
                        round_fn=round_fn if args.get("batched", True) else None)
    final = create(typ, _machine_table(typ, args, best, False))
    _, metrics = train_tm(typ, final, args, best, final_iters,
                          final_patience if final_patience > 0 else None, tolerance, metric_fn,
                          each_cb, {"is_final": True})
    return final, metrics, best


def classifier(args):
    """optimize.classifier (optimize.lua:838)"""
    return _optimize_tm(args, "classifier")


def encoder(args):
    """optimize.encoder (optimize.lua:842)"""
    return _optimize_tm(args, "encoder")
