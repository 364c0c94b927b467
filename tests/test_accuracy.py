"""Accuracy of the CUDA path against the reference's own training structure.

The reference trains with one generator stream and one shuffle per OpenMP
thread (capi.c:1136-1167); its generator (santoku's tk_fast_random) is not
available, so the oracle's `refstruct` mode stands in for it (same loop
structure, per-thread streams seeded by thread id, a 64-bit multiplicative
congruential generator).  Over 5 seeds, the mean test accuracy of the CUDA
path (Philox draw contract) must be within 1 point of the reference
structure's on the plain-classifier workload (10 classes, 784 features,
256 clauses per class, specificity 10, target 50, 10 epochs), on data made
harder than the benchmark's so that accuracy is not saturated: class
prototypes share a base pattern and differ in 24 features each, with 35 %
bit noise; 4,000 train and 5,000 test samples.
"""
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

CFG = dict(classes=10, features=784, clauses=256, clause_tolerance=64, clause_maximum=64,
           target=50, specificity=10.0)


def data(seed):
    from santoku_tsetlin import datagen
    rs = np.random.default_rng(4242)
    base = rs.random(784) < 0.2
    protos = np.repeat(base[None], 10, axis=0)
    for c in range(10):
        protos[c, rs.choice(784, size=24, replace=False)] ^= True
    x, y, _ = datagen.prototype_classifier(9000, classes=10, features=784, flip=0.35, seed=seed,
                                           prototypes=protos)
    return x[:4000], y[:4000], x[4000:], y[4000:]


def test_accuracy_within_one_point_of_reference_structure(tm):
    threads = os.cpu_count() or 4
    gpu, ref = [], []
    for seed in range(5):
        x, y, xt, yt = data(100 + seed)
        t = tm.create("classifier", dict(CFG, seed=seed))
        t.train({"samples": len(y), "problems": x.ravel(), "solutions": y, "iterations": 10})
        gpu.append(float((t.predict(xt.ravel(), len(yt)) == yt).mean()))
        m = O.Machine(type="classifier", **CFG)
        m.train(x.ravel(), len(y), 10, labels=y, seed=seed, mode=O.REFSTRUCT, threads=threads)
        ref.append(float((m.predict(xt.ravel(), len(yt), threads=threads) == yt).mean()))
    g, r = 100 * np.mean(gpu), 100 * np.mean(ref)
    print("accuracy over 5 seeds: cuda %.2f %%  reference structure %.2f %%" % (g, r))
    assert 50.0 < r < 99.9, "data must not saturate accuracy"
    assert abs(g - r) <= 1.0
