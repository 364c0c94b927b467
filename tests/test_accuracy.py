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


def test_sparse_classifier_accuracy_within_one_point(tm):
    """The large sparse classifier's data (20 classes, 16,384 Zipf(1.1)
    features at ~1.5 % density, each class boosting 200 features 8x) with
    128 clauses per class: units are independent 8-clause chunks, so the
    per-unit rules are those of the 2,048-clause machine.  3,000 train /
    3,000 test samples, 6 epochs, 5 seeds."""
    from santoku_tsetlin import datagen
    threads = os.cpu_count() or 4
    cfg = dict(classes=20, features=16384, clauses=128, clause_tolerance=64, clause_maximum=64,
               specificity=25.0, target=200)
    gpu, ref = [], []
    for seed in range(5):
        x, y = datagen.sparse_classifier(6000, classes=20, features=16384, seed=10 + seed)
        x, y, xt, yt = x[:3000], y[:3000], x[3000:], y[3000:]
        t = tm.create("classifier", dict(cfg, seed=seed))
        t.train({"samples": 3000, "problems": x.ravel(), "solutions": y, "iterations": 6})
        pred = t.predict(xt.ravel(), 3000)
        gpu.append(float((pred == yt).mean()))
        t.destroy()
        m = O.Machine(which="ref" if O.ref_available() else "oracle", type="classifier", **cfg)
        m.train(x.ravel(), 3000, 6, labels=y, seed=seed, mode=O.REFSTRUCT, threads=threads)
        ref.append(float((m.predict(xt.ravel(), 3000, threads=threads) == yt).mean()))
    g, r = 100 * np.mean(gpu), 100 * np.mean(ref)
    print("sparse classifier accuracy over 5 seeds: cuda %.2f %%  reference %.2f %%" % (g, r))
    assert 50.0 < r < 99.9
    assert abs(g - r) <= 1.0


def test_encoder_hamming_within_one_point(tm):
    """The encoder's data (4,096 visible bits as signs of 64-dim Gaussian
    latents under a random projection plus 5 % bit noise; codes the signs
    of a second projection) with 32 hidden bits and 16 clauses per bit.
    Hamming error per bit on a 2,000-sample holdout -- counted on the GPU by
    the evaluator's encoding_accuracy (evaluator/capi.c:497-574) for the
    CUDA path -- over 5 seeds, 3,000 train samples, 4 epochs."""
    from santoku_tsetlin import datagen
    threads = os.cpu_count() or 4
    hidden = 32
    cfg = dict(features=4096, clauses=16, clause_tolerance=64, clause_maximum=64,
               specificity=15.0, target=100)
    gpu, ref = [], []
    for seed in range(5):
        x, c = datagen.latent_encoder(5000, visible=4096, hidden=hidden, seed=20 + seed)
        x, c, xt, ct = x[:3000], c[:3000], x[3000:], c[3000:]
        t = tm.create("encoder", dict(hidden=hidden, visible=cfg["features"],
                                      **{k: v for k, v in cfg.items() if k != "features"},
                                      seed=seed))
        t.train({"samples": 3000, "sentences": x.ravel(), "codes": c.ravel(), "iterations": 4})
        pred = t.predict(xt.ravel(), 2000)
        # the evaluator's `mean_hamming` is one minus the mean bit error rate
        gpu.append(1.0 - tm.encoding_accuracy(pred, ct.ravel(), 2000, hidden)["mean_hamming"])
        t.destroy()
        m = O.Machine(which="ref" if O.ref_available() else "oracle", type="encoder",
                      classes=hidden, **cfg)
        m.train(x.ravel(), 3000, 4, codes=c.ravel(), seed=seed, mode=O.REFSTRUCT, threads=threads)
        p = m.predict(xt.ravel(), 2000, threads=threads).reshape(2000, -1)
        bp = np.unpackbits(p, axis=1, bitorder="little")[:, :hidden]
        bt = np.unpackbits(ct, axis=1, bitorder="little")[:, :hidden]
        ref.append(float((bp != bt).mean()))
    g, r = 100 * np.mean(gpu), 100 * np.mean(ref)
    print("encoder Hamming error over 5 seeds: cuda %.2f %%  reference %.2f %%" % (g, r))
    assert 1.0 < r < 45.0
    assert abs(g - r) <= 1.0
