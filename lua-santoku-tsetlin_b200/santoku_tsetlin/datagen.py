"""Seeded synthetic workloads with the shapes and value distributions of the
benchmark configurations (the reference ships none; its tests read MNIST /
20news / IMDB, which stand outside the hot path).

Every generator returns flip-packed samples: for F features, bits 0..F-1
hold the features and bits F..2F-1 their complements, LSB-first within each
byte, ceil(2F/8) bytes per sample -- the layout santoku-matrix's
`bits_to_cvec(n, F, true)` produces for the reference (doc/sth.md:70-78,
test/spec/santoku/tsetlin/classify/mnist.lua:60).
"""
import numpy as np


def pack_bits(bits):
    """bool (n, B) -> uint8 (n, ceil(B/8)), LSB-first."""
    bits = np.ascontiguousarray(bits, dtype=bool)
    return np.packbits(bits, axis=1, bitorder="little")


def flip_pack(bits):
    """bool (n, F) -> flip-interleaved uint8 (n, ceil(2F/8))."""
    bits = np.asarray(bits, dtype=bool)
    return pack_bits(np.concatenate([bits, ~bits], axis=1))


def unpack_bits(packed, nbits):
    return np.unpackbits(packed, axis=1, bitorder="little", count=nbits).astype(bool)


def balanced_labels(n, classes, rng):
    y = np.arange(n, dtype=np.int64) % classes
    rng.shuffle(y)
    return y


def prototype_classifier(n, classes=10, features=784, density=0.2, flip=0.1, seed=0,
                         negated=True, prototypes=None):
    """Plain classifier workload: each class has a prototype of iid
    Bernoulli(density) bits; each sample flips each bit of its class
    prototype with probability `flip`; balanced labels.  With negated=False
    the raw F bits are packed as a machine of F/2 features (the literal
    space is exactly the F raw bits)."""
    rng = np.random.default_rng(seed)
    if prototypes is None:
        prototypes = np.random.default_rng(seed + 7919).random((classes, features)) < density
    y = balanced_labels(n, classes, rng)
    out = []
    step = 8192
    for i in range(0, n, step):
        yy = y[i:i + step]
        noise = rng.random((len(yy), features), dtype=np.float32) < flip
        bits = prototypes[yy] ^ noise
        out.append(flip_pack(bits) if negated else pack_bits(bits))
    x = np.concatenate(out, axis=0) if out else np.zeros((0, (2 * features + 7) // 8), np.uint8)
    return np.ascontiguousarray(x), y, prototypes


def sparse_classifier(n, classes=20, features=16384, density=0.015, zipf=1.1, boost=8.0,
                      subset=200, seed=1, spec_seed=None):
    """Large sparse classifier workload: feature activation probabilities
    follow Zipf(zipf) over a random feature rank, scaled to `density` mean;
    each class boosts a random `subset`-feature set by `boost` (clipped to
    1)."""
    srng = np.random.default_rng(seed + 104729 if spec_seed is None else spec_seed)
    rank = srng.permutation(features)
    base = 1.0 / np.power(rank + 1.0, zipf)
    lo, hi = 0.0, 1.0 / base.min()
    for _ in range(100):  # scale so that the clipped mean is `density`
        mid = 0.5 * (lo + hi)
        if np.minimum(base * mid, 1.0).mean() < density:
            lo = mid
        else:
            hi = mid
    p = np.minimum(base * hi, 1.0)
    boosts = [srng.choice(features, size=subset, replace=False) for _ in range(classes)]
    pc = np.repeat(p[None, :], classes, axis=0)
    for c in range(classes):
        pc[c, boosts[c]] = np.minimum(pc[c, boosts[c]] * boost, 1.0)
    pc = pc.astype(np.float32)
    rng = np.random.default_rng(seed)
    y = balanced_labels(n, classes, rng)
    nb = (2 * features + 7) // 8
    x = np.empty((n, nb), dtype=np.uint8)
    step = 2048
    for i in range(0, n, step):
        yy = y[i:i + step]
        bits = rng.random((len(yy), features), dtype=np.float32) < pc[yy]
        x[i:i + len(yy)] = flip_pack(bits)
    return x, y


def latent_encoder(n, visible=4096, hidden=256, latent=64, noise=0.05, seed=2):
    """Encoder workload: visible bits are the sign of N(0, I_latent) latents
    under a random latent->visible Gaussian projection plus `noise` bit
    flips; target codes are the sign of the same latents under a separate
    latent->hidden projection (LSB-first, ceil(hidden/8) bytes)."""
    prng = np.random.default_rng(seed + 15485863)
    px = prng.standard_normal((latent, visible)).astype(np.float32)
    pcode = prng.standard_normal((latent, hidden)).astype(np.float32)
    rng = np.random.default_rng(seed)
    nb = (2 * visible + 7) // 8
    x = np.empty((n, nb), dtype=np.uint8)
    codes = np.empty((n, (hidden + 7) // 8), dtype=np.uint8)
    step = 4096
    for i in range(0, n, step):
        m = min(step, n - i)
        z = rng.standard_normal((m, latent)).astype(np.float32)
        bits = (z @ px) > 0
        bits ^= rng.random((m, visible), dtype=np.float32) < noise
        x[i:i + m] = flip_pack(bits)
        codes[i:i + m] = pack_bits((z @ pcode) > 0)
    return x, codes


def search_machines(count=64, classes=10, features=784, seed=3):
    """Per-machine hyper-parameters of the batched search workload: clauses
    per class log-uniform over [64, 4096] rounded to 8, specificity uniform
    over [2, 40], target uniform over [20, 400], negated literals on or off."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        clauses = int(np.exp(rng.uniform(np.log(64), np.log(4096))))
        clauses = max(8, int(round(clauses / 8.0)) * 8)
        negated = bool(rng.random() < 0.5)
        out.append(dict(
            classes=classes,
            features=features if negated else features // 2,
            negated=negated,
            clauses=clauses,
            specificity=float(rng.uniform(2.0, 40.0)),
            target=float(int(rng.uniform(20.0, 400.0))),
            clause_tolerance=64,
            clause_maximum=64,
            seed=i,
        ))
    return out
