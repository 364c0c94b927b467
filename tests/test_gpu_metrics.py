"""Device evaluator metrics and input packing against their CPU
restatements (oracle/evaluator_ref.py): counts exact, doubles equal to the
last bit (both evaluate the reference's formulas in its order with one
rounding per operation), packed rows bit-exact."""
import numpy as np
import pytest

import evaluator_ref as R

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,classes", [(1, 1), (1000, 10), (20000, 20), (777, 37)])
def test_class_accuracy(tm, n, classes):
    rng = np.random.default_rng(n + classes)
    yt = rng.integers(0, classes, size=n).astype(np.int64)
    yp = np.where(rng.random(n) < 0.7, yt, rng.integers(0, classes + 2, size=n)).astype(np.int64)
    yp[::11] = -1  # out of range: skipped, as in the reference
    got = tm.class_accuracy(yp, yt, n, classes)
    want = R.class_accuracy(yp, yt, n, classes)
    assert got == want


@pytest.mark.parametrize("n,hidden", [(1, 1), (500, 13), (20000, 256)])
def test_encoding_accuracy(tm, n, hidden):
    rng = np.random.default_rng(n + hidden)
    nb = (hidden + 7) // 8
    e = rng.integers(0, 256, size=n * nb).astype(np.uint8)
    flips = np.packbits(rng.random((n, nb * 8)) < 0.07, axis=1, bitorder="little").ravel()
    p = e ^ flips
    got = tm.encoding_accuracy(p, e, n, hidden)
    want = R.encoding_accuracy(p, e, n, hidden)
    assert got == want


@pytest.mark.parametrize("n,features,flip", [(3, 5, True), (100, 784, True), (57, 100, False),
                                             (10, 16384, True)])
def test_bits_to_cvec(tm, n, features, flip):
    rng = np.random.default_rng(features)
    bits = rng.random((n, features)) < 0.1
    s, f = np.nonzero(bits)
    idx = (s * features + f).astype(np.int64)
    idx = np.concatenate([idx, idx[:5], [-1]])  # duplicates and a negative entry
    rng.shuffle(idx)
    got = tm.bits_to_cvec(idx, n, features, flip)
    assert np.array_equal(got, R.bits_to_cvec(idx, n, features, flip))
    if flip:
        from santoku_tsetlin import datagen
        assert np.array_equal(got, datagen.flip_pack(bits).ravel())
