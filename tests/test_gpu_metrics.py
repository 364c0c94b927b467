"""Device evaluator metrics and input packing against their CPU
restatements (oracle/evaluator_ref.py): counts exact, doubles equal to the
last bit (both evaluate the reference's formulas in its order with one
rounding per operation), packed rows bit-exact; and the metrics against the
outputs recorded from the reference's own evaluator functions."""
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


def test_metrics_match_reference_fixtures(tm):
    """The device metrics against the outputs recorded from the reference's
    own tm_class_accuracy and tm_encoding_accuracy (evaluator/capi.c:119-202,
    497-574; tests/golden/make_golden_evaluator.py): every number equal, on
    cases with out-of-range predictions, a class without support, one class,
    one hidden bit and codes with no or every byte changed."""
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                             "evaluator.npz"))
    for key in sorted(k for k in z.files if k.endswith("_out")):
        kind, k = key.split("_")[:2]
        n, dims = (int(v) for v in z["%s_%s_meta" % (kind, k)])
        p, t = z["%s_%s_pred" % (kind, k)], z["%s_%s_true" % (kind, k)]
        if kind == "class":
            r = tm.class_accuracy(p, t, n, dims)
            got = [r["precision"], r["recall"], r["f1"]] + \
                [v for c in r["classes"] for v in (c["precision"], c["recall"], c["f1"])]
        else:
            r = tm.encoding_accuracy(p, t, n, dims)
            got = [r["mean_hamming"], r["ber_min"], r["ber_max"], r["ber_std"]] + list(r["bits"])
        assert np.array_equal(np.array(got, dtype=np.float64), z[key]), key


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


def _ind_lists(rng, n, ks, density):
    """Per-dimension set-bit lists, as bits_individualize hands them over."""
    lists, bits = [], []
    for k in ks:
        b = rng.random((n, k)) < density
        s, f = np.nonzero(b)
        lst = (s * k + f).astype(np.int64)
        if lst.size:
            lst = np.concatenate([lst, lst[:3], [-1]])  # duplicates, a negative entry
        rng.shuffle(lst)
        lists.append(lst)
        bits.append(b)
    io = np.concatenate([[0], np.cumsum([len(x) for x in lists])]).astype(np.int64)
    fo = np.concatenate([[0], np.cumsum(ks)]).astype(np.int64)
    idx = np.concatenate(lists) if lists else np.zeros(0, np.int64)
    return idx, io, fo, bits


@pytest.mark.parametrize("n,ks,flip", [(5, [1, 7, 8, 9], True), (300, [40, 0, 33, 64, 100], True),
                                       (64, [31, 32, 5], False), (1000, [300] * 20, True)])
def test_bits_to_cvec_ind(tm, n, ks, flip):
    rng = np.random.default_rng(n + len(ks))
    idx, io, fo, bits = _ind_lists(rng, n, ks, 0.15)
    got, doff = tm.bits_to_cvec_ind(idx, io, fo, n, flip)
    want, woff = R.bits_to_cvec_ind(idx, io, fo, n, flip)
    assert np.array_equal(doff, woff)
    assert np.array_equal(got, want)
    if flip:  # the golden fixtures' individualized layout: flip_pack per block
        from santoku_tsetlin import datagen
        blocks = [datagen.flip_pack(b).ravel() for b, k in zip(bits, ks) if k]
        assert np.array_equal(got, np.concatenate(blocks))


def test_bits_to_cvec_ind_device_and_train(tm):
    """Device lists in, device bitmap out; the bitmap trains an individualized
    classifier exactly as the same rows packed on the host do."""
    import torch
    rng = np.random.default_rng(77)
    n, ks = 400, [60, 23, 90, 41]
    idx, io, fo, bits = _ind_lists(rng, n, ks, 0.2)
    got, doff = tm.bits_to_cvec_ind(torch.from_numpy(idx).cuda(), io, fo, n, True)
    want, _ = R.bits_to_cvec_ind(idx, io, fo, n, True)
    assert np.array_equal(got.cpu().numpy(), want)
    y = rng.integers(0, len(ks), size=n).astype(np.int64)
    outs = []
    for x, yy in ((got, torch.from_numpy(y).cuda()), (want, y)):
        t = tm.create("classifier", dict(classes=len(ks), clauses=16,
                                         clause_tolerance=8, clause_maximum=16, target=8,
                                         specificity=5, individualized=True, feat_offsets=fo,
                                         reusable=True, seed=3))
        t.train(dict(samples=n, problems=x, solutions=yy, iterations=2, dim_offsets=doff[:-1]))
        outs.append(np.asarray(t.predict(want, doff[:-1], n)))
        t.destroy()
    assert np.array_equal(outs[0], outs[1])


def test_bits_to_cvec_ind_rejects_short_list(tm):
    with pytest.raises(tm.TsetlinError):
        tm.bits_to_cvec_ind(np.zeros(3, np.int64), [0, 5], [0, 8], 4, True)


def test_int_peaks_are_sane(tm):
    """The integer-pipe microbenchmarks return plausible rates: POPC runs
    at a fraction of the logic-op rate, and all are far above zero."""
    pk = tm.int_peaks()
    assert all(v > 1e11 for v in pk.values())
    assert pk["popc"] < pk["lop3"]
