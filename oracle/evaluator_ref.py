"""CPU restatements of the evaluator metrics and of the input packing.

TEST INFRASTRUCTURE ONLY (the checker for tm_class_accuracy,
tm_encoding_accuracy, tm_bits_to_cvec and tm_bits_to_cvec_ind).  Counting uses numpy; the
floating-point finish is a plain Python loop in the reference's order, so
every operation rounds once, as in the reference's C without contraction.
The two metrics are pinned to the reference's own functions, compiled by
eval_harness.c (fixtures in tests/golden/evaluator.npz).
"""
import math

import numpy as np


def class_accuracy(predicted, expected, n, classes):
    """evaluator/capi.c:119-202 (tm_class_accuracy)."""
    yp = np.asarray(predicted, dtype=np.int64)[:n].astype(np.uint32)
    yt = np.asarray(expected, dtype=np.int64)[:n].astype(np.uint32)
    tp = [0] * classes
    fp = [0] * classes
    fn = [0] * classes
    for a, b in zip(yp.tolist(), yt.tolist()):         # capi.c:141-153
        if a >= classes or b >= classes:
            continue
        if a == b:
            tp[b] += 1
        else:
            fp[a] += 1
            fn[b] += 1
    out = {"classes": []}
    pa = ra = fa = 0.0
    for c in range(classes):                            # capi.c:155-172
        t, f, g = tp[c], fp[c], fn[c]
        p = t / (t + f) if (t + f) > 0 else 0.0
        r = t / (t + g) if (t + g) > 0 else 0.0
        f1 = 2.0 * p * r / (p + r) if (p + r) > 0 else 0.0
        out["classes"].append({"precision": p, "recall": r, "f1": f1})
        pa += p
        ra += r
        fa += f1
    out["precision"] = pa / classes
    out["recall"] = ra / classes
    out["f1"] = fa / classes
    return out


def encoding_accuracy(predicted, expected, n, hidden):
    """evaluator/capi.c:497-574 (tm_encoding_accuracy)."""
    nb = (hidden + 7) // 8
    p = np.asarray(predicted, dtype=np.uint8)[:n * nb].reshape(n, nb)
    e = np.asarray(expected, dtype=np.uint8)[:n * nb].reshape(n, nb)
    diff = np.unpackbits(p ^ e, axis=1, bitorder="little", count=hidden)
    bd = diff.sum(axis=0).astype(np.int64).tolist()    # capi.c:520-535
    total = sum(bd)
    mn, mx = 1.0, 0.0
    bits = []
    for j in range(hidden):                             # capi.c:544-555
        t = bd[j] / n
        mn = min(mn, t) if t < mn else mn
        mx = t if t > mx else mx
        bits.append(t)
    mean = total / (n * hidden)
    var = 0.0
    for j in range(hidden):                             # capi.c:557-561
        ber = bd[j] / n
        var += (ber - mean) * (ber - mean)
    std = math.sqrt(var / (hidden - 1)) if hidden > 1 else 0.0
    return {"bits": bits, "mean_hamming": 1.0 - mean, "ber_min": 1.0 - mn,
            "ber_max": 1.0 - mx, "ber_std": std}


def bits_to_cvec(set_bits, n, features, flip):
    """santoku-matrix's bits_to_cvec on a list of `sample * features +
    feature` indices (dataset.lua:11-41), flip-interleaved when `flip`
    (doc/sth.md:70-78)."""
    width = 2 * features if flip else features
    rows = np.zeros((n, width), dtype=bool)
    idx = np.asarray(set_bits, dtype=np.int64)
    idx = idx[idx >= 0]
    s, f = idx // features, idx % features
    keep = s < n
    rows[s[keep], f[keep]] = True
    if flip:
        rows[:, features:] = ~rows[:, :features]
    return np.packbits(rows, axis=1, bitorder="little").ravel()


def bits_to_cvec_ind(set_bits, ind_offsets, feat_offsets, n, flip):
    """santoku-matrix's bits_to_cvec_ind: dimension h's list
    set_bits[ind_offsets[h]:ind_offsets[h+1]] (entries sample * k_h +
    feature, k_h = feat_offsets[h+1] - feat_offsets[h]) packed as n rows of
    its own width, blocks concatenated in dimension order (doc/sth.md:42-54;
    the reader is capi.c:1344-1354).  Returns (bitmap, dim_offsets) with
    dims + 1 offsets, the last the total size."""
    io = np.asarray(ind_offsets, dtype=np.int64)
    fo = np.asarray(feat_offsets, dtype=np.int64)
    idx = np.asarray(set_bits, dtype=np.int64)
    blocks, offs, off = [], [], 0
    for h in range(len(fo) - 1):
        k = int(fo[h + 1] - fo[h])
        offs.append(off)
        if k == 0:
            continue
        lst = idx[io[h] - io[0]:io[h + 1] - io[0]]
        b = bits_to_cvec(lst, n, k, flip)
        blocks.append(b)
        off += b.size
    offs.append(off)
    bm = np.concatenate(blocks) if blocks else np.zeros(0, np.uint8)
    return bm, np.array(offs, dtype=np.int64)
