"""Generates tests/golden/evaluator.npz from the reference's own evaluator.

Runs only where the reference tree is present: it drives the evaluator
harness (oracle/_ref/libeval_ref.so, built by `make -C oracle` from the
reference's lib/santoku/tsetlin/evaluator/capi.c: tm_class_accuracy,
:119-202, and tm_encoding_accuracy, :497-574) and records, for each seeded
case, the inputs and the reference's outputs:

  class_<k>_pred / _true / _meta (n, classes) / _out
      out = precision, recall, f1, then (precision, recall, f1) per class
  enc_<k>_pred / _true / _meta (n, hidden) / _out
      out = mean_hamming, ber_min, ber_max, ber_std, then the per-bit rates

Usage:  python tests/golden/make_golden_evaluator.py
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SO = os.path.join(ROOT, "oracle", "_ref", "libeval_ref.so")

# (n, classes, kind): "mixed" = 70 % correct, the rest uniform over
# [-2, classes + 2) (predictions and labels out of range are skipped by the
# reference); "absent" = one class never predicted nor present; "perfect"
CLASS_CASES = [(1, 1, "mixed"), (7, 3, "mixed"), (500, 10, "mixed"), (333, 20, "absent"),
               (64, 2, "perfect"), (1000, 37, "mixed"), (5, 8, "absent")]
# (n, hidden, flip probability of a code byte)
ENC_CASES = [(1, 1, 0.5), (9, 7, 0.3), (200, 64, 0.05), (150, 256, 0.2), (33, 13, 0.0),
             (80, 100, 1.0), (2, 2, 0.5)]


def lib():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    if not os.path.exists(SO):
        raise SystemExit("evaluator harness not built (reference tree absent)")
    return ctypes.CDLL(SO)


def ref_class(L, pred, true, n, classes):
    out = np.zeros(3 + 3 * classes)
    p = ctypes.c_void_p
    L.ref_eval_class_accuracy(pred.ctypes.data_as(p), true.ctypes.data_as(p), ctypes.c_uint32(n),
                              ctypes.c_uint32(classes), out.ctypes.data_as(p))
    return out


def ref_encoding(L, pred, true, n, hidden):
    out = np.zeros(4 + hidden)
    p = ctypes.c_void_p
    L.ref_eval_encoding_accuracy(pred.ctypes.data_as(p), true.ctypes.data_as(p),
                                 ctypes.c_uint32(n), ctypes.c_uint32(hidden),
                                 out.ctypes.data_as(p))
    return out


def class_inputs(rng, n, classes, kind):
    true = rng.integers(0, classes, size=n).astype(np.int64)
    if kind == "perfect":
        return true.copy(), true
    pred = rng.integers(-2, classes + 2, size=n).astype(np.int64)
    pred = np.where(rng.random(n) < 0.7, true, pred)
    if kind == "absent" and classes > 1:
        gone = classes - 1
        true = np.where(true == gone, 0, true)
        pred = np.where(pred == gone, 0, pred)
    return pred, true


def enc_inputs(rng, n, hidden, flip):
    nb = (hidden + 7) // 8
    true = rng.integers(0, 256, size=n * nb, dtype=np.uint8)
    pred = true.copy()
    sel = rng.random(n * nb) < flip
    pred[sel] ^= rng.integers(1, 256, size=int(sel.sum()), dtype=np.uint8)
    return pred, true


def main():
    L = lib()
    rng = np.random.default_rng(2027)
    rec = {}
    for k, (n, classes, kind) in enumerate(CLASS_CASES):
        pred, true = class_inputs(rng, n, classes, kind)
        rec["class_%d_pred" % k] = pred
        rec["class_%d_true" % k] = true
        rec["class_%d_meta" % k] = np.array([n, classes], dtype=np.int64)
        rec["class_%d_out" % k] = ref_class(L, pred, true, n, classes)
    for k, (n, hidden, flip) in enumerate(ENC_CASES):
        pred, true = enc_inputs(rng, n, hidden, flip)
        rec["enc_%d_pred" % k] = pred
        rec["enc_%d_true" % k] = true
        rec["enc_%d_meta" % k] = np.array([n, hidden], dtype=np.int64)
        rec["enc_%d_out" % k] = ref_encoding(L, pred, true, n, hidden)
    np.savez_compressed(os.path.join(HERE, "evaluator.npz"), **rec)
    print("wrote", os.path.join(HERE, "evaluator.npz"), len(CLASS_CASES) + len(ENC_CASES),
          "cases")


if __name__ == "__main__":
    main()
