"""The CPU oracle, pinned against the reference's own code.

* Philox4x32-10 against the Random123 known-answer vectors.
* Every golden fixture (generated from the reference's capi.c/automata.h by
  tests/golden/make_golden.py) reproduced bit-for-bit: derived parameters,
  actions, count planes, vote sums, predictions, persisted bytes.
* Where the reference harness is built (oracle/_ref), random machines
  cross-checked oracle vs reference code in both draw modes.
* The evaluator restatement (oracle/evaluator_ref.py, the checker of the
  device metrics) against the reference's own tm_class_accuracy and
  tm_encoding_accuracy (evaluator/capi.c:119-202, 497-574): bit for bit on
  the fixtures tests/golden/make_golden_evaluator.py recorded from them,
  and, where the evaluator harness is built (oracle/_ref/libeval_ref.so),
  on fresh random cases.
"""
import ctypes
import hashlib
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from cases import CASES, make_inputs  # noqa: E402

import oracle as O  # noqa: E402



def test_philox_known_answers(oracle_lib):
    kat = [
        ([0, 0, 0, 0], 0, [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
        ([0xFFFFFFFF] * 4, 0xFFFFFFFFFFFFFFFF, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
        ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], (0x299F31D0 << 32) | 0xA4093822,
         [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
    ]
    for ctr, key, want in kat:
        assert list(O.philox(ctr, key)) == want


def test_perm_is_permutation(oracle_lib):
    for n in (0, 1, 2, 17, 1000):
        p = O.perm(7, 3, n)
        assert sorted(p.tolist()) == list(range(n))
    a, b = O.perm(7, 3, 500), O.perm(7, 4, 500)
    assert not np.array_equal(a, b)
    assert np.array_equal(a, O.perm(7, 3, 500))


def load_fixture(name):
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_fixture(oracle_lib, case):
    case = dict(case, create=dict(case["create"]))
    inp = make_inputs(case)
    fx = load_fixture(case["name"])
    m = O.Machine(**case["create"])
    tr = case["train"]
    m.train(inp["x"], inp["n"], tr["epochs"], labels=inp.get("labels"), codes=inp.get("codes"),
            dim_offsets=inp.get("dim_offsets"), seed=tr["seed"],
            mode=O.REFSTRUCT if tr.get("refstruct") else O.PHILOX, threads=1)
    info = dict(zip(fx["info_keys"].tolist(), fx["info_vals"].tolist()))
    assert m.info == info
    assert np.array_equal(inp["x"], fx["in_x"])
    assert np.array_equal(m.actions(), fx["actions"])
    st = m.state()
    assert hashlib.sha256(st.tobytes()).digest() == fx["state_sha256"].tobytes()
    out, scores = m.predict(inp["xt"], inp["nt"], dim_offsets=inp.get("dim_offsets_t"),
                            scores=True, threads=1)
    assert np.array_equal(scores, fx["scores"])
    assert np.array_equal(out, fx["out"])
    assert m.persist() == fx["persist"].tobytes()


def test_oracle_multithreaded_philox_is_deterministic(oracle_lib):
    case = dict(CASES[9], create=dict(CASES[9]["create"]))
    inp = make_inputs(case)
    res = []
    for threads in (1, 4):
        m = O.Machine(**case["create"])
        m.train(inp["x"], inp["n"], 2, labels=inp["labels"], seed=20, threads=threads)
        res.append((m.actions(), m.state()))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


def test_persist_load_roundtrip(oracle_lib):
    case = dict(CASES[3], create=dict(CASES[3]["create"]))
    inp = make_inputs(case)
    m = O.Machine(**case["create"])
    m.train(inp["x"], inp["n"], 2, codes=inp["codes"], seed=3)
    blob = m.persist()
    m2 = O.Machine.load(blob)
    assert m2.info["has_state"] == 0
    assert np.array_equal(m2.actions(), m.actions())
    assert np.array_equal(m2.predict(inp["xt"], inp["nt"]), m.predict(inp["xt"], inp["nt"]))
    assert m2.persist() == blob


def test_oracle_reconfigure_and_restrict(oracle_lib):
    m = O.Machine(type="classifier", classes=3, features=16, clauses=16, clause_tolerance=8,
                  clause_maximum=8, specificity=4.0, reusable=True)
    m.reconfigure(clauses=20, clause_tolerance=4, clause_maximum=10, specificity=2.0, target=0.5)
    assert m.info["clauses"] == 24 and m.info["target"] == 12
    fo = np.array([0, 3, 8, 10], dtype=np.int64)
    mi = O.Machine(type="encoder", classes=3, clauses=8, clause_tolerance=4, clause_maximum=4,
                   specificity=2.0, individualized=True, feat_offsets=fo)
    a = mi.actions()
    mi.restrict([2, 0])
    assert mi.info["classes"] == 2
    assert mi.info["action_chunks"] == 8 * 1 + 8 * 1


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built here")
@pytest.mark.parametrize("seed", range(6))
def test_oracle_vs_reference_random(oracle_lib, seed):
    rng = np.random.default_rng(1000 + seed)
    kind = "classifier" if seed % 2 == 0 else "encoder"
    F = int(rng.integers(3, 90))
    classes = int(rng.integers(2, 7))
    kw = dict(type=kind, classes=classes, features=F, clauses=int(rng.integers(1, 4)) * 8,
              clause_tolerance=int(rng.integers(1, 20)), clause_maximum=int(rng.integers(1, 40)),
              state=int(rng.integers(2, 9)), include_bits=int(rng.integers(1, 4)),
              target=float(rng.choice([-1.0, 0.25, 7.0])), specificity=float(rng.uniform(1.5, 9)))
    n = 50
    x = np.packbits(np.concatenate([(b := rng.random((n, F)) < 0.35), ~b], axis=1), axis=1,
                    bitorder="little").ravel()
    labels = rng.integers(0, classes, size=n).astype(np.int64)
    codes = np.packbits(rng.random((n, classes)) < 0.5, axis=1, bitorder="little").ravel()
    for mode in (O.PHILOX, O.REFSTRUCT):
        res = []
        for which in ("oracle", "ref"):
            m = O.Machine(which=which, **kw)
            m.train(x, n, 3, labels=labels if kind == "classifier" else None,
                    codes=codes if kind == "encoder" else None, seed=seed, mode=mode, threads=1)
            res.append((m.actions(), m.state(), m.predict(x, n, scores=True)[1], m.persist()))
        assert np.array_equal(res[0][0], res[1][0])
        assert np.array_equal(res[0][1], res[1][1])
        assert np.array_equal(res[0][2], res[1][2])
        assert res[0][3] == res[1][3]


@pytest.mark.parametrize("case", ["cls_ind", "enc_ind"])
def test_bits_to_cvec_ind_restatement_matches_fixture_layout(case):
    """The restated bits_to_cvec_ind rebuilds the individualized inputs that
    the reference-code fixtures were trained and predicted on: per-block
    flip-interleaved rows at the recorded dim_offsets."""
    import evaluator_ref as R
    d = np.load(os.path.join(HERE, "golden", case + ".npz"))
    fo = d["in_feat_offsets"]
    for xk, ok, n in (("in_x", "in_dim_offsets", max(int(d["in_n"]), 1)),
                      ("in_xt", "in_dim_offsets_t", int(d["in_nt"]))):
        x, offs = d[xk], d[ok]
        lists = []
        for h in range(len(fo) - 1):
            k = int(fo[h + 1] - fo[h])
            nb = (2 * k + 7) // 8
            blk = x[offs[h]:offs[h] + n * nb].reshape(n, nb)
            bits = np.unpackbits(blk, axis=1, bitorder="little", count=k).astype(bool)
            s, f = np.nonzero(bits)
            lists.append((s * k + f).astype(np.int64))
        io = np.concatenate([[0], np.cumsum([len(v) for v in lists])]).astype(np.int64)
        got, doff = R.bits_to_cvec_ind(np.concatenate(lists), io, fo, n, True)
        assert np.array_equal(doff[:-1], offs)
        assert np.array_equal(got, x)


def _class_vec(r):
    return np.array([r["precision"], r["recall"], r["f1"]] +
                    [v for c in r["classes"] for v in (c["precision"], c["recall"], c["f1"])])


def _enc_vec(r):
    return np.array([r["mean_hamming"], r["ber_min"], r["ber_max"], r["ber_std"]] + r["bits"])


def test_evaluator_restatement_matches_reference_fixtures():
    """Every recorded case of the reference's evaluator reproduced to the
    last bit: per-class and macro precision / recall / F1 (out-of-range
    predictions and labels skipped, classes without support at 0), and
    mean Hamming accuracy, the per-bit error rates, their extremes and
    standard deviation (one bit: 0)."""
    import evaluator_ref as R
    z = np.load(os.path.join(HERE, "golden", "evaluator.npz"))
    kinds = {"class": (R.class_accuracy, _class_vec), "enc": (R.encoding_accuracy, _enc_vec)}
    seen = 0
    for key in sorted(k for k in z.files if k.endswith("_out")):
        kind, k = key.split("_")[:2]
        fn, vec = kinds[kind]
        n, dims = (int(v) for v in z["%s_%s_meta" % (kind, k)])
        got = vec(fn(z["%s_%s_pred" % (kind, k)], z["%s_%s_true" % (kind, k)], n, dims))
        assert np.array_equal(got, z[key]), key
        seen += 1
    assert seen >= 14


EVAL_SO = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libeval_ref.so")


@pytest.mark.skipif(not os.path.exists(EVAL_SO), reason="evaluator harness not built")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_evaluator_restatement_vs_reference_random(seed):
    import evaluator_ref as R
    L = ctypes.CDLL(EVAL_SO)
    vp = ctypes.c_void_p
    rng = np.random.default_rng(seed)
    for _ in range(40):
        classes, n = int(rng.integers(1, 50)), int(rng.integers(1, 4000))
        yt = rng.integers(0, classes + 1, size=n).astype(np.int64)
        yp = np.where(rng.random(n) < rng.random(), yt,
                      rng.integers(-3, classes + 3, size=n)).astype(np.int64)
        out = np.zeros(3 + 3 * classes)
        L.ref_eval_class_accuracy(yp.ctypes.data_as(vp), yt.ctypes.data_as(vp),
                                  ctypes.c_uint32(n), ctypes.c_uint32(classes),
                                  out.ctypes.data_as(vp))
        assert np.array_equal(_class_vec(R.class_accuracy(yp, yt, n, classes)), out)
        hidden, n = int(rng.integers(1, 400)), int(rng.integers(1, 2000))
        nb = (hidden + 7) // 8
        e = rng.integers(0, 256, size=n * nb, dtype=np.uint8)
        p = e.copy()
        sel = rng.random(n * nb) < rng.random()
        p[sel] ^= rng.integers(1, 256, size=int(sel.sum()), dtype=np.uint8)
        out = np.zeros(4 + hidden)
        L.ref_eval_encoding_accuracy(p.ctypes.data_as(vp), e.ctypes.data_as(vp),
                                     ctypes.c_uint32(n), ctypes.c_uint32(hidden),
                                     out.ctypes.data_as(vp))
        assert np.array_equal(_enc_vec(R.encoding_accuracy(p, e, n, hidden)), out)
