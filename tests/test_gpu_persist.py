"""Versioned save with state (tm_save / tm_save_buf) and its load.

The container's bytes equal the restatement in oracle/persist_ref.py built
from the machine's own reference record (tm_persist, whose bytes the parity
tests pin to the reference) and exported count planes.  A machine loaded
from it is the saved machine: same info, actions, count planes and
predictions, and -- because `negative`, the seed and the reusable flag
travel too -- the same result when trained again.  Corrupt, truncated and
future-version data are refused.
"""
import os
import struct
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from cases import CASES, make_inputs  # noqa: E402

import persist_ref as P  # noqa: E402

pytestmark = pytest.mark.gpu

CASE_IDS = ["cls_f61_q2", "enc_v20_b3", "cls_ind", "enc_ind", "cls_c0_shape"]


def _machine(tm, name, negative=None):
    base = next(c for c in CASES if c["name"] == name)
    case = dict(base, create=dict(base["create"]))
    inp = make_inputs(case)
    c = dict(case["create"])
    kind = c.pop("type")
    t = {}
    if kind == "encoder":
        t["hidden"] = c.pop("classes")
        if "features" in c:
            t["visible"] = c.pop("features")
    t.update(c)
    t.update(reusable=True, seed=11)
    if negative is not None and kind == "classifier":
        t["negative"] = negative
    return kind, t, inp


def _train_tbl(kind, inp, epochs):
    t = {"samples": inp["n"], "iterations": epochs}
    if kind == "classifier":
        t["problems"], t["solutions"] = inp["x"], inp["labels"]
    else:
        t["sentences"], t["codes"] = inp["x"], inp["codes"]
    if inp.get("dim_offsets") is not None:
        t["dim_offsets"] = inp["dim_offsets"]
    return t


def _pargs(inp):
    if inp.get("dim_offsets_t") is not None:
        return (inp["xt"], inp["dim_offsets_t"], inp["nt"])
    return (inp["xt"], inp["nt"])


@pytest.mark.parametrize("name", CASE_IDS)
def test_save_with_state_round_trip(tm, name, tmp_path):
    kind, tbl, inp = _machine(tm, name, negative=0.37)
    t = tm.create(kind, tbl)
    t.train(_train_tbl(kind, inp, 2))
    acts, state = t.export_state()
    blob = t.save()
    neg = 0.37 if kind == "classifier" else 1.0 / t.info()["classes"]
    assert blob == P.container(t.persist(), state.tobytes(), neg, 11, True)
    path = str(tmp_path / "m.stmv")
    t.save(path)
    assert open(path, "rb").read() == blob
    for t2 in (tm.load(blob, True), tm.load(path)):
        assert t2.info() == t.info()
        a2, s2 = t2.export_state()
        assert np.array_equal(a2, acts) and np.array_equal(s2, state)
        assert np.array_equal(np.asarray(t2.predict(*_pargs(inp))),
                              np.asarray(t.predict(*_pargs(inp))))
        assert t2.persist() == t.persist()
        assert t2.save() == blob
        t2.destroy()
    # negative, seed and reusable travel: training both again ends equal
    t3 = tm.load(blob, True)
    t.train(_train_tbl(kind, inp, 1))
    t3.train(_train_tbl(kind, inp, 1))
    for x, y in zip(t.export_state(), t3.export_state()):
        assert np.array_equal(x, y)
    t3.reconfigure(dict(clauses=tbl["clauses"], clause_tolerance=tbl["clause_tolerance"],
                        clause_maximum=tbl["clause_maximum"], target=tbl.get("target", 8),
                        specificity=tbl["specificity"]))
    t.destroy()
    t3.destroy()


def test_save_without_state_and_refusals(tm):
    kind, tbl, inp = _machine(tm, "enc_v64_ib3")
    t = tm.create(kind, tbl)
    t.train(_train_tbl(kind, inp, 2))
    blob = t.save(state=False)
    version, flags, _, seed, record, st = P.parse(blob)
    assert (version, flags, seed, st) == (1, 2, 11, None)
    assert record == t.persist()
    t2 = tm.load(blob, True)
    assert t2.info()["has_state"] == 0 and t2.info()["reusable"] == 1
    assert np.array_equal(np.asarray(t2.predict(*_pargs(inp))), np.asarray(t.predict(*_pargs(inp))))
    with pytest.raises(tm.TsetlinError, match="without state"):
        t2.train(_train_tbl(kind, inp, 1))
    with pytest.raises(tm.TsetlinError, match="no state"):
        t2.save(state=True)
    full = t.save()
    bad = bytearray(full)
    bad[60] ^= 1
    with pytest.raises(tm.TsetlinError, match="checksum"):
        tm.load(bytes(bad), True)
    with pytest.raises(tm.TsetlinError, match="truncated|checksum"):
        tm.load(full[:-20], True)
    _, fl, neg, sd, rec, stt = P.parse(full)
    future = P.container(rec, stt, neg, sd, bool(fl & 2), version=2)
    with pytest.raises(tm.TsetlinError, match="version 2"):
        tm.load(future, True)
    # trailing bytes inside a valid checksum
    body = full[:-8] + b"\0"
    with pytest.raises(tm.TsetlinError, match="trailing"):
        tm.load(body + struct.pack("<Q", P.fnv1a64(body)), True)
    t.destroy()
    t2.destroy()


def test_non_reusable_machine_saves_without_state(tm):
    kind, tbl, inp = _machine(tm, "cls_f61_q2")
    tbl["reusable"] = False
    t = tm.create(kind, tbl)
    t.train(_train_tbl(kind, inp, 1))
    with pytest.raises(tm.TsetlinError, match="no state"):
        t.save()
    t2 = tm.load(t.save(state=False), True)
    assert t2.persist() == t.persist()
    t.destroy()
    t2.destroy()
