"""Large-batch predict through the 8-bit GEMM (failed literals F = L - A.x
from a tensor-core product of action bytes and literal bytes, votes and
class sums in the library's own epilogue) against the oracle's bitwise
evaluation (capi.c:97-161): vote sums and outputs identical, bit for bit,
in the device's default encoding and, in a child process, in the other
one (e4m3 operands with fp32 accumulation)."""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from test_gpu_parity import ref_table  # noqa: E402

import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu


def _machine_pair(tm, kind, classes, F, clauses, dens, seed):
    rng = np.random.default_rng(seed)
    cfg = dict(type=kind, classes=classes, features=F, clauses=clauses, clause_tolerance=48,
               clause_maximum=64, specificity=25.0)
    m = O.Machine(**cfg)
    acts = np.packbits(rng.random(m.info["action_chunks"] * 8) < dens, bitorder="little")
    m.load_state(actions=acts)
    kind2, tbl = ref_table(cfg)
    t = tm.create(kind2, tbl)
    t.import_state(actions=acts)
    return m, t, rng


@pytest.mark.parametrize("kind,classes,F,clauses,dens,sizes", [
    ("classifier", 20, 16384, 136, 0.0005, (97, 300, 1000)),  # clauses of ~16 literals
    ("classifier", 20, 16384, 136, 0.01, (300,)),
    ("classifier", 7, 16000, 40, 0.001, (2500,)),             # 1,000-word rows, tail mask
    ("encoder", 24, 4096, 48, 0.01, (1200,)),
], ids=["c1_rows_short", "c1_rows", "tail", "encoder"])
def test_gemm_predict_matches_oracle(tm, kind, classes, F, clauses, dens, sizes):
    m, t, rng = _machine_pair(tm, kind, classes, F, clauses, dens, classes * F + clauses)
    t.stats_enable(True)
    for n in sizes:
        b = rng.random((n, F)) < 0.02
        x = np.packbits(np.concatenate([b, ~b], axis=1), axis=1, bitorder="little").ravel()
        want_out, want = m.predict(x, n, scores=True)
        assert np.array_equal(t.predict_scores(x, n), want), n
        assert t.stats()["predict_gemm"] in (1, 2), n
        assert np.array_equal(np.asarray(t.predict(x, n)).ravel(), np.asarray(want_out).ravel()), n
    t.destroy()


def test_gemm_predict_other_encoding_matches_oracle(tm):
    """The encoding the device did not choose by default, pinned with
    TSETLIN_B200_GEMM in a child process (the choice is made once per
    process)."""
    code = r'''
import sys, numpy as np
sys.path[:0] = [{oracle!r}, {pkg!r}, {tests!r}]
import santoku_tsetlin as tm
import oracle as O
from test_gpu_gemm_predict import _machine_pair
m, t, rng = _machine_pair(tm, "classifier", 20, 16384, 136, 0.0005, 99)
b = rng.random((400, 16384)) < 0.02
x = np.packbits(np.concatenate([b, ~b], axis=1), axis=1, bitorder="little").ravel()
want = m.predict(x, 400, scores=True)[1]
t.stats_enable(True)
got = t.predict_scores(x, 400)
print("ENC", t.stats()["predict_gemm"], "EQ", bool(np.array_equal(got, want)))
'''
    root = os.path.dirname(HERE)
    env = dict(os.environ, TSETLIN_B200_GEMM="fp8")
    r = subprocess.run([sys.executable, "-c", code.format(
        oracle=os.path.join(root, "oracle"), pkg=os.path.join(root, "lua-santoku-tsetlin_b200"),
        tests=HERE)],
        env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("ENC")][-1]
    enc, eq = line.split()[1], line.split()[3]
    assert eq == "True", line
    assert enc in ("0", "2"), line  # e4m3, or the bitwise kernels if the library has no e4m3 GEMM
