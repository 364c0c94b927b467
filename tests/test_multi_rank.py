"""Multi-rank host path on CPU: world size 2 over gloo.

The per-rank device work is replaced by the oracle's vote sums for the
rank's class range (test infrastructure); what is under test is the
partitioning, the exchange of per-class sums, the reference's argmax / sign
finish (capi.c:934-942, 982-990) and the max-over-ranks timing reduction.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path.insert(0, os.path.join(root, "lua-santoku-tsetlin_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    import oracle as O
    from santoku_tsetlin import multi
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = {}
        for kind, classes in (("classifier", 7), ("encoder", 13)):
            rng = np.random.default_rng(3)
            F, n = 40, 60
            m = O.Machine(type=kind, classes=classes, features=F, clauses=16, clause_tolerance=6,
                          clause_maximum=12, specificity=4.0)
            x = np.packbits(np.concatenate([(b := rng.random((n, F)) < 0.3), ~b], axis=1),
                            axis=1, bitorder="little").ravel()
            lab = rng.integers(0, classes, size=n).astype(np.int64)
            cod = np.packbits(rng.random((n, classes)) < 0.5, axis=1, bitorder="little").ravel()
            m.train(x, n, 2, labels=lab if kind == "classifier" else None,
                    codes=cod if kind == "encoder" else None, seed=5)
            want, scores = m.predict(x, n, scores=True)
            lo, hi = multi.class_range(classes, world, rank)
            got, full = multi.gather_predict(scores[:, lo:hi], classes, kind)
            res[kind] = (np.array_equal(got, want.ravel()), np.array_equal(full, scores))
        res["max"] = multi.max_over_ranks(10.0 + rank)
        res["parts"] = multi.partition_lpt([5, 1, 4, 4, 2, 9, 3], world)
        out[rank] = res
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_gloo(oracle_lib):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    for r in range(world):
        res = out[r]
        assert res["classifier"] == (True, True)
        assert res["encoder"] == (True, True)
        assert res["max"] == 11.0
        assert res["parts"] == out[0]["parts"]
    parts = out[0]["parts"]
    assert sorted(parts[0] + parts[1]) == list(range(7))


def test_partition_and_ranges():
    from santoku_tsetlin import multi
    p = multi.partition_lpt([8, 1, 1, 1, 1, 1, 1, 1, 1], 2)
    assert p == [[0], [1, 2, 3, 4, 5, 6, 7, 8]]
    covered = []
    for r in range(3):
        lo, hi = multi.class_range(10, 3, r)
        covered += list(range(lo, hi))
    assert covered == list(range(10))


class _OracleRangeMachine:
    """Stand-in for a device machine in `multi.train_sharded` (test
    infrastructure): training a class range is the oracle's full training
    with every class outside the range put back to its initial state --
    units are independent, so that is what class-range training leaves."""

    def __init__(self, O, cfg, x, lab, n):
        self.m = O.Machine(**cfg)
        self.x, self.lab, self.n = x, lab, n
        self.a0, self.s0 = self.m.actions(), self.m.state()

    def info(self):
        return dict(self.m.info)

    def train(self, tbl):
        lo, hi = tbl["class_range"]
        self.m.train(self.x, self.n, tbl["iterations"], labels=self.lab, seed=5)
        a, s = self.m.actions(), self.m.state()
        C = self.m.info["classes"]
        pa, ps = len(a) // C, len(s) // C
        for h in range(C):
            if not lo <= h < hi:
                a[h * pa:(h + 1) * pa] = self.a0[h * pa:(h + 1) * pa]
                s[h * ps:(h + 1) * ps] = self.s0[h * ps:(h + 1) * ps]
        self.m.load_state(a, s)

    def export_state(self):
        return self.m.actions(), self.m.state()

    def import_state(self, a, s):
        self.m.load_state(a, s)

    # the class-slice interface of santoku_tsetlin.Machine, on host tensors
    def class_bytes(self, lo, hi):
        C = self.m.info["classes"]
        pa, ps = len(self.a0) // C, len(self.s0) // C
        return (hi - lo) * pa, (hi - lo) * ps

    def export_classes(self, lo, hi, out):
        a, s = self.export_state()
        na, ns = self.class_bytes(lo, hi)
        pa, ps = self.class_bytes(0, 1)
        out[:na] = __import__("torch").from_numpy(a[lo * pa:lo * pa + na].copy())
        out[na:na + ns] = __import__("torch").from_numpy(s[lo * ps:lo * ps + ns].copy())
        return out

    def import_classes(self, lo, hi, buf):
        a, s = self.export_state()
        na, ns = self.class_bytes(lo, hi)
        pa, ps = self.class_bytes(0, 1)
        b = buf.numpy()
        a[lo * pa:lo * pa + na] = b[:na]
        s[lo * ps:lo * ps + ns] = b[na:na + ns]
        self.import_state(a, s)


def _sharded_worker(rank, world, port, out, classes):
    import sys
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path.insert(0, os.path.join(root, "lua-santoku-tsetlin_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    import oracle as O
    from santoku_tsetlin import multi
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(8)
        F, n = 30, 50
        cfg = dict(type="classifier", classes=classes, features=F, clauses=16,
                   clause_tolerance=6, clause_maximum=12, specificity=4.0)
        b = rng.random((n, F)) < 0.3
        x = np.packbits(np.concatenate([b, ~b], axis=1), axis=1, bitorder="little").ravel()
        lab = rng.integers(0, classes, size=n).astype(np.int64)
        sm = _OracleRangeMachine(O, cfg, x, lab, n)
        multi.train_sharded(sm, dict(iterations=2))
        full = O.Machine(**cfg)
        full.train(x, n, 2, labels=lab, seed=5)
        a, s = sm.export_state()
        out[rank] = (np.array_equal(a, full.actions()), np.array_equal(s, full.state()))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("world,classes", [(2, 5), (3, 2)])
def test_train_sharded_gathers_every_class(oracle_lib, world, classes):
    """gloo ranks on CPU: each rank holds every class's automata after
    `train_sharded`, equal to one process training the whole machine --
    also with more ranks than classes, where a rank trains nothing but must
    still join the exchange (otherwise the others would wait for it)."""
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_sharded_worker, args=(r, world, port, out, classes))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    for r in range(world):
        assert out[r] == (True, True)
