"""One machine trained across two ranks (gloo, host exchange) on the one
GPU available: each rank trains its class range, the ranks all-gather the
automata, and both end bit-identical to the machine trained by one process.
The ranks' kernels never wait on each other; the only exchange is the
host-side all-gather after training."""
import hashlib
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG = dict(classes=5, features=600, clauses=48, clause_tolerance=16, clause_maximum=60,
           specificity=8.0, target=20, reusable=True, seed=13)


def _data():
    from santoku_tsetlin import datagen
    x, y, _ = datagen.prototype_classifier(900, classes=5, features=600, seed=21)
    return x.ravel(), y.astype(np.int64)


def _digest(t):
    a, s = t.export_state()
    return hashlib.sha256(a.tobytes() + s.tobytes()).hexdigest()


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
        import santoku_tsetlin as tm
        from santoku_tsetlin import multi
        x, y = _data()
        t = tm.create("classifier", dict(CFG))
        multi.train_sharded(t, dict(samples=len(y), problems=x, solutions=y, iterations=3))
        q.put((rank, _digest(t), [int(v) for v in t.predict(x, 64)]))
        t.destroy()
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        q.put((rank, "error: %r" % (e,), None))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_class_sharded_training_equals_single_process(tm):
    x, y = _data()
    t = tm.create("classifier", dict(CFG))
    t.train(dict(samples=len(y), problems=x, solutions=y, iterations=3))
    want = _digest(t)
    want_pred = [int(v) for v in t.predict(x, 64)]
    # a class range alone trains only those classes: the others stay initial
    u = tm.create("classifier", dict(CFG))
    u.train(dict(samples=len(y), problems=x, solutions=y, iterations=3, class_range=(1, 3)))
    ua, _ = u.export_state()
    ta, _ = t.export_state()
    per = len(ta) // CFG["classes"]
    assert np.array_equal(ua[per:3 * per], ta[per:3 * per])
    assert not ua[:per].any() and not ua[3 * per:].any()
    with pytest.raises(tm.TsetlinError):
        u.train(dict(samples=len(y), problems=x, solutions=y, iterations=1, class_range=(3, 9)))
    u.destroy()
    t.destroy()

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in procs:
            rank, digest, pred = q.get(timeout=600)
            got[rank] = (digest, pred)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.terminate()
    for rank in (0, 1):
        assert got[rank][0] == want, got[rank][0]
        assert got[rank][1] == want_pred


@pytest.mark.parametrize("on_device", [True, False])
def test_class_slices_round_trip(tm, on_device):
    """export_classes / import_classes move exactly the slice of the
    reference byte layout that a class range occupies, device to device (the
    NCCL exchange of train_sharded) or through host memory (gloo)."""
    import torch
    x, y = _data()
    t = tm.create("classifier", dict(CFG))
    t.train(dict(samples=len(y), problems=x, solutions=y, iterations=2))
    ta, ts = t.export_state()
    C = CFG["classes"]
    pa, ps = len(ta) // C, len(ts) // C
    u = tm.create("classifier", dict(CFG, seed=99))
    for lo, hi in ((0, 2), (2, 5)):
        a, s = t.class_bytes(lo, hi)
        assert (a, s) == ((hi - lo) * pa, (hi - lo) * ps)
        buf = torch.zeros(a + s + 5, dtype=torch.uint8, device="cuda" if on_device else "cpu")
        t.export_classes(lo, hi, buf)
        got = buf.cpu().numpy()
        assert np.array_equal(got[:a], ta[lo * pa:hi * pa])
        assert np.array_equal(got[a:a + s], ts[lo * ps:hi * ps])
        u.import_classes(lo, hi, buf)
    ua, us = u.export_state()
    assert np.array_equal(ua, ta) and np.array_equal(us, ts)
    assert np.array_equal(u.predict(x, 64), t.predict(x, 64))
    with pytest.raises(tm.TsetlinError):
        t.export_classes(3, 9, torch.zeros(1 << 20, dtype=torch.uint8))
    t.destroy()
    u.destroy()
