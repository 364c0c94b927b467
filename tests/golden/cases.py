"""Golden-fixture cases: small machines that together cover every branch of
the reference's hot path -- classifier / encoder, dense / individualized,
tail masks (2F % 8 != 0), the 128-bit tail path (input_chunks % 16 == 0
with 2F % 8 != 0), state_bits 2..8, include_bits 1..3, clause_maximum
below and above the literal counts, target < 1, out-of-range labels,
empty training sets, random padding bits in the tail byte, and a
config-0-shaped machine (784 features, 49-word rows)."""
import numpy as np


def flip_pack(bits):
    bits = np.asarray(bits, dtype=bool)
    return np.packbits(np.concatenate([bits, ~bits], axis=1), axis=1, bitorder="little")


def _c(name, create, train, data):
    return dict(name=name, create=create, train=train, data=data)


CASES = [
    _c("cls_f16", dict(type="classifier", classes=3, features=16, clauses=16, clause_tolerance=8,
                       clause_maximum=8, specificity=4.0),
       dict(epochs=2, seed=11), dict(n=60, nt=40, density=0.3, seed=1)),
    _c("cls_f13_tail_ib2", dict(type="classifier", classes=3, features=13, clauses=16,
                                clause_tolerance=8, clause_maximum=8, include_bits=2,
                                specificity=4.0),
       dict(epochs=3, seed=12), dict(n=60, nt=40, density=0.3, seed=2, pad_noise=True,
                                     bad_labels=True)),
    _c("cls_f61_q2", dict(type="classifier", classes=2, features=61, clauses=8,
                          clause_tolerance=5, clause_maximum=20, state=4, include_bits=2,
                          target=10, specificity=3.0),
       dict(epochs=3, seed=13), dict(n=50, nt=30, density=0.3, seed=3, pad_noise=True)),
    _c("enc_v20_b3", dict(type="encoder", classes=9, features=20, clauses=8,
                          clause_tolerance=3, clause_maximum=6, state=3, include_bits=2,
                          target=0.3, specificity=5.0),
       dict(epochs=2, seed=14), dict(n=50, nt=30, density=0.3, seed=4)),
    _c("enc_v64_ib3", dict(type="encoder", classes=5, features=64, clauses=24,
                           clause_tolerance=16, clause_maximum=16, include_bits=3,
                           specificity=2.0),
       dict(epochs=2, seed=15), dict(n=40, nt=30, density=0.4, seed=5)),
    _c("cls_f100_b2", dict(type="classifier", classes=4, features=100, clauses=16,
                           clause_tolerance=10, clause_maximum=50, state=2, target=6,
                           specificity=8.0),
       dict(epochs=2, seed=16), dict(n=40, nt=30, density=0.3, seed=6)),
    _c("cls_ind", dict(type="classifier", classes=4, clauses=16, clause_tolerance=8,
                       clause_maximum=8, specificity=4.0, individualized=True),
       dict(epochs=2, seed=17), dict(n=50, nt=30, density=0.3, seed=7, ind_max=12)),
    _c("enc_ind", dict(type="encoder", classes=4, clauses=16, clause_tolerance=8,
                       clause_maximum=8, include_bits=2, specificity=3.0, individualized=True),
       dict(epochs=2, seed=18), dict(n=50, nt=30, density=0.3, seed=8, ind_max=12)),
    _c("cls_empty", dict(type="classifier", classes=3, features=10, clauses=8,
                         clause_tolerance=4, clause_maximum=4, specificity=2.0),
       dict(epochs=2, seed=19), dict(n=0, nt=10, density=0.3, seed=9)),
    _c("cls_c0_shape", dict(type="classifier", classes=10, features=784, clauses=32,
                            clause_tolerance=64, clause_maximum=64, target=50,
                            specificity=10.0),
       dict(epochs=2, seed=20), dict(n=200, nt=100, seed=10, prototypes=True)),
    _c("cls_refstruct", dict(type="classifier", classes=3, features=16, clauses=16,
                             clause_tolerance=8, clause_maximum=8, specificity=4.0),
       dict(epochs=2, seed=0, refstruct=True), dict(n=60, nt=40, density=0.3, seed=1)),
    _c("enc_refstruct", dict(type="encoder", classes=5, features=61, clauses=16,
                             clause_tolerance=8, clause_maximum=8, state=5, include_bits=2,
                             specificity=4.0),
       dict(epochs=2, seed=0, refstruct=True), dict(n=60, nt=40, density=0.3, seed=2)),
]


def make_inputs(c):
    d = c["data"]
    cr = c["create"]
    rng = np.random.default_rng(d["seed"])
    n, nt = d["n"], d["nt"]
    classes = cr["classes"]
    out = dict(n=n, nt=nt)
    if cr.get("individualized"):
        ks = rng.integers(1, d["ind_max"] + 1, size=classes)
        fo = np.concatenate([[0], np.cumsum(ks)]).astype(np.int64)
        cr["feat_offsets"] = fo
        out["feat_offsets"] = fo

        def pack(nn):
            blocks, offs, off = [], [], 0
            for h in range(classes):
                xb = flip_pack(rng.random((nn, ks[h])) < d["density"])
                offs.append(off)
                off += xb.size
                blocks.append(xb.ravel())
            return (np.concatenate(blocks) if blocks else np.zeros(0, np.uint8),
                    np.array(offs, dtype=np.int64))
        out["x"], out["dim_offsets"] = pack(max(n, 1))
        out["xt"], out["dim_offsets_t"] = pack(nt)
    else:
        F = cr["features"]
        if d.get("prototypes"):
            protos = np.random.default_rng(d["seed"] + 99).random((classes, F)) < 0.2

            def gen(nn, y):
                return flip_pack(protos[y] ^ (rng.random((nn, F)) < 0.1))
            y = rng.integers(0, classes, size=n)
            yt = rng.integers(0, classes, size=nt)
            out["x"], out["xt"] = gen(n, y), gen(nt, yt)
            out["labels"] = y.astype(np.int64)
        else:
            out["x"] = flip_pack(rng.random((max(n, 1), F)) < d["density"])
            out["xt"] = flip_pack(rng.random((nt, F)) < d["density"])
        if d.get("pad_noise") and (2 * F) % 8:
            pm = np.uint8(~((1 << ((2 * F) % 8)) - 1) & 0xFF)
            out["x"][:, -1] |= rng.integers(0, 256, size=out["x"].shape[0]).astype(np.uint8) & pm
            out["xt"][:, -1] |= rng.integers(0, 256, size=nt).astype(np.uint8) & pm
        out["x"] = np.ascontiguousarray(out["x"]).ravel()
        out["xt"] = np.ascontiguousarray(out["xt"]).ravel()
    if cr["type"] == "classifier":
        if "labels" not in out:
            y = rng.integers(0, classes, size=max(n, 1)).astype(np.int64)
            if d.get("bad_labels"):
                y[::7] = -1
            out["labels"] = y
    else:
        out["codes"] = np.packbits(rng.random((max(n, 1), classes)) < 0.5, axis=1,
                                   bitorder="little").ravel()
    return out
