"""Generates the golden fixtures under tests/golden/ from the reference's own
code.

Runs only where the reference tree is present: it drives the reference-code
harness (oracle/_ref/libtm_ref.so, built by `make -C oracle` from the
reference's lib/santoku/tsetlin/capi.c and automata.h) and records, for each
case, the inputs and the reference's outputs:

  * derived parameters (capi.c:449-606),
  * actions and count planes after training under the Philox draw contract
    (capi.c:85-402 driven per sample, automata.h),
  * per-class vote sums, predictions / codes (capi.c:903-1086),
  * persisted bytes (capi.c:1509-1562),
  * for the `refstruct` cases, the same after training with the reference's
    own per-thread structure on one thread (stand-in generator).

Usage:  python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import oracle as O  # noqa: E402
from cases import CASES, make_inputs  # noqa: E402


def main():
    O.build()
    if not O.ref_available():
        raise SystemExit("reference harness not built (reference tree absent)")
    for c in CASES:
        inp = make_inputs(c)
        m = O.Machine(which="ref", **c["create"])
        tr = c["train"]
        kw = dict(labels=inp.get("labels"), codes=inp.get("codes"),
                  dim_offsets=inp.get("dim_offsets"), seed=tr["seed"],
                  mode=O.REFSTRUCT if tr.get("refstruct") else O.PHILOX, threads=1)
        m.train(inp["x"], inp["n"], tr["epochs"], **kw)
        out, scores = m.predict(inp["xt"], inp["nt"], dim_offsets=inp.get("dim_offsets_t"),
                                scores=True, threads=1)
        acts = m.actions()
        state = m.state()
        blob = m.persist()
        info = m.info
        rec = dict(
            info_keys=np.array(list(info.keys())),
            info_vals=np.array(list(info.values()), dtype=np.uint64),
            actions=acts,
            state_sha256=np.frombuffer(hashlib.sha256(state.tobytes()).digest(), dtype=np.uint8),
            scores=scores,
            out=out,
            persist=np.frombuffer(blob, dtype=np.uint8),
        )
        if state.size <= 65536:
            rec["state"] = state
        for k, v in inp.items():
            if v is None:
                continue
            rec["in_" + k] = np.asarray(v)
        path = os.path.join(HERE, c["name"] + ".npz")
        np.savez_compressed(path, **rec)
        print("%-28s actions %7d B  state %8d B  ones %d" % (c["name"], acts.size, state.size,
                                                           int(np.unpackbits(acts).sum())))


if __name__ == "__main__":
    main()
