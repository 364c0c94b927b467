"""ctypes loader for the CPU oracle (liboracle.so) and, where it was built,
the reference-code harness (_ref/libtm_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg, never by the product package.

Both libraries expose the same machine operations, so tests can run one
scenario through either and compare the reference byte layouts they export.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtm_ref.so")

PHILOX = 0
REFSTRUCT = 1

INFO_KEYS = ("type", "classes", "features", "clauses", "clause_tolerance",
             "clause_maximum", "target", "state_bits", "include_bits",
             "input_bits", "input_chunks", "clause_chunks", "class_chunks",
             "state_chunks", "action_chunks", "tail_mask", "individualized",
             "reusable", "has_state")

_u8p = ctypes.POINTER(ctypes.c_uint8)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_vp = ctypes.c_void_p


def build():
    """Build liboracle.so (and _ref/ when the reference tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _ptr(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def _setup(lib, prefix):
    f = lambda n: getattr(lib, prefix + n)  # noqa: E731
    f("create").restype = _vp
    f("create").argtypes = [ctypes.c_int] + [ctypes.c_uint32] * 7 + [
        ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_int, _i64p]
    f("destroy").argtypes = [_vp]
    f("info").argtypes = [_vp, _u64p]
    f("train").restype = ctypes.c_int
    f("train").argtypes = [_vp, _u8p, _i64p, _u8p, _i64p, ctypes.c_uint64,
                           ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32,
                           ctypes.c_int, ctypes.c_int]
    f("predict").restype = ctypes.c_int
    f("predict").argtypes = [_vp, _u8p, _i64p, ctypes.c_uint64, _i64p, _u8p,
                             _i64p, ctypes.c_int]
    f("export").argtypes = [_vp, _u8p, _u8p]
    f("import").argtypes = [_vp, _u8p, _u8p]
    f("persist").restype = ctypes.c_int
    f("persist").argtypes = [_vp, _u8p, ctypes.c_uint64, _u64p]
    f("load").restype = _vp
    f("load").argtypes = [_u8p, ctypes.c_uint64]
    f("setup").argtypes = [_vp]


_libs = {}


def lib(which="oracle"):
    if which in _libs:
        return _libs[which]
    if which == "oracle":
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        _setup(L, "orc_")
        L.orc_perm.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, _u32p]
        L.orc_philox.argtypes = [_u32p, ctypes.c_uint64, _u32p]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_clause_eval.argtypes = [_vp, _u8p, _i64p, ctypes.c_uint64, _u32p, _u32p]
        L.orc_reconfigure.argtypes = [_vp, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.c_uint32, ctypes.c_int64, ctypes.c_double,
                                      ctypes.c_double]
        L.orc_restrict.argtypes = [_vp, _i64p, ctypes.c_uint64]
        L.orc_negative.restype = ctypes.c_double
        L.orc_negative.argtypes = [_vp]
    else:
        if not os.path.exists(REF_SO):
            return None
        L = ctypes.CDLL(REF_SO)
        _setup(L, "ref_")
        L.ref_negative.restype = ctypes.c_double
        L.ref_negative.argtypes = [_vp]
    _libs[which] = L
    return L


def ref_available():
    return os.path.exists(REF_SO)


class Machine:
    """One machine in the oracle ("oracle") or the reference harness ("ref")."""

    def __init__(self, type="classifier", classes=2, features=8, clauses=8,
                 clause_tolerance=8, clause_maximum=8, state=8, include_bits=1,
                 target=-1.0, negative=-1.0, specificity=10.0, reusable=False,
                 individualized=False, feat_offsets=None, which="oracle", _handle=None):
        self.which = which
        self.L = lib(which)
        self.p = "orc_" if which == "oracle" else "ref_"
        if _handle is not None:
            self.h = _handle
        else:
            fo = None
            if individualized:
                fo = np.ascontiguousarray(feat_offsets, dtype=np.int64)
            t = 0 if type == "classifier" else 1
            self.h = self._f("create")(t, classes, features, clauses, clause_tolerance,
                                       clause_maximum, state, include_bits, float(target),
                                       float(negative), float(specificity),
                                       int(bool(reusable)), int(bool(individualized)),
                                       _ptr(fo, _i64p))
            if not self.h:
                err = self.L.orc_last_error().decode() if which == "oracle" else "create failed"
                raise ValueError(err)
        self.info = self._info()

    def _f(self, n):
        return getattr(self.L, self.p + n)

    def _info(self):
        o = np.zeros(19, dtype=np.uint64)
        self._f("info")(self.h, _ptr(o, _u64p))
        return {k: int(v) for k, v in zip(INFO_KEYS, o)}

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def train(self, x, n, epochs, labels=None, codes=None, dim_offsets=None, seed=0,
              epoch_base=0, mode=PHILOX, threads=0):
        x = np.ascontiguousarray(x, dtype=np.uint8)
        lab = None if labels is None else np.ascontiguousarray(labels, dtype=np.int64)
        cod = None if codes is None else np.ascontiguousarray(codes, dtype=np.uint8)
        dof = None if dim_offsets is None else np.ascontiguousarray(dim_offsets, dtype=np.int64)
        rc = self._f("train")(self.h, _ptr(x, _u8p), _ptr(lab, _i64p), _ptr(cod, _u8p),
                              _ptr(dof, _i64p), n, epochs, seed, epoch_base, mode, threads)
        if rc != 0:
            raise RuntimeError("train failed")
        self.info = self._info()

    def predict(self, x, n, dim_offsets=None, threads=0, scores=False):
        x = np.ascontiguousarray(x, dtype=np.uint8)
        dof = None if dim_offsets is None else np.ascontiguousarray(dim_offsets, dtype=np.int64)
        C = self.info["classes"]
        sc = np.zeros((n, C), dtype=np.int64)
        if self.info["type"] == 0:
            out = np.zeros(n, dtype=np.int64)
            self._f("predict")(self.h, _ptr(x, _u8p), _ptr(dof, _i64p), n, _ptr(out, _i64p),
                               None, _ptr(sc, _i64p), threads)
        else:
            out = np.zeros((n, self.info["class_chunks"]), dtype=np.uint8)
            self._f("predict")(self.h, _ptr(x, _u8p), _ptr(dof, _i64p), n, None,
                               _ptr(out, _u8p), _ptr(sc, _i64p), threads)
        return (out, sc) if scores else out

    def actions(self):
        a = np.zeros(self.info["action_chunks"], dtype=np.uint8)
        self._f("export")(self.h, _ptr(a, _u8p), None)
        return a

    def state(self):
        s = np.zeros(self.info["state_chunks"], dtype=np.uint8)
        self._f("export")(self.h, None, _ptr(s, _u8p))
        return s

    def load_state(self, actions=None, state=None):
        a = None if actions is None else np.ascontiguousarray(actions, dtype=np.uint8)
        s = None if state is None else np.ascontiguousarray(state, dtype=np.uint8)
        self._f("import")(self.h, _ptr(a, _u8p), _ptr(s, _u8p))

    def setup(self):
        self._f("setup")(self.h)

    def persist(self):
        n = ctypes.c_uint64(0)
        self._f("persist")(self.h, None, 0, ctypes.byref(n))
        buf = np.zeros(n.value, dtype=np.uint8)
        rc = self._f("persist")(self.h, _ptr(buf, _u8p), n.value, ctypes.byref(n))
        if rc != 0:
            raise RuntimeError("persist failed")
        return bytes(buf)

    @classmethod
    def load(cls, data, which="oracle"):
        L = lib(which)
        p = "orc_" if which == "oracle" else "ref_"
        b = np.frombuffer(data, dtype=np.uint8).copy()
        h = getattr(L, p + "load")(_ptr(b, _u8p), len(b))
        if not h:
            raise ValueError("load failed")
        return cls(which=which, _handle=h)

    def clause_eval(self, x, n, dim_offsets=None):
        assert self.which == "oracle"
        ncl = self.info["classes"] * self.info["clauses"]
        lit = np.zeros((n, ncl), dtype=np.uint32)
        vot = np.zeros((n, ncl), dtype=np.uint32)
        x = np.ascontiguousarray(x, dtype=np.uint8)
        dof = None if dim_offsets is None else np.ascontiguousarray(dim_offsets, dtype=np.int64)
        self.L.orc_clause_eval(self.h, _ptr(x, _u8p), _ptr(dof, _i64p), n,
                               _ptr(lit, _u32p), _ptr(vot, _u32p))
        return lit, vot

    def reconfigure(self, clauses, clause_tolerance, clause_maximum, specificity,
                    include_bits=-1, target=-1.0):
        assert self.which == "oracle"
        rc = self.L.orc_reconfigure(self.h, clauses, clause_tolerance, clause_maximum,
                                    include_bits, float(target), float(specificity))
        if rc != 0:
            raise RuntimeError(self.L.orc_last_error().decode())
        self.info = self._info()

    def restrict(self, dims):
        assert self.which == "oracle"
        d = np.ascontiguousarray(dims, dtype=np.int64)
        rc = self.L.orc_restrict(self.h, _ptr(d, _i64p), len(d))
        if rc != 0:
            raise RuntimeError(self.L.orc_last_error().decode())
        self.info = self._info()


def philox(ctr, key):
    L = lib("oracle")
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    L.orc_philox(_ptr(c, _u32p), key, _ptr(o, _u32p))
    return o


def perm(seed, epoch, n):
    L = lib("oracle")
    o = np.zeros(max(n, 1), dtype=np.uint32)
    L.orc_perm(seed, epoch, n, _ptr(o, _u32p))
    return o[:n]
