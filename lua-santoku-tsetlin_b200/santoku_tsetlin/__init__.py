"""santoku.tsetlin on B200.

A Python mirror of the reference's Lua module `santoku.tsetlin`
(lib/santoku/tsetlin/capi.c:1790-1803 and the methods of capi.c:419-431),
bound with ctypes to the C ABI of libtsetlin_b200.so
(include/tsetlin_b200.h).  Names, table keys, argument order and error
behaviour follow the reference:

    import santoku_tsetlin as tm
    t = tm.create("classifier", {"features": 784, "classes": 10, "clauses": 256,
                                 "clause_tolerance": 64, "clause_maximum": 64,
                                 "specificity": 10, "target": 50})
    t.train({"samples": n, "problems": x, "solutions": y, "iterations": 10})
    yhat = t.predict(x_test, n_test)
    blob = t.persist()
    t2 = tm.load(blob, True)

All computation runs in the CUDA library; there is no CPU path.  Importing
works without a GPU, creating a machine needs one.

Inputs may be numpy arrays, bytes / bytearray, or torch tensors; CUDA
tensors are passed to the library as device pointers.
"""
import ctypes
import os
import sys

import numpy as np

from . import datagen  # noqa: F401  (workload generators)

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "libtsetlin_b200.so")

align = 8

CLASSIFIER = 0
ENCODER = 1
SAVE_STATE = 1  # tm_save flag: include the count planes


class TsetlinError(RuntimeError):
    """Raised where the reference raises a Lua error."""


class _Params(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int32),
        ("classes", ctypes.c_uint32),
        ("features", ctypes.c_uint32),
        ("clauses", ctypes.c_uint32),
        ("clause_tolerance", ctypes.c_uint32),
        ("clause_maximum", ctypes.c_uint32),
        ("state_bits", ctypes.c_uint32),
        ("include_bits", ctypes.c_uint32),
        ("target", ctypes.c_double),
        ("negative", ctypes.c_double),
        ("specificity", ctypes.c_double),
        ("reusable", ctypes.c_int32),
        ("individualized", ctypes.c_int32),
        ("feat_offsets", ctypes.POINTER(ctypes.c_int64)),
        ("seed", ctypes.c_uint64),
        ("device", ctypes.c_int32),
    ]


EPOCH_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32)
SEARCH_EPOCH_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32,
                                   ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_int32),
                                   ctypes.POINTER(ctypes.c_int32), ctypes.c_uint32)
METRICS = {"f1": 0, "accuracy": 1, "mean_hamming": 2}
BATCH_EPOCH_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32,
                                  ctypes.POINTER(ctypes.c_int32), ctypes.c_uint32)


class _TrainArgs(ctypes.Structure):
    _fields_ = [
        ("samples", ctypes.c_uint64),
        ("problems", ctypes.c_void_p),
        ("solutions", ctypes.c_void_p),
        ("codes", ctypes.c_void_p),
        ("dim_offsets", ctypes.c_void_p),
        ("iterations", ctypes.c_uint32),
        ("each", EPOCH_CB),
        ("each_user", ctypes.c_void_p),
        ("on_device", ctypes.c_int32),
        ("has_seed", ctypes.c_int32),
        ("seed", ctypes.c_uint64),
        ("class_begin", ctypes.c_uint32),
        ("class_end", ctypes.c_uint32),
    ]


class _Reconfig(ctypes.Structure):
    _fields_ = [
        ("clauses", ctypes.c_uint32),
        ("clause_tolerance", ctypes.c_uint32),
        ("clause_maximum", ctypes.c_uint32),
        ("include_bits", ctypes.c_int64),
        ("target", ctypes.c_double),
        ("specificity", ctypes.c_double),
    ]


class _SearchArgs(ctypes.Structure):
    _fields_ = [
        ("test_samples", ctypes.c_uint64),
        ("test_problems", ctypes.c_void_p),
        ("test_solutions", ctypes.c_void_p),
        ("test_codes", ctypes.c_void_p),
        ("test_dim_offsets", ctypes.c_void_p),
        ("test_each", ctypes.c_void_p),
        ("on_device", ctypes.c_int32),
        ("metric", ctypes.c_int32),
        ("patience", ctypes.c_uint32),
        ("tolerance", ctypes.c_double),
        ("each", SEARCH_EPOCH_CB),
        ("each_user", ctypes.c_void_p),
        ("scores", ctypes.c_void_p),
        ("final_scores", ctypes.c_void_p),
        ("best_scores", ctypes.c_void_p),
        ("epochs_run", ctypes.c_void_p),
        ("best_epochs", ctypes.c_void_p),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("train_launches", ctypes.c_uint64),
        ("train_kernel_ms", ctypes.c_double),
        ("predict_launches", ctypes.c_uint64),
        ("predict_kernel_ms", ctypes.c_double),
        ("kernel_launches", ctypes.c_uint64),
        ("train_unit_steps", ctypes.c_uint64),
        ("train_mode", ctypes.c_int32),
        ("train_autotuned", ctypes.c_int32),
        ("train_cpw", ctypes.c_int32),
        ("predict_gemm", ctypes.c_int32),
        ("train_active_pairs", ctypes.c_uint64),
        ("search_epoch_ms", ctypes.c_double),
        ("search_epochs", ctypes.c_uint64),
        ("search_train_ms", ctypes.c_double),
        ("train_resident", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class _ServerConfig(ctypes.Structure):
    _fields_ = [
        ("hbm_budget_bytes", ctypes.c_uint64),
        ("max_inflight", ctypes.c_uint32),
        ("max_batch_samples", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("max_queued_samples", ctypes.c_uint64),
    ]


_lib = None
EXPORTS = (
    "tm_params_init", "tm_create", "tm_train", "tm_train_batch", "tm_train_batch_each",
    "tm_train_batch_search",
    "tm_predict",
    "tm_predict_scores", "tm_persist", "tm_persist_buf", "tm_save", "tm_save_buf", "tm_free",
    "tm_load",
    "tm_checkpoint", "tm_restore", "tm_reconfigure", "tm_restrict", "tm_type",
    "tm_destroy", "tm_last_error", "tm_align", "tm_get_info", "tm_export_state",
    "tm_import_state", "tm_export_classes", "tm_import_classes", "tm_class_accuracy", "tm_encoding_accuracy", "tm_bits_to_cvec", "tm_bits_to_cvec_ind",
    "tm_predict_noalloc", "tm_int_peaks", "tm_debug_fail_alloc", "tm_set_autotune", "tm_force_variant", "tm_stats_enable", "tm_get_stats", "tm_reset_stats", "tm_serve_open", "tm_serve_submit", "tm_serve_poll",
    "tm_serve_latency_us", "tm_serve_phases_us", "tm_serve_stats", "tm_serve_close",
)


def lib():
    """The loaded CUDA library.  Fails loudly when it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise TsetlinError(
            "libtsetlin_b200.so is not built (run `make -C lua-santoku-tsetlin_b200/csrc`)")
    L = ctypes.CDLL(LIB_PATH)
    vp, u64, u32, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int32
    L.tm_params_init.argtypes = [ctypes.POINTER(_Params)]
    L.tm_create.argtypes = [ctypes.POINTER(_Params), ctypes.POINTER(vp)]
    L.tm_train.argtypes = [vp, ctypes.POINTER(_TrainArgs)]
    L.tm_train_batch.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(_TrainArgs), u32]
    L.tm_train_batch_each.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(_TrainArgs), u32,
                                      BATCH_EPOCH_CB, vp]
    L.tm_train_batch_search.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(_TrainArgs), u32,
                                        ctypes.POINTER(_SearchArgs)]
    L.tm_predict.argtypes = [vp, vp, vp, u64, vp, vp, i32]
    L.tm_predict_scores.argtypes = [vp, vp, vp, u64, vp, i32]
    L.tm_persist.argtypes = [vp, ctypes.c_char_p]
    L.tm_persist_buf.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(u64)]
    L.tm_save.argtypes = [vp, ctypes.c_char_p, u32]
    L.tm_save_buf.argtypes = [vp, u32, ctypes.POINTER(vp), ctypes.POINTER(u64)]
    L.tm_free.argtypes = [vp]
    L.tm_load.argtypes = [vp, u64, i32, i32, ctypes.POINTER(vp)]
    L.tm_checkpoint.argtypes = [vp, vp, u64, ctypes.POINTER(u64)]
    L.tm_restore.argtypes = [vp, vp, u64]
    L.tm_reconfigure.argtypes = [vp, ctypes.POINTER(_Reconfig)]
    L.tm_restrict.argtypes = [vp, vp, u64]
    L.tm_type.argtypes = [vp]
    L.tm_destroy.argtypes = [vp]
    L.tm_destroy.restype = None
    L.tm_last_error.restype = ctypes.c_char_p
    L.tm_align.restype = u32
    L.tm_get_info.argtypes = [vp, vp]
    L.tm_export_state.argtypes = [vp, vp, vp]
    L.tm_import_state.argtypes = [vp, vp, vp]
    L.tm_export_classes.argtypes = [vp, u32, u32, vp, vp, i32]
    L.tm_import_classes.argtypes = [vp, u32, u32, vp, vp, i32]
    L.tm_predict_noalloc.argtypes = [vp, vp, u64, vp, vp]
    L.tm_int_peaks.argtypes = [i32, vp]
    L.tm_debug_fail_alloc.argtypes = [ctypes.c_int64]
    L.tm_set_autotune.argtypes = [vp, i32]
    L.tm_force_variant.argtypes = [vp, i32, i32]
    L.tm_class_accuracy.argtypes = [vp, vp, u64, u32, i32, i32, vp]
    L.tm_encoding_accuracy.argtypes = [vp, vp, u64, u32, i32, i32, vp]
    L.tm_bits_to_cvec.argtypes = [vp, u64, u64, u32, i32, i32, i32, vp]
    L.tm_bits_to_cvec_ind.argtypes = [vp, vp, vp, u32, u64, i32, i32, i32, vp, u64, vp]
    L.tm_stats_enable.argtypes = [vp, i32]
    L.tm_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    L.tm_reset_stats.argtypes = [vp]
    L.tm_serve_open.argtypes = [ctypes.POINTER(_ServerConfig), ctypes.POINTER(vp), u32,
                                ctypes.POINTER(vp)]
    L.tm_serve_submit.argtypes = [vp, u32, vp, u64, ctypes.POINTER(u64)]
    L.tm_serve_poll.argtypes = [vp, u64, vp, vp, u64]
    L.tm_serve_latency_us.argtypes = [vp, u64, ctypes.POINTER(ctypes.c_double)]
    L.tm_serve_phases_us.argtypes = [vp, u64, ctypes.POINTER(ctypes.c_double)]
    L.tm_serve_stats.argtypes = [vp, vp]
    L.tm_serve_close.argtypes = [vp]
    _lib = L
    return L


def _check(rc):
    if rc < 0:
        raise TsetlinError(lib().tm_last_error().decode())
    return rc


# ---------------------------------------------------------------------------
# buffers
# ---------------------------------------------------------------------------
class _Buf:
    """A pointer to caller data (kept alive), host or device."""

    def __init__(self, obj, dtype):
        self.keep = obj
        self.device = False
        if obj is None:
            self.ptr = None
            self.nbytes = 0
            return
        mod = type(obj).__module__
        if mod.startswith("torch"):
            t = obj.contiguous()
            self.keep = t
            self.device = bool(t.is_cuda)
            self.ptr = t.data_ptr()
            self.nbytes = t.numel() * t.element_size()
            return
        if isinstance(obj, (bytes, bytearray, memoryview)):
            a = np.frombuffer(obj, dtype=np.uint8)
            if dtype != np.uint8:
                a = a.view(dtype)
        else:
            a = np.ascontiguousarray(obj)
            if a.dtype != dtype:
                a = a.astype(dtype)
        self.keep = a
        self.ptr = a.ctypes.data if a.size else None
        self.nbytes = a.nbytes


def _opt(tbl, key, default):
    v = tbl.get(key, None) if tbl is not None else None
    return default if v is None else v


# ---------------------------------------------------------------------------
# machine
# ---------------------------------------------------------------------------
INFO_KEYS = ("type", "classes", "features", "clauses", "clause_tolerance",
             "clause_maximum", "target", "state_bits", "include_bits",
             "input_bits", "input_chunks", "clause_chunks", "class_chunks",
             "state_chunks", "action_chunks", "tail_mask", "individualized",
             "reusable", "has_state")


class Machine:
    """A Tsetlin machine resident on one GPU (the reference's userdata,
    metatable "santoku_tsetlin", capi.c:39, 419-431)."""

    def __init__(self, handle, device=0):
        self._h = ctypes.c_void_p(handle)
        self.device = device

    # -- bookkeeping -------------------------------------------------------
    @property
    def handle(self):
        if not self._h:
            raise TsetlinError("machine destroyed")
        return self._h

    def info(self):
        o = np.zeros(19, dtype=np.uint64)
        _check(lib().tm_get_info(self.handle, o.ctypes.data))
        return {k: int(v) for k, v in zip(INFO_KEYS, o)}

    def type(self):
        """capi.c:1774-1788"""
        return "classifier" if _check(lib().tm_type(self.handle)) == CLASSIFIER else "encoder"

    def destroy(self):
        """capi.c:744-750"""
        if self._h:
            lib().tm_destroy(self._h)
            self._h = ctypes.c_void_p(None)

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # -- train -------------------------------------------------------------
    def _train_args(self, tbl):
        info = self.info()
        n = int(tbl["samples"])
        if info["type"] == CLASSIFIER:
            prob = _Buf(tbl["problems"], np.uint8)
            sol = _Buf(tbl["solutions"], np.int64)
            cod = _Buf(None, np.uint8)
        else:
            prob = _Buf(tbl["sentences"], np.uint8)
            cod = _Buf(tbl["codes"], np.uint8)
            sol = _Buf(None, np.int64)
        dof = _Buf(tbl.get("dim_offsets"), np.int64)
        if dof.device:
            raise TsetlinError("dim_offsets must be host memory")
        a = _TrainArgs()
        a.samples = n
        a.problems = prob.ptr
        a.solutions = sol.ptr
        a.codes = cod.ptr
        a.dim_offsets = dof.ptr
        a.iterations = int(tbl["iterations"])
        a.on_device = 1 if prob.device else 0
        if prob.device and ((sol.keep is not None and not sol.device) or
                            (cod.keep is not None and not cod.device)):
            raise TsetlinError("problems and labels must both be host or both device memory")
        if "seed" in tbl and tbl["seed"] is not None:
            a.has_seed = 1
            a.seed = int(tbl["seed"])
        if tbl.get("class_range") is not None:
            # train only these classes' units (multi.train_sharded)
            a.class_begin, a.class_end = (int(v) for v in tbl["class_range"])
        return a, (prob, sol, cod, dof)

    def train(self, tbl):
        """capi.c:1484-1507.  `each(epoch)` returning False stops training;
        an exception in `each` is reported on stderr and stops training, as
        the reference does with a Lua error (capi.c:1171-1175)."""
        a, keep = self._train_args(tbl)
        each = tbl.get("each")
        cb = None
        if each is not None:
            def _cb(_user, epoch):
                try:
                    r = each(int(epoch))
                except Exception as e:  # noqa: BLE001
                    sys.stderr.write("Error in callback: %s\n" % (e,))
                    return 1
                return 1 if r is False else 0
            cb = EPOCH_CB(_cb)
            a.each = cb
        _check(lib().tm_train(self.handle, ctypes.byref(a)))
        del keep, cb

    # -- predict -----------------------------------------------------------
    def predict(self, problems, *args):
        """predict(problems, n) or, individualized, predict(problems,
        dim_offsets, n) (capi.c:1088-1110).  Classifier: int64 class per
        sample.  Encoder: uint8 codes, ceil(hidden/8) bytes per sample."""
        dof, n = (None, args[0]) if len(args) == 1 else (args[0], args[1])
        n = int(n)
        info = self.info()
        x = _Buf(problems, np.uint8)
        d = _Buf(dof, np.int64)
        if x.device:
            import torch
            dev = torch.device("cuda", self.device)
            if info["type"] == CLASSIFIER:
                out = torch.empty(n, dtype=torch.int64, device=dev)
                _check(lib().tm_predict(self.handle, x.ptr, d.ptr, n, out.data_ptr(), None, 1))
            else:
                out = torch.empty(n * info["class_chunks"], dtype=torch.uint8, device=dev)
                _check(lib().tm_predict(self.handle, x.ptr, d.ptr, n, None, out.data_ptr(), 1))
            return out
        if info["type"] == CLASSIFIER:
            out = np.zeros(n, dtype=np.int64)
            _check(lib().tm_predict(self.handle, x.ptr, d.ptr, n, out.ctypes.data, None, 0))
        else:
            out = np.zeros(n * info["class_chunks"], dtype=np.uint8)
            _check(lib().tm_predict(self.handle, x.ptr, d.ptr, n, None, out.ctypes.data, 0))
        return out

    def predict_scores(self, problems, *args):
        """Per-class vote sums (int64, n x classes) behind predict."""
        dof, n = (None, args[0]) if len(args) == 1 else (args[0], args[1])
        n = int(n)
        C = self.info()["classes"]
        x = _Buf(problems, np.uint8)
        d = _Buf(dof, np.int64)
        out = np.zeros((n, C), dtype=np.int64)
        if x.device:
            raise TsetlinError("predict_scores takes host inputs")
        _check(lib().tm_predict_scores(self.handle, x.ptr, d.ptr, n, out.ctypes.data, 0))
        return out

    # -- persistence -------------------------------------------------------
    def persist(self, path=None):
        """capi.c:1538-1562: writes `path`, or returns the bytes."""
        if path is not None:
            _check(lib().tm_persist(self.handle, os.fsencode(path)))
            return None
        p = ctypes.c_void_p()
        n = ctypes.c_uint64()
        _check(lib().tm_persist_buf(self.handle, ctypes.byref(p), ctypes.byref(n)))
        try:
            return ctypes.string_at(p, n.value)
        finally:
            lib().tm_free(p)

    def save(self, path=None, state=True):
        """Versioned container (no counterpart in the reference): the
        reference's persisted record plus `negative`, the default seed, the
        reusable flag and, with `state`, the count planes, under a format
        version and a checksum.  `load` reads it back; a machine saved with
        its state can train again.  Writes `path`, or returns the bytes."""
        flags = SAVE_STATE if state else 0
        if path is not None:
            _check(lib().tm_save(self.handle, os.fsencode(path), flags))
            return None
        p = ctypes.c_void_p()
        n = ctypes.c_uint64()
        _check(lib().tm_save_buf(self.handle, flags, ctypes.byref(p), ctypes.byref(n)))
        try:
            return ctypes.string_at(p, n.value)
        finally:
            lib().tm_free(p)

    def checkpoint(self, buf=None):
        """capi.c:1564-1576: the action bytes.  Fills a bytearray in place
        when one is given, else returns a new one."""
        n = ctypes.c_uint64()
        _check(lib().tm_checkpoint(self.handle, None, 0, ctypes.byref(n)))
        if buf is None:
            buf = bytearray(n.value)
        elif len(buf) != n.value:
            buf[:] = bytes(n.value)
        a = (ctypes.c_uint8 * n.value).from_buffer(buf) if n.value else None
        _check(lib().tm_checkpoint(self.handle, a, n.value, ctypes.byref(n)))
        return buf

    def restore(self, buf):
        """capi.c:1578-1588"""
        b = _Buf(bytes(buf), np.uint8)
        _check(lib().tm_restore(self.handle, b.ptr, b.nbytes))

    def reconfigure(self, tbl):
        """capi.c:1590-1673"""
        r = _Reconfig()
        for k in ("clauses", "clause_tolerance", "clause_maximum", "specificity"):
            if tbl.get(k) is None:
                raise TsetlinError("reconfigure: %s is required" % k)
        r.clauses = int(tbl["clauses"])
        r.clause_tolerance = int(tbl["clause_tolerance"])
        r.clause_maximum = int(tbl["clause_maximum"])
        r.include_bits = int(_opt(tbl, "include_bits", -1))
        r.target = float(_opt(tbl, "target", -1.0))
        r.specificity = float(tbl["specificity"])
        _check(lib().tm_reconfigure(self.handle, ctypes.byref(r)))

    def restrict(self, dims):
        """capi.c:752-901"""
        d = _Buf(dims, np.int64)
        _check(lib().tm_restrict(self.handle, d.ptr, d.nbytes // 8))

    # -- instrumentation ---------------------------------------------------
    def stats_enable(self, on=True):
        _check(lib().tm_stats_enable(self.handle, 1 if on else 0))

    def set_autotune(self, mode=1):
        """Train-kernel variant choice: 0 heuristic, 1 tuned once per launch
        shape (default), 2 tuned on every train call.  Results are the same
        in every mode."""
        _check(lib().tm_set_autotune(self.handle, int(mode)))

    def force_variant(self, mode=-1, cpw=1):
        """Pin the train-kernel variant (0 shared planes, 1 global planes,
        2 cluster pair, 3 warp per unit; cpw clauses per warp); -1 returns
        to the automatic choice."""
        _check(lib().tm_force_variant(self.handle, int(mode), int(cpw)))

    def stats(self):
        st = Stats()
        _check(lib().tm_get_stats(self.handle, ctypes.byref(st)))
        return st.as_dict()

    def reset_stats(self):
        _check(lib().tm_reset_stats(self.handle))

    # -- raw state (reference byte layouts) --------------------------------
    def export_state(self):
        info = self.info()
        a = np.zeros(info["action_chunks"], dtype=np.uint8)
        s = np.zeros(info["state_chunks"], dtype=np.uint8) if info["has_state"] else None
        _check(lib().tm_export_state(self.handle, a.ctypes.data,
                                     None if s is None else s.ctypes.data))
        return a, s

    def import_state(self, actions=None, state=None):
        a = _Buf(actions, np.uint8)
        s = _Buf(state, np.uint8)
        _check(lib().tm_import_state(self.handle, a.ptr, s.ptr))

    def class_bytes(self, lo, hi):
        """Bytes of classes [lo, hi) in the action and count-plane layouts
        of export_state."""
        info = self.info()
        per = info["action_chunks"] // max(1, info["classes"])
        if info["individualized"]:
            raise TsetlinError("class_bytes: individualized machines have uneven class blocks")
        a = (hi - lo) * per
        return a, a * (info["state_bits"] - 1)

    def export_classes(self, lo, hi, out):
        """Copy classes [lo, hi) (actions, then count planes) into `out`, a
        uint8 buffer of sum(class_bytes(lo, hi)) bytes: a CUDA tensor on this
        machine's device (copied on the device) or host memory."""
        a, s = self.class_bytes(lo, hi)
        b = _Buf(out, np.uint8)
        if b.nbytes < a + s:
            raise TsetlinError("export_classes: buffer too small")
        base = b.ptr or 0
        _check(lib().tm_export_classes(self.handle, lo, hi, base if a else None,
                                       base + a if s else None, 1 if b.device else 0))
        return out

    def import_classes(self, lo, hi, buf):
        """Inverse of export_classes."""
        a, s = self.class_bytes(lo, hi)
        b = _Buf(buf, np.uint8)
        if b.nbytes < a + s:
            raise TsetlinError("import_classes: buffer too small")
        base = b.ptr or 0
        _check(lib().tm_import_classes(self.handle, lo, hi, base if a else None,
                                       base + a if s else None, 1 if b.device else 0))


def _params(type_, tbl):
    p = _Params()
    lib().tm_params_init(ctypes.byref(p))
    if type_ == "classifier":
        p.type = CLASSIFIER
        p.classes = int(tbl["classes"])
        p.features = int(_opt(tbl, "features", 0))
    elif type_ == "encoder":
        p.type = ENCODER
        p.classes = int(tbl["hidden"])
        p.features = int(_opt(tbl, "visible", 0))
    else:
        raise TsetlinError("unexpected tsetlin machine type in create")
    for k in ("clauses", "clause_tolerance", "clause_maximum", "specificity"):
        if tbl.get(k) is None:
            raise TsetlinError("create %s: %s is required" % (type_, k))
    p.clauses = int(tbl["clauses"])
    p.clause_tolerance = int(tbl["clause_tolerance"])
    p.clause_maximum = int(tbl["clause_maximum"])
    p.state_bits = int(_opt(tbl, "state", 8))
    p.include_bits = int(_opt(tbl, "include_bits", 1))
    p.target = float(_opt(tbl, "target", -1.0))
    p.negative = float(_opt(tbl, "negative", -1.0))
    p.specificity = float(tbl["specificity"])
    p.reusable = 1 if tbl.get("reusable") else 0
    p.individualized = 1 if tbl.get("individualized") else 0
    keep = None
    if p.individualized:
        fo = np.ascontiguousarray(tbl["feat_offsets"], dtype=np.int64)
        if len(fo) != p.classes + 1:
            raise TsetlinError("create %s: feat_offsets must have classes + 1 elements" % type_)
        keep = fo
        p.feat_offsets = fo.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    p.seed = int(_opt(tbl, "seed", 0))
    p.device = int(_opt(tbl, "device", 0))
    return p, keep


def create(type_, tbl):
    """tsetlin.create("classifier"|"encoder", tbl) (capi.c:701-716)."""
    p, keep = _params(type_, tbl)
    h = ctypes.c_void_p()
    _check(lib().tm_create(ctypes.byref(p), ctypes.byref(h)))
    del keep
    return Machine(h.value, p.device)


def classifier(tbl):
    return create("classifier", tbl)


def encoder(tbl):
    return create("encoder", tbl)


def load(data, from_string=False, device=0):
    """tsetlin.load(path) / tsetlin.load(data, true) (capi.c:1751-1772)."""
    h = ctypes.c_void_p()
    if from_string:
        b = bytes(data)
        _check(lib().tm_load(b, len(b), 1, device, ctypes.byref(h)))
    else:
        _check(lib().tm_load(os.fsencode(data), 0, 0, device, ctypes.byref(h)))
    return Machine(h.value, device)


def train_batch(machines, tbls, each=None):
    """Train many machines in one persistent launch; each ends exactly as
    its own train(tbl) would leave it.  With `each(epoch)`: called after
    every epoch; return False to stop all, or a sequence of per-machine
    flags (true = stop that machine), or None to continue."""
    if len(machines) != len(tbls):
        raise TsetlinError("train_batch: one table per machine")
    arr = (_TrainArgs * len(tbls))()
    keeps = []
    for i, (m, t) in enumerate(zip(machines, tbls)):
        if t.get("each") is not None:
            raise TsetlinError("train_batch: per-epoch callbacks are not supported")
        a, keep = m._train_args(t)
        arr[i] = a
        keeps.append(keep)
    hs = (ctypes.c_void_p * len(machines))(*[m.handle.value for m in machines])
    if each is None:
        _check(lib().tm_train_batch(hs, arr, len(machines)))
    else:
        def _cb(_user, epoch, stop, count):
            try:
                r = each(int(epoch))
            except Exception as e:  # noqa: BLE001
                sys.stderr.write("Error in callback: %s\n" % (e,))
                return 1
            if r is False:
                return 1
            if r is not None:
                for i, flag in enumerate(r):
                    if i < count and flag:
                        stop[i] = 1
            return 0
        cb = BATCH_EPOCH_CB(_cb)
        _check(lib().tm_train_batch_each(hs, arr, len(machines), cb, None))
        del cb
    del keeps


def train_batch_search(machines, tbls, test, patience=0, tolerance=1e-8, metric=None,
                       each=None):
    """One device-resident round of the reference's search
    (optimize.lua:424-471 with train_tm's epoch logic, :586-653): every
    machine trains on its table, is scored on `test` after each epoch on the
    GPU (metric "f1" -- evaluator.class_accuracy(...).f1, the reference's
    usual search_metric --, "accuracy", or "mean_hamming" for encoders),
    keeps a checkpoint of its best epoch when patience > 0, stops after
    `patience` epochs without improving by more than `tolerance`, and ends
    restored to its best checkpoint.  One CUDA graph replay per epoch.
    `test`: {"samples", "problems", "solutions"} or {"samples", "sentences",
    "codes"} (+ "dim_offsets"); "problems_each" (one holdout per machine, for
    machines whose literal layouts differ) replaces "problems".
    `each(epoch, scores, training)` may return False (stop all) or
    per-machine stop flags.  Returns per-machine numpy arrays: scores
    [machines, epochs] (NaN where untrained), final, best, epochs,
    best_epoch."""
    if len(machines) != len(tbls):
        raise TsetlinError("train_batch_search: one table per machine")
    count = len(machines)
    if count == 0:
        return {}
    arr = (_TrainArgs * count)()
    keeps = []
    for i, (m, t) in enumerate(zip(machines, tbls)):
        if t.get("each") is not None:
            raise TsetlinError("train_batch_search: per-epoch callbacks go in `each`")
        a, keep = m._train_args(t)
        arr[i] = a
        keeps.append(keep)
    enc = machines[0].info()["type"] == ENCODER
    if metric is None:
        metric = "mean_hamming" if enc else "f1"
    if metric not in METRICS:
        raise TsetlinError("train_batch_search: metric is one of %s" % sorted(METRICS))
    n = int(test["samples"])
    each_x = test.get("problems_each")
    x = _Buf(test.get("sentences" if enc else "problems"), np.uint8)
    xs = [_Buf(v, np.uint8) for v in each_x] if each_x is not None else []
    if each_x is not None and len(xs) != count:
        raise TsetlinError("train_batch_search: one holdout per machine in problems_each")
    truth = _Buf(test["codes"], np.uint8) if enc else _Buf(test["solutions"], np.int64)
    dof = _Buf(test.get("dim_offsets"), np.int64)
    on_dev = xs[0].device if xs else x.device
    if on_dev != truth.device or any(b.device != on_dev for b in xs):
        raise TsetlinError("train_batch_search: test inputs on different devices")
    tx_arr = (ctypes.c_void_p * count)(*[b.ptr for b in xs]) if xs else None
    E = max(int(t["iterations"]) for t in tbls)
    out = {"scores": np.full((count, max(E, 1)), np.nan), "final": np.zeros(count),
           "best": np.zeros(count), "epochs": np.zeros(count, dtype=np.uint32),
           "best_epoch": np.zeros(count, dtype=np.uint32)}
    sa = _SearchArgs()
    sa.test_samples = n
    sa.test_problems = x.ptr
    sa.test_solutions = None if enc else truth.ptr
    sa.test_codes = truth.ptr if enc else None
    sa.test_dim_offsets = dof.ptr
    sa.test_each = ctypes.cast(tx_arr, ctypes.c_void_p) if tx_arr is not None else None
    sa.on_device = 1 if on_dev else 0
    sa.metric = METRICS[metric]
    sa.patience = int(patience or 0)
    sa.tolerance = float(tolerance)
    sa.scores = out["scores"].ctypes.data
    sa.final_scores = out["final"].ctypes.data
    sa.best_scores = out["best"].ctypes.data
    sa.epochs_run = out["epochs"].ctypes.data
    sa.best_epochs = out["best_epoch"].ctypes.data
    cb = None
    if each is not None:
        def _cb(_user, epoch, scores, training, stop, cnt):
            try:
                sc = np.ctypeslib.as_array(scores, shape=(cnt,)).copy()
                tr = np.ctypeslib.as_array(training, shape=(cnt,)).astype(bool)
                r = each(int(epoch), sc, tr)
            except Exception as e:  # noqa: BLE001
                sys.stderr.write("Error in callback: %s\n" % (e,))
                return 1
            if r is False:
                return 1
            if r is not None:
                for i, flag in enumerate(r):
                    if i < cnt and flag:
                        stop[i] = 1
            return 0
        cb = SEARCH_EPOCH_CB(_cb)
        sa.each = cb
    hs = (ctypes.c_void_p * count)(*[m.handle.value for m in machines])
    _check(lib().tm_train_batch_search(hs, arr, count, ctypes.byref(sa)))
    del keeps, cb, xs, tx_arr
    if E:
        out["scores"] = out["scores"][:, :E]
    return out


# ---------------------------------------------------------------------------
# evaluator metrics (santoku.tsetlin.evaluator) and input packing
# ---------------------------------------------------------------------------
def class_accuracy(predicted, expected, n_samples, n_classes, device=0):
    """evaluator.class_accuracy (evaluator/capi.c:119-202), counted on the
    GPU: {"classes": [{"precision", "recall", "f1"}, ...], "precision",
    "recall", "f1"} (macro averages)."""
    p = _Buf(predicted, np.int64)
    e = _Buf(expected, np.int64)
    if p.device != e.device:
        raise TsetlinError("class_accuracy: predicted and expected on different devices")
    out = np.zeros(3 + 3 * int(n_classes), dtype=np.float64)
    _check(lib().tm_class_accuracy(p.ptr, e.ptr, int(n_samples), int(n_classes),
                                   1 if p.device else 0, device, out.ctypes.data))
    per = out[3:].reshape(-1, 3)
    return {"classes": [{"precision": float(a), "recall": float(b), "f1": float(c)}
                        for a, b, c in per],
            "precision": float(out[0]), "recall": float(out[1]), "f1": float(out[2])}


def encoding_accuracy(predicted, expected, n_samples, n_hidden, device=0):
    """evaluator.encoding_accuracy (evaluator/capi.c:497-574), counted on the
    GPU: {"bits": [...], "mean_hamming", "ber_min", "ber_max", "ber_std"}."""
    p = _Buf(predicted, np.uint8)
    e = _Buf(expected, np.uint8)
    if p.device != e.device:
        raise TsetlinError("encoding_accuracy: predicted and expected on different devices")
    out = np.zeros(4 + int(n_hidden), dtype=np.float64)
    _check(lib().tm_encoding_accuracy(p.ptr, e.ptr, int(n_samples), int(n_hidden),
                                      1 if p.device else 0, device, out.ctypes.data))
    return {"bits": [float(v) for v in out[4:]], "mean_hamming": float(out[0]),
            "ber_min": float(out[1]), "ber_max": float(out[2]), "ber_std": float(out[3])}


def int_peaks(device=0):
    """Measured integer-pipe peaks of the GPU (thread-operations/s):
    {"lop3": .., "popc": .., "iadd": ..}."""
    o = np.zeros(3, dtype=np.float64)
    _check(lib().tm_int_peaks(int(device), o.ctypes.data))
    return {"lop3": float(o[0]), "popc": float(o[1]), "iadd": float(o[2])}


def bits_to_cvec(set_bits, n_samples, n_features, flip=False, device=0):
    """santoku-matrix's bits_to_cvec on the GPU: set-bit list (sample *
    n_features + feature) -> packed rows, flip-interleaved when `flip`."""
    b = _Buf(set_bits, np.int64)
    nb = ((2 if flip else 1) * int(n_features) + 7) // 8
    if b.device:
        import torch
        out = torch.empty(int(n_samples) * nb, dtype=torch.uint8,
                          device=torch.device("cuda", device))
        _check(lib().tm_bits_to_cvec(b.ptr, b.nbytes // 8, int(n_samples), int(n_features),
                                     1 if flip else 0, 1, device, out.data_ptr()))
        return out
    out = np.zeros(int(n_samples) * nb, dtype=np.uint8)
    _check(lib().tm_bits_to_cvec(b.ptr, b.nbytes // 8, int(n_samples), int(n_features),
                                 1 if flip else 0, 0, device, out.ctypes.data))
    return out


def bits_to_cvec_ind(set_bits, ind_offsets, feat_offsets, n_samples, flip=False, device=0):
    """santoku-matrix's bits_to_cvec_ind on the GPU: per-dimension set-bit
    lists (dimension h: set_bits[ind_offsets[h]:ind_offsets[h+1]], entries
    sample * k_h + feature) -> (bitmap, dim_offsets), the individualized
    layout `train` / `predict` take with `dim_offsets` (capi.c:1344-1354).
    dim_offsets has one entry per dimension plus the total size."""
    io = np.ascontiguousarray(ind_offsets, dtype=np.int64)
    fo = np.ascontiguousarray(feat_offsets, dtype=np.int64)
    if io.ndim != 1 or fo.ndim != 1 or len(io) != len(fo) or len(io) < 2:
        raise TsetlinError("ind_offsets and feat_offsets need dims + 1 entries each")
    dims = len(fo) - 1
    b = _Buf(set_bits, np.int64)
    if b.nbytes // 8 < int(io[-1] - io[0]):
        raise TsetlinError("set_bits is shorter than ind_offsets says")
    doff = np.zeros(dims + 1, dtype=np.int64)
    L = lib()
    _check(L.tm_bits_to_cvec_ind(None, io.ctypes.data, fo.ctypes.data, dims, int(n_samples),
                                 1 if flip else 0, 0, device, None, 0, doff.ctypes.data))
    total = int(doff[-1])
    if b.device:
        import torch
        out = torch.empty(max(total, 1), dtype=torch.uint8, device=torch.device("cuda", device))
        _check(L.tm_bits_to_cvec_ind(b.ptr, io.ctypes.data, fo.ctypes.data, dims,
                                     int(n_samples), 1 if flip else 0, 1, device,
                                     out.data_ptr(), total, doff.ctypes.data))
        return out[:total], doff
    out = np.zeros(max(total, 1), dtype=np.uint8)
    _check(L.tm_bits_to_cvec_ind(b.ptr, io.ctypes.data, fo.ctypes.data, dims, int(n_samples),
                                 1 if flip else 0, 0, device, out.ctypes.data, total,
                                 doff.ctypes.data))
    return out[:total], doff
