"""ctypes bindings to ``libeinfold_b200.so`` (declared in ``include/einfold_b200.h``).

Loading fails loudly when the library is missing: there is no fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libeinfold_b200.so")

# Status codes (einfold_status).
OK, DECLINED, BUDGET, INVALID, COMPUTE, DEVICE, TIMEOUT = range(7)
STATUS_NAMES = {OK: "ok", DECLINED: "declined", BUDGET: "budget", INVALID: "invalid", COMPUTE: "compute",
                DEVICE: "device", TIMEOUT: "timeout"}
ALGORITHMS = {0: None, 1: "dense", 2: "discriminate", 3: "fused"}


class ArrowSchema(ctypes.Structure):
    pass


ArrowSchema._fields_ = [
    ("format", ctypes.c_char_p), ("name", ctypes.c_char_p), ("metadata", ctypes.c_char_p),
    ("flags", ctypes.c_int64), ("n_children", ctypes.c_int64),
    ("children", ctypes.POINTER(ctypes.POINTER(ArrowSchema))), ("dictionary", ctypes.POINTER(ArrowSchema)),
    ("release", ctypes.c_void_p), ("private_data", ctypes.c_void_p)]


class ArrowArray(ctypes.Structure):
    pass


ArrowArray._fields_ = [
    ("length", ctypes.c_int64), ("null_count", ctypes.c_int64), ("offset", ctypes.c_int64),
    ("n_buffers", ctypes.c_int64), ("n_children", ctypes.c_int64),
    ("buffers", ctypes.POINTER(ctypes.c_void_p)), ("children", ctypes.POINTER(ctypes.POINTER(ArrowArray))),
    ("dictionary", ctypes.POINTER(ArrowArray)), ("release", ctypes.c_void_p), ("private_data", ctypes.c_void_p)]


class Key(ctypes.Structure):
    _fields_ = [("dimension", ctypes.c_int32), ("column", ctypes.c_int32)]


class Operand(ctypes.Structure):
    _fields_ = [("n_keys", ctypes.c_int32), ("keys", ctypes.POINTER(Key)), ("factor", ctypes.c_int32)]


class Output(ctypes.Structure):
    _fields_ = [("dimension", ctypes.c_int32), ("domain_column", ctypes.c_int32),
                ("domain_equality", ctypes.c_int32)]


class Condition(ctypes.Structure):
    _fields_ = [("left", ctypes.c_int32), ("comparison", ctypes.c_int32), ("right", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("offset", ctypes.c_int64)]


class Domain(ctypes.Structure):
    _fields_ = [("n_carry", ctypes.c_int32), ("carry", ctypes.POINTER(ctypes.c_int32)),
                ("has_missing", ctypes.c_int32), ("pad", ctypes.c_int32), ("missing", ctypes.c_double)]


class ExprNode(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("a", ctypes.c_int32), ("b", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("value", ctypes.c_double)]


class Expression(ctypes.Structure):
    _fields_ = [("n_nodes", ctypes.c_int32), ("nodes", ctypes.POINTER(ExprNode))]


class FoldDesc(ctypes.Structure):
    _fields_ = [("n_dimensions", ctypes.c_int32), ("equality", ctypes.POINTER(ctypes.c_int32)),
                ("n_operands", ctypes.c_int32), ("operands", ctypes.POINTER(Operand)),
                ("n_outputs", ctypes.c_int32), ("outputs", ctypes.POINTER(Output)),
                ("row_is_expression", ctypes.c_int32), ("row", Expression),
                ("domain", ctypes.POINTER(Domain)),
                ("n_conditions", ctypes.c_int32), ("conditions", ctypes.POINTER(Condition))]


class PipelineDesc(ctypes.Structure):
    _fields_ = [("producer", ctypes.POINTER(FoldDesc)), ("weight_is_expression", ctypes.c_int32),
                ("scale_kind", ctypes.c_int32), ("scale_c", ctypes.c_double), ("shift", ctypes.c_int32),
                ("normalizer", ctypes.c_int32), ("weight", Expression), ("n_dimensions", ctypes.c_int32),
                ("equality", ctypes.POINTER(ctypes.c_int32)), ("values", Operand), ("n_outputs", ctypes.c_int32),
                ("outputs", ctypes.POINTER(ctypes.c_int32))]


class Relation(ctypes.Structure):
    _fields_ = [("schema", ctypes.POINTER(ArrowSchema)), ("n_batches", ctypes.c_int64),
                ("batches", ctypes.POINTER(ctypes.POINTER(ArrowArray))), ("device", ctypes.c_int32),
                ("pad", ctypes.c_int32)]


GROW = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint64)
SHRINK = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_uint64)


class Options(ctypes.Structure):
    _fields_ = [("float_keys", ctypes.c_int32), ("threads", ctypes.c_int32), ("domain_rows", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("slices", ctypes.c_int32), ("result_on_device", ctypes.c_int32),
                ("budget_ctx", ctypes.c_void_p), ("budget_grow", GROW), ("budget_shrink", SHRINK)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("algorithm", ctypes.c_int32), ("n_batches", ctypes.c_int64),
                ("batches", ctypes.POINTER(ArrowArray)), ("schema", ctypes.POINTER(ArrowSchema)),
                ("tiles_visited", ctypes.c_uint64), ("tiles", ctypes.c_uint64),
                ("kernels_launched", ctypes.c_uint64), ("device_ms", ctypes.c_double),
                ("product_ms", ctypes.c_double), ("product_ops", ctypes.c_double),
                ("schedule", ctypes.c_int32), ("graph", ctypes.c_int32),
                ("message", ctypes.c_char * 480)]



class DenseShape(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("pad", ctypes.c_int32), ("batches", ctypes.c_int64),
                ("rows", ctypes.c_int64), ("inner", ctypes.c_int64), ("columns", ctypes.c_int64),
                ("keys", ctypes.c_int64)]


class DenseWork(ctypes.Structure):
    _fields_ = [("shape", DenseShape), ("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("q", ctypes.c_void_p),
                ("kt", ctypes.c_void_p), ("v", ctypes.c_void_p), ("scale_kind", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("scale_c", ctypes.c_double), ("allowed", ctypes.c_void_p),
                ("device", ctypes.c_int32), ("pad2", ctypes.c_int32)]

# Every symbol the header declares, with its signature.
SIGNATURES = {
    "einfold_context_create": (ctypes.c_void_p, [ctypes.c_int32]),
    "einfold_context_destroy": (None, [ctypes.c_void_p]),
    "einfold_last_error": (ctypes.c_char_p, []),
    "einfold_version": (ctypes.c_char_p, []),
    "einfold_fold": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(FoldDesc), ctypes.POINTER(Relation),
                                      ctypes.POINTER(Relation), ctypes.POINTER(Relation), ctypes.POINTER(Options),
                                      ctypes.POINTER(Result)]),
    "einfold_fold_dense": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(FoldDesc), ctypes.POINTER(Relation),
                                            ctypes.POINTER(Relation), ctypes.POINTER(Relation),
                                            ctypes.POINTER(Options), ctypes.POINTER(Result)]),
    "einfold_fold_chain": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(FoldDesc), ctypes.POINTER(Relation),
                                            ctypes.POINTER(Options), ctypes.POINTER(Result)]),
    "einfold_pipeline": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(PipelineDesc), ctypes.POINTER(Relation),
                                          ctypes.POINTER(Options), ctypes.POINTER(Result)]),
    "einfold_pipeline_backward": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(PipelineDesc),
                                                   ctypes.POINTER(Relation), ctypes.POINTER(Relation),
                                                   ctypes.POINTER(Options), ctypes.POINTER(Result)]),
    "einfold_schema": (ctypes.c_int32, [ctypes.POINTER(FoldDesc), ctypes.POINTER(ctypes.POINTER(ArrowSchema)),
                                        ctypes.c_int32, ctypes.POINTER(ArrowSchema), ctypes.POINTER(ArrowSchema),
                                        ctypes.c_char_p, ctypes.c_int32]),
    "einfold_pipeline_schema": (ctypes.c_int32, [ctypes.POINTER(PipelineDesc),
                                                 ctypes.POINTER(ctypes.POINTER(ArrowSchema)),
                                                 ctypes.POINTER(ArrowSchema), ctypes.c_char_p, ctypes.c_int32]),
    "einfold_result_release": (None, [ctypes.POINTER(Result)]),
    "einfold_rank_words": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]),
    "einfold_rank_columns": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(Relation), ctypes.c_int32,
                                              ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.POINTER(ctypes.c_int64)]),
    "einfold_check_wait": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    "einfold_exp_weights": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                             ctypes.c_int32, ctypes.c_void_p]),
    "einfold_evaluate_pairs": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(Expression), ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p]),
    "einfold_backend_may_run": (ctypes.c_int32, [ctypes.POINTER(DenseShape)]),
    "einfold_backend_run": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(DenseWork), ctypes.c_void_p,
                                             ctypes.POINTER(Result)]),
    "einfold_split_gemm": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                            ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    "einfold_split_gemm_static": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                                   ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32,
                                                   ctypes.c_int32, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32]),
    "einfold_attention_forward": (ctypes.c_int32, [ctypes.c_void_p] + [ctypes.c_void_p] * 5 + [ctypes.c_int64] * 5 +
                                  [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int32,
                                   ctypes.c_int32, ctypes.c_void_p, ctypes.POINTER(Result)]),
    "einfold_attention_backward": (ctypes.c_int32, [ctypes.c_void_p] + [ctypes.c_void_p] * 9 + [ctypes.c_int64] * 5 +
                                   [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int32,
                                    ctypes.c_void_p, ctypes.POINTER(Result)]),
    "einfold_attention_forward_ragged": (ctypes.c_int32, [ctypes.c_void_p] + [ctypes.c_void_p] * 5 +
                                         [ctypes.c_int64] * 5 + [ctypes.c_void_p] * 2 +
                                         [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                          ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.POINTER(Result)]),
    "einfold_attention_backward_ragged": (ctypes.c_int32, [ctypes.c_void_p] + [ctypes.c_void_p] * 9 +
                                          [ctypes.c_int64] * 5 + [ctypes.c_void_p] * 2 +
                                          [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                           ctypes.c_int32, ctypes.c_void_p, ctypes.POINTER(Result)]),
    "einfold_fp64_gemm": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                           ctypes.c_int32, ctypes.c_void_p]),
}

_lib = None
_lock = threading.Lock()


def load():
    """The library, loaded once. Raises if it hasn't been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m einfold_b200.build` "
                    "(the kernels have no CPU fallback)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def declared_symbols(header: str) -> list:
    """The function names ``include/einfold_b200.h`` declares."""
    import re
    text = open(header).read()
    return sorted(set(re.findall(r"\b(einfold_[a-z_0-9]+)\s*\(", text)) - {"einfold_status"})


_contexts = {}


def context(device: int = 0) -> int:
    """A shared context (one stream) per device."""
    lib = load()
    with _lock:
        ctx = _contexts.get(device)
        if ctx is None:
            ctx = lib.einfold_context_create(device)
            if not ctx:
                raise RuntimeError("einfold_context_create failed: " + lib.einfold_last_error().decode())
            _contexts[device] = ctx
    return ctx
