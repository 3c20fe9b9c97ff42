"""einfold's kernel layer on a B200: the Python face of the C ABI.

The functions mirror ``einfold_kernels`` (``crates/einfold-kernels/src/lib.rs:43-48``)
name for name: :func:`fold`, :func:`fold_dense`, :func:`fold_chain`,
:func:`pipeline`, :func:`schema`, :func:`pipeline_schema`, with :class:`Options`,
:class:`Budget`, :class:`Host`, :class:`FloatKeys`, :class:`DomainRows`,
:class:`Relation`, :class:`Folded`, :class:`Piped` and :class:`Algorithm`.
Relations are pyarrow record batches; they cross into the library through the
Arrow C Data Interface, and every computation runs on the GPU. Where the
reference returns ``Ok(None)`` (the caller runs the host's plan) these return
``None``; its ``ArrowError`` variants are the exceptions below.
"""
from __future__ import annotations

import ctypes
import enum
import threading
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import pyarrow as pa

from . import _lib, ir


class ArrowMemoryError(MemoryError):
    """``ArrowError::MemoryError``: the budget refused (``options.rs:101-108``)."""


class ArrowInvalidArgumentError(ValueError):
    """``ArrowError::InvalidArgumentError`` (``lib.rs:54-56``)."""


class ArrowComputeError(RuntimeError):
    """``ArrowError::ComputeError`` (``discriminate.rs:383-387``)."""


class DeviceError(RuntimeError):
    """A CUDA error or a device-side wait that ran out."""


class FloatKeys(enum.IntEnum):
    BITWISE = 0
    SIGNED_ZEROS_EQUAL = 1


@dataclass(frozen=True)
class Host:
    float_keys: FloatKeys = FloatKeys.BITWISE


class DomainRows(enum.IntEnum):
    ANY = 0
    UNIQUE_KEYS = 1


class Budget:
    """The memory a kernel may take beyond its inputs (``options.rs:56-65``)."""

    def grow(self, nbytes: int) -> bool:  # pragma: no cover - interface
        return True

    def shrink(self, nbytes: int) -> None:
        pass


class Precision(enum.Enum):
    """How dense products are computed: int8 slices on the tensor cores with
    exact integer sums and an FP64 combine (``SPLIT``), or FP64 on the CUDA
    cores in the reference's order of additions (``FP64``)."""

    SPLIT = 0
    FP64 = 1


@dataclass
class Options:
    host: Host = field(default_factory=Host)
    threads: int = 1
    domain_rows: DomainRows = DomainRows.ANY
    budget: Optional[Budget] = None
    precision: Precision = Precision.SPLIT
    slices: int = 0
    device: int = 0
    # Leave the result's buffers in HBM: the functions then return DeviceBatch
    # objects instead of pyarrow record batches.
    result_on_device: bool = False
    # The context the call runs on (None: the device's shared one). Calls on
    # one context are serialized; calls on different contexts of a device
    # may run at the same time from different threads.
    context: Optional["Context"] = None


class Context:
    """A context of its own on ``device`` (``einfold_context_create``): its
    own stream and scratch; calls on it are serialized, while calls on other
    contexts run beside them from other threads."""

    def __init__(self, device: int = 0):
        lib = _lib.load()
        self.device = device
        self.handle = lib.einfold_context_create(device)
        if not self.handle:
            raise RuntimeError("einfold_context_create failed: " + lib.einfold_last_error().decode())

    def close(self) -> None:
        if self.handle:
            _lib.load().einfold_context_destroy(self.handle)
            self.handle = None

    def __enter__(self) -> "Context":
        return self

    def __exit__(self, *exc) -> None:
        self.close()


def _ctx(options: "Options"):
    if options.context is not None:
        if not options.context.handle:
            raise ValueError("a closed context")
        return options.context.handle
    return _lib.context(options.device)


class Algorithm(enum.Enum):
    DENSE = "dense"
    DISCRIMINATE = "discriminate"
    FUSED = "fused"


@dataclass
class Relation:
    schema: pa.Schema
    batches: List[pa.RecordBatch]


_FORMATS = {pa.int8(): b"c", pa.uint8(): b"C", pa.int16(): b"s", pa.uint16(): b"S", pa.int32(): b"i",
            pa.uint32(): b"I", pa.int64(): b"l", pa.uint64(): b"L", pa.float32(): b"f", pa.float64(): b"g"}


class DeviceRelation:
    """One batch whose columns are CUDA tensors already in HBM (the Arrow C
    Device Data Interface's CUDA placement): fixed-width columns, each with an
    optional validity bitmap tensor (uint8, bit i = row i) and its null count."""

    def __init__(self, schema: pa.Schema, columns: Sequence, validity: Optional[Sequence] = None,
                 null_counts: Optional[Sequence[int]] = None, device: int = 0):
        self.schema = schema
        self.columns = list(columns)
        self.validity = list(validity) if validity is not None else [None] * len(self.columns)
        self.null_counts = list(null_counts) if null_counts is not None else [0] * len(self.columns)
        self.device = device
        self.rows = int(self.columns[0].numel()) if self.columns else 0
        for f in schema:
            if f.type not in _FORMATS:
                raise ArrowInvalidArgumentError(f"a device column of type {f.type}")


class _CudaArray:
    """A device buffer seen through __cuda_array_interface__ (for torch.as_tensor)."""

    def __init__(self, ptr: int, n: int, typestr: str, owner):
        self.owner = owner
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "strides": None}


class _DeviceResult:
    """A library result whose buffers are in HBM, released once."""

    def __init__(self, res):
        self.res = res

    def release(self):
        if self.res is not None:
            _lib.load().einfold_result_release(ctypes.byref(self.res))
            self.res = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class DeviceBatch:
    """A result batch whose buffers are in HBM, owned until :meth:`release`
    (which frees every batch of the same result)."""

    _TYPESTR = {b"c": "|i1", b"C": "|u1", b"s": "<i2", b"S": "<u2", b"i": "<i4", b"I": "<u4", b"l": "<i8",
                b"L": "<u8", b"f": "<f4", b"g": "<f8"}

    def __init__(self, res, index: int = 0, owner: Optional[_DeviceResult] = None):
        self._owner = owner or _DeviceResult(res)
        self._i = index
        self.rows = int(res.batches[index].length) if index < res.n_batches else 0
        self.formats = []
        s = res.schema.contents
        for i in range(s.n_children):
            self.formats.append(s.children[i].contents.format)

    @property
    def _res(self):
        return self._owner.res

    def column(self, i: int):
        """Column i's values as a CUDA tensor sharing the result's memory
        (fixed-width columns; see :meth:`strings` for string and binary)."""
        import torch

        if self.formats[i] not in self._TYPESTR:
            raise TypeError(f"column {i} has Arrow format {self.formats[i]!r}: use strings({i})")
        arr = self._res.batches[self._i].children[i].contents
        ptr = arr.buffers[1]
        return torch.as_tensor(_CudaArray(ptr or 0, self.rows, self._TYPESTR[self.formats[i]], self), device="cuda")

    def strings(self, i: int):
        """A string or binary column's Arrow offsets (rows + 1, int32, or int64
        for the large kinds) and bytes (uint8) as CUDA tensors sharing the
        result's memory."""
        import torch

        fmt = self.formats[i]
        if fmt not in (b"u", b"z", b"U", b"Z"):
            raise TypeError(f"column {i} has Arrow format {fmt!r}, not a string or binary one")
        arr = self._res.batches[self._i].children[i].contents
        wide = fmt in (b"U", b"Z")
        offsets = torch.as_tensor(_CudaArray(arr.buffers[1] or 0, self.rows + 1, "<i8" if wide else "<i4", self),
                                  device="cuda")
        total = int(offsets[-1].item()) if self.rows else 0
        data = torch.as_tensor(_CudaArray(arr.buffers[2] or 0, total, "|u1", self), device="cuda")
        return offsets, data

    def null_count(self, i: int) -> int:
        return int(self._res.batches[self._i].children[i].contents.null_count)

    def release(self):
        self._owner.release()


def _device_batches(res) -> List[DeviceBatch]:
    """A result's batches left in HBM (at least one, perhaps of no rows)."""
    owner = _DeviceResult(res)
    return [DeviceBatch(res, i, owner) for i in range(max(1, int(res.n_batches)))]


@dataclass
class Folded:
    algorithm: Algorithm
    batches: List[pa.RecordBatch]


@dataclass
class Piped:
    batches: List[pa.RecordBatch]
    tiles_visited: int
    tiles: int


# ---------------------------------------------------------------------------
# Marshalling
# ---------------------------------------------------------------------------


class _Keep:
    """Holds the ctypes objects a call's pointers refer to."""

    def __init__(self):
        self.items = []
        self.exported_arrays = []
        self.exported_schemas = []

    def add(self, x):
        self.items.append(x)
        return x

    def release(self):
        rel_a = ctypes.CFUNCTYPE(None, ctypes.POINTER(_lib.ArrowArray))
        rel_s = ctypes.CFUNCTYPE(None, ctypes.POINTER(_lib.ArrowSchema))
        for a in self.exported_arrays:
            if a.release:
                rel_a(a.release)(ctypes.byref(a))
        for s in self.exported_schemas:
            if s.release:
                rel_s(s.release)(ctypes.byref(s))
        self.exported_arrays.clear()
        self.exported_schemas.clear()


def _array(ctype, values):
    arr = (ctype * max(len(values), 1))()
    for i, v in enumerate(values):
        arr[i] = v
    return arr


def _expression(e: Optional[ir.Expression], keep: _Keep) -> _lib.Expression:
    if e is None:
        return _lib.Expression(0, None)
    nodes = [_lib.ExprNode(k, a, b, 0, v) for (k, a, b, v) in e.postfix()]
    arr = keep.add(_array(_lib.ExprNode, nodes))
    return _lib.Expression(len(nodes), arr)


def _operand(op: ir.Operand, keep: _Keep) -> _lib.Operand:
    keys = keep.add(_array(_lib.Key, [_lib.Key(k.dimension, k.column) for k in op.keys]))
    return _lib.Operand(len(op.keys), keys, -1 if op.factor is None else op.factor)


def _fold_desc(f: ir.Fold, keep: _Keep) -> _lib.FoldDesc:
    eq = keep.add(_array(ctypes.c_int32, [int(d.equality) for d in f.dimensions()]))
    ops = keep.add(_array(_lib.Operand, [_operand(o, keep) for o in f.operands()]))
    outs = keep.add(_array(_lib.Output, [
        _lib.Output(o.dimension, -1 if o.domain_key is None else o.domain_key.column,
                    0 if o.domain_key is None else int(o.domain_key.equality)) for o in f.outputs()]))
    conds = keep.add(_array(_lib.Condition, [
        _lib.Condition(c.left, int(c.comparison), c.right, 0, c.offset) for c in f.conditions()]))
    dom = None
    if f.domain() is not None:
        carry = keep.add(_array(ctypes.c_int32, list(f.domain().carry)))
        missing = f.domain().missing
        dom = keep.add(_lib.Domain(len(f.domain().carry), carry, 0 if missing is None else 1, 0,
                                   0.0 if missing is None else missing))
    row = f.row()
    desc = _lib.FoldDesc(len(f.dimensions()), eq, len(f.operands()), ops, len(f.outputs()), outs,
                         0 if row.is_product else 1, _expression(row.expression, keep),
                         ctypes.pointer(dom) if dom is not None else None, len(f.conditions()), conds)
    return keep.add(desc)


def _pipeline_desc(p: ir.Pipeline, keep: _Keep) -> _lib.PipelineDesc:
    prod = _fold_desc(p.producer(), keep)
    w = p.weight()
    eq = keep.add(_array(ctypes.c_int32, [int(d.equality) for d in p.dimensions()]))
    outs = keep.add(_array(ctypes.c_int32, list(p.outputs())))
    if w.is_exp:
        desc = _lib.PipelineDesc(ctypes.pointer(prod), 0, w.scale.kind, w.scale.c, int(w.shift),
                                 int(p.normalizer()), _lib.Expression(0, None), len(p.dimensions()), eq,
                                 _operand(p.values(), keep), len(p.outputs()), outs)
    else:
        desc = _lib.PipelineDesc(ctypes.pointer(prod), 1, 0, 1.0, 0, int(p.normalizer()),
                                 _expression(w.of, keep), len(p.dimensions()), eq, _operand(p.values(), keep),
                                 len(p.outputs()), outs)
    return keep.add(desc)


def _export_schema(s: pa.Schema, keep: _Keep) -> _lib.ArrowSchema:
    c = keep.add(_lib.ArrowSchema())
    s._export_to_c(ctypes.addressof(c))
    keep.exported_schemas.append(c)
    return c


def _device_relation(r: "DeviceRelation", keep: _Keep) -> _lib.Relation:
    cs = _export_schema(r.schema, keep)
    children = []
    for col, valid, nulls in zip(r.columns, r.validity, r.null_counts):
        bufs = keep.add(_array(ctypes.c_void_p, [valid.data_ptr() if valid is not None else None, col.data_ptr()]))
        child = keep.add(_lib.ArrowArray(int(col.numel()), int(nulls), 0, 2, 0, bufs, None, None, None, None))
        children.append(ctypes.pointer(child))
    kids = keep.add(_array(ctypes.POINTER(_lib.ArrowArray), children))
    top_bufs = keep.add(_array(ctypes.c_void_p, [None]))
    top = keep.add(_lib.ArrowArray(r.rows, 0, 0, 1, len(children), top_bufs, kids, None, None, None))
    ptrs = keep.add(_array(ctypes.POINTER(_lib.ArrowArray), [ctypes.pointer(top)]))
    return keep.add(_lib.Relation(ctypes.pointer(cs), 1, ptrs, r.device, 0))


def _relation(r, keep: _Keep) -> _lib.Relation:
    if isinstance(r, DeviceRelation):
        return _device_relation(r, keep)
    if isinstance(r, Relation):
        schema, batches = r.schema, list(r.batches)
    elif isinstance(r, pa.Table):
        schema, batches = r.schema, r.to_batches()
    elif isinstance(r, pa.RecordBatch):
        schema, batches = r.schema, [r]
    else:
        batches = list(r)
        if not batches:
            raise ArrowInvalidArgumentError("a relation of no batches needs its schema: pass a Relation")
        schema = batches[0].schema
    cs = _export_schema(schema, keep)
    arrays = []
    for b in batches:
        a = keep.add(_lib.ArrowArray())
        b._export_to_c(ctypes.addressof(a))
        keep.exported_arrays.append(a)
        arrays.append(ctypes.pointer(a))
    ptrs = keep.add(_array(ctypes.POINTER(_lib.ArrowArray), arrays))
    return keep.add(_lib.Relation(ctypes.pointer(cs), len(batches), ptrs, -1, 0))


def _options(o: Options, keep: _Keep) -> _lib.Options:
    grow = _lib.GROW(0)
    shrink = _lib.SHRINK(0)
    if o.budget is not None:
        budget = o.budget
        grow = keep.add(_lib.GROW(lambda _ctx, n: 1 if budget.grow(int(n)) else 0))
        shrink = keep.add(_lib.SHRINK(lambda _ctx, n: budget.shrink(int(n))))
    return keep.add(_lib.Options(int(o.host.float_keys), max(int(o.threads), 1), int(o.domain_rows),
                                 int(o.precision.value), int(o.slices), int(bool(o.result_on_device)), None, grow,
                                 shrink))


def _raise(status: int, message: str):
    if status == _lib.BUDGET:
        raise ArrowMemoryError(message)
    if status == _lib.INVALID:
        raise ArrowInvalidArgumentError(message)
    if status == _lib.COMPUTE:
        raise ArrowComputeError(message)
    raise DeviceError(f"{_lib.STATUS_NAMES.get(status, status)}: {message}")


@dataclass
class CallInfo:
    """What the last call on this thread did on the device."""

    kernels_launched: int = 0
    device_ms: float = 0.0
    product_ms: float = 0.0
    product_ops: float = 0.0
    # Split attention forwards: the schedule (0 a block per item, 1
    # persistent by key tiles, 2 persistent by batch; -1 other calls) and the
    # graph launch (0 direct, arguments seen for the first time; 1 replayed;
    # 2 updated, 3 instantiated, arguments seen a second time).
    schedule: int = -1
    graph: int = 0
    message: str = ""


class _ThreadCalls(threading.local):
    def __init__(self):
        self.info = CallInfo()


_calls = _ThreadCalls()


def __getattr__(name):
    # ``last_call``: the calling thread's CallInfo.
    if name == "last_call":
        return _calls.info
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


def _collect(res: _lib.Result) -> List[pa.RecordBatch]:
    lib = _lib.load()
    try:
        schema = pa.Schema._import_from_c(ctypes.addressof(res.schema.contents))
        return [pa.RecordBatch._import_from_c(ctypes.addressof(res.batches[i]), schema)
                for i in range(res.n_batches)]
    finally:
        lib.einfold_result_release(ctypes.byref(res))


def _after_torch(*relations) -> None:
    """The Arrow entry points run on the context's own stream, which does not
    wait for torch's: operands in HBM are first finished on torch's current
    stream."""
    for r in relations:
        if isinstance(r, DeviceRelation):
            import torch

            torch.cuda.current_stream(r.device).synchronize()


def _call(fn, *args) -> Optional[_lib.Result]:
    res = _lib.Result()
    status = fn(args[-1], *args[:-1], ctypes.byref(res))
    msg = res.message.decode(errors="replace")
    _calls.info.kernels_launched = res.kernels_launched
    _calls.info.device_ms = res.device_ms
    _calls.info.product_ms = res.product_ms
    _calls.info.product_ops = res.product_ops
    _calls.info.schedule = res.schedule
    _calls.info.graph = res.graph
    _calls.info.message = msg
    if status == _lib.DECLINED:
        return None
    if status != _lib.OK:
        _raise(status, msg)
    return res


# ---------------------------------------------------------------------------
# The kernel layer's functions (crates/einfold-kernels/src/algorithm.rs)
# ---------------------------------------------------------------------------


def fold(f: ir.Fold, a, b, domain=None, schema: Optional[pa.Schema] = None,
         options: Optional[Options] = None) -> Folded:
    """``einfold_kernels::fold`` (algorithm.rs:97-133): dense when its
    requirements hold, else discrimination."""
    options = options or Options()
    _after_torch(a, b, domain)
    keep = _Keep()
    try:
        res = _call(_lib.load().einfold_fold, ctypes.byref(_fold_desc(f, keep)), ctypes.byref(_relation(a, keep)),
                    ctypes.byref(_relation(b, keep)),
                    ctypes.byref(_relation(domain, keep)) if domain is not None else None,
                    ctypes.byref(_options(options, keep)), _ctx(options))
        if res is None:
            raise ArrowComputeError("the fold declined")
        alg = Algorithm(_lib.ALGORITHMS[res.algorithm])
        if options.result_on_device:
            return Folded(alg, _device_batches(res))
        return Folded(alg, _collect(res))
    finally:
        keep.release()


def fold_dense(f: ir.Fold, a, b, domain=None, schema: Optional[pa.Schema] = None,
               options: Optional[Options] = None) -> Optional[List[pa.RecordBatch]]:
    """``einfold_kernels::fold_dense`` (algorithm.rs:52-62)."""
    options = options or Options()
    _after_torch(a, b, domain)
    keep = _Keep()
    try:
        res = _call(_lib.load().einfold_fold_dense, ctypes.byref(_fold_desc(f, keep)),
                    ctypes.byref(_relation(a, keep)), ctypes.byref(_relation(b, keep)),
                    ctypes.byref(_relation(domain, keep)) if domain is not None else None,
                    ctypes.byref(_options(options, keep)), _ctx(options))
        if res is None:
            return None
        return _device_batches(res) if options.result_on_device else _collect(res)
    finally:
        keep.release()


def fold_chain(f: ir.Fold, operands: Sequence, schema: Optional[pa.Schema] = None,
               options: Optional[Options] = None) -> Optional[List[pa.RecordBatch]]:
    """``einfold_kernels::fold_chain`` (algorithm.rs:76-83)."""
    options = options or Options()
    _after_torch(*operands)
    keep = _Keep()
    try:
        rels = keep.add(_array(_lib.Relation, [_relation(r, keep) for r in operands]))
        res = _call(_lib.load().einfold_fold_chain, ctypes.byref(_fold_desc(f, keep)), rels,
                    ctypes.byref(_options(options, keep)), _ctx(options))
        if res is None:
            return None
        return _device_batches(res) if options.result_on_device else _collect(res)
    finally:
        keep.release()


def pipeline(p: ir.Pipeline, operands: Sequence, schema: Optional[pa.Schema] = None,
             options: Optional[Options] = None) -> Optional[Piped]:
    """``einfold_kernels::pipeline`` (algorithm.rs:146-160) over ``[q, k, v]``."""
    options = options or Options()
    _after_torch(*operands)
    keep = _Keep()
    try:
        rels = keep.add(_array(_lib.Relation, [_relation(r, keep) for r in operands]))
        res = _call(_lib.load().einfold_pipeline, ctypes.byref(_pipeline_desc(p, keep)), rels,
                    ctypes.byref(_options(options, keep)), _ctx(options))
        if res is None:
            return None
        visited, tiles = int(res.tiles_visited), int(res.tiles)
        return Piped(_device_batches(res) if options.result_on_device else _collect(res), visited, tiles)
    finally:
        keep.release()


def pipeline_backward(p: ir.Pipeline, operands: Sequence, d_out: Relation,
                      options: Optional[Options] = None) -> Optional[List[List[pa.RecordBatch]]]:
    """The gradients of ``pipeline``'s result with respect to q's, k's and v's
    factors (``einfold_pipeline_backward``): ``d_out`` holds the result's key
    columns and a DOUBLE gradient per result row; returns, per operand, its
    key columns and a ``grad`` column, a row per placed cell; None where the
    pipeline isn't attention-shaped."""
    options = options or Options()
    _after_torch(*operands, d_out)
    keep = _Keep()
    lib = _lib.load()
    try:
        rels = keep.add(_array(_lib.Relation, [_relation(r, keep) for r in operands]))
        results = (_lib.Result * 3)()
        status = lib.einfold_pipeline_backward(_ctx(options), ctypes.byref(_pipeline_desc(p, keep)),
                                               rels, ctypes.byref(_relation(d_out, keep)),
                                               ctypes.byref(_options(options, keep)), results)
        msg = results[0].message.decode(errors="replace")
        _calls.info.kernels_launched = results[0].kernels_launched
        _calls.info.device_ms = results[0].device_ms
        _calls.info.product_ms = results[0].product_ms
        _calls.info.product_ops = results[0].product_ops
        _calls.info.message = msg
        if status == _lib.DECLINED:
            return None
        if status != _lib.OK:
            _raise(status, msg)
        if options.result_on_device:
            return [_device_batches(results[i]) for i in range(3)]
        return [_collect(results[i]) for i in range(3)]
    finally:
        keep.release()


@dataclass
class Ranks:
    """Each row's rank among the distinct keys, and the first row of each rank."""

    rank: np.ndarray  # uint32 per row
    first: np.ndarray  # uint32 per distinct key


def evaluate_pairs(e: ir.Expression, a, a_valid, b, b_valid, options: Optional[Options] = None):
    """``Expression::evaluate`` (expression.rs) on the device, as the tile
    kernels evaluate row expressions (``einfold_evaluate_pairs``), for every
    pair of a row of ``a`` and a row of ``b``: CUDA float64 tensors of
    ``cols`` values a row, with uint8 validity tensors of the same shape
    (1: valid). Returns the values and their validity, ``[len(a)][len(b)]``
    (0 and 0 where a column the expression reads is NULL)."""
    import torch

    options = options or Options()
    if a.dim() != 2 or b.dim() != 2 or a.shape[1] != b.shape[1]:
        raise ValueError("a and b must be [rows][cols] with the same cols")
    a, b = a.contiguous(), b.contiguous()
    a_valid, b_valid = a_valid.contiguous().to(torch.uint8), b_valid.contiguous().to(torch.uint8)
    na, nb, cols = a.shape[0], b.shape[0], a.shape[1]
    out = torch.empty((na, nb), dtype=torch.float64, device=a.device)
    valid = torch.empty((na, nb), dtype=torch.uint8, device=a.device)
    keep = _Keep()
    try:
        expr = _expression(e, keep)
        torch.cuda.current_stream(a.device).synchronize()
        st = _lib.load().einfold_evaluate_pairs(_ctx(options), ctypes.byref(expr), a.data_ptr(), a_valid.data_ptr(),
                                                na, b.data_ptr(), b_valid.data_ptr(), nb, cols, out.data_ptr(),
                                                valid.data_ptr(), None)
    finally:
        keep.release()
    if st != _lib.OK:
        _raise(st, _lib.load().einfold_last_error().decode())
    return out, valid


def rank_columns(relation: Relation, columns: Sequence[int], float_keys: FloatKeys = FloatKeys.BITWISE,
                 device: int = 0) -> Ranks:
    """``rank_columns`` (discriminate.rs:240-277) on the device: the ranks of
    the keys in ``columns`` of a host relation, in the order of Arrow's row
    format, keys of any length."""
    n = sum(b.num_rows for b in relation.batches)
    rank = np.zeros(max(n, 1), dtype=np.uint32)
    first = np.zeros(max(n, 1), dtype=np.uint32)
    cols = np.asarray(list(columns), dtype=np.int32)
    k = ctypes.c_int64(0)
    keep = _Keep()
    try:
        st = _lib.load().einfold_rank_columns(_lib.context(device), ctypes.byref(_relation(relation, keep)),
                                              len(cols), cols.ctypes.data if len(cols) else None, int(float_keys),
                                              rank.ctypes.data, first.ctypes.data, ctypes.byref(k))
    finally:
        keep.release()
    if st != _lib.OK:
        if st == _lib.DECLINED:
            raise ArrowComputeError("the ranking declined: " + _lib.load().einfold_last_error().decode())
        _raise(st, _lib.load().einfold_last_error().decode())
    return Ranks(rank[:n], first[: k.value].copy())


def schema(f: ir.Fold, operands: Sequence[pa.Schema], domain: Optional[pa.Schema] = None) -> pa.Schema:
    """``einfold_kernels::schema`` (schema.rs:31-36)."""
    keep = _Keep()
    try:
        ptrs = keep.add(_array(ctypes.POINTER(_lib.ArrowSchema),
                               [ctypes.pointer(_export_schema(s, keep)) for s in operands]))
        dom = ctypes.pointer(_export_schema(domain, keep)) if domain is not None else None
        out = _lib.ArrowSchema()
        msg = ctypes.create_string_buffer(480)
        st = _lib.load().einfold_schema(ctypes.byref(_fold_desc(f, keep)), ptrs, len(operands), dom,
                                        ctypes.byref(out), msg, 480)
        if st != _lib.OK:
            _raise(st, msg.value.decode())
        return pa.Schema._import_from_c(ctypes.addressof(out))
    finally:
        keep.release()


def pipeline_schema(p: ir.Pipeline, inputs: Sequence[pa.Schema]) -> pa.Schema:
    """``einfold_kernels::pipeline_schema`` (schema.rs:155-206)."""
    keep = _Keep()
    try:
        ptrs = keep.add(_array(ctypes.POINTER(_lib.ArrowSchema),
                               [ctypes.pointer(_export_schema(s, keep)) for s in inputs]))
        out = _lib.ArrowSchema()
        msg = ctypes.create_string_buffer(480)
        st = _lib.load().einfold_pipeline_schema(ctypes.byref(_pipeline_desc(p, keep)), ptrs, ctypes.byref(out),
                                                 msg, 480)
        if st != _lib.OK:
            _raise(st, msg.value.decode())
        return pa.Schema._import_from_c(ctypes.addressof(out))
    finally:
        keep.release()
