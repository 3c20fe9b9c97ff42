"""The C ABI library loads, exports what the header declares, and computes
schemas on the host (no GPU needed)."""
import ctypes
import os

import pyarrow as pa
import pytest

from einfold_b200 import _lib, ir, kernels as K

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "einfold_b200.h")


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    declared = _lib.declared_symbols(HEADER)
    assert len(declared) >= 14
    for name in declared:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"
    assert lib.einfold_version().startswith(b"einfold_b200")


def _matmul():
    e = ir.EQ
    return ir.Fold([e, e, e], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)],
                   [ir.Output(0), ir.Output(2)])


def test_schema_follows_the_key_types():
    sa = pa.schema([("i", pa.int32()), ("j", pa.int64()), ("v", pa.float64())])
    sb = pa.schema([("j", pa.int64()), ("k", pa.uint16()), ("v", pa.float64())])
    s = K.schema(_matmul(), [sa, sb])
    assert [f.type for f in s] == [pa.int32(), pa.uint16(), pa.float64()]
    assert [f.name for f in s] == ["0", "1", "2"]


@pytest.mark.parametrize("i_type,k_type", [
    (pa.decimal32(9, 2), pa.decimal64(18, 3)),
    (pa.decimal128(38, 4), pa.decimal256(76, 5)),
    (pa.binary(12), pa.binary(1)),
    (pa.date32(), pa.timestamp("us", tz="UTC")),
    (pa.time64("ns"), pa.duration("ms")),
    (pa.dictionary(pa.int8(), pa.decimal256(76, 5)), pa.dictionary(pa.int32(), pa.binary(4))),
])
def test_schema_keeps_every_key_type(i_type, k_type):
    sa = pa.schema([("i", i_type), ("j", pa.int64()), ("v", pa.float64())])
    sb = pa.schema([("j", pa.int64()), ("k", k_type), ("v", pa.float64())])
    s = K.schema(_matmul(), [sa, sb])
    assert [f.type for f in s] == [i_type, k_type, pa.float64()]


def test_schema_rejects_decimals_of_another_scale_on_one_dimension():
    sa = pa.schema([("i", pa.int64()), ("j", pa.decimal128(10, 2)), ("v", pa.float64())])
    sb = pa.schema([("j", pa.decimal128(10, 3)), ("k", pa.int64()), ("v", pa.float64())])
    with pytest.raises(K.ArrowInvalidArgumentError):
        K.schema(_matmul(), [sa, sb])


def test_schema_rejects_mismatched_keys_and_non_float_values():
    sa = pa.schema([("i", pa.int64()), ("j", pa.int64()), ("v", pa.float64())])
    sb = pa.schema([("j", pa.int32()), ("k", pa.int64()), ("v", pa.float64())])
    with pytest.raises(K.ArrowInvalidArgumentError):
        K.schema(_matmul(), [sa, sb])
    sb = pa.schema([("j", pa.int64()), ("k", pa.int64()), ("v", pa.float32())])
    with pytest.raises(K.ArrowInvalidArgumentError):
        K.schema(_matmul(), [sa, sb])


def test_domain_schema_carries_columns_and_a_non_null_default():
    e = ir.EQ
    f = ir.Fold([e, e, e], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)],
                [ir.Output(0, ir.DomainKey(1)), ir.Output(2, ir.DomainKey(2))], domain=ir.Domain((0, 1, 2), 0.0))
    sa = pa.schema([("i", pa.int64()), ("j", pa.int64()), ("v", pa.float64())])
    sb = pa.schema([("j", pa.int64()), ("k", pa.int64()), ("v", pa.float64())])
    sd = pa.schema([("tag", pa.string()), ("i", pa.int64()), ("k", pa.int64())])
    s = K.schema(f, [sa, sb], sd)
    assert [f.type for f in s] == [pa.string(), pa.int64(), pa.int64(), pa.float64()]
    assert not s.field(3).nullable


def test_invalid_folds_are_rejected_by_the_ir():
    e = ir.EQ
    with pytest.raises(ir.InvalidFold):
        ir.Fold([e, e], [ir.Operand([(0, 0)], 1)], [ir.Output(0)])  # dimension 1 held by no operand
    with pytest.raises(ir.InvalidFold):
        ir.Fold([e], [ir.Operand([(0, 0), (0, 1)], 2)], [ir.Output(0)])
    with pytest.raises(ir.InvalidFold):
        _matmul().with_conditions([ir.Condition(0, ir.Comparison.LESS, 0, 0)])


def test_pipeline_schema():
    e = ir.EQ
    scores = ir.Fold([e, e, e], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(2, 0), (1, 1)], 2)],
                     [ir.Output(0), ir.Output(2)])
    p = ir.Pipeline(scores, ir.Weight.exp(), [e], ir.Operand([(2, 0), (3, 1)], 2), [0, 3], ir.Normalizer.KEPT_GROUPS)
    q = pa.schema([("t", pa.int64()), ("d", pa.int64()), ("x", pa.float64())])
    v = pa.schema([("t", pa.int64()), ("c", pa.int32()), ("x", pa.float64())])
    s = K.pipeline_schema(p, [q, q, v])
    assert [f.type for f in s] == [pa.int64(), pa.int32(), pa.float64()]


# The C structs of the header and their ctypes mirrors (einfold_b200/_lib.py).
_MIRRORS = {
    "einfold_key": "Key", "einfold_operand": "Operand", "einfold_output": "Output",
    "einfold_condition": "Condition", "einfold_domain": "Domain", "einfold_expr_node": "ExprNode",
    "einfold_expression": "Expression", "einfold_fold_desc": "FoldDesc", "einfold_pipeline_desc": "PipelineDesc",
    "einfold_relation": "Relation", "einfold_options": "Options", "einfold_result": "Result",
    "struct ArrowSchema": "ArrowSchema", "struct ArrowArray": "ArrowArray",
    "einfold_dense_shape": "DenseShape", "einfold_dense_work": "DenseWork",
}


def test_ctypes_mirrors_have_the_headers_layout(tmp_path):
    # Sizes and field offsets as a C compiler lays the header's structs out.
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "einfold_b200.h"', "int main(void) {"]
    for cname, pyname in _MIRRORS.items():
        cls = getattr(_lib, pyname)
        lines.append(f'  printf("{pyname} %zu\\n", sizeof({cname}));')
        for field in cls._fields_:
            lines.append(f'  printf("{pyname}.{field[0]} %zu\\n", offsetof({cname}, {field[0]}));')
    lines += ["  return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines))
    subprocess.run([cc, "-std=c11", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    c_layout = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                            text=True).stdout.splitlines())
    import ctypes

    for pyname in _MIRRORS.values():
        cls = getattr(_lib, pyname)
        assert int(c_layout[pyname]) == ctypes.sizeof(cls), f"sizeof {pyname}"
        for field in cls._fields_:
            assert int(c_layout[f"{pyname}.{field[0]}"]) == getattr(cls, field[0]).offset, f"{pyname}.{field[0]}"


def test_smoother_pipeline_schema():
    # The Gaussian smoother's pipeline is valid and its output is (b, t, value).
    from einfold_b200 import cases as C

    q = pa.schema([("b", pa.int64()), ("t", pa.int64()), ("d", pa.int64()), ("x", pa.float64())])
    v = pa.schema([("b", pa.int64()), ("t", pa.int64()), ("x", pa.float64())])
    s = K.pipeline_schema(C.smoother_pipeline(0.01), [q, q, v])
    assert [f.type for f in s] == [pa.int64(), pa.int64(), pa.float64()]


def test_small_fold_tables_have_the_stated_shape():
    # 512 x 512 and 512 x 256 rows, every key tuple once, in four batches,
    # with about 1% of b's values NULL when asked (and none otherwise).
    import numpy as np

    from einfold_b200 import cases as C

    for nulls in (True, False):
        (sa, a), (sb, b) = C.small_fold_tables(nulls)
        assert len(a) == 4 and len(b) == 4
        ta, tb = pa.Table.from_batches(a), pa.Table.from_batches(b)
        assert ta.num_rows == 512 * 512 and tb.num_rows == 512 * 256
        keys = ta.column(0).to_numpy() * 512 + ta.column(1).to_numpy()
        assert np.array_equal(np.sort(keys), np.arange(512 * 512))
        n_null = tb.column(2).null_count
        assert (0.008 * tb.num_rows < n_null < 0.012 * tb.num_rows) if nulls else n_null == 0
        assert ta.column(2).null_count == 0


def test_backend_may_run_takes_products_and_attention_only():
    # DenseBackend::may_run (backend.rs:124-132): the kinds this backend
    # knows, with non-negative extents; no device is touched.
    lib = _lib.load()
    for kind, want in ((0, 1), (1, 1), (2, 0), (-1, 0)):
        shape = _lib.DenseShape(kind, 0, 2, 3, 4, 5, 6)
        assert lib.einfold_backend_may_run(ctypes.byref(shape)) == want
    assert lib.einfold_backend_may_run(ctypes.byref(_lib.DenseShape(0, 0, 1, -1, 4, 5, 0))) == 0
    assert lib.einfold_backend_may_run(None) == 0


def test_last_call_is_per_thread():
    import threading

    from einfold_b200 import kernels as K

    K.last_call.message = "main"
    seen = []

    def other():
        seen.append(K.last_call.message)
        K.last_call.message = "other"
        seen.append(K.last_call.message)

    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert seen == ["", "other"] and K.last_call.message == "main"
