"""Contexts of their own (``K.Context``, einfold_context_create): calls on
two contexts from two threads at once give the same rows and bits as on the
shared context, and each thread reads its own ``last_call``."""
import threading

import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle
from tests import pipelines as P
from tests.tables import rows_of

pytestmark = pytest.mark.gpu

E = ir.Dimension(ir.KeyEquality.EQUAL)


def _matmul(n, seed):
    rng = oracle.Rng.seeded(seed, 0)
    ii, jj = np.indices((n, n)).reshape(2, -1)
    a = pa.record_batch([pa.array(ii), pa.array(jj), pa.array(rng.units(n * n) * 2 - 1)], names=["i", "j", "v"])
    b = pa.record_batch([pa.array(ii), pa.array(jj), pa.array(rng.units(n * n) * 2 - 1)], names=["j", "k", "v"])
    f = ir.Fold([E, E, E], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)],
                [ir.Output(0), ir.Output(2)])
    return f, K.Relation(a.schema, [a]), K.Relation(b.schema, [b])


def test_two_contexts_from_two_threads_give_the_shared_contexts_bits():
    f, a, b = _matmul(300, 41)
    case = P.attention(200, d=16, nb=2, weight=ir.Weight.exp(ir.Scale.one(), ir.Shift.KEPT_MAXIMUM),
                       q_value=lambda n: oracle.Rng.seeded(42, 2).units(n) * 2 - 1,
                       k_value=lambda n: oracle.Rng.seeded(43, 2).units(n) * 2 - 1,
                       v_value=lambda n: oracle.Rng.seeded(44, 2).units(n) * 2 - 1)
    ops = [K.Relation(*case.q), K.Relation(*case.k), K.Relation(*case.v)]
    want_fold = rows_of(K.fold(f, a, b).batches)
    want_pipe = rows_of(K.pipeline(case.pipeline, ops).batches)
    got, algos, errors = {}, {}, []
    with K.Context(0) as c1, K.Context(0) as c2:
        def folds():
            try:
                for i in range(3):
                    got[("fold", i)] = rows_of(K.fold(f, a, b, options=K.Options(context=c1)).batches)
                algos["fold"] = K.last_call.kernels_launched
            except BaseException as e:
                errors.append(e)

        def pipes():
            try:
                for i in range(3):
                    got[("pipe", i)] = rows_of(K.pipeline(case.pipeline, ops, options=K.Options(context=c2)).batches)
                algos["pipe"] = K.last_call.kernels_launched
            except BaseException as e:
                errors.append(e)

        threads = [threading.Thread(target=folds), threading.Thread(target=pipes)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    assert not errors, errors
    for i in range(3):
        assert got[("fold", i)].equals(want_fold)
        assert got[("pipe", i)].equals(want_pipe)
    assert algos["fold"] > 0 and algos["pipe"] > 0


def test_a_closed_context_is_refused():
    c = K.Context(0)
    c.close()
    f, a, b = _matmul(8, 45)
    with pytest.raises(ValueError):
        K.fold(f, a, b, options=K.Options(context=c))
