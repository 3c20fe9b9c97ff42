"""The discrimination fold's result in bounded batches: with at most
EINFOLD_GROUPS_PER_BATCH groups a batch, the fold's groups come out as
several batches of consecutive x blocks (discriminate.rs:548-584 sums each
block of x apart), which together are the oracle's rows bit for bit, and
each holds at most that many groups; with results left in HBM as well."""
import os
import subprocess
import sys
import textwrap

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = textwrap.dedent("""
    import sys
    import numpy as np
    import pyarrow as pa
    sys.path.insert(0, %r)
    from einfold_b200 import kernels as K, synthetic as S
    from oracle import oracle
    from tests.tables import assert_same_rows, matmul_fold, rows_of
    oracle.build()
    a, b = S.sorting_tables(8_000, pool=20_000, names=3_000)
    f = matmul_fold()
    got = K.fold(f, K.Relation(a.schema, [a]), K.Relation(b.schema, [b]))
    want = oracle.fold(f, a.schema, [a], b.schema, [b], None, oracle.schema(f, [a.schema, b.schema]))
    assert len(got.batches) > 3, len(got.batches)
    assert max(x.num_rows for x in got.batches) <= 50_000
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)
    dev = K.fold(f, K.Relation(a.schema, [a]), K.Relation(b.schema, [b]), options=K.Options(result_on_device=True))
    assert len(dev.batches) == len(got.batches)
    for d, h in zip(dev.batches, got.batches):
        assert d.rows == h.num_rows
        assert np.array_equal(d.column(2).cpu().numpy(), h.column(2).to_numpy(zero_copy_only=False))
    dev.batches[0].release()  # the result's batches share one release
    print("ok", len(got.batches))
""") % ROOT


def test_groups_in_bounded_batches_are_the_oracles_rows():
    env = dict(os.environ, EINFOLD_GROUPS_PER_BATCH="50000")
    r = subprocess.run([sys.executable, "-c", SCRIPT], env=env, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout[-2000:] + r.stderr[-4000:]
