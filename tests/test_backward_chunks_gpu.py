"""The split attention backward under an export limit: batches go in chunks
whose exports (P's digits and dS, for the allowed tiles only) fit
EINFOLD_BACKWARD_EXPORT_MB, alternating
between two streams, and give the same bits as one chunk of every batch; a
limit below one batch's exports takes the kernels that recompute the scores,
with the same bits again (same digits, scales and order of summation)."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = textwrap.dedent("""
    import sys
    import numpy as np
    import torch
    sys.path.insert(0, %r)
    from einfold_b200 import autograd as A
    from einfold_b200.kernels import Precision
    g = torch.Generator(device="cuda").manual_seed(11)
    q, k, v, d = (torch.randn(12, 1024, 64, dtype=torch.float64, device="cuda", generator=g) * s
                  for s in (0.125, 0.125, 0.125, 1.0))
    out, lse = A.attention_forward(q, k, v, A.causal(), 1.0, Precision.SPLIT)
    grads = A.attention_backward(q, k, v, out, lse, d, A.causal(), 1.0, Precision.SPLIT)
    np.save(sys.argv[1], torch.stack(grads).cpu().numpy())
""") % ROOT


def _grads(tmp_path, limit_mb):
    path = str(tmp_path / f"grads_{limit_mb}.npy")
    env = dict(os.environ)
    if limit_mb is None:
        env.pop("EINFOLD_BACKWARD_EXPORT_MB", None)
    else:
        env["EINFOLD_BACKWARD_EXPORT_MB"] = str(limit_mb)
    r = subprocess.run([sys.executable, "-c", SCRIPT, path], env=env, capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-4000:]
    return np.load(path)


def test_chunked_exports_give_the_same_bits(tmp_path):
    # A batch's exports at T = 1024, causal: the 72 allowed P tiles (48 KB
    # each, and their rows' exponents) and 72 dS tiles (64 KB), about 8.3 MB;
    # 12 batches in one chunk by default, 2 a chunk (two buffers) under
    # 40 MB, and the recomputing kernels under 12 MB.
    whole = _grads(tmp_path, None)
    chunked = _grads(tmp_path, 40)
    recomputed = _grads(tmp_path, 12)
    assert np.isfinite(whole).all()
    assert np.array_equal(whole.view(np.uint64), chunked.view(np.uint64))
    assert np.array_equal(whole.view(np.uint64), recomputed.view(np.uint64))
