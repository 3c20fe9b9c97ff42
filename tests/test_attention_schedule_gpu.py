"""The split attention forward under each launch schedule: a block per
(query tile, batch) item, persistent blocks claiming the items by key tiles,
and persistent blocks taking them batch by batch; the schedule the first
call of a shape times fastest; and the tile phase replayed from a CUDA graph.
Every item's sums are exact integers combined in a fixed order, so all of
them give the same bits."""
import pytest
import torch

from einfold_b200 import _lib
from einfold_b200 import autograd as A
from einfold_b200.kernels import ArrowInvalidArgumentError, Precision, last_call
from tests.test_ragged_gpu import _ragged

pytestmark = pytest.mark.gpu

SCHEDULES = {"grid": 0, "tiles": 1, "batches": 2}

CASES = {
    # batches or group lengths, padded length, d, dv, conditions, scale. More
    # items than SMs, so persistent blocks run several each.
    "causal_24x1024_d64": (24, 1024, 64, 64, A.causal(), 1.0),
    "ragged_window_d128_dv128": ([1500, 90, 1024, 700, 1, 333, 1200, 640] * 5, 1500, 128, 128, A.window(200),
                                 0.0884),
    "full_12x700_d32_dv96": (12, 700, 32, 96, [], 0.5),
}


def _case(name):
    lengths, lmax, d, dv, cond, scale = CASES[name]
    if isinstance(lengths, int):
        q, k, v = _ragged([lmax] * lengths, lmax, d, dv, seed=7)
        ql = None
    else:
        q, k, v = _ragged(lengths, lmax, d, dv, seed=8)
        ql = torch.tensor(lengths, dtype=torch.int64)
    return q, k, v, ql, cond, scale


def _equal(a, b):
    return torch.equal(a.nan_to_num(123.0), b.nan_to_num(123.0)) and torch.equal(torch.isnan(a), torch.isnan(b))


@pytest.mark.parametrize("name", list(CASES))
def test_every_schedule_gives_the_same_bits(monkeypatch, name):
    q, k, v, ql, cond, scale = _case(name)
    ref = None
    for schedule, code in SCHEDULES.items():
        monkeypatch.setenv("EINFOLD_ATTENTION_SCHEDULE", schedule)
        out, lse = A.attention_forward(q, k, v, cond, scale, Precision.SPLIT, q_lengths=ql, k_lengths=ql)
        assert last_call.schedule == code
        if ref is None:
            ref = (out, lse)
        else:
            assert _equal(out, ref[0]), f"out under {schedule}"
            assert _equal(lse, ref[1]), f"lse under {schedule}"
    monkeypatch.delenv("EINFOLD_ATTENTION_SCHEDULE")
    out64, _ = A.attention_forward(q, k, v, cond, scale, Precision.FP64, q_lengths=ql, k_lengths=ql)
    seen = ~torch.isnan(out64)
    assert torch.equal(seen, ~torch.isnan(ref[0]))
    # Scores spread over tens of units (operands of deviation 0.5, d up to
    # 128): the weights' relative error grows with the spread.
    assert (ref[0][seen] - out64[seen]).abs().max().item() <= 1e-10 * out64[seen].abs().max().item()


def test_the_tuned_schedule_and_graph_replays(monkeypatch):
    # The first call of a shape times the three schedules and keeps the
    # fastest. Arguments seen for the first time launch directly; seen
    # again, the tile phase is captured as a graph (new output buffers update
    # the graph of that shape), and then replayed.
    monkeypatch.delenv("EINFOLD_ATTENTION_SCHEDULE", raising=False)
    monkeypatch.delenv("EINFOLD_GRAPHS", raising=False)
    q, k, v, _, cond, scale = _case("causal_24x1024_d64")
    q = q[:20].contiguous()  # a shape no other test has timed
    k, v = k[:20].contiguous(), v[:20].contiguous()
    b, lq, d = q.shape
    dv = v.shape[-1]
    lib = _lib.load()
    n, cmp, off = A._conditions(cond)

    def forward(out, lse):
        A._call(lib.einfold_attention_forward, 0, q.data_ptr(), k.data_ptr(), v.data_ptr(), out.data_ptr(),
                lse.data_ptr(), b, lq, lq, d, dv, n, cmp, off, float(scale), Precision.SPLIT.value, 0)
        return last_call.schedule, last_call.graph

    def buffers():
        return (torch.full((b, lq, dv), float("nan"), dtype=torch.float64, device="cuda"),
                torch.full((b, lq), float("nan"), dtype=torch.float64, device="cuda"))

    out, lse = buffers()
    schedule, graph = forward(out, lse)
    assert schedule in SCHEDULES.values() and graph == 0
    first = (out.clone(), lse.clone())
    graphs = [forward(out, lse)[1] for _ in range(3)]
    assert graphs[0] in (2, 3) and graphs[1:] == [1, 1], f"graph launches {graphs}"
    assert _equal(out, first[0]) and _equal(lse, first[1])
    out2, lse2 = buffers()
    assert [forward(out2, lse2) for _ in range(3)] == [(schedule, 0), (schedule, 2), (schedule, 1)]
    assert _equal(out2, first[0]) and _equal(lse2, first[1])
    monkeypatch.setenv("EINFOLD_GRAPHS", "0")
    out3, lse3 = buffers()
    assert forward(out3, lse3) == (schedule, 0)
    assert _equal(out3, first[0]) and _equal(lse3, first[1])


def test_an_unknown_schedule_is_refused(monkeypatch):
    q, k, v, _, cond, scale = _case("full_12x700_d32_dv96")
    monkeypatch.setenv("EINFOLD_ATTENTION_SCHEDULE", "sideways")
    with pytest.raises(ArrowInvalidArgumentError, match="EINFOLD_ATTENTION_SCHEDULE"):
        A.attention_forward(q, k, v, cond, scale, Precision.SPLIT)


def test_new_lengths_of_a_timed_shape_are_not_timed_again(monkeypatch):
    # The schedule is timed once per padded shape: a later call with other
    # ragged lengths (a training loop's next batch) launches the tile kernel
    # once, not the six timing runs again.
    monkeypatch.delenv("EINFOLD_ATTENTION_SCHEDULE", raising=False)
    lmax, d, dv = 512, 32, 40  # a shape no other test uses
    runs = []
    for lengths in ([300, 17, 512, 64, 200], [100, 512, 3, 250, 511]):
        q, k, v = _ragged(lengths, lmax, d, dv, seed=len(runs) + 11)
        ql = torch.tensor(lengths, dtype=torch.int64)
        out, _ = A.attention_forward(q, k, v, A.window(30), 0.3, Precision.SPLIT, q_lengths=ql, k_lengths=ql)
        runs.append((last_call.kernels_launched, last_call.schedule))
        alone, _ = A.attention_forward(q[1:2, :lengths[1]], k[1:2, :lengths[1]], v[1:2, :lengths[1]], A.window(30),
                                       0.3, Precision.SPLIT)
        assert _equal(out[1, :lengths[1]], alone[0])
    assert runs[0][1] == runs[1][1]
    assert runs[0][0] - runs[1][0] == 6, runs
