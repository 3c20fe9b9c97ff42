"""Benchmark of einfold's kernel layer on B200s.

One step is the metric's workload, in the split form (int8 digit products
on the tensor cores with exact integer sums and an FP64 combine):

* a dense matrix-product fold of 8192x8192 by 8192x8192 FP64 tables through
  the C ABI (``SUM(a.v * b.v) ... GROUP BY a.i, b.k`` over a(i, j, v) and
  b(j, k, v), 67.1M rows each): 2·n³ FLOP;
* causal attention over q, k, v (b 0..3, h 0..15, t 0..4095, d 0..63),
  values normal(0, 1/8): the forward pass (scores, online softmax, weighted
  values over the T(T+1)/2 allowed pairs of each of the 64 groups, 4·d FLOP
  a pair) and the backward pass from the saved log-sum-exp for an upstream
  gradient normal(0, 1) (five products, 10·d FLOP a pair).

The metric is the step's FP64-equivalent throughput, next to the plain FP64
GPU form of the same step (cuBLAS DGEMM for the fold, the faster of torch's
float64 attention and this library's FP64 tile kernels for attention) and
the errors against it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (under torchrun, one process per GPU) every rank runs its own
step: replicas, no collective on the data path. ``--impl reference`` times
the reference's CPU algorithms (their C restatements in ``oracle/``, as the
reference's Rust can't be built here) on a bounded sample of the same step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "attn fwd+bwd & matmul fold TFLOP/s: split-BF16 vs FP64 GPU at equal error"
N = 8192
B, H, T, D = 4, 16, 4096, 64
SEED = 0
# The split attention forward's launch schedules and graph launches, by the
# codes the library reports.
SCHEDULE_NAMES = {0: "grid", 1: "tiles", 2: "batches"}
GRAPH_NAMES = {0: "direct", 1: "replayed", 2: "updated", 3: "instantiated"}
PAIRS = B * H * T * (T + 1) // 2
ATT_FWD = 4.0 * D * PAIRS
ATT_BWD = 10.0 * D * PAIRS
FOLD = 2.0 * N ** 3


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["bf16_tflops"]), float(p["hbm_gbs"]), "measured"
    except Exception:
        return 1590.0, 6650.0, "fallback"


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() in ("active", "1"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(ms, dist, device):
    """The slowest rank's time: every rank contributes its own and receives
    the largest (an all-reduce of one value; the only collective of the
    replicas besides the barriers)."""
    if dist is None:
        return ms
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(world, flop_per_step, steps, ms):
    """TFLOP/s of the whole job: every rank runs `steps` steps of the same
    work (weak scaling), in `ms` milliseconds on the slowest rank."""
    return world * flop_per_step * steps / (ms / 1e3) / 1e12


def _matmul_fold():
    from einfold_b200 import ir

    e = ir.EQ
    return ir.Fold([e, e, e], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)],
                   [ir.Output(0), ir.Output(2)])


def _tables(device):
    """a(i, j, v) and b(j, k, v), keys in row-major order, v uniform[-1, 1]
    from SplitMix64 (seed 0; salts 1 and 2)."""
    import torch

    from einfold_b200 import synthetic as S

    i, j = S.grid_keys([N, N], device)
    av = S.uniform(SEED, 1, N * N, device=device)
    bv = S.uniform(SEED, 2, N * N, device=device)
    if str(device).startswith("cuda"):
        torch.cuda.synchronize()
    return (i, j, av), (i.clone(), j.clone(), bv)


def _attention_inputs(device, groups=B * H):
    """q, k, v [groups][T][D] normal(0, 1/8) and d_out normal(0, 1) from
    SplitMix64 (seed 0; salts 3 to 6)."""
    from einfold_b200 import synthetic as S

    n = groups * T * D
    q, k, v = (S.normal(SEED, salt, n, 1.0 / 8, device=device).view(groups, T, D) for salt in (3, 4, 5))
    d_out = S.normal(SEED, 6, n, 1.0, device=device).view(groups, T, D)
    return q, k, v, d_out


def _attention_pipeline(causal=True):
    """Config 3 as einfold's pipeline: q(b, h, t, d, x), k(b, h, t, d, x),
    v(b, h, t, c, x); scores SUM(q.x * k.x) over d, weights exp(s - MAX(s))
    over (b, h, tq) normalised by their sum, out(b, h, tq, c) = SUM(w * v.x);
    causal mask tq >= tk. Dimensions: 0 b, 1 h, 2 tq, 3 d, 4 tk, 5 c."""
    from einfold_b200 import ir

    e = ir.EQ
    q = ir.Operand([(0, 0), (1, 1), (2, 2), (3, 3)], 4)
    k = ir.Operand([(0, 0), (1, 1), (4, 2), (3, 3)], 4)
    producer = ir.Fold([e] * 5, [q, k], [ir.Output(0), ir.Output(1), ir.Output(2), ir.Output(4)])
    if causal:
        producer = producer.with_conditions([ir.Condition(2, ir.Comparison.GREATER_OR_EQUAL, 4, 0)])
    values = ir.Operand([(0, 0), (1, 1), (4, 2), (5, 3)], 4)
    return ir.Pipeline(producer, ir.Weight.exp(), [e], values, [0, 1, 2, 5], ir.Normalizer.KEPT_GROUPS)


def _host_table(names, extents, values, pinned):
    """A host Arrow table in pinned memory: every key tuple of `extents`
    (first slowest) and a value per row, from a device tensor."""
    import pyarrow as pa
    import torch

    from einfold_b200 import synthetic as S

    def col(t):
        h = torch.empty(t.numel(), dtype=t.dtype, pin_memory=True)
        h.copy_(t.reshape(-1))
        pinned.append(h)
        return pa.Array.from_buffers(pa.int64() if t.dtype == torch.int64 else pa.float64(), t.numel(),
                                     [None, pa.foreign_buffer(h.data_ptr(), h.numel() * 8, base=h)])

    keys = S.grid_keys(extents, values.device)
    cols = [col(x) for x in keys] + [col(values)]
    del keys
    return pa.record_batch(cols, names=list(names) + ["x"])


def _cpu_fold_sample(a_cols, b_cols, rows=1024, cols=2048):
    """A bounded sample of the fold for the CPU: a's first `rows` values of i
    against b's first `cols` values of k, every j: 2·rows·n·cols FLOP."""
    import pyarrow as pa

    ai, aj, av = (t[: rows * N].cpu().numpy() for t in a_cols)
    bj, bk, bv = (t.view(N, N)[:, :cols].reshape(-1).cpu().numpy() for t in b_cols)
    a = pa.record_batch([pa.array(ai), pa.array(aj), pa.array(av)], names=["i", "j", "v"])
    b = pa.record_batch([pa.array(bj), pa.array(bk), pa.array(bv)], names=["j", "k", "v"])
    return a, b, 2.0 * rows * N * cols


def _cpu_attention_sample(q, k, v):
    """One (b, h) group of the attention as Arrow tables q(t, d, x), k(t, d, x),
    v(t, c, x) and the causal pipeline over them: 4·d·T(T+1)/2 FLOP."""
    import numpy as np
    import pyarrow as pa

    from einfold_b200 import ir

    t, d = np.indices((T, D)).reshape(2, -1)

    def table(x, names):
        return [pa.record_batch([pa.array(t), pa.array(d), pa.array(x.reshape(-1).cpu().numpy())], names=names)]

    e = ir.EQ
    producer = ir.Fold([e, e, e], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(2, 0), (1, 1)], 2)],
                       [ir.Output(0), ir.Output(2)]).with_conditions(
        [ir.Condition(0, ir.Comparison.GREATER_OR_EQUAL, 2, 0)])
    p = ir.Pipeline(producer, ir.Weight.exp(), [e], ir.Operand([(2, 0), (3, 1)], 2), [0, 3], ir.Normalizer.KEPT_GROUPS)
    return p, table(q[0], ["t", "d", "x"]), table(k[0], ["t", "d", "x"]), table(v[0], ["t", "c", "x"]), \
        4.0 * D * T * (T + 1) / 2


def _time_cpu_fold(a, b, threads, steps=1):
    from oracle import oracle

    f = _matmul_fold()
    s = oracle.schema(f, [a.schema, b.schema])
    opts = oracle.Options(threads=threads)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        out = oracle.dense_fold(f, [a], [b], None, s, opts)
        times.append(time.perf_counter() - t0)
        assert out is not None
    return times


def _time_cpu_attention(sample, threads, steps=1):
    from oracle import oracle

    p, q, k, v, _ = sample
    s = oracle.pipeline_schema(p, [q[0].schema, k[0].schema, v[0].schema])
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        out = oracle.pipeline(p, q, k, v, s, oracle.Options(threads=threads))
        times.append(time.perf_counter() - t0)
        assert out is not None
    return times


def _cpu_baseline(cols_a, cols_b, qkv, threads, steps):
    """The oracle's C restatements of dense::fold and fused::pipeline on a
    bounded sample of the step; FLOP per second over both."""
    a, b, fold_flops = _cpu_fold_sample(cols_a, cols_b)
    att = _cpu_attention_sample(*qkv)
    _time_cpu_fold(a, b, threads, 1)
    tf = _time_cpu_fold(a, b, threads, steps)
    ta = _time_cpu_attention(att, threads, steps)
    flops = (fold_flops + att[4]) * steps
    return flops / (sum(tf) + sum(ta)) / 1e12, 1e3 * (sum(tf) + sum(ta)) / steps


CPU_SAMPLE = ("dense fold 1024x8192 . 8192x2048 and the causal attention forward of one (b, h) group, "
              "T=4096, d=64 (oracle/ C restatements of dense::fold and fused::pipeline; the reference has "
              "no backward pass for its fused pipeline)")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle

    oracle.build()
    a_cols, b_cols = _tables("cpu")
    q, k, v, _ = _attention_inputs("cpu", groups=1)
    threads = os.cpu_count() or 1
    value, ms = _cpu_baseline(a_cols, b_cols, (q, k, v), threads, max(args.steps, 1))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"dense matrix-product fold {N}x{N} . {N}x{N} and causal attention "
                               f"B={B} H={H} T={T} d={D}; each step a bounded sample: " + CPU_SAMPLE,
                   "global_batch": 1, "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": threads, "kind": "port", "sample": CPU_SAMPLE},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _rel(a, b):
    return ((a - b).norm() / b.norm()).item()


def run_ours(args):
    import numpy as np
    import pyarrow as pa
    import torch

    from einfold_b200 import autograd as A
    from einfold_b200 import kernels as K

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def event():
        return torch.cuda.Event(enable_timing=True)

    f = _matmul_fold()
    (ai, aj, av), (bj, bk, bv) = _tables(dev)
    sa = pa.schema([("i", pa.int64()), ("j", pa.int64()), ("v", pa.float64())])
    sb = pa.schema([("j", pa.int64()), ("k", pa.int64()), ("v", pa.float64())])
    ra = K.DeviceRelation(sa, [ai, aj, av], device=local)
    rb = K.DeviceRelation(sb, [bj, bk, bv], device=local)
    opts = K.Options(slices=args.slices, device=local, result_on_device=True)
    q, k, v, d_out = _attention_inputs(dev)
    causal = A.causal()
    split, fp64 = K.Precision.SPLIT, K.Precision.FP64

    # One step; per component: the product kernels' time and digit ops, and
    # the kernels launched.
    stats = {"fold": [], "attn_fwd": [], "attn_bwd": []}
    launches = [0]
    fwd_launch = {}

    def note(name):
        stats[name].append((K.last_call.product_ms, K.last_call.product_ops))
        launches[0] += K.last_call.kernels_launched
        if name == "attn_fwd":
            fwd_launch.update(schedule=SCHEDULE_NAMES.get(K.last_call.schedule),
                              graph=GRAPH_NAMES.get(K.last_call.graph))

    def step(record=False):
        K.fold(f, ra, rb, options=opts).batches[0].release()
        if record:
            note("fold")
        out, lse = A.attention_forward(q, k, v, causal, 1.0, split)
        if record:
            note("attn_fwd")
        grads = A.attention_backward(q, k, v, out, lse, d_out, causal, 1.0, split)
        if record:
            note("attn_bwd")
        return out, grads

    # The plain FP64 GPU form of the same step, and the errors against it.
    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = event(), event()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    A_, B_ = av.view(N, N), bv.view(N, N)
    ref = torch.matmul(A_, B_)
    dgemm_ms = timed(lambda: torch.matmul(A_, B_, out=ref), 3)
    folded = K.fold(f, ra, rb, options=opts)
    got = folded.batches[0].column(2).view(N, N)
    fold_err = ((got - ref).abs().max() / ref.abs().max()).item()
    keys_ok = bool((folded.batches[0].column(0).view(N, N)[:, 0] == torch.arange(N, device=dev)).all()) and \
        bool((folded.batches[0].column(1).view(N, N)[0] == torch.arange(N, device=dev)).all())
    folded.batches[0].release()
    del ref, got

    mask = torch.ones(T, T, dtype=torch.bool, device=dev).tril()

    def torch_attention():
        qr, kr, vr = (t.detach().requires_grad_(True) for t in (q, k, v))
        s = (qr @ kr.transpose(-1, -2)).masked_fill(~mask, float("-inf"))
        out = torch.softmax(s, -1) @ vr
        grads = torch.autograd.grad(out, (qr, kr, vr), d_out)
        return out.detach(), grads

    torch_ms = timed(torch_attention, 1)
    out_t, grads_t = torch_attention()
    out_s, grads_s = step()
    attn_err = {"out": _rel(out_s, out_t), "d_q": _rel(grads_s[0], grads_t[0]), "d_k": _rel(grads_s[1], grads_t[1]),
                "d_v": _rel(grads_s[2], grads_t[2])}
    del out_t, grads_t, out_s, grads_s
    torch.cuda.empty_cache()

    # This library's FP64 form: the forward and backward kernels on the FP64
    # tensor pipe (mma.sync f64), the scores recomputed from the saved lse.
    fp64_state = {}

    def fp64_forward():
        fp64_state["out"], fp64_state["lse"] = A.attention_forward(q, k, v, causal, 1.0, fp64)

    def fp64_backward():
        A.attention_backward(q, k, v, fp64_state["out"], fp64_state["lse"], d_out, causal, 1.0, fp64)

    fp64_fwd_ms = timed(fp64_forward, 2)
    fp64_bwd_ms = timed(fp64_backward, 2)
    fp64_state.clear()

    def split_attention():
        out, lse = A.attention_forward(q, k, v, causal, 1.0, split)
        A.attention_backward(q, k, v, out, lse, d_out, causal, 1.0, split)

    split_attention_ms = timed(split_attention, 2)
    split_fold_ms = timed(lambda: K.fold(f, ra, rb, options=opts).batches[0].release(), 2)
    tiles_ms = fp64_fwd_ms + fp64_bwd_ms
    fp64_attention_ms = min(torch_ms, tiles_ms)
    fp64_step_ms = dgemm_ms + fp64_attention_ms

    for _ in range(args.warmup):
        step()
    barrier()
    with Clocks(local) as clocks:
        t0, t1 = event(), event()
        barrier()
        t0.record()
        for _ in range(args.steps):
            step(record=True)
        t1.record()
        barrier()
    ms = max_over_ranks(t0.elapsed_time(t1), dist, dev)
    ms_per_step = ms / args.steps
    flops = FOLD + ATT_FWD + ATT_BWD
    value = replicas_value(world, flops, args.steps, ms)

    # End to end: the public API from pinned host memory, results read back:
    # the fold through einfold_fold from host Arrow tables, attention through
    # einfold_pipeline (forward) and einfold_pipeline_backward (gradients,
    # which recomputes the forward for its log-sum-exp) from host Arrow
    # tables q, k, v and d_out of 16.8M rows each.
    e2e = None
    if not args.no_e2e:
        pinned = []

        def host_col(t):
            h = torch.empty(t.numel(), dtype=t.dtype, pin_memory=True)
            h.copy_(t)
            pinned.append(h)
            return pa.Array.from_buffers(pa.int64() if t.dtype == torch.int64 else pa.float64(), t.numel(),
                                         [None, pa.foreign_buffer(h.data_ptr(), h.numel() * 8, base=h)])

        ha = pa.record_batch([host_col(ai), host_col(aj), host_col(av)], schema=sa)
        hb = pa.record_batch([host_col(bj), host_col(bk), host_col(bv)], schema=sb)
        ext = [B, H, T, D]
        hq = _host_table(["b", "h", "t", "d"], ext, q, pinned)
        hk = _host_table(["b", "h", "t", "d"], ext, k, pinned)
        hv = _host_table(["b", "h", "t", "c"], ext, v, pinned)
        hd = _host_table(["b", "h", "t", "c"], ext, d_out, pinned)
        pipe = _attention_pipeline()
        hopts = K.Options(slices=args.slices, device=local)
        rel = lambda t: K.Relation(t.schema, [t])
        phases = {}

        def e2e_step(record=False):
            res = K.fold(f, K.Relation(sa, [ha]), K.Relation(sb, [hb]), options=hopts)
            if record:
                phases["fold_ms"] = K.last_call.device_ms
            piped = K.pipeline(pipe, [rel(hq), rel(hk), rel(hv)], options=hopts)
            if record:
                phases["pipeline_ms"] = K.last_call.device_ms
                phases["pipeline_product_ms"] = K.last_call.product_ms
            grads = K.pipeline_backward(pipe, [rel(hq), rel(hk), rel(hv)], rel(hd), options=hopts)
            if record:
                phases["pipeline_backward_ms"] = K.last_call.device_ms
                phases["pipeline_backward_product_ms"] = K.last_call.product_ms
            return res, piped, grads

        res, piped, grads = e2e_step(record=True)
        assert piped is not None and grads is not None, K.last_call.message
        outs = list(res.batches) + list(piped.batches) + [b for g in grads for b in g]
        d2h = sum(buf.size for batch in outs for col in batch.columns for buf in col.buffers() if buf)
        h2d = sum(buf.size for batch in (ha, hb, hq, hk, hv, hq, hk, hv, hd) for col in batch.columns
                  for buf in col.buffers() if buf)
        # The same attention output as the device-array leg's (bits).
        o_host = np.asarray(piped.batches[0].column(4).to_numpy(zero_copy_only=False))
        o_dev = A.attention_forward(q, k, v, causal, 1.0, split)[0].reshape(-1).cpu().numpy()
        same_as_kernel_leg = bool(np.array_equal(o_host.view(np.uint64), o_dev.view(np.uint64)))
        # (no view of a result may outlive this: it would keep the result's
        # pinned buffers from the library's pool while the timed steps run)
        del res, piped, grads, outs, o_host, o_dev
        e2e_steps = max(1, min(args.steps, 3))
        barrier()
        t0.record()
        for i in range(e2e_steps):
            out_ = e2e_step(record=i == e2e_steps - 1)
            del out_
        t1.record()
        barrier()
        ems = max_over_ranks(t0.elapsed_time(t1), dist, dev)
        # Per call of the last timed step: each call's time on the device
        # (its copies in and out of pinned host memory included) and, for
        # attention, its product kernels' share; the rest of an attention
        # call is staging, placement and the result's assembly.
        phases["attention_staging_placement_and_result_ms"] = (
            phases["pipeline_ms"] - phases["pipeline_product_ms"] + phases["pipeline_backward_ms"] -
            phases["pipeline_backward_product_ms"])
        e2e = {"value": replicas_value(world, flops, e2e_steps, ems), "unit": "TFLOP/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
               "ms_per_step": ems / e2e_steps,
               "path": "einfold_fold + einfold_pipeline + einfold_pipeline_backward from host Arrow tables "
                       "(a(i,j,v), b(j,k,v) 67.1M rows; q, k, v, d_out 16.8M rows), results to host Arrow",
               "phases_ms": phases, "attention_out_same_bits_as_device_array_leg": same_as_kernel_leg}
        del ha, hb, hq, hk, hv, hd, pinned

    # Rooflines of the three product kernels: digit ops executed on the
    # tensor cores per second against the int8 dense peak.
    bf16, hbm, basis = _peaks()
    int8_peak = 2.0 * bf16
    names = {"fold": "split_gemm_kernel<6>", "attn_fwd": "attn_fwd_split<6,1>",
             "attn_bwd": "grad_split<d_k> + grad_tiles<d_v> + grad_tiles<d_q>"}
    kernels = {}
    for key, recs in stats.items():
        p_ms = statistics.mean(r[0] for r in recs)
        p_ops = statistics.mean(r[1] for r in recs)
        achieved = p_ops / (p_ms / 1e3) / 1e12 if p_ms else None
        kernels[key] = {"kernel": names[key], "ms": p_ms, "ops_per_step": p_ops, "achieved": achieved,
                        "frac": achieved / int8_peak if achieved else None, "share": p_ms / ms_per_step}
    top = max(kernels, key=lambda k_: kernels[k_]["ms"])
    roofline = {"bound": "tensor", "kernel": kernels[top]["kernel"], "achieved": kernels[top]["achieved"],
                "peak": int8_peak, "unit": "TFLOP/s", "frac": kernels[top]["frac"],
                "traffic": _profiled_traffic(top), "peak_basis": f"int8 dense = 2 x {basis} bf16 burst ({bf16} TFLOP/s)",
                "kernel_ms": kernels[top]["ms"], "ops_per_launch": kernels[top]["ops_per_step"], "kernels": kernels}

    ranking = _ranking(hbm, basis) if not args.no_ranking else None
    ragged = _ragged() if not args.no_ragged else None
    sparse = _sparse(cpu=rank == 0 and world == 1 and not args.no_cpu) if not args.no_sparse else None
    smoother = _smoother(cpu=rank == 0 and world == 1 and not args.no_cpu) if not args.no_smoother else None
    small_fold = _small_fold(cpu=rank == 0 and world == 1 and not args.no_cpu) if not args.no_small_fold else None
    gradients = _gradients() if not args.no_gradients else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle

        oracle.build()
        threads = os.cpu_count() or 1
        cval, _ = _cpu_baseline((ai, aj, av), (bj, bk, bv), (q[:1].cpu(), k[:1].cpu(), v[:1].cpu()), threads, 1)
        cpu = {"value": cval, "unit": "TFLOP/s", "cores": threads, "kind": "port", "sample": CPU_SAMPLE}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int8 slices (exact int32 sums) -> f64", "data": "synthetic",
            "config": {"workload": f"dense matrix-product fold {N}x{N} . {N}x{N} through einfold_fold (a(i,j,v), "
                                   f"b(j,k,v), {N * N} rows each, FP64 uniform[-1,1]) + causal attention "
                                   f"B={B} H={H} T={T} d={D} forward and backward (values normal(0,1/8), "
                                   f"d_out normal(0,1)), SplitMix64 seed 0",
                       "flop_per_step": {"fold": FOLD, "attention_forward": ATT_FWD, "attention_backward": ATT_BWD},
                       "slices": args.slices, "l2": "inputs larger than L2 (3.2 GB of tables, 0.5 GB of q,k,v,d_out)",
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "errors_vs_fp64": {"fold_max_rel": fold_err, "attention_norm_rel": attn_err},
                       "keys_exact": keys_ok},
            "fp64_gpu": {"value": flops / (fp64_step_ms / 1e3) / 1e12, "unit": "TFLOP/s", "ms": fp64_step_ms,
                         "form": "cuBLAS DGEMM (fold) + the faster of torch float64 attention (unfused, with "
                                 "autograd) and this library's FP64 attention on the FP64 tensor pipe",
                         "fold_dgemm_ms": dgemm_ms, "attention_torch_f64_ms": torch_ms,
                         "attention_fp64_mma_ms": tiles_ms,
                         "attention_fp64_mma_forward_ms": fp64_fwd_ms, "attention_fp64_mma_backward_ms": fp64_bwd_ms,
                         "attention_fp64_mma_tflops": (ATT_FWD + ATT_BWD) / (tiles_ms / 1e3) / 1e12,
                         "attention_split_ms": split_attention_ms,
                         "ratio_attention_split_over_fp64_mma": tiles_ms / split_attention_ms,
                         "ratio_fold_split_over_dgemm": dgemm_ms / split_fold_ms, "fold_split_ms": split_fold_ms,
                         "ratio_split_over_fp64": fp64_step_ms / ms_per_step},
            "roofline": roofline,
            "ranking": ranking,
            "ragged": ragged,
            "sparse": sparse,
            "smoother": smoother,
            "small_fold": small_fold,
            "gradients": gradients,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "attention_forward_launch": fwd_launch,
            "gpu_launches": launches[0],
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def _ranking(hbm, basis):
    """einfold_rank_words on random 64-bit keys (each drawn from a pool of
    n/2), timed with CUDA events: 2^28 keys (passes of 6 GB, beyond L2) and
    4M keys (the sorting path's join column over a and b). Two fractions of
    HBM bandwidth: over the bytes the kernels move, per key 8 read for the
    byte histograms, per 8-bit pass 12 read and 12 written (the first pass
    reads no row numbers), then 12 read and 4 written for the ranks (beyond
    4M keys 8 more written and read again: the (row, rank) pairs partitioned
    by row bucket) plus 4 per distinct key for the first rows; and over the
    algorithmic bytes of
    the ranking itself, 8 B of key read, 4 B of rank and 4 B of first row
    written per key."""
    import ctypes

    import torch

    from einfold_b200 import _lib
    from einfold_b200 import synthetic as S

    lib = _lib.load()
    out = {}
    for n in (1 << 28, 1 << 22):
        pool = S.u64(SEED, 7, n // 2)
        words = pool[(S.u64(SEED, 8, n) % (n // 2)).to(torch.int64)].contiguous()
        del pool
        w64 = words.view(torch.int64)
        varying = 0
        for b in range(8):
            byte = (w64 >> (8 * b)) & 255
            varying += int(byte.min().item() != byte.max().item())
            del byte
        rank_ = torch.empty(n, dtype=torch.int32, device="cuda")
        first = torch.empty(n, dtype=torch.int32, device="cuda")
        k = ctypes.c_int64(0)
        times = []
        for _ in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            st = lib.einfold_rank_words(_lib.context(torch.cuda.current_device()), words.data_ptr(), n,
                                        rank_.data_ptr(), first.data_ptr(), ctypes.byref(k), None)
            e1.record()
            torch.cuda.synchronize()
            assert st == _lib.OK
            times.append(e0.elapsed_time(e1))
        ms = statistics.median(times[1:])
        passes = varying
        finish = 32 if n > (1 << 22) else 16
        moved = n * (8 + (20 + (passes - 1) * 24 if passes else 0) + finish) + k.value * 4
        algorithmic = n * 16
        out[f"n{n}"] = {"keys": n, "distinct": k.value, "ms": ms, "gkeys_per_s": n / ms / 1e6, "passes": passes,
                        "moved_gb_per_s": moved / ms / 1e6, "frac_of_hbm": moved / ms / 1e6 / hbm,
                        "algorithmic_gb_per_s": algorithmic / ms / 1e6,
                        "frac_of_hbm_algorithmic": algorithmic / ms / 1e6 / hbm}
        del words, rank_, first, w64
        torch.cuda.empty_cache()
    out["peak"] = {"hbm_gb_per_s": hbm, "basis": basis}
    return out


def _ragged():
    """Ragged batches (64 groups, d=128, lengths log-uniform in [128, 8192],
    window |tq - tk| <= 512, values normal(0, 1/sqrt(128)), padded to the
    longest): the attention forward in the split form (the query tiles that
    join some key, under the launch schedule its first call timed fastest,
    replayed from a CUDA graph) and in the FP64 form, timed with CUDA
    events, FLOP = 4·d per allowed pair; the split result's error against
    the FP64 one (max |diff| / max |out|); the split forward under each
    schedule."""
    import torch

    from einfold_b200 import autograd as A
    from einfold_b200 import cases as C
    from einfold_b200 import kernels as K
    from einfold_b200.kernels import Precision

    groups, d, radius = 64, 128, 512
    q, k, v, lengths = C.ragged_inputs(groups, d, seed=SEED)
    flop = 4.0 * d * C.allowed_pairs(lengths, radius)
    out = {"groups": groups, "d": d, "window": radius, "rows": int(lengths.sum()), "padded_to": int(lengths.max()),
           "flop": flop}
    results = {}
    for name, prec in (("split", Precision.SPLIT), ("fp64", Precision.FP64)):
        # An untimed first call: the split form times its launch schedules on
        # a shape's first call.
        A.attention_forward(q, k, v, A.window(radius), d ** -0.5, prec, q_lengths=lengths, k_lengths=lengths)
        times, o = [], None
        for _ in range(4):
            o = None  # the previous output's memory back to torch's cache before the call
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            o, _ = A.attention_forward(q, k, v, A.window(radius), d ** -0.5, prec, q_lengths=lengths,
                                       k_lengths=lengths)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        results[name] = o
        ms = statistics.median(times)
        out[name] = {"ms": ms, "tflop_per_s": flop / ms / 1e9}
    seen = ~torch.isnan(results["fp64"])
    out["split_max_rel_err"] = ((results["split"][seen] - results["fp64"][seen]).abs().max() /
                                results["fp64"][seen].abs().max()).item()
    out["ratio_split_over_fp64"] = out["fp64"]["ms"] / out["split"]["ms"]
    # The split forward under each launch schedule (forced), against the one
    # its first call timed fastest.
    A.attention_forward(q, k, v, A.window(radius), d ** -0.5, Precision.SPLIT, q_lengths=lengths, k_lengths=lengths)
    out["tuned_schedule"] = SCHEDULE_NAMES.get(K.last_call.schedule)
    out["graph"] = GRAPH_NAMES.get(K.last_call.graph)
    out["schedules_ms"] = {}
    try:
        for name in ("grid", "tiles", "batches"):
            os.environ["EINFOLD_ATTENTION_SCHEDULE"] = name
            times = []
            for _ in range(4):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                A.attention_forward(q, k, v, A.window(radius), d ** -0.5, Precision.SPLIT, q_lengths=lengths,
                                    k_lengths=lengths)
                e1.record()
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1))
            out["schedules_ms"][name] = statistics.median(times[1:])
    finally:
        os.environ.pop("EINFOLD_ATTENTION_SCHEDULE", None)
    del q, k, v, results
    torch.cuda.empty_cache()
    return out


def _sparse_tables():
    """The sorting path's tables at 1/40 of their size (synthetic.sorting_tables:
    a(i, j, v) and b(j, k, v), 50,000 rows each; i and k 16-hex-digit strings
    from 50,000 distinct, j 63-bit hashes from a pool of 200,000 drawn with
    Zipf(1.1) frequencies, v normal(0, 1)), and the regridding variant's
    weight table at 1/40 (w(src, dst, wt), 100,000 rows, src from the same
    pool and law, dst from 50,000 int64 cells, wt uniform[0, 1))."""
    import pyarrow as pa

    from einfold_b200 import synthetic as S

    a, b = S.sorting_tables(50_000, seed=SEED)
    wt = S.regrid_table(100_000, seed=SEED)
    w = pa.record_batch([wt.column(0), wt.column(1), wt.column(2)], names=["j", "k", "v"])
    pairs = S.joined_pairs(a.column(1).to_numpy(), b.column(0).to_numpy())
    regrid_pairs = S.joined_pairs(a.column(1).to_numpy(), w.column(0).to_numpy())
    return a, b, pairs, w, regrid_pairs


def _sparse(cpu=False):
    """The discrimination fold (ranking, counting sorts, the Gustavson
    product, grouped output) on the sorting path's tables scaled to 50,000
    rows an operand, and on the regridding variant (a weighted by w on
    j = src, grouped by i and dst), results left in HBM, timed with CUDA
    events: pair products (one per pair of rows joining on j) per second."""
    import torch

    from einfold_b200 import kernels as K

    a, b, pairs, w, regrid_pairs = _sparse_tables()
    f = _matmul_fold()
    opts = K.Options(result_on_device=True)

    def run(left, right, n_pairs):
        ra, rb = K.Relation(left.schema, [left]), K.Relation(right.schema, [right])
        times, groups, alg = [], 0, None
        for _ in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            got = K.fold(f, ra, rb, options=opts)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            alg = got.algorithm.name.lower()
            groups = sum(batch.rows for batch in got.batches)
            for batch in got.batches:
                batch.release()
        ms = statistics.median(times[1:])
        return {"rows": [left.num_rows, right.num_rows], "pairs": n_pairs, "groups": groups, "algorithm": alg,
                "ms": ms, "gpairs_per_s": n_pairs / ms / 1e6,
                "host_to_device": "the Arrow tables are copied in each call"}

    out = run(a, b, pairs)
    out["rows_per_operand"] = a.num_rows
    out["regrid"] = run(a, w, regrid_pairs)
    if cpu:
        # The CPU baseline leg: the oracle's restatement of discriminate::fold
        # (one host thread), on the same tables.
        from oracle import oracle

        oracle.build()
        t0 = time.perf_counter()
        want = oracle.fold(f, a.schema, [a], b.schema, [b], None, oracle.schema(f, [a.schema, b.schema]))
        sec = time.perf_counter() - t0
        out["cpu_oracle"] = {"seconds": sec, "gpairs_per_s": pairs / sec / 1e9, "cores": 1,
                             "groups": sum(x.num_rows for x in want.batches)}
    return out


def _smoother(cpu=False):
    """The Gaussian smoother: per group (64), 2^20
    query positions x and 256 key positions y uniform[0, 1) and values v
    normal(0, 1); out(b, x) = sum_y w v / sum_y w with FP64 weights
    w = exp(-power(x - y, 2) / h), h = 0.01, as a pipeline whose scores are
    the row expression -power(q.x - k.x, 2) over one feature and whose
    weight is exp(s / h) without a shift. The tables (b, t, d, x) are in
    HBM (2.1 GB of q); the result stays there. Pairs per second, timed with
    CUDA events; the error of group 0's first 4,096 rows against torch
    float64."""
    import pyarrow as pa
    import torch

    from einfold_b200 import cases as C
    from einfold_b200 import kernels as K

    groups, nx, ny, h = 64, 1 << 20, 256, 0.01
    pipe = C.smoother_pipeline(h)
    q, k, v, xs, ys, vs = C.smoother_tables(groups, nx, ny, SEED)
    pairs = groups * nx * ny
    opts = K.Options(result_on_device=True)
    times, got = [], None
    for _ in range(4):
        if got is not None:
            for batch in got.batches:
                batch.release()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        got = K.pipeline(pipe, [q, k, v], options=opts)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = statistics.median(times[1:])
    vals = got.batches[0].column(2)
    rows = 4096
    x0, y0, v0 = xs[:rows], ys[:ny], vs[:ny]
    w = torch.exp(-(x0[:, None] - y0[None, :]) ** 2 / h)
    want = (w @ v0) / w.sum(1)
    err = ((vals[:rows] - want).abs().max() / want.abs().max()).item()
    out = {"groups": groups, "x_per_group": nx, "y_per_group": ny, "h": h, "pairs": pairs, "ms": ms,
           "gpairs_per_s": pairs / ms / 1e6, "rows_out": sum(b.rows for b in got.batches),
           "tiles_visited": got.tiles_visited, "max_rel_err_vs_torch_f64": err,
           "kernel": "fused_unshifted (FP64 scores and weights on the CUDA cores, no per-tile reductions)"}
    for batch in got.batches:
        batch.release()
    if cpu:
        # The CPU leg: the oracle's restatement of fused::pipeline on group
        # 0's first 16,384 positions (one host thread a call).
        from oracle import oracle

        oracle.build()
        n = 16384

        def host(cols, names):
            return [pa.record_batch([pa.array(c.cpu().numpy()) for c in cols], names=names)]

        zeros = torch.zeros(n, dtype=torch.int64)
        qa = host([zeros, torch.arange(n), zeros, xs[:n]], ["b", "t", "d", "x"])
        ka = host([zeros[:ny], torch.arange(ny), zeros[:ny], ys[:ny]], ["b", "t", "d", "x"])
        va = host([zeros[:ny], torch.arange(ny), vs[:ny]], ["b", "t", "x"])
        schema = oracle.pipeline_schema(pipe, [qa[0].schema, ka[0].schema, va[0].schema])
        t0 = time.perf_counter()
        oracle.pipeline(pipe, qa, ka, va, schema, oracle.Options(threads=1))
        sec = time.perf_counter() - t0
        out["cpu_oracle"] = {"seconds": sec, "pairs": n * ny, "gpairs_per_s": n * ny / sec / 1e9, "cores": 1}
    del q, k, v, xs, ys, vs
    torch.cuda.empty_cache()
    return out


def _small_fold(cpu=False):
    """The plain matmul fold at 512 x 512 . 512 x 256 (2·512·512·256 FLOP)
    through einfold_fold from host Arrow tables (rows shuffled, four batches
    an operand) to host results, timed end to end on the host clock around
    each call (the copies in, the kernels, the copies out): with 1% of b's
    values NULL (the reference sends that to its discrimination algorithm,
    and so does this library) and complete (the dense product). The CPU leg
    runs the oracle's restatement of the same fold on one host thread."""
    import torch

    from einfold_b200 import cases as C
    from einfold_b200 import kernels as K

    f = _matmul_fold()
    flop = 2.0 * 512 * 512 * 256
    out = {"flop": flop}
    for name, nulls in (("nulls_in_b", True), ("complete", False)):
        (sa, a), (sb, b) = C.small_fold_tables(nulls, SEED)
        ra, rb = K.Relation(sa, a), K.Relation(sb, b)
        times, device_ms, got = [], [], None
        for _ in range(6):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            got = K.fold(f, ra, rb)
            torch.cuda.synchronize()
            times.append((time.perf_counter() - t0) * 1e3)
            device_ms.append(K.last_call.device_ms)
        ms = statistics.median(times[1:])
        leg = {"algorithm": got.algorithm.name.lower(), "rows_out": sum(x.num_rows for x in got.batches),
               "e2e_ms": ms, "e2e_gflop_per_s": flop / ms / 1e6, "device_ms": statistics.median(device_ms[1:])}
        if cpu:
            from oracle import oracle

            oracle.build()
            t0 = time.perf_counter()
            want = oracle.fold(f, sa, a, sb, b, None, oracle.schema(f, [sa, sb]))
            sec = time.perf_counter() - t0
            leg["cpu_oracle"] = {"seconds": sec, "gflop_per_s": flop / sec / 1e9, "cores": 1,
                                 "rows_out": sum(x.num_rows for x in want.batches)}
        out[name] = leg
    return out


def _gradients():
    """The gradient shapes at their own sizes: the causal attention backward
    at B=2 H=16 T=2048 d=64 (q, k, v normal(0, 1/8), d_out normal(0, 1);
    FLOP 2.5 x the forward's 4·B·H·T²·d·(T+1)/(2T)) and the matmul fold's
    forward and gradients at 4096² (dA = dC·Bᵀ, dB = Aᵀ·dC: 3 x 2·4096³
    FLOP; a, b uniform[-1, 1], dC normal(0, 1)), each in the split form and
    the FP64 forms, timed with CUDA events (median of 3 after a first call),
    with the split results' normwise errors against the FP64 ones."""
    import torch

    from einfold_b200 import autograd as A
    from einfold_b200 import synthetic as S
    from einfold_b200.kernels import Precision

    def timed(fn):
        fn()
        times = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = fn()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        return statistics.median(times), r

    def rel(x, y):
        return ((x - y).norm() / y.norm()).item()

    b_, h_, t_, d_ = 2, 16, 2048, 64
    n = b_ * h_ * t_ * d_
    q, k, v = (S.normal(SEED, salt, n, 1.0 / 8).view(b_, h_, t_, d_) for salt in (41, 42, 43))
    d_out = S.normal(SEED, 44, n, 1.0).view(b_, h_, t_, d_)
    causal = A.causal()
    bwd_flop = 2.5 * 4.0 * b_ * h_ * t_ * t_ * d_ * (t_ + 1) / (2 * t_)
    att = {"shape": {"B": b_, "H": h_, "T": t_, "d": d_}, "flop": bwd_flop}
    grads = {}
    for name, prec in (("split", Precision.SPLIT), ("fp64_tensor_pipe", Precision.FP64)):
        out, lse = A.attention_forward(q, k, v, causal, 1.0, prec)
        ms, g = timed(lambda: A.attention_backward(q, k, v, out, lse, d_out, causal, 1.0, prec))
        grads[name] = g
        att[name] = {"ms": ms, "tflop_per_s": bwd_flop / ms / 1e9}
    att["split_norm_rel_err"] = {x: rel(a, b) for x, a, b in zip(("d_q", "d_k", "d_v"), grads["split"],
                                                                   grads["fp64_tensor_pipe"])}
    att["ratio_split_over_fp64"] = att["fp64_tensor_pipe"]["ms"] / att["split"]["ms"]
    del q, k, v, d_out, grads
    m = 4096
    a = S.uniform(SEED, 45, m * m).view(m, m)
    b = S.uniform(SEED, 46, m * m).view(m, m)
    dc = S.normal(SEED, 47, m * m).view(m, m)
    mm_flop = 3 * 2.0 * m ** 3
    mm = {"n": m, "flop": mm_flop}
    res = {}
    for name, prec in (("split", Precision.SPLIT), ("fp64_reference_order", Precision.FP64), ("cublas_dgemm", None)):
        def step():
            x, y = a.clone().requires_grad_(), b.clone().requires_grad_()
            c = A.matmul(x, y, prec) if prec is not None else x @ y
            c.backward(dc)
            return c.detach(), x.grad, y.grad
        ms, r = timed(step)
        res[name] = r
        mm[name] = {"ms": ms, "tflop_per_s": mm_flop / ms / 1e9}
    mm["split_norm_rel_err"] = {x: rel(p_, q_) for x, p_, q_ in zip(("c", "d_a", "d_b"), res["split"],
                                                                     res["cublas_dgemm"])}
    mm["ratio_split_over_dgemm"] = mm["cublas_dgemm"]["ms"] / mm["split"]["ms"]
    del a, b, dc, res
    torch.cuda.empty_cache()
    return {"attention_backward": att, "matmul_gradients": mm}


def _profiled_traffic(component):
    """DRAM bytes per step of a component's product kernel, from the committed
    ncu summary (`traffic_bytes_per_launch:` line), or None."""
    files = {"fold": "split_gemm_kernel_matmul8192.txt", "attn_fwd": "attn_fwd_split_causal_T4096.txt",
             "attn_bwd": "attention_backward_kernels_causal_T4096.txt"}
    path = os.path.join(ROOT, "profiles", files[component])
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--slices", type=int, default=6)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-ranking", action="store_true")
    p.add_argument("--no-ragged", action="store_true")
    p.add_argument("--no-sparse", action="store_true")
    p.add_argument("--no-smoother", action="store_true")
    p.add_argument("--no-small-fold", action="store_true")
    p.add_argument("--no-gradients", action="store_true")
    args = p.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
