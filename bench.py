"""Benchmark of einfold's kernel layer on B200s.

One step is one dense matrix-product fold of 8192x8192 by 8192x8192 FP64
tables through the C ABI (``SUM(a.v * b.v) ... GROUP BY a.i, b.k`` over
a(i, j, v) and b(j, k, v), 67.1M rows each), computed in the split form:
int8 slices on the tensor cores with exact integer sums and an FP64 combine.
The metric is its FP64-equivalent throughput (2·n³ per step), next to the
plain FP64 GPU form (cuBLAS DGEMM on the same matrices) and the error against
it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (under torchrun, one process per GPU) every rank folds its own
tables: replicas, no collective on the data path. ``--impl reference`` times
the reference's CPU algorithm (its C restatement in ``oracle/``, as the
reference's Rust can't be built here) on a bounded sample of the same fold.
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
SEED = 0


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


def _matmul_fold():
    from einfold_b200 import ir

    e = ir.EQ
    return ir.Fold([e, e, e], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)],
                   [ir.Output(0), ir.Output(2)])


def _tables(device):
    """a(i, j, v) and b(j, k, v) on the device, keys in row-major order, v
    uniform[-1, 1] from SplitMix64 (seed 0; salts 1 and 2)."""
    import torch

    from einfold_b200 import synthetic as S

    i, j = S.grid_keys([N, N], device)
    av = S.uniform(SEED, 1, N * N, device=device)
    bv = S.uniform(SEED, 2, N * N, device=device)
    if str(device).startswith("cuda"):
        torch.cuda.synchronize()
    return (i, j, av), (i.clone(), j.clone(), bv)


def _cpu_sample(a_cols, b_cols, rows=1024, cols=2048):
    """A bounded sample of the fold for the CPU: a's first `rows` values of i
    against b's first `cols` values of k, every j: 2·rows·n·cols FLOP."""
    import numpy as np
    import pyarrow as pa

    ai, aj, av = (t[: rows * N].cpu().numpy() for t in a_cols)
    bj, bk, bv = (t.view(N, N)[:, :cols].reshape(-1).cpu().numpy() for t in b_cols)
    a = pa.record_batch([pa.array(ai), pa.array(aj), pa.array(av)], names=["i", "j", "v"])
    b = pa.record_batch([pa.array(bj), pa.array(bk), pa.array(bv)], names=["j", "k", "v"])
    return a, b, 2.0 * rows * N * cols


def _time_cpu(a, b, flops, threads, steps=1):
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


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch

    from oracle import oracle

    oracle.build()
    a_cols, b_cols = _tables("cpu")
    a, b, flops = _cpu_sample(a_cols, b_cols)
    threads = os.cpu_count() or 1
    _time_cpu(a, b, flops, threads, steps=args.warmup)
    times = _time_cpu(a, b, flops, threads, steps=args.steps)
    t = sum(times)
    value = flops * len(times) / t / 1e12
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"dense matrix-product fold {N}x{N} . {N}x{N}, FP64 uniform[-1,1] (seed 0); "
                               f"each step a bounded sample: 1024 values of i x 2048 of k, every j",
                   "global_batch": 1, "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": threads, "kind": "port",
                         "sample": "dense fold 1024x8192 . 8192x2048 (oracle/ C restatement of dense::fold)"},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import pyarrow as pa
    import torch

    from einfold_b200 import kernels as K

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
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

    f = _matmul_fold()
    (ai, aj, av), (bj, bk, bv) = _tables(f"cuda:{local}")
    sa = pa.schema([("i", pa.int64()), ("j", pa.int64()), ("v", pa.float64())])
    sb = pa.schema([("j", pa.int64()), ("k", pa.int64()), ("v", pa.float64())])
    ra = K.DeviceRelation(sa, [ai, aj, av], device=local)
    rb = K.DeviceRelation(sb, [bj, bk, bv], device=local)
    opts = K.Options(slices=args.slices, device=local, result_on_device=True)
    flops = 2.0 * N ** 3

    # The plain FP64 GPU form: cuBLAS DGEMM on the same matrices, and the error.
    A = av.view(N, N)
    B = bv.view(N, N)
    ref = torch.matmul(A, B)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(3):
        torch.matmul(A, B, out=ref)
    e1.record()
    torch.cuda.synchronize()
    fp64_ms = e0.elapsed_time(e1) / 3
    out = K.fold(f, ra, rb, options=opts)
    got = out.batches[0].column(2).view(N, N)
    err = ((got - ref).abs().max() / ref.abs().max()).item()
    keys_ok = bool((out.batches[0].column(0).view(N, N)[:, 0] == torch.arange(N, device=got.device)).all()) and \
        bool((out.batches[0].column(1).view(N, N)[0] == torch.arange(N, device=got.device)).all())
    out.batches[0].release()
    del ref, got

    for _ in range(args.warmup):
        K.fold(f, ra, rb, options=opts).batches[0].release()
    barrier()
    product_ms, product_ops, launches = [], [], 0
    with Clocks(local) as clocks:
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        t0.record()
        for _ in range(args.steps):
            r = K.fold(f, ra, rb, options=opts)
            product_ms.append(K.last_call.product_ms)
            product_ops.append(K.last_call.product_ops)
            launches += K.last_call.kernels_launched
            r.batches[0].release()
        t1.record()
        barrier()
    ms = t0.elapsed_time(t1)
    if dist is not None:
        tt = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    ms_per_step = ms / args.steps
    value = world * flops * args.steps / (ms / 1e3) / 1e12

    # End to end: the public API with host Arrow buffers in pinned memory.
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
        hopts = K.Options(slices=args.slices, device=local)
        res = K.fold(f, K.Relation(sa, [ha]), K.Relation(sb, [hb]), options=hopts)
        d2h = sum(buf.size for batch in res.batches for col in batch.columns for buf in col.buffers() if buf)
        h2d = sum(buf.size for batch in (ha, hb) for col in batch.columns for buf in col.buffers() if buf)
        del res
        e2e_steps = max(1, min(args.steps, 3))
        barrier()
        t0.record()
        for _ in range(e2e_steps):
            res = K.fold(f, K.Relation(sa, [ha]), K.Relation(sb, [hb]), options=hopts)
            del res
        t1.record()
        barrier()
        ems = t0.elapsed_time(t1)
        if dist is not None:
            tt = torch.tensor([ems], device=f"cuda:{local}")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ems = float(tt.item())
        e2e = {"value": world * flops * e2e_steps / (ems / 1e3) / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
               "ms_per_step": ems / e2e_steps}
        del ha, hb, pinned

    bf16, hbm, basis = _peaks()
    int8_peak = 2.0 * bf16
    p_ms = statistics.mean(product_ms) if product_ms else None
    p_ops = statistics.mean(product_ops) if product_ops else None
    achieved = p_ops / (p_ms / 1e3) / 1e12 if p_ms else None
    traffic = _profiled_traffic()
    roofline = {"bound": "tensor", "kernel": "split_gemm_kernel<6>", "achieved": achieved, "peak": int8_peak,
                "unit": "TFLOP/s", "frac": achieved / int8_peak if achieved else None, "traffic": traffic,
                "peak_basis": f"int8 dense = 2 x {basis} bf16 burst ({bf16} TFLOP/s)",
                "kernel_ms": p_ms, "ops_per_launch": p_ops}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle

        oracle.build()
        a, b, sflops = _cpu_sample((ai, aj, av), (bj, bk, bv))
        threads = os.cpu_count() or 1
        times = _time_cpu(a, b, sflops, threads, steps=1)
        cpu = {"value": sflops / times[0] / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": "port",
               "sample": "dense fold 1024x8192 . 8192x2048 (oracle/ C restatement of dense::fold)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int8 slices (exact int32 sums) -> f64", "data": "synthetic",
            "config": {"workload": f"dense matrix-product fold {N}x{N} . {N}x{N} through einfold_fold, "
                                   f"a(i,j,v) and b(j,k,v) with {N * N} rows each, FP64 uniform[-1,1] (seed 0)",
                       "slices": args.slices, "l2": "inputs larger than L2 (3.2 GB of tables per step)",
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "max_rel_error_vs_fp64": err, "keys_exact": keys_ok},
            "fp64_gpu": {"value": flops / (fp64_ms / 1e3) / 1e12, "unit": "TFLOP/s", "form": "cuBLAS DGEMM (torch)",
                         "ms": fp64_ms, "ratio_split_over_fp64": (flops / (ms_per_step / 1e3)) / (flops / (fp64_ms / 1e3))},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def _profiled_traffic():
    """DRAM bytes per launch of the product kernel, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "split_gemm_kernel_matmul8192.txt")
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
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--slices", type=int, default=6)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    args = p.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
