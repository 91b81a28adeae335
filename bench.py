#!/usr/bin/env python
"""Benchmark of the B200 hash groupby (libgbx) on the 100M-row workload.

Workload (one "step"): four plain groupbys of 100,000,000 rows each, one per
key cardinality C in {1e2, 1e4, 1e6, 1e8}: int64 key uniform over C values;
value `a` int64 uniform in [-1e6, 1e6]; value `b` float32 ~N(0,1) with 10%
nulls; SUM, COUNT, MIN, MAX, MEAN, VAR on both values.  Inputs are seeded
synthetic data (no public dataset), generated on the device.  Inputs (2.01 GB
per groupby) are larger than L2 (126 MB), so no L2 flush is needed.

  value  -- rows/s over the whole job with inputs resident in HBM, through the
            public API (cudf_b200.GroupBy.aggregate), CUDA events on the stream
  e2e    -- same metric with host (pinned) inputs: every step copies inputs
            host->device and reads all results back device->host, the four
            calls pipelined over PCIe (uploads on one copy stream, read-backs
            on another, overlapping the other calls' transfers and compute)
  roofline -- the whole aggregate() call (every kernel of the four calls):
            algorithmic bytes (20.125 B per row read + 85.75 B per group
            written) / the step's device time, against the measured HBM
            copy bandwidth; per-cardinality fractions over each call's own
            event time; `traffic` = ncu DRAM bytes of all of a call's kernels
  checks -- size-independent properties of the timed calls' results at full
            size (group count, COUNT totals, exact int64 SUM total, extremes)

Further sections in the same JSON line: config1 (10M rows, 1e3 groups, with
the oracle, pandas and pyarrow over the same rows), config3 (200M rows,
Zipf(1.2) composite key with null keys), sorted (the sort-path kinds MEDIAN,
QUANTILE, NUNIQUE, NTH_ELEMENT and M2 over the 100M-row columns at 1e4
groups), batched (4,096 instances in one
graph launch against a plain loop and an async 4-stream plain loop) and
served (Poisson arrivals at three rates, plus each form's capacity).

`--impl reference` times the reference's CPU algorithm (the oracle
restatement, all host threads) on a bounded sample of the same workload.
Multi-GPU (torchrun): N independent replicas ("replicas only": a hash groupby
of one input does not shard without an exchange step); value sums all ranks'
rows over the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

CARDS = [100, 10_000, 1_000_000, 100_000_000]
ROWS = 100_000_000
BYTES_PER_ROW_IN = 8 + 8 + 4 + 1.0 / 8  # key + a + b + b's validity bit
# output bytes per group: key 8; a: sum 8, count 4, min 8, max 8, mean 8, var 8;
# b: sum 4, count 4, min 4, max 4, mean 8, var 8; validity bits
BYTES_PER_GROUP_OUT = 8 + (8 + 4 + 8 + 8 + 8 + 8) + (4 + 4 + 4 + 4 + 8 + 8) + 6.0 / 8
METRIC = "groupby rows/s (plain hash groupby, 100M rows, int64 key, cardinality 1e2/1e4/1e6/1e8)"
PARTITIONED = 3  # gbx_strategy of the radix-partitioned path
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) of every
# kernel of one 100M-row call, per cardinality: 20M-row captures scaled by
# rows (None: not captured)
WHOLE_CALL_DRAM_BYTES = {100: 2.07e9, 10_000: 6.95e9, 1_000_000: 14.48e9, 100_000_000: 20.63e9}
STRATEGY_NAMES = {1: "privatized", 2: "global", 3: "partitioned", 4: "warp", 5: "bucketed"}
# bytes of one row's copies in a radix pass: packed key 8 + a 8 + b 4 + b's validity byte 1
PART_BYTES_PER_ROW = 21


def parse_args(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--rows", type=int, default=ROWS)
    p.add_argument("--cards", type=str, default=",".join(str(c) for c in CARDS))
    p.add_argument("--cpu-sample-rows", type=int, default=2_000_000)
    p.add_argument("--strategy", choices=["auto", "warp", "privatized", "global", "partitioned", "bucketed"], default="auto",
                   help="force one aggregation strategy (default: chosen per call)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--c3-rows", type=int, default=200_000_000)
    p.add_argument("--sections", type=str, default="plain,config1,config3,sorted,batched,served",
                   help="comma list of: plain (the headline line), config1 (10M rows, 1e3 groups), config3 "
                        "(200M rows, Zipf composite key), sorted (MEDIAN / QUANTILE / NUNIQUE / NTH_ELEMENT / "
                        "M2 over the 100M-row columns), batched (4,096-instance batch), served (Poisson "
                        "request stream)")
    p.add_argument("--batch-instances", type=int, default=4096)
    p.add_argument("--batch-tune", choices=["off", "cached", "missing", "all"], default="missing")
    p.add_argument("--batch-tune-save", type=str, default=None,
                   help="write the tuning table the batch used (and extended) to this path")
    p.add_argument("--served-requests", type=int, default=200)
    # 4 workers (measured on B200 against 8 and 16 on this request mix) and
    # requests of at most 32K rows merged (no merging, 32K and 128K all kept
    # p99 below the per-request loop's at the three rates; few requests of
    # this mix are small enough to merge)
    p.add_argument("--served-workers", type=int, default=4)
    p.add_argument("--served-batch-rows", type=int, default=32_768)
    p.add_argument("--served-large-rows", type=int, default=0,
                   help="served: requests of at least this many rows run one at a time (0: library default, "
                        "-1: none)")
    return p.parse_args(argv)


# --------------------------------------------------------------- distributed

def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Max of a per-rank float over all ranks (identity when world == 1)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm_sorted = sorted(sm)
        return {"sm_mhz": sm_sorted[len(sm_sorted) // 2], "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# -------------------------------------------------------------------- data

def device_inputs(card: int, n: int, seed: int, device):
    """The 100M-row workload's columns generated on the device (seeded)."""
    from cudf_b200 import workloads as W

    return W.plain_100m_device(card, n, seed, device)


def pack_mask_torch(valid):
    """Bool tensor -> cudf bitmask words (int32, LSB-first) padded to 64 bytes."""
    from cudf_b200 import workloads as W

    return W._bitmask_device(valid)


def aggs():
    from cudf_b200 import aggregation as agg

    return [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean(), agg.variance()]


# --------------------------------------------------------------- our arm

def check_plain_results(n, cols, kt, res):
    """Size-independent properties of one timed call's results, on the
    device: the group count equals the distinct keys, COUNTs add up to the
    (valid) rows, the int64 SUMs add up exactly to the column's sum, and the
    extreme MIN / MAX equal the column's extremes."""
    import torch

    k, a, b = cols
    G = kt.num_rows()

    def typed(col, dt):
        return col.data[: G * torch.empty(0, dtype=dt).element_size()].view(dt)

    def valid_rows(col, size):
        words = col.mask[: (size + 31) // 32].to(torch.int64) & 0xFFFFFFFF
        bits = (words.view(-1, 1) >> torch.arange(32, device=words.device)) & 1
        return bits.view(-1)[:size].bool()

    kd, ad, bd = k.data[:n], a.data[:n], b.data[:n]
    bvalid = valid_rows(b, n)
    ra, rb = res[0].columns(), res[1].columns()
    out = {
        "groups": G == int(torch.unique(kd).numel()),
        "count_a": int(typed(ra[1], torch.int32).to(torch.int64).sum()) == n,
        "count_b": int(typed(rb[1], torch.int32).to(torch.int64).sum()) == int(bvalid.sum()),
        "sum_a_exact": int(typed(ra[0], torch.int64).sum()) == int(ad.sum()),
        "min_a": int(typed(ra[2], torch.int64).min()) == int(ad.min()),
        "max_a": int(typed(ra[3], torch.int64).max()) == int(ad.max()),
    }
    gvalid = valid_rows(rb[2], G)
    bv = bd[bvalid]
    out["min_b"] = float(typed(rb[2], torch.float32)[gvalid].min()) == float(bv.min())
    out["max_b"] = float(typed(rb[3], torch.float32)[valid_rows(rb[3], G)].max()) == float(bv.max())
    out["ok"] = all(out.values())
    return out


def run_ours(args, rank, world, local):
    import torch

    from cudf_b200 import Column, GroupBy, GroupByRequest, Table, TorchAllocator

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)
    cards = [int(c) for c in args.cards.split(",")]
    n = args.rows
    stream = torch.cuda.current_stream()
    alloc = TorchAllocator(device)

    data = {c: device_inputs(c, n, 20241003 + 2 + rank, device) for c in cards}
    gbs = {}
    reqs = {}
    for c in cards:
        k, a, b = data[c]
        gb = GroupBy(Table([k]))
        gb.set_timing(True)
        if args.strategy != "auto":
            from cudf_b200 import Strategy

            gb.set_strategy(Strategy[args.strategy.upper()])
        gbs[c] = gb
        reqs[c] = [GroupByRequest(a, aggs()), GroupByRequest(b, aggs())]
    torch.cuda.synchronize()

    def step(record=None):
        for c in cards:
            kt, res = gbs[c].aggregate(reqs[c], stream=stream, allocator=alloc)
            if record is not None:
                record.append((c, gbs[c].last_stats(), kt.num_rows()))
            del kt, res

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    rec = []
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step(rec)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms_local = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms_local, world, device)
    rows_per_step = n * len(cards)
    value = world * rows_per_step * args.steps / (ms / 1e3)

    # the timed calls' results, checked once more after the timed region
    checks = {}
    for c in cards:
        kt, res = gbs[c].aggregate(reqs[c], stream=stream, allocator=alloc)
        checks[f"{c:g}"] = check_plain_results(n, data[c], kt, res)
        del kt, res

    # whole-call roofline: every kernel of every aggregate() call.  Algorithmic
    # bytes per call = rows read (20.125 B) + groups written (85.75 B), over
    # the step's device time (ms_per_step, host gaps between calls included);
    # per cardinality over that call's own first-to-last event time.
    peaks = _load_peaks()
    per = {}
    launches = 0
    for c, st, g in rec:
        d = per.setdefault(c, {"calls": 0, "total_ms": 0.0, "groups": g, "strategy": st["strategy"],
                               "phases_ms": {}, "partition_bits": st["partition_bits"],
                               "bucket_slots": st["bucket_slots"]})
        d["calls"] += 1
        d["total_ms"] += st["total_ms"]
        for ph in ("sample_ms", "init_ms", "partition_ms", "aggregate_ms", "compact_ms", "finalize_ms"):
            d["phases_ms"][ph] = d["phases_ms"].get(ph, 0.0) + st[ph]
        launches += st["kernel_launches"]
    per_out = {}
    alg_step = 0.0
    for c, d in per.items():
        calls = d["calls"]
        call_ms = d["total_ms"] / calls
        groups = d["groups"]
        alg = n * BYTES_PER_ROW_IN + groups * BYTES_PER_GROUP_OUT
        alg_step += alg
        per_out[f"{c:g}"] = {
            "groups": groups, "strategy": STRATEGY_NAMES.get(d["strategy"], d["strategy"]),
            "partition_bits": d["partition_bits"], "bucket_slots": d["bucket_slots"],
            "ms_per_call": round(call_ms, 4),
            "rows_per_s": n / (call_ms / 1e3),
            "algorithmic_bytes": alg,
            "hbm_frac_whole_call": (alg / (call_ms / 1e3)) / 1e9 / peaks["hbm_gbs"],
            "dram_traffic_bytes": WHOLE_CALL_DRAM_BYTES.get(c),
            "phases_ms": {k: round(v / calls, 4) for k, v in d["phases_ms"].items()},
        }
    step_s = ms / args.steps / 1e3
    achieved = alg_step / step_s / 1e9
    traffic = [WHOLE_CALL_DRAM_BYTES.get(c) for c in cards]
    roofline = {
        "bound": "hbm",
        "kernel": "whole aggregate() call: every kernel of the four 100M-row calls (1e2, 1e4, 1e6, 1e8)",
        "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
        "peak_source": peaks["source"],
        "algorithmic_bytes_per_launch": alg_step / len(cards),
        "algorithmic_bytes_per_step": alg_step,
        "bytes_per_row_in": BYTES_PER_ROW_IN, "bytes_per_group_out": BYTES_PER_GROUP_OUT,
        "per_cardinality_frac": {k: v["hbm_frac_whole_call"] for k, v in per_out.items()},
        # ncu dram__bytes_read.sum + dram__bytes_write.sum summed over every
        # kernel of one call (20M-row captures scaled by rows to 100M)
        "traffic": (sum(traffic) / len(traffic)) if all(t is not None for t in traffic) else None,
        "traffic_per_cardinality": {f"{c:g}": WHOLE_CALL_DRAM_BYTES.get(c) for c in cards},
    }
    # the dominant kernel (k_radix_scatter_bulk, a third of the sweep's GPU
    # time): the partition phase of the partitioned calls, its bytes the
    # copies each radix pass must move (21 B a row read + 21 B written)
    pbytes = pms = 0.0
    for c, st, g in rec:
        if st["strategy"] == PARTITIONED and st["partition_ms"] > 0:
            passes = (st["partition_bits"] + 7) // 8
            pbytes += passes * n * 2 * PART_BYTES_PER_ROW
            pms += st["partition_ms"]
    if pms > 0:
        pa = pbytes / (pms / 1e3) / 1e9
        roofline["dominant_kernel"] = {
            "kernel": "k_radix_scatter_bulk (the partition phase of the 1e6 / 1e8 calls: histograms, scans, passes)",
            "achieved": pa, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": pa / peaks["hbm_gbs"],
            "bytes_per_row_per_pass": 2 * PART_BYTES_PER_ROW}

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, cards, data, gbs, reqs, alloc, stream, world, device)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, cards)

    # release the plain workload before the other sections
    del gbs, reqs, data
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    sections = args.sections.split(",")
    extra = {}
    for name, fn in (("config1", run_config1), ("config3", run_config3), ("sorted", run_sorted),
                     ("batched", run_batched), ("served", run_served)):
        if name not in sections:
            continue
        if name == "served":
            extra[name] = fn(args, rank, device, stream)
        else:
            extra[name] = fn(args, rank, world, device, stream, alloc)
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    out = {
        "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64+f32 (f64 accumulation)",
        "data": "synthetic (seeded, generated on device)",
        "config": {"workload": "plain groupby, 100M rows x 4 cardinalities", "rows": n, "cardinalities": cards,
                   "key": "int64", "values": ["int64 U[-1e6,1e6]", "float32 N(0,1) 10% nulls"],
                   "aggregations": ["SUM", "COUNT", "MIN", "MAX", "MEAN", "VAR"],
                   "l2": "inputs (2.01 GB per groupby) larger than L2; no flush",
                   "parallelism": f"replicas x{world}"},
        "per_cardinality": per_out,
        "checks": checks,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    out.update(extra)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_e2e(args, cards, data, gbs, reqs, alloc, stream, world, device):
    """Host-resident inputs: H2D copies and D2H result reads inside the timed region."""
    import torch

    from cudf_b200 import Column, GroupBy, GroupByRequest, Table

    host = {}
    dev = {}
    for c in cards:
        k, a, b = data[c]
        host[c] = [k.data.cpu().pin_memory(), a.data.cpu().pin_memory(), b.data.cpu().pin_memory(),
                   b.mask.cpu().pin_memory()]
        dev[c] = [torch.empty_like(t, device=device) for t in host[c]]
    h2d = sum(t.numel() * t.element_size() for c in cards for t in host[c])
    d2h_bytes = [0]
    from cudf_b200.column import storage_dtype

    # one pinned host buffer receives every result column of a step
    max_groups = max(args.rows, 1)
    out_host = torch.empty(int(max_groups * BYTES_PER_GROUP_OUT * 1.1) + (1 << 20), dtype=torch.uint8,
                           pin_memory=True)

    def read_back(outs, off):
        """D2H of each column's rows (data and mask) into the pinned buffer from
        byte `off` on; returns the offset after them."""
        for col in outs:
            if col.size == 0:
                continue
            if col.data is not None:
                nb = col.size * storage_dtype(col.type_id).itemsize
                out_host[off:off + nb].copy_(col.data.view(torch.uint8)[:nb], non_blocking=True)
                off += nb
            if col.mask is not None:
                nb = ((col.size + 31) // 32) * 4
                out_host[off:off + nb].copy_(col.mask.view(torch.uint8)[:nb], non_blocking=True)
                off += nb
        return off

    # The step's four groupbys are pipelined over PCIe, which carries both
    # directions at once: every upload is queued on one copy stream, each
    # call starts when its own inputs have landed, and its results are read
    # back on a second copy stream while the later calls upload and compute.
    # The call with the most output goes first, so that its read-back
    # overlaps the other uploads.
    order = sorted(cards, key=lambda c: -c)
    up = torch.cuda.Stream(device)
    down = torch.cuda.Stream(device)

    def step():
        up.wait_stream(stream)
        landed = {}
        with torch.cuda.stream(up):
            for c in order:
                for s_, d_ in zip(host[c], dev[c]):
                    d_.copy_(s_, non_blocking=True)
                landed[c] = torch.cuda.Event()
                landed[c].record(up)
        off = 0
        keep = []
        for c in order:
            dk, da, db, dm = dev[c]
            stream.wait_event(landed[c])
            n = dk.numel()
            kc = Column(data[c][0].type_id, n, dk)
            ac = Column(data[c][1].type_id, n, da)
            bc = Column(data[c][2].type_id, n, db, dm, 0, data[c][2]._null_count)
            gb = GroupBy(Table([kc]))
            kt, res = gb.aggregate([GroupByRequest(ac, aggs()), GroupByRequest(bc, aggs())], stream=stream,
                                   allocator=alloc)
            outs = [col for col in kt.columns()] + [col for t in res for col in t.columns()]
            down.wait_stream(stream)
            with torch.cuda.stream(down):
                off = read_back(outs, off)
            keep.append(outs)  # alive until the read-back is ordered before reuse
        stream.wait_stream(down)
        d2h_bytes[0] = off

    step()
    torch.cuda.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    steps = max(1, min(args.steps, 2))
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world, device)
    rows = args.rows * len(cards) * steps * world
    return {"value": rows / (ms / 1e3), "unit": "rows/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h_bytes[0],
            "steps": steps, "ms_per_step": ms / steps}


# ------------------------------------------------- configs 1 and 3 (plain)

C1_ROWS = 10_000_000
C1_BYTES_PER_ROW = 4 + 8                    # int32 key + float64 value
C1_BYTES_PER_GROUP = 4 + 8 + 4 + 8 + 8 + 8  # key, SUM, COUNT, MEAN, MIN, MAX
C3_ROWS = 200_000_000
C3_BYTES_PER_ROW = 4 + 2 + 0.125 + 0.125 + 8  # int32 + int16 keys, their validity bits, float64 value
C3_BYTES_PER_GROUP = 4 + 2 + 8 + 8            # keys (EXCLUDE: no null keys out), SUM, MEAN


def _time_calls(gb, reqs, stream, alloc, warmup, steps):
    """CUDA-event time per aggregate() call (ms) and the last call's stats."""
    import torch

    for _ in range(warmup):
        kt, res = gb.aggregate(reqs, stream=stream, allocator=alloc)
        del kt, res
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        kt, res = gb.aggregate(reqs, stream=stream, allocator=alloc)
        groups = kt.num_rows()
        del kt, res
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, gb.last_stats(), groups


def _host_cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def _cpu_baselines(keys, vals, kinds, rows, pandas_aggs, arrow_aggs, oracle_threads=1):
    """The oracle (single thread), pandas (single thread by construction) and
    pyarrow (all host threads) on the same host sample; rows/s each."""
    import numpy as np

    from oracle import oracle as orc

    t0 = time.perf_counter()
    orc.groupby(keys, vals, 0, threads=oracle_threads)
    out = {"value": rows / (time.perf_counter() - t0), "unit": "rows/s", "cores": oracle_threads, "kind": "port"}
    cols = {}  # pandas: nulls as NaN (what cudf.pandas' CPU fallback holds)
    masked = []  # pyarrow: nulls as a validity mask
    for i, k in enumerate(keys):
        v = k.values.astype(np.float64) if k.valid is not None else k.values
        cols[f"k{i}"] = np.where(k.valid, v, np.nan) if k.valid is not None else v
        masked.append((f"k{i}", k.values, k.valid))
    for j, (hv, _) in enumerate(vals):
        cols[f"v{j}"] = np.where(hv.valid, hv.values, np.nan) if hv.valid is not None else hv.values
        masked.append((f"v{j}", hv.values, hv.valid))
    try:
        import pandas as pd

        df = pd.DataFrame(cols)
        t0 = time.perf_counter()
        df.groupby([f"k{i}" for i in range(len(keys))], sort=False, dropna=True).agg(pandas_aggs)
        out["pandas_rows_per_s"] = rows / (time.perf_counter() - t0)
        out["pandas_version"] = pd.__version__
    except Exception as e:  # pragma: no cover
        out["pandas_error"] = str(e)
    try:
        import pyarrow as pa

        tbl = pa.table({name: pa.array(v, mask=None if m is None else ~m) for name, v, m in masked})
        t0 = time.perf_counter()
        tbl.group_by([f"k{i}" for i in range(len(keys))], use_threads=True).aggregate(arrow_aggs)
        out["pyarrow_rows_per_s"] = rows / (time.perf_counter() - t0)
        out["pyarrow_threads"] = pa.cpu_count()
        out["pyarrow_version"] = pa.__version__
    except Exception as e:  # pragma: no cover
        out["pyarrow_error"] = str(e)
    out["host_cpu_count"] = os.cpu_count()
    out["host_cpu_model"] = _host_cpu_model()
    return out


def run_config1(args, rank, world, device, stream, alloc):
    """The CPU-runnable config at full size: 10M rows, int32 key uniform over
    1,000 values, float64 N(0,1), SUM/COUNT/MEAN/MIN/MAX -- on the GPU and,
    over the same 10M rows, the oracle, pandas and pyarrow."""
    import torch

    from cudf_b200 import Column, GroupBy, GroupByRequest, Table
    from cudf_b200 import aggregation as agg
    from cudf_b200 import workloads as W
    from cudf_b200._abi import Kind
    from oracle.oracle import HostCol

    d = W.plain_10m(n=C1_ROWS)
    k = Column.from_numpy(d.keys[0], device=device)
    v = Column.from_numpy(d.values[0], device=device)
    gb = GroupBy(Table([k]))
    gb.set_timing(True)
    reqs = [GroupByRequest(v, [agg.sum(), agg.count(), agg.mean(), agg.min(), agg.max()])]
    ms, st, groups = _time_calls(gb, reqs, stream, alloc, max(args.warmup, 3), max(args.steps, 10))
    peaks = _load_peaks()
    alg = C1_ROWS * C1_BYTES_PER_ROW + groups * C1_BYTES_PER_GROUP
    out = {"metric": "groupby rows/s (10M rows, int32 key, 1e3 groups, float64 value)", "value": C1_ROWS / (ms / 1e3),
           "unit": "rows/s", "ms_per_call": ms, "groups": groups,
           "strategy": STRATEGY_NAMES.get(st["strategy"], st["strategy"]),
           "hbm_frac_whole_call": alg / (ms / 1e3) / 1e9 / peaks["hbm_gbs"],
           "config": {"rows": C1_ROWS, "key": "int32 U[0, 1000)", "value": "float64 N(0,1)",
                      "aggregations": ["SUM", "COUNT", "MEAN", "MIN", "MAX"],
                      "l2": "inputs (120 MB) about the size of L2; no flush (a repeated call re-reads L2-resident rows)"}}
    del gb, reqs, k, v
    if rank == 0 and not args.no_cpu:
        aggs5 = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MEAN, 0), (Kind.MIN, 0), (Kind.MAX, 0)]
        cpu = _cpu_baselines([HostCol(d.keys[0])], [(HostCol(d.values[0]), aggs5)], aggs5, C1_ROWS,
                             {"v0": ["sum", "count", "mean", "min", "max"]},
                             [("v0", "sum"), ("v0", "count"), ("v0", "mean"), ("v0", "min"), ("v0", "max")])
        cpu["sample"] = "the whole 10M-row workload"
        out["cpu_baseline"] = cpu
        out["speedup_vs_pandas"] = out["value"] / cpu["pandas_rows_per_s"] if "pandas_rows_per_s" in cpu else None
    return out


def run_config3(args, rank, world, device, stream, alloc):
    """200M rows, (int32, int16) key with 2% nulls per column, Zipf(1.2) over
    1e5 pairs, float64 LogNormal(0, 1), SUM and MEAN (EXCLUDE)."""
    import numpy as np
    import torch

    from cudf_b200 import GroupBy, GroupByRequest, Table
    from cudf_b200 import aggregation as agg
    from cudf_b200 import workloads as W
    from cudf_b200._abi import Kind
    from oracle.oracle import HostCol

    n = args.c3_rows
    k1, k2, v = W.plain_200m_device(n, W.SEED0 + 3 + rank, device)
    gb = GroupBy(Table([k1, k2]))
    gb.set_timing(True)
    reqs = [GroupByRequest(v, [agg.sum(), agg.mean()])]
    with ClockSampler(device.index) as clk:
        ms, st, groups = _time_calls(gb, reqs, stream, alloc, max(args.warmup, 3), max(args.steps, 5))
    peaks = _load_peaks()
    alg = n * C3_BYTES_PER_ROW + groups * C3_BYTES_PER_GROUP
    out = {"metric": "groupby rows/s (200M rows, (int32, int16) key Zipf(1.2) over 1e5 pairs, 2% null keys)",
           "value": n / (ms / 1e3), "unit": "rows/s", "ms_per_call": ms, "groups": groups,
           "strategy": STRATEGY_NAMES.get(st["strategy"], st["strategy"]),
           "estimated_groups": st["estimated_groups"],
           "phases_ms": {p: st[p] for p in ("sample_ms", "init_ms", "partition_ms", "aggregate_ms", "compact_ms",
                                            "finalize_ms")},
           "roofline": {"bound": "hbm", "kernel": "whole aggregate() call", "achieved": alg / (ms / 1e3) / 1e9,
                        "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": alg / (ms / 1e3) / 1e9 / peaks["hbm_gbs"], "peak_source": peaks["source"],
                        "algorithmic_bytes_per_launch": alg, "bytes_per_row_in": C3_BYTES_PER_ROW,
                        "bytes_per_group_out": C3_BYTES_PER_GROUP},
           "config": {"rows": n, "key": "(int32, int16), 2% nulls each, Zipf(1.2) over 1e5 distinct pairs",
                      "value": "float64 LogNormal(0,1)", "aggregations": ["SUM", "MEAN"], "null_policy": "EXCLUDE",
                      "l2": "inputs (%.2f GB) larger than L2; no flush" % (n * C3_BYTES_PER_ROW / 1e9)},
           "clocks": clk.summary()}
    del gb, reqs, k1, k2, v
    if rank == 0 and not args.no_cpu:
        rows = min(args.cpu_sample_rows, n)
        d = W.plain_200m(n=rows)
        keys = [HostCol(d.keys[0], d.key_valid[0]), HostCol(d.keys[1], d.key_valid[1])]
        a2 = [(Kind.SUM, 0), (Kind.MEAN, 0)]
        cpu = _cpu_baselines(keys, [(HostCol(d.values[0]), a2)], a2, rows, {"v0": ["sum", "mean"]},
                             [("v0", "sum"), ("v0", "mean")])
        cpu["sample"] = f"{rows} rows of the same distribution (numpy seed)"
        out["cpu_baseline"] = cpu
    return out


# --------------------------------------------------- sort-path kinds (plain)

SORTED_CARD = 10_000
SORTED_QS = (0.25, 0.5, 0.75)


def run_sorted(args, rank, world, device, stream, alloc):
    """The kinds libcudf computes on its sort path, over the 100M-row
    workload's columns at 1e4 groups: MEDIAN, QUANTILE {.25, .5, .75} and
    NUNIQUE of the int64 column a, NTH_ELEMENT(0) and M2 of the float32
    column b (10% nulls).  Checks at full size: QUANTILE 0.5 equals MEDIAN,
    quantiles ascend within a group, NUNIQUE <= the group's row count."""
    import numpy as np
    import torch

    from cudf_b200 import GroupBy, GroupByRequest, Table
    from cudf_b200 import aggregation as agg
    from cudf_b200 import workloads as W
    from cudf_b200._abi import Kind, NullPolicy
    from oracle.oracle import HostCol

    n = args.rows
    k, a, b = W.plain_100m_device(SORTED_CARD, n, W.SEED0 + 11 + rank, device)
    gb = GroupBy(Table([k]))
    gb.set_timing(True)
    reqs = [GroupByRequest(a, [agg.median(), agg.quantile(SORTED_QS), agg.nunique(), agg.count()]),
            GroupByRequest(b, [agg.nth_element(0), agg.m2()])]
    with ClockSampler(device.index) as clk:
        ms, st, groups = _time_calls(gb, reqs, stream, alloc, max(args.warmup, 3), max(args.steps, 5))
    kt, res = gb.aggregate(reqs, stream=stream, allocator=alloc)
    med = res[0].columns()[0].to_numpy()[0]
    qv = res[0].columns()[1].to_numpy()[0].reshape(-1, len(SORTED_QS))
    nu = res[0].columns()[2].to_numpy()[0]
    cnt = res[0].columns()[3].to_numpy()[0]
    checks = {"groups": int(kt.num_rows()),
              "median_equals_quantile_0.5": bool(np.array_equal(med, qv[:, 1])),
              "quantiles_ascend": bool(np.all(np.diff(qv, axis=1) >= 0)),
              "nunique_le_rows": bool(np.all((nu >= 1) & (nu <= cnt))),
              "rows_total": int(cnt.sum()) == n}
    del kt, res
    peaks = _load_peaks()
    alg = n * (8 + 8 + 4 + 0.125) + groups * (8 + 8 + 8 * len(SORTED_QS) + 4 + 4 + 4 + 8)
    out = {"metric": "groupby rows/s (100M rows, int64 key, 1e4 groups; MEDIAN, QUANTILE x3, NUNIQUE, "
                     "NTH_ELEMENT, M2)",
           "value": n / (ms / 1e3), "unit": "rows/s", "ms_per_call": ms, "groups": groups,
           "strategy": STRATEGY_NAMES.get(st["strategy"], st["strategy"]),
           "kernel_launches": st["kernel_launches"],
           "phases_ms": {p: st[p] for p in ("sample_ms", "init_ms", "aggregate_ms", "compact_ms", "finalize_ms")},
           "hbm_frac_whole_call": alg / (ms / 1e3) / 1e9 / peaks["hbm_gbs"],
           "checks": checks,
           "config": {"rows": n, "key": "int64 U[0, 1e4)", "values": ["int64 U[-1e6,1e6]", "float32 N(0,1) 10% nulls"],
                      "aggregations": ["MEDIAN(a)", "QUANTILE(a, .25/.5/.75, LINEAR)", "NUNIQUE(a)", "COUNT(a)",
                                       "NTH_ELEMENT(b, 0)", "M2(b)"],
                      "note": "finalize_ms holds the labels, the radix sorts of (group, value) records and the "
                              "selections"},
           "clocks": clk.summary()}
    del gb, reqs, k, a, b
    if rank == 0 and not args.no_cpu:
        rows = min(args.cpu_sample_rows, 2_000_000)
        d = W.plain_100m(SORTED_CARD, n=rows)
        aggs_a = [(Kind.MEDIAN, 0), (Kind.QUANTILE, 0, {"quantiles": list(SORTED_QS)}), (Kind.NUNIQUE, 0),
                  (Kind.COUNT_VALID, 0)]
        aggs_b = [(Kind.NTH_ELEMENT, 0, {"null_policy": NullPolicy.INCLUDE}), (Kind.M2, 0)]
        from oracle import oracle as orc

        t0 = time.perf_counter()
        orc.groupby([HostCol(d.keys[0])], [(HostCol(d.values[0]), aggs_a),
                                            (HostCol(d.values[1], d.value_valid[1]), aggs_b)])
        cpu = {"value": rows / (time.perf_counter() - t0), "unit": "rows/s", "cores": 1, "kind": "port",
               "sample": f"{rows} rows of the same distribution (numpy seed)"}
        try:
            import pandas as pd

            df = pd.DataFrame({"k": d.keys[0], "a": d.values[0],
                               "b": np.where(d.value_valid[1], d.values[1], np.nan)})
            t0 = time.perf_counter()
            g = df.groupby("k", sort=False)
            g["a"].median(), g["a"].quantile(list(SORTED_QS)), g["a"].nunique(), g["a"].count()
            g["b"].nth(0), g["b"].var(ddof=0)
            cpu["pandas_rows_per_s"] = rows / (time.perf_counter() - t0)
        except Exception as e:  # pragma: no cover
            cpu["pandas_error"] = str(e)
        out["cpu_baseline"] = cpu
    return out


# ------------------------------------------------------------- batched form

BATCH_BYTES_PER_ROW = 4 + 8            # int32 key + int64 value
BATCH_BYTES_PER_GROUP = 4 + 8 + 4 + 8  # key, SUM (int64), COUNT (int32), MAX (int64)
TUNE_TABLE = os.path.join(ROOT, "cudf_b200", "tuning", "batch_tune.txt")


def _segmented_inputs(spec, device, seed, key_dtype, value_kind):
    """Every instance's columns in two device buffers (instance i at rows
    [start_i, start_i + rows_i)): key uniform in [0, C_i); value int64
    uniform in [0, 1e9] ("int") or float64 N(0, 1) ("normal")."""
    import numpy as np
    import torch

    rows = torch.from_numpy(spec.rows).to(device)
    total = int(spec.rows.sum())
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    cards = torch.repeat_interleave(torch.from_numpy(spec.cards.astype(np.float64)).to(device), rows)
    k = (torch.rand(total, generator=g, device=device, dtype=torch.float64) * cards).floor_().to(key_dtype)
    del cards
    if value_kind == "int":
        v = torch.randint(0, 1_000_000_001, (total,), generator=g, device=device, dtype=torch.int64)
    else:
        v = torch.randn(total, generator=g, device=device, dtype=torch.float64)
    starts = np.concatenate([[0], np.cumsum(spec.rows)[:-1]]).astype(np.int64)
    return k, v, starts


def _percentiles(xs):
    import numpy as np

    a = np.asarray(xs, dtype=np.float64)
    return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)), "max": float(a.max())}


def run_batched(args, rank, world, device, stream, alloc):
    """4,096 independent groupbys (rows log-uniform in [1e3, 1e6], cardinality
    log-uniform in [10, 1e4], int32 key, int64 value, SUM/COUNT/MAX) as one
    graph launch, against a loop of the plain form over the same instances."""
    import shutil
    import tempfile

    import torch

    from cudf_b200 import BatchGroupBy, BatchInstance, Column, GroupBy, GroupByRequest, Table, Tune, TypeId
    from cudf_b200 import aggregation as agg
    from cudf_b200 import workloads as W
    from cudf_b200.column import storage_dtype

    spec = W.batched_spec(args.batch_instances)
    k, v, starts = _segmented_inputs(spec, device, 20241003 + 4 + rank, torch.int32, "int")
    total = spec.total_rows
    insts = []
    for i in range(spec.num_instances):
        n, s = int(spec.rows[i]), int(starts[i])
        insts.append(BatchInstance(Table([Column(TypeId.INT32, n, k, None, s)]),
                                   [GroupByRequest(Column(TypeId.INT64, n, v, None, s),
                                                   [agg.sum(), agg.count(), agg.max()])]))
    tune = {"off": Tune.OFF, "cached": Tune.CACHED, "missing": Tune.MISSING, "all": Tune.ALL}[args.batch_tune]
    tune_copy = None
    if tune != Tune.OFF:
        fd, tune_copy = tempfile.mkstemp(suffix=".txt")
        os.close(fd)
        if os.path.exists(TUNE_TABLE):
            shutil.copyfile(TUNE_TABLE, tune_copy)
    t0 = time.perf_counter()
    b = BatchGroupBy(insts, tune=tune, tune_file=tune_copy, stream=stream, allocator=alloc)
    create_s = time.perf_counter() - t0
    st0 = b.stats()
    if args.batch_tune_save and tune_copy:
        shutil.copyfile(tune_copy, args.batch_tune_save)

    for _ in range(args.warmup):
        b.execute(stream)
    torch.cuda.synchronize()
    lat_ms, agg_ms = [], []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    steps = max(args.steps, 5)
    with ClockSampler(device.index) as clk:
        e0.record(stream)
        for _ in range(steps):
            res = b.execute(stream)
            s = b.stats()
            lat_ms.append(s["execute_ms"])
            agg_ms.append(s["aggregate_ms"])
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    stats = b.stats()
    groups = res.num_groups
    peaks = _load_peaks()
    agg_avg = sum(agg_ms) / len(agg_ms)
    achieved = total * BATCH_BYTES_PER_ROW / (agg_avg / 1e3) / 1e9
    batch_rows_s = total / (ms / 1e3)

    # e2e: host (pinned) inputs copied in place each step, results read back
    hk = k.cpu().pin_memory()
    hv = v.cpu().pin_memory()
    out_host = torch.empty(int(groups * BATCH_BYTES_PER_GROUP * 1.05) + (1 << 20), dtype=torch.uint8,
                           pin_memory=True)

    def e2e_step():
        k.copy_(hk, non_blocking=True)
        v.copy_(hv, non_blocking=True)
        r = b.execute(stream)
        off = 0
        for col in list(r.keys.columns()) + [c for t in r.results for c in t.columns()]:
            nb = col.size * storage_dtype(col.type_id).itemsize
            out_host[off:off + nb].copy_(col.data.view(torch.uint8)[:nb], non_blocking=True)
            off += nb
        stream.synchronize()
        return off

    e2e_step()
    e2e_steps = 3
    e0.record(stream)
    for _ in range(e2e_steps):
        d2h = e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    h2d = hk.numel() * hk.element_size() + hv.numel() * hv.element_size()
    del hk, hv

    # the plain form, one aggregate() per instance, on the same GPU
    gbs = [GroupBy(x.keys) for x in insts]

    def loop_pass(record):
        t_start = time.perf_counter()
        for gb, x in zip(gbs, insts):
            kt, rs = gb.aggregate(x.requests, stream=stream, allocator=alloc)
            if record is not None:
                record.append((time.perf_counter() - t_start) * 1e3)
            del kt, rs
        return (time.perf_counter() - t_start) * 1e3

    loop_pass(None)
    torch.cuda.synchronize()
    done_ms = []
    loop_ms = loop_pass(done_ms)
    loop_rows_s = total / (loop_ms / 1e3)

    # the plain form issued asynchronously: 4 host threads, each with its own
    # stream and allocator, split the instances round-robin (calls overlap on
    # the GPU while others wait for their group counts)
    import threading

    from cudf_b200 import TorchAllocator

    workers = 4
    streams = [torch.cuda.Stream(device) for _ in range(workers)]
    allocs = [TorchAllocator(device) for _ in range(workers)]

    def async_pass():
        def work(w):
            with torch.cuda.stream(streams[w]):
                for i in range(w, len(insts), workers):
                    kt, rs = gbs[i].aggregate(insts[i].requests, stream=streams[w], allocator=allocs[w])
                    del kt, rs
                streams[w].synchronize()

        t_start = time.perf_counter()
        ts = [threading.Thread(target=work, args=(w,)) for w in range(workers)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        return (time.perf_counter() - t_start) * 1e3

    async_pass()
    async_ms = async_pass()
    async_rows_s = total / (async_ms / 1e3)

    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = _batched_cpu(spec)
    b.close()
    if tune_copy:
        os.unlink(tune_copy)
    return {
        "metric": "batched groupby rows/s (4,096 instances, one graph launch)",
        "config": {"instances": spec.num_instances, "total_rows": total, "rows": "log-uniform [1e3, 1e6]",
                   "cardinality": "log-uniform [10, 1e4]", "key": "int32", "value": "int64 U[0, 1e9]",
                   "aggregations": ["SUM", "COUNT", "MAX"], "tune": args.batch_tune,
                   "l2": "inputs (%.1f GB) larger than L2; no flush" % (total * BATCH_BYTES_PER_ROW / 1e9)},
        "value": batch_rows_s, "unit": "rows/s", "ms_per_step": ms, "steps": steps, "groups": groups,
        "latency_ms": {"batched": {"p50": float(_percentiles(lat_ms)["p50"]), "p99": _percentiles(lat_ms)["p99"],
                                   "note": "every instance completes when the launch does"},
                       "plain_loop": dict(_percentiles(done_ms),
                                          note="completion time of instance i when all arrive at once")},
        "plain_loop": {"value": loop_rows_s, "unit": "rows/s", "ms_per_pass": loop_ms, "calls": spec.num_instances},
        "speedup_vs_plain_loop": batch_rows_s / loop_rows_s,
        "plain_async_loop": {"value": async_rows_s, "unit": "rows/s", "ms_per_pass": async_ms,
                             "calls": spec.num_instances, "host_threads": workers, "streams": workers},
        "speedup_vs_plain_async_loop": batch_rows_s / async_rows_s,
        "phases_ms": {"init": stats["init_ms"], "aggregate": agg_avg, "output": stats["output_ms"],
                      "launch": stats["execute_ms"]},
        "roofline": {"bound": "hbm", "kernel": "k_batch_agg", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                     "algorithmic_bytes_per_launch": total * BATCH_BYTES_PER_ROW},
        "e2e": {"value": total / (e2e_ms / 1e3), "unit": "rows/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
        "tuner": {"create_s": create_s, "tune_ms": st0["tune_ms"], "classes": st0["classes"],
                  "classes_measured": st0["classes_measured"], "classes_cached": st0["classes_cached"],
                  "block_threads": stats["block_threads"], "grid": stats["grid"],
                  "mode_count": {"shared": stats["mode_count"][1], "warp": stats["mode_count"][2],
                                 "global": stats["mode_count"][3]},
                  "work_items": stats["work_items"], "dynamic_smem": stats["dynamic_smem"]},
        "gpu_launches": stats["kernels_per_execute"] * steps,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }


def _batched_cpu(spec, sample_instances=48):
    """Oracle (single thread) and pandas on the first instances of the batch."""
    from cudf_b200 import workloads as W
    from cudf_b200._abi import Kind
    from oracle import oracle as orc
    from oracle.oracle import HostCol

    data = [W.batched_instance(spec, i) for i in range(min(sample_instances, spec.num_instances))]
    rows = sum(len(kk) for kk, _ in data)
    t0 = time.perf_counter()
    for kk, vv in data:
        orc.groupby([HostCol(kk)], [(HostCol(vv), [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MAX, 0)])], 0,
                    threads=1)
    out = {"value": rows / (time.perf_counter() - t0), "unit": "rows/s", "cores": 1, "kind": "port",
           "sample": f"the first {len(data)} instances ({rows} rows)"}
    try:
        import pandas as pd

        frames = [pd.DataFrame({"k": kk, "v": vv}) for kk, vv in data]
        t0 = time.perf_counter()
        for df in frames:
            df.groupby("k", sort=False).agg({"v": ["sum", "count", "max"]})
        out["pandas_rows_per_s"] = rows / (time.perf_counter() - t0)
    except Exception as e:  # pragma: no cover
        out["pandas_error"] = str(e)
    out["host_cpu_count"] = os.cpu_count()
    return out


# -------------------------------------------------------------- served form

def _serve_run(lib, srv, prepared, arrivals):
    """Submits request i at arrivals[i] (seconds from the run's start) from one
    thread, waits for every result in another; returns per-request latency in
    ms (done - scheduled arrival), the run's span in s and merged requests."""
    import ctypes as C
    import threading

    from cudf_b200 import _abi

    n = len(prepared)
    tickets = [0] * n
    done = [0.0] * n
    batched = [1] * n
    ready = [threading.Event() for _ in range(n)]
    errors = []
    start = lib.gbx_server_now(srv) + 0.002

    def submitter():
        for i, (tv, reqs, nreq, _) in enumerate(prepared):
            t_arr = start + arrivals[i]
            while True:
                d = t_arr - lib.gbx_server_now(srv)
                if d <= 0:
                    break
                time.sleep(d if d > 0.002 else 0)
            t = C.c_uint64()
            if lib.gbx_server_submit(srv, C.byref(tv), reqs, nreq, C.byref(t)) != 0:
                errors.append(lib.gbx_last_error())
            tickets[i] = t.value
            ready[i].set()

    def waiter():
        for i in range(n):
            ready[i].wait()
            if not tickets[i]:
                continue
            out = C.POINTER(_abi.gbx_result)()
            tm = _abi.gbx_server_timing()
            if lib.gbx_server_wait(srv, tickets[i], -1.0, C.byref(out), C.byref(tm)) != 0:
                errors.append(lib.gbx_last_error())
                continue
            done[i] = tm.done_s
            batched[i] = tm.batched
            lib.gbx_result_release(out)

    ts = [threading.Thread(target=submitter), threading.Thread(target=waiter)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errors:
        raise RuntimeError(f"served run failed: {errors[0]}")
    lat = [(done[i] - (start + arrivals[i])) * 1e3 for i in range(n)]
    return lat, max(done) - start, sum(1 for b in batched if b > 1)


def run_served(args, rank, device, stream):
    """A Poisson stream of groupby requests (rows log-uniform in [1e4, 5e7],
    cardinality log-uniform in [1e2, 1e7], int64 key, float64 N(0,1) value,
    SUM/COUNT/MEAN) over device-resident columns, at 0.5x, 0.9x and 1.2x of
    the plain loop's capacity: the served form (continuous batching, HBM
    admission) against a per-request loop of the plain form (one worker, no
    merging) on the same arrivals."""
    import ctypes as C

    import numpy as np
    import torch

    from cudf_b200 import Column, GroupByRequest, Table, TypeId, _abi, _lib
    from cudf_b200 import aggregation as agg
    from cudf_b200 import workloads as W
    from cudf_b200.server import request_array

    spec = W.batched_spec(args.served_requests, rows_range=(1e4, 5e7), card_range=(1e2, 1e7), seed=20241003 + 5)
    k, v, starts = _segmented_inputs(spec, device, 20241003 + 5 + rank, torch.int64, "normal")
    torch.cuda.synchronize()
    lib = _lib.lib()
    prepared = []
    for i in range(spec.num_instances):
        n, s = int(spec.rows[i]), int(starts[i])
        kt = Table([Column(TypeId.INT64, n, k, None, s)])
        rq = [GroupByRequest(Column(TypeId.FLOAT64, n, v, None, s), [agg.sum(), agg.count(), agg.mean()])]
        tv, cols = kt.view()
        reqs, keep = request_array(rq)
        prepared.append((tv, reqs, len(rq), (kt, rq, cols, keep)))
    total_rows = spec.total_rows

    def server(workers, batch_rows):
        opts = _abi.gbx_server_options(workers=workers, null_policy=0, hbm_budget_bytes=150 << 30,
                                       batch_max_rows=batch_rows, batch_max_requests=64,
                                       large_rows=args.served_large_rows if workers > 1 else -1)
        h = C.c_void_p()
        _lib.check(lib.gbx_server_create(C.byref(opts), C.byref(h)))
        return h

    served_cfg = (args.served_workers, args.served_batch_rows)
    loop_cfg = (1, 0)
    # warm-up: every request once per configuration, so that the stream-ordered
    # pool has grown to what concurrent requests hold and modules are loaded
    for cfg in (served_cfg, loop_cfg):
        h = server(*cfg)
        _serve_run(lib, h, prepared, [0.0] * len(prepared))
        lib.gbx_server_destroy(h)
    # the plain loop's capacity: every request queued at t = 0
    h = server(*loop_cfg)
    _, span0, _ = _serve_run(lib, h, prepared, [0.0] * len(prepared))
    lib.gbx_server_destroy(h)
    capacity_rps = len(prepared) / span0
    # the served configuration's own capacity, every request queued at t = 0
    h = server(*served_cfg)
    _, span_served, _ = _serve_run(lib, h, prepared, [0.0] * len(prepared))
    lib.gbx_server_destroy(h)
    rng = np.random.default_rng(20241003 + 5)
    gaps = rng.exponential(1.0, len(prepared))
    rates = {}
    with ClockSampler(device.index) as clk:
        for mult in (0.5, 0.9, 1.2):
            lam = mult * capacity_rps
            arrivals = np.cumsum(gaps / lam) - gaps[0] / lam
            res = {"arrival_rate_per_s": lam}
            for name, cfg in (("served", served_cfg), ("plain_loop", loop_cfg)):
                h = server(*cfg)
                lat, span, merged = _serve_run(lib, h, prepared, arrivals)
                st = _abi.gbx_server_stats()
                lib.gbx_server_last_stats(h, C.byref(st))
                lib.gbx_server_destroy(h)
                p = _percentiles(lat)
                res[name] = {"p50_ms": p["p50"], "p99_ms": p["p99"], "rows_per_s": total_rows / span,
                             "max_in_flight": st.max_in_flight, "merged_requests": merged,
                             "batched_launches": st.batches, "peak_reserved_gb": st.peak_reserved_bytes / 1e9}
            res["p99_speedup"] = res["plain_loop"]["p99_ms"] / res["served"]["p99_ms"]
            res["rows_per_s_speedup"] = res["served"]["rows_per_s"] / res["plain_loop"]["rows_per_s"]
            rates[f"{mult}x"] = res
    del prepared
    return {
        "metric": "served groupby p50/p99 latency and rows/s at 3 Poisson arrival rates",
        "config": {"requests": spec.num_instances, "total_rows": total_rows, "rows": "log-uniform [1e4, 5e7]",
                   "cardinality": "log-uniform [1e2, 1e7]", "key": "int64", "value": "float64 N(0,1)",
                   "aggregations": ["SUM", "COUNT", "MEAN"], "hbm_budget_gb": 150,
                   "served": {"workers": served_cfg[0], "merge_rows_max": served_cfg[1]},
                   "plain_loop": "one worker, one request at a time, arrival order",
                   "rates": "0.5x, 0.9x, 1.2x of the plain loop's capacity (requests/s with all queued at t=0)"},
        "plain_loop_capacity_requests_per_s": capacity_rps,
        "plain_loop_capacity_rows_per_s": total_rows / span0,
        "served_capacity_requests_per_s": spec.num_instances / span_served,
        "served_capacity_rows_per_s": total_rows / span_served,
        "capacity_speedup": span0 / span_served,
        "rates": rates,
        "clocks": clk.summary(),
    }


# ----------------------------------------------------------- CPU baselines

def _sample_inputs(cards, rows):
    from cudf_b200 import workloads as W

    return {c: W.plain_100m(c, n=rows) for c in cards}


def _oracle_requests(d):
    from cudf_b200._abi import Kind
    from oracle.oracle import HostCol

    a6 = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MIN, 0), (Kind.MAX, 0), (Kind.MEAN, 0), (Kind.VARIANCE, 1)]
    return [HostCol(d.keys[0])], [(HostCol(d.values[0]), a6), (HostCol(d.values[1], d.value_valid[1]), a6)]


def cpu_baseline(args, cards):
    """The oracle (a C restatement of the reference's hash groupby, single
    thread), pandas (single thread) and pyarrow (all host threads) on a
    bounded sample of the workload: `cpu_sample_rows` rows of each
    cardinality, same distributions."""
    rows = args.cpu_sample_rows
    samples = _sample_inputs(cards, rows)
    names = ["sum", "count", "min", "max", "mean", "var"]
    pandas_aggs = {"v0": names, "v1": names}
    arrow_aggs = [(f"v{j}", a if a != "var" else "variance") for j in range(2) for a in names]
    secs = {"value": 0.0, "pandas_rows_per_s": 0.0, "pyarrow_rows_per_s": 0.0}
    last = {}
    for c in cards:
        keys, reqs = _oracle_requests(samples[c])
        r = _cpu_baselines(keys, reqs, None, rows, pandas_aggs, arrow_aggs)
        for k in secs:
            if k in r:
                secs[k] += rows / r[k]
        last = r
    out = dict(last)
    for k, t in secs.items():
        if t > 0:
            out[k] = rows * len(cards) / t
    out["sample"] = f"{rows} rows of each of the {len(cards)} cardinalities (same distributions, numpy seed)"
    return out


def run_reference(args, rank, world):
    """Reference arm: the reference's CPU algorithm (the oracle restatement)
    with all host threads, on a bounded sample of the same workload."""
    if rank != 0:
        return
    from oracle import oracle as orc

    cards = [int(c) for c in args.cards.split(",")]
    rows = args.cpu_sample_rows
    samples = _sample_inputs(cards, rows)
    threads = os.cpu_count() or 1
    prepared = {c: _oracle_requests(samples[c]) for c in cards}

    def step():
        for c in cards:
            keys, reqs = prepared[c]
            orc.groupby(keys, reqs, 0, threads=threads)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = rows * len(cards) * args.steps / dt
    out = {"metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "int64+f32 (long double accumulation)",
           "data": "synthetic (seeded numpy)", "impl": "reference",
           "config": {"workload": "plain groupby, 100M rows x 4 cardinalities (bounded CPU sample)",
                      "rows": rows, "cardinalities": cards},
           "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                            "sample": f"{rows} rows per cardinality per step"},
           "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------- peaks

def _load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return {"hbm_gbs": float(p["hbm_gbs"]), "source": "measured (MEASURED_PEAKS.json)"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "source": "fallback 6.65 TB/s"}


def replica_command(n: int, argv, port: int):
    """The torchrun command that runs this benchmark as n replicas (one rank
    per GPU), as the driver launches it."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
            "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *argv]


def _free_port() -> int:
    import socket

    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    args = parse_args(argv)
    rank, world, local = dist_env()
    launched = "WORLD_SIZE" in os.environ
    if launched and world != args.gpus:
        print(f"bench.py: --gpus {args.gpus} does not match WORLD_SIZE={world}", file=sys.stderr)
        sys.exit(2)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if not launched and args.gpus > 1:
        # N replicas: relaunch under torchrun, one rank per GPU
        r = subprocess.run(replica_command(args.gpus, argv, _free_port()))
        sys.exit(r.returncode)
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
