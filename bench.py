"""Compaction throughput benchmark (one JSON line on rank 0).

Workload: the L1->L2 compaction at size (1 L1 table of 2 MiB over 32 L2 tables
of 2 MiB, Zipf(0.99) keys of 8-64 bytes, lognormal values, 3 snapshots, 5%
deletion markers, L3 grandparents over half the key range), synthetic and
seeded.  One step = one compaction job through the engine's C ABI.

* value: MiB of input compacted per second with the input tables already in
  HBM and the outputs left in HBM (lc_job_desc.inputs_on_device /
  outputs_on_device); L2 is flushed between steps.
* e2e: the same job through lc_compact with the tables in pinned host memory:
  the host->device copy of the inputs and the device->host copy of every
  output file are inside each step.
* roofline: the slowest of the three bandwidth-bound kernels (decode, merge,
  data-block encode), timed live with CUDA events on the job's own stream,
  against the measured HBM copy bandwidth.
* cpu_baseline: the reference's own CPU DoCompactionWork on one host core.

--impl reference times the reference's CPU compaction on all usable host
cores (one job per thread) on the same workload instead.

Multi-GPU (torchrun): every rank compacts its own job stream on its own GPU
(replicas; no collective on the data path); value sums all ranks' input bytes
over the slowest rank's time.
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
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "compaction MB/s in->out (byte-exact); p50/p99 job latency, batched vs plain"
UNIT = "MiB/s"
WORKLOAD = "l1_l2_at_size"
MiB = float(1 << 20)


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=400)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="luda", choices=["luda", "reference"])
    p.add_argument("--scale", type=float, default=1.0)
    p.add_argument("--cpu-seconds", type=float, default=10.0,
                   help="bound on the CPU baseline sample")
    p.add_argument("--no-graphs", action="store_true",
                   help="launch every kernel directly instead of replaying CUDA graphs")
    p.add_argument("--batch-jobs", type=int, default=64)
    p.add_argument("--served-dbs", type=int, default=16)
    p.add_argument("--served-flushes", type=int, default=16,
                   help="flushes per database (0: skip the served leg)")
    p.add_argument("--served-loads", type=float, nargs="*", default=[0.5, 0.9])
    p.add_argument("--batch-steps", type=int, default=5,
                   help="timed repetitions of the 64-job set (0: skip the batched leg)")
    return p.parse_args()


# DRAM bytes (read + write) per launch from one ncu capture of each kernel on
# this workload at scale 1 (profiles/k_encode_blocks_l1_l2_at_size.md,
# profiles/k_block_decode_l1_l2_at_size.md).
NCU_TRAFFIC = {"encode_blocks": 88.962560e6 + 32.451328e6, "decode": 68.024832e6 + 3.235840e6}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples (every 50 ms, written to a file) of SM clock and
    throttle reasons; summary() keeps the samples taken while the timed region
    ran (mark_start/mark_end)."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        import tempfile
        self.device = device
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")
        self.proc = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            time.sleep(0.5)
        except Exception:
            self.proc = None
        return self

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        import datetime
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) < 10:
                        continue
                    try:
                        ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    except ValueError:
                        continue
                    rows.append((ts, parts))
        except OSError:
            pass
        if self.t0 is not None:
            win = [p for ts, p in rows if self.t0 - 0.06 <= ts <= (self.t1 or ts) + 0.06]
        else:
            win = [p for _, p in rows]
        if not win:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"],
                    "samples": 0, "samples_total": len(rows)}
        sm = [float(p[2]) for p in win if p[2].replace(".", "").isdigit()]
        mx = [float(p[3]) for p in win if p[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for p in win:
            for n, v in zip(names, p[6:10]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(win)}


def make_job(scale: float, seed: int):
    from luda_b200 import workloads
    return workloads.l1_l2_at_size(seed=seed, scale=scale)


def reference_arm(args, rank):
    if rank != 0:
        return
    import oracle
    if not oracle.has_ref():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU build (oracle/_ref) not present"}))
        return
    job = make_job(args.scale, 1)
    job.materialize(lambda e, o: oracle.build_table(e, o, "ref"))
    mib = job.input_bytes() / MiB
    cores = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
        cores = max(1, min(cores, int(avail // (8 * job.input_bytes()))))
    except Exception:
        pass
    cores = min(cores, 64)
    for _ in range(args.warmup):
        oracle.ref_compact_parallel(job, cores)
    secs = []
    for _ in range(args.steps):
        secs.append(oracle.ref_compact_parallel(job, cores))
    total = sum(secs)
    value = args.steps * cores * mib / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "input_mib": mib, "jobs_per_step": cores,
                   "scale": args.scale},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{cores} concurrent copies of the {mib:.1f} MiB job per step "
                                   f"(reference CPU DoCompactionWork, one DB per thread)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def cpu_baseline(job, bound_s):
    import oracle
    kind = "reference" if oracle.has_ref() else "port"
    mib = job.input_bytes() / MiB
    secs = []
    t_end = time.perf_counter() + bound_s
    while time.perf_counter() < t_end and len(secs) < 50:
        if kind == "reference":
            _, s = oracle.ref_compact_timed(job)
        else:
            _, s = oracle.oracle_compact_timed(job)
        secs.append(s)
    med = float(np.median(secs))
    return {"value": mib / med, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{len(secs)} runs of the full {mib:.1f} MiB job, median "
                      f"DoCompactionWork time {med * 1e3:.1f} ms"}


def _upload(tables, torch):
    """Input tables back to back in one device buffer (16-byte aligned starts)."""
    offs, total = [], 0
    for f in tables:
        offs.append(total)
        total += (len(f.data) + 15) // 16 * 16
    buf = torch.zeros(total + 16, dtype=torch.uint8, device="cuda")
    for f, o in zip(tables, offs):
        buf[o:o + len(f.data)] = torch.frombuffer(bytearray(f.data), dtype=torch.uint8).to("cuda")
    return buf, [buf.data_ptr() + o for o in offs]


def _pin(tables, torch):
    keep = []
    for f in tables:
        t = torch.empty(max(1, len(f.data)), dtype=torch.uint8).pin_memory()
        t[:len(f.data)].copy_(torch.frombuffer(bytearray(f.data), dtype=torch.uint8))
        keep.append(t)
        f.data = t[:len(f.data)].numpy()
    return keep


def _pct(v, q):
    return float(np.percentile(np.asarray(v, dtype=np.float64), q)) if len(v) else None


def batched_leg(eng, args, rank, flush, torch):
    """64 independent jobs (log-uniform 1-64 MiB input, 2-12 tables, 16-byte
    keys and 100-byte values), all submitted at once: run one after another
    through lc_compact (plain) and as batches through lc_compact_batch after
    the autotuner has picked the launch settings.  A job's latency is the
    time from the common start to its own completion."""
    from luda_b200 import workloads
    jobs = [workloads.batched_job(s + 1000 * rank) for s in range(args.batch_jobs)]
    for j in jobs:
        j.materialize(lambda e, o: eng.build_table(e, o))
    in_bytes = [j.input_bytes() for j in jobs]
    total_in = float(sum(in_bytes))
    bufs, prep_dev = [], []
    for j in jobs:
        buf, ptrs = _upload(j.input_tables(), torch)
        bufs.append(buf)
        prep_dev.append(eng.prepare(j, device_tables=ptrs, outputs_on_device=True))
    pins = []
    for j in jobs:
        pins += _pin(j.input_tables(), torch)
    prep_host = [eng.prepare(j) for j in jobs]
    torch.cuda.synchronize()
    # same bytes alone and batched (untimed)
    alone = [eng.run(p) for p in prep_host[:8]]
    batched = eng.run_batch(prep_host[:8])
    assert [a.file_bytes() for a in alone] == [b.file_bytes() for b in batched]
    for r in alone + batched:
        r.release()
    tuning = eng.autotune(prep_dev, repeats=1)
    steps = max(1, args.batch_steps)

    def plain_step(preps):
        lat = []
        t0 = time.perf_counter()
        launches = 0
        for p in preps:
            r = eng.run(p)
            lat.append((time.perf_counter() - t0) * 1e3)
            launches += r.kernel_launches
            r.release()
        return lat, launches

    def batch_step(preps):
        t0 = time.perf_counter()
        rs = eng.run_batch(preps)
        ms = (time.perf_counter() - t0) * 1e3
        launches = rs[0].kernel_launches if rs else 0
        for r in rs:
            r.release()
        return [ms] * len(preps), launches

    out = {}
    for name, fn, preps in (("plain", plain_step, prep_dev), ("batched", batch_step, prep_dev),
                            ("plain_e2e", plain_step, prep_host),
                            ("batched_e2e", batch_step, prep_host)):
        for _ in range(3):  # untimed: graphs, slabs and pinned memory for every part
            fn(preps)
        dev_ms, lats, launches = [], [], 0
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            lat, nl = fn(preps)
            e1.record()
            torch.cuda.synchronize()
            dev_ms.append(e0.elapsed_time(e1))
            lats += lat
            launches += nl
        ms = float(np.sum(dev_ms))
        out[name] = {"value": steps * total_in / MiB / (ms / 1e3), "unit": UNIT,
                     "ms_per_step": ms / steps, "p50_ms": _pct(lats, 50), "p99_ms": _pct(lats, 99),
                     "kernel_launches_per_step": launches / steps}
    for b in bufs:
        del b
    return {
        "workload": "batched_64 (log-uniform 1-64 MiB per job, 2-12 tables, 16 B keys, 100 B values)",
        "jobs": len(jobs), "input_mib": total_in / MiB,
        "job_mib_min": min(in_bytes) / MiB, "job_mib_max": max(in_bytes) / MiB,
        "steps": steps, "tuning": tuning, **out,
        "speedup_batched_vs_plain": out["batched"]["value"] / out["plain"]["value"],
        "speedup_batched_vs_plain_e2e": out["batched_e2e"]["value"] / out["plain_e2e"]["value"],
        "note": "device-resident inputs and outputs for plain/batched; host pinned buffers for *_e2e; "
                "all jobs start together, latency = completion time from the common start",
    }


def served_leg(args, local, rank, torch):
    """Served compaction: simulated databases fed by a random-fill stream
    (4 MiB flushes of 16-byte keys uniform over 2^26 and 100-byte values)
    whose level-0 -> level-1 and deeper compactions run through one engine.
    Capacity is measured closed-loop (every flush available at once); then
    flushes arrive as a Poisson process at fractions of the served capacity.
    The plain drop-in (one compaction at a time, host buffers) runs the same
    traces.  Both engines are long-lived, as a server keeps them."""
    from luda_b200 import served
    from luda_b200.device_buffers import TorchUploader
    from luda_b200.engine import Engine
    builder = Engine(local, max_inflight=1)
    flushes = served.make_flushes(args.served_dbs, args.served_flushes,
                                  lambda e, o: builder.build_table(e, o), seed=3 + 100 * rank)
    builder.close()
    for fl in flushes:  # pinned host copies: an arriving table is in host memory
        for f in fl:
            t = torch.empty(len(f.data), dtype=torch.uint8).pin_memory()
            t.copy_(torch.frombuffer(bytearray(f.data), dtype=torch.uint8))
            f.data = t.numpy()
    up = TorchUploader(local)
    # phase timing: per-phase CUDA events of each batch, reported for the slowest jobs
    engines = {"served": Engine(local, max_inflight=4, pinned_reserve=4 << 30, phase_timing=True),
               "plain": Engine(local, max_inflight=1, max_batch=1, pinned_reserve=4 << 30,
                               phase_timing=True)}

    def run(mode, rate):
        eng = engines[mode]
        if mode == "served":
            srv = served.Server(eng, len(flushes), mode="served", upload=up.upload, free=up.free,
                                ready=up.ready)
        else:
            srv = served.Server(eng, len(flushes), mode="plain")
        s0 = eng.stats()
        try:
            st = srv.run(served.schedule(flushes, rate))
        finally:
            srv.close()
        s1 = eng.stats()
        out = st.summary()
        out["offered_flushes_per_s"] = rate
        out["engine"] = {k: s1[k] - s0[k] for k in (
            "batches", "graph_captures", "graph_replays", "direct_tails", "block_takes",
            "block_take_us", "staging_grows", "pinned_slab_grows", "scratch_slab_grows",
            "device_out_slab_grows", "exact_reruns")}
        # over the engine's life so far
        out["engine"]["setup_us_max"] = s1["setup_us_max"]
        for k in ("pinned", "scratch", "scratch_peak", "device_out", "device_out_peak"):
            out["engine"][k + "_mib"] = s1[k + "_bytes"] / float(1 << 20)
        return out

    # warm-up: graphs, memory pools, pinned slabs, at every arrival pattern
    run("served", None)
    run("plain", None)
    cap = run("served", None)
    plain_cap = run("plain", None)
    flush_rate = cap["flushes"] / cap["makespan_s"]
    for rho in args.served_loads:
        run("served", rho * flush_rate)
    loads = {}
    for rho in args.served_loads:
        rate = rho * flush_rate
        loads[f"{rho:g}"] = {"served": run("served", rate), "plain": run("plain", rate)}
    for e in engines.values():
        e.close()
    n_flushes = sum(len(f) for f in flushes)
    return {
        "workload": f"served ({args.served_dbs} databases x {args.served_flushes} flushes of 4 MiB, "
                    "random fill, 16 B keys uniform over 2^26, 100 B values)",
        "flushes": n_flushes, "flush_mib": n_flushes * 4.0,
        "capacity": {"served": cap, "plain": plain_cap,
                     "speedup_served_vs_plain": cap["value"] / plain_cap["value"]},
        "loads": loads,
        "note": "job latency = engine submit -> completion; value = compaction input MiB / makespan; "
                "loads are fractions of the closed-loop served capacity in flushes/s",
    }


def reduce_over_ranks(dist, device, total_ms, e2e_total, in_bytes):
    """Whole-job figures over the ranks (replicas, one job stream per GPU):
    the slowest rank's timed totals and the input bytes of all ranks, so that
    value = all bytes / slowest time.  ``dist`` None: one process."""
    if dist is None:
        return float(total_ms), float(e2e_total), float(in_bytes)
    import torch
    t = torch.tensor([total_ms, e2e_total], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    b = torch.tensor([float(in_bytes)], device=device, dtype=torch.float64)
    dist.all_reduce(b)
    return float(t[0]), float(t[1]), float(b[0])


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import torch
    from luda_b200.engine import Engine

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    job = make_job(args.scale, 1 + 1000 * rank)
    eng = Engine(local, phase_timing=True, max_inflight=4, graphs=not args.no_graphs)
    # input tables built by the engine's own flush encoder
    job.materialize(lambda e, o: eng.build_table(e, o))
    tables = job.input_tables()
    in_bytes = job.input_bytes()
    offs, total = [], 0
    for f in tables:
        offs.append(total)
        total += (len(f.data) + 15) // 16 * 16
    dev_in = torch.zeros(total + 16, dtype=torch.uint8, device="cuda")
    for f, o in zip(tables, offs):
        dev_in[o:o + len(f.data)] = torch.frombuffer(bytearray(f.data), dtype=torch.uint8).to("cuda")
    ptrs = [dev_in.data_ptr() + o for o in offs]
    # pinned host copies for the end-to-end leg
    pinned = []
    for f in tables:
        t = torch.empty(len(f.data), dtype=torch.uint8).pin_memory()
        t.copy_(torch.frombuffer(bytearray(f.data), dtype=torch.uint8))
        pinned.append(t)
    for f, t in zip(tables, pinned):
        f.data = t.numpy()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()

    # consistency of the two paths (untimed): same file sizes
    prep_dev = eng.prepare(job, device_tables=ptrs, outputs_on_device=True)
    prep_host = eng.prepare(job)
    host_res = eng.run(prep_host)
    dev_res = eng.run(prep_dev)
    assert dev_res.bytes_out == host_res.bytes_out and len(dev_res.files) == len(host_res.files)
    host_res.release()
    dev_res.release()

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        eng.run(prep_dev).release()
    barrier()
    torch.cuda.synchronize()
    ms_steps, phases, launches = [], [], 0
    bytes_out = 0
    # the timed call is the bare C ABI (lc_compact); the Python result
    # objects are built from the last step only, outside the timed region
    with ClockSampler(local) as clocks:
        clocks.mark_start()
        for step in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            jh, out = eng.run_raw(prep_dev)
            e1.record()
            torch.cuda.synchronize()
            ms_steps.append(e0.elapsed_time(e1))
            phases.append({out.phase_name[i].decode(): out.phase_ms[i] for i in range(out.n_phases)})
            launches += out.kernel_launches
            bytes_out = out.bytes_out
            eng.release_raw(jh)
        clocks.mark_end()
    r = eng.run(prep_dev)
    r.release()
    barrier()
    torch.cuda.synchronize()
    total_ms = float(sum(ms_steps))

    # end to end through host buffers: K jobs through the asynchronous C ABI
    # (lc_job_submit / lc_job_wait), at most `depth` in flight, so that one
    # job's host<->device copies overlap another job's kernels.  Every job
    # copies its own inputs in and its own outputs out.
    depth = 4

    def pipelined(n):
        inflight, done, submitted, d2h = [], 0, 0, 0
        while done < n:
            while submitted < n and len(inflight) < depth:
                inflight.append(eng.submit_prepared(prep_host))
                submitted += 1
            r = inflight.pop(0).wait()
            d2h = r.bytes_out
            r.release()
            done += 1
        return d2h

    # warm-up of the same pipelined path (worker slots, pools, pinned slabs)
    pipelined(max(2 * depth, args.warmup))
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    d2h = pipelined(args.steps)
    e1.record()
    torch.cuda.synchronize()
    e2e_total = e0.elapsed_time(e1)
    # the same, one job at a time (lc_compact), for reference
    seq_ms = []
    for _ in range(min(args.steps, 20)):
        t0 = time.perf_counter()
        r = eng.run(prep_host)
        seq_ms.append((time.perf_counter() - t0) * 1e3)
        r.release()

    batched = None
    if args.batch_steps > 0:
        batched = batched_leg(eng, args, rank, flush, torch)
    served_res = None
    if args.served_flushes > 0:
        served_res = served_leg(args, local, rank, torch)

    total_ms, e2e_total, all_in = reduce_over_ranks(dist, "cuda", total_ms, e2e_total, in_bytes)
    value = args.steps * all_in / MiB / (total_ms / 1e3)
    e2e_value = args.steps * all_in / MiB / (e2e_total / 1e3)

    # roofline: algorithmic bytes of the three bandwidth-bound kernels
    n_in = r.entries_in
    k_in = r.key_bytes_in
    n_keep = r.entries_out
    alg = {
        "decode": in_bytes + k_in + 16 * n_in,
        "merge": k_in + 16 * n_in + 4 * n_in,
        "encode_blocks": r.key_bytes_out + r.value_bytes_out + bytes_out,
    }
    mean_ph = {k: float(np.mean([p[k] for p in phases])) for k in phases[0]}
    dominant = max(alg, key=lambda k: mean_ph[k])
    peak, peak_kind = measured_peak()
    achieved = alg[dominant] / (mean_ph[dominant] / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (NCU_TRAFFIC.get(dominant) if args.scale == 1.0 else None),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch",
                "algorithmic_bytes": alg[dominant],
                "phase_ms": mean_ph,
                "per_kernel_gbs": {k: alg[k] / (mean_ph[k] / 1e3) / 1e9 for k in alg
                                   if mean_ph[k] > 0}}

    if rank == 0:
        cpu = None
        if world == 1 and args.cpu_seconds > 0:
            try:
                cpu = cpu_baseline(job, args.cpu_seconds)
            except Exception as ex:  # the baseline is reported, never required
                cpu = {"error": str(ex)}
        lat = np.array(ms_steps)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": WORKLOAD, "input_mib": in_bytes / MiB,
                       "output_mib": bytes_out / MiB, "entries_in": n_in, "entries_out": n_keep,
                       "output_files": len(r.files), "parallelism": f"replicas{world}",
                       "l2": "flushed between steps (256 MiB write)", "scale": args.scale},
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p99": float(np.percentile(lat, 99))},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": in_bytes,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_total / args.steps,
                    "jobs_in_flight": depth,
                    "sequential_ms_per_step": float(np.mean(seq_ms)),
                    "sequential_value": in_bytes / MiB / (float(np.mean(seq_ms)) / 1e3)},
            "roofline": roofline,
            "batched": batched,
            "served": served_res,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "gpu_launches": launches,
            "host": {"cpus": os.cpu_count()},
        }
        print(json.dumps(line))
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
