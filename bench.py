"""Compaction throughput benchmark (one JSON line on rank 0).

Headline workload: the large L2->L3 compaction (1 + 15 tables of 64 MiB,
1 GiB of input; run A: 8-byte big-endian keys with 1 KiB values, one
snapshot, 1% deletion markers, 64 MiB output files), synthetic and seeded.
One step = one compaction job through the engine's C ABI.

* value: MiB of input compacted per second with the input tables already in
  HBM and the outputs left in HBM (lc_job_desc.inputs_on_device /
  outputs_on_device), timed with CUDA events around the bare lc_compact call
  on an engine without phase timing.  The input (1 GiB) is larger than L2,
  and L2 is also flushed between steps.
* e2e: the same job through the asynchronous C ABI (lc_job_submit /
  lc_job_wait) with the tables in pinned host memory, four jobs in flight:
  every job's host->device copy of its inputs and device->host copy of its
  output files are inside the timed region.
* pcie: host<->device copy bandwidth of the job's bytes measured on their
  own, and the engine's own upload and download phases.
* roofline: the slowest of the three bandwidth-bound kernels (decode, merge,
  data-block encode), from a separate pass of the same steps on an engine
  that records per-phase CUDA events on the job's stream, against the
  measured HBM copy bandwidth; per_kernel_gbs for every phase.
* parity: the SHA-256 of every output file of the last timed step (and of
  the host-buffer path) must equal the reference's, recorded in
  tests/golden/golden.json; a mismatch fails the run.
* legs: run B (24-byte keys, 32-byte values: 16M entries), the L1->L2
  compaction at size (66 MiB) and the plain L0->L1 compaction, measured the
  same way; the batched (64 uneven jobs) and served (request loop) legs.
* cpu_baseline: the reference's own CPU DoCompactionWork on one host core on
  the same job (and, for the batched and served legs, the reference on the
  same jobs and traces).

--impl reference times the reference's CPU compaction on all usable host
cores (one job per thread) on the headline job instead.

Multi-GPU (torchrun): every rank compacts its own job stream on its own GPU
(replicas; no collective on the data path); value sums all ranks' input bytes
over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import hashlib
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
MiB = float(1 << 20)
GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.json")

# name -> (generator in luda_b200.workloads, its arguments, description)
WORKLOADS = {
    "large_A": ("large_l2_l3", {"run": "A", "seed": 4},
                "large_l2_l3 run A: L2->L3, 1 + 15 tables of 64 MiB (1 GiB), 8-byte big-endian "
                "uniform u64 keys, 1 KiB values, 1 snapshot, 1% deletion markers, 64 MiB files"),
    "large_B": ("large_l2_l3", {"run": "B", "seed": 4},
                "large_l2_l3 run B: L2->L3, 1 + 15 tables of 64 MiB (1 GiB), 24-byte keys, "
                "32-byte values (about 16M entries), 1 snapshot, 1% deletion markers"),
    "l1_l2_at_size": ("l1_l2_at_size", {"seed": 1},
                      "l1_l2_at_size: 1 L1 table of 2 MiB over 32 L2 tables of 2 MiB, Zipf(0.99) "
                      "keys of 8-64 bytes, lognormal values, 3 snapshots, 5% deletion markers"),
    "plain_l0_l1": ("plain_l0_l1", {"seed": 0},
                    "plain_l0_l1: 2 L0 + 2 L1 tables of ~20k entries, %016d keys, 100-byte values"),
}
HEADLINE = "large_A"
LEGS = ["large_B", "l1_l2_at_size", "plain_l0_l1"]


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="luda", choices=["luda", "reference"])
    p.add_argument("--scale", type=float, default=1.0,
                   help="table size scale of every workload (1: full size)")
    p.add_argument("--cpu-seconds", type=float, default=10.0,
                   help="bound on each CPU baseline sample")
    p.add_argument("--no-graphs", action="store_true",
                   help="launch every kernel directly instead of replaying CUDA graphs")
    p.add_argument("--legs", nargs="*", default=LEGS,
                   help="extra single-job legs, measured like the headline")
    p.add_argument("--leg-steps", type=int, default=10)
    p.add_argument("--batch-jobs", type=int, default=64)
    p.add_argument("--served-dbs", type=int, default=16)
    p.add_argument("--served-flushes", type=int, default=16,
                   help="flushes per database (0: skip the served leg)")
    p.add_argument("--served-loads", type=float, nargs="*", default=[0.5, 0.9])
    p.add_argument("--batch-steps", type=int, default=5,
                   help="timed repetitions of the 64-job set (0: skip the batched leg)")
    return p.parse_args()


# DRAM bytes (read + write) per launch of each kernel, from one ncu capture
# on each workload: (workload, kernel) -> bytes; None where none was taken.
# large_A's capture ran at scale 0.25 (profiles/k_encode_blocks_large_A.md:
# 276.8 + 222.3 MB); the kernel's traffic grows with the bytes it moves, so
# the full-size figure is four times that.
NCU_TRAFFIC = {
    ("large_A", "encode_blocks"): 4 * (276.840960e6 + 223.603712e6),
}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_job(name: str, scale: float):
    from luda_b200 import workloads
    gen, kw, _ = WORKLOADS[name]
    return getattr(workloads, gen)(**kw, scale=scale)


def golden_case(name: str, scale: float):
    """The fixture case recorded from the reference for this workload, if any."""
    gen, kw, _ = WORKLOADS[name]
    try:
        with open(GOLDEN) as f:
            cases = json.load(f)["cases"]
    except OSError:
        return None
    want = {"workload": gen, "kwargs": {**kw, "scale": scale}}
    for c in cases:
        if c.get("spec") == want:
            return c
    return None


def sha(b) -> str:
    return hashlib.sha256(b).hexdigest()


def check_outputs(case, blobs, what):
    """Raises unless the output files hash to the reference's."""
    got = [(len(b), sha(b)) for b in blobs]
    want = [(g["size"], g["sha256"]) for g in case["outputs"]]
    if got != want:
        raise SystemExit(f"bench: {what}: output differs from the reference's "
                         f"({len(got)} files vs {len(want)})")


def device_bytes(ptr, n):
    from cuda.bindings import runtime as rt
    out = np.empty(max(1, n), np.uint8)
    if n:
        err, = rt.cudaMemcpy(out.ctypes.data, ptr, n, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == rt.cudaError_t.cudaSuccess, err
    return out[:n]


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



def reference_arm(args, rank):
    """The reference's own CPU DoCompactionWork (oracle/_ref) on the headline
    job: per step, one copy of the job per usable host core, each on its own
    in-memory DB in its own thread."""
    if rank != 0:
        return
    import oracle
    if not oracle.has_ref():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU build (oracle/_ref) not present"}))
        return
    job = make_job(HEADLINE, args.scale)
    job.materialize(lambda e, o: oracle.build_table(e, o, "ref"))
    mib = job.input_bytes() / MiB
    cores = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
        cores = max(1, min(cores, int(avail // (4 * job.input_bytes()))))
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
        "config": {"workload": WORKLOADS[HEADLINE][2], "input_mib": mib, "jobs_per_step": cores,
                   "scale": args.scale},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{cores} concurrent copies of the {mib:.1f} MiB job per step "
                                   f"(reference CPU DoCompactionWork, one DB per thread)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def cpu_baseline(job, bound_s):
    """The reference's DoCompactionWork on one core, repeated for about
    bound_s seconds (at least once); the median run."""
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


def _pct(v, q):
    return float(np.percentile(np.asarray(v, dtype=np.float64), q)) if len(v) else None


def alg_bytes(r, in_bytes):
    """Algorithmic bytes per launch of each phase: what the phase must read
    and write at the least.  S_in input bytes, N_in / K_in input entries and
    their key bytes, N_keep / K_keep / V_keep survivors and their key and
    value bytes, S_out output bytes."""
    n_in, k_in = r.entries_in, r.key_bytes_in
    n_keep, k_keep, v_keep = r.entries_out, r.key_bytes_out, r.value_bytes_out
    return {
        # the decode reads the 32-byte sectors holding the entry headers and
        # key deltas (values are not read; at most the whole input), writes
        # the keys and 32 bytes of entry arrays, and passes a 16-byte record
        # per entry from its header walk to its key pass
        "decode": min(in_bytes, 32 * n_in + k_in) + k_in + 32 * n_in + 32 * n_in,
        "merge": k_in + 16 * n_in + 4 * n_in,
        # merged ids, key offsets and lengths, tags, prefixes; keep flags and
        # grandparent counts written
        "drop": 33 * n_in,
        "partition": k_keep + 24 * n_keep,
        "encode_blocks": k_keep + v_keep + r.bytes_out,
    }


def job_leg(name, args, eng, eng_ph, flush, torch, steps, warmup, clocks=None, pcie=False,
            cpu=True):
    """One workload, one job per step: device-resident timing on `eng`
    (no phase events), a phase pass on `eng_ph`, end to end through host
    buffers, parity of the timed outputs against the reference's hashes."""
    job = make_job(name, args.scale)
    job.materialize(lambda e, o: eng.build_table(e, o))
    tables = job.input_tables()
    in_bytes = job.input_bytes()
    case = golden_case(name, args.scale)
    if case is not None and [sha(f.data) for f in tables] != case["inputs"]:
        raise SystemExit(f"bench: {name}: input tables differ from the reference's")
    offs, total = [], 0
    for f in tables:
        offs.append(total)
        total += (len(f.data) + 15) // 16 * 16
    dev_in = torch.zeros(total + 16, dtype=torch.uint8, device="cuda")
    for f, o in zip(tables, offs):
        dev_in[o:o + len(f.data)] = torch.frombuffer(bytearray(f.data), dtype=torch.uint8).to("cuda")
    ptrs = [dev_in.data_ptr() + o for o in offs]
    pinned = []
    for f in tables:
        t = torch.empty(max(1, len(f.data)), dtype=torch.uint8).pin_memory()
        t[:len(f.data)].copy_(torch.frombuffer(bytearray(f.data), dtype=torch.uint8))
        pinned.append(t)
    for f, t in zip(tables, pinned):
        f.data = t[:len(f.data)].numpy()
    torch.cuda.synchronize()
    prep_dev = eng.prepare(job, device_tables=ptrs, outputs_on_device=True)
    prep_host = eng.prepare(job)

    # parity of both paths before timing (host buffers here; the timed
    # device-resident path on its last step below)
    host_res = eng.run(prep_host)
    if case is not None:
        check_outputs(case, host_res.file_bytes(), f"{name} (host buffers)")
    host_res.release()

    # warm-up keeps outputs alive the way the timed loop does (a step's output
    # is released after the next step has run), so that the engine's device
    # memory for two outputs is taken before timing
    last = None
    for _ in range(warmup):
        w = eng.run_raw(prep_dev)
        if last is not None:
            eng.release_raw(last[0])
        last = w
    torch.cuda.synchronize()
    ms_steps, launches = [], 0
    if clocks:
        clocks.mark_start()
    for step in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        jh, out = eng.run_raw(prep_dev)
        e1.record()
        torch.cuda.synchronize()
        ms_steps.append(e0.elapsed_time(e1))
        launches += out.kernel_launches
        if last is not None:
            eng.release_raw(last[0])
        last = (jh, out)
    if clocks:
        clocks.mark_end()
    jh, out = last
    blobs = []
    if case is not None:
        whole = device_bytes(out.device_data, out.bytes_out)
        blobs = [whole[out.file_offset[i]:out.file_offset[i] + out.file_size[i]].tobytes()
                 for i in range(out.n_files)]
        check_outputs(case, blobs, f"{name} (last timed step, device-resident)")
    parity = ({"checked": True, "files": out.n_files,
               "against": "SHA-256 of every output file recorded from the reference's CPU "
                          "DoCompactionWork (tests/golden/golden.json)"}
              if case is not None else {"checked": False, "why": "no fixture at this scale"})
    eng.release_raw(jh)
    del blobs

    # phase pass: same steps, per-phase CUDA events on the job's stream
    prep_ph = eng_ph.prepare(job, device_tables=ptrs, outputs_on_device=True)
    for _ in range(max(1, warmup)):
        eng_ph.run(prep_ph).release()
    phases, ph_ms, stats_r = [], [], None
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        r = eng_ph.run(prep_ph)
        phases.append(r.phase_ms)
        ph_ms.append(r.device_ms)
        stats_r = r
        r.release()
    mean_ph = {k: float(np.mean([p[k] for p in phases])) for k in phases[0]}

    # end to end through host buffers: jobs through lc_job_submit /
    # lc_job_wait, at most `depth` in flight, so that one job's copies
    # overlap another job's kernels; every job copies its own inputs in and
    # its own outputs out
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

    pipelined(max(2 * depth, warmup))
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    d2h = pipelined(steps)
    e1.record()
    torch.cuda.synchronize()
    e2e_total = e0.elapsed_time(e1)
    seq_ms = []
    for _ in range(min(steps, 10)):
        t0 = time.perf_counter()
        r = eng.run(prep_host)
        seq_ms.append((time.perf_counter() - t0) * 1e3)
        r.release()

    # host<->device links: the job's bytes on their own, and the engine's
    # own upload / download phases (phase events, one job from host buffers)
    link = None
    if pcie:
        src = torch.cat([t[:len(f.data)] for f, t in zip(tables, pinned)])
        src = src.pin_memory()
        dst = torch.empty_like(src, device="cuda")
        back = torch.empty(d2h, dtype=torch.uint8).pin_memory()
        h2d, dh = [], []
        for _ in range(3):
            a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a.record()
            dst.copy_(src, non_blocking=True)
            b.record()
            back.copy_(dst[:d2h], non_blocking=True)
            c.record()
            torch.cuda.synchronize()
            h2d.append(a.elapsed_time(b))
            dh.append(b.elapsed_time(c))
        p_host = eng_ph.prepare(job)
        eng_ph.run(p_host).release()  # pinned output memory taken once, outside the figure
        r = eng_ph.run(p_host)
        up_ms, down_ms = r.phase_ms["upload"], r.phase_ms["download"]
        r.release()
        link = {"h2d_gbs": src.numel() / (min(h2d) / 1e3) / 1e9,
                "d2h_gbs": d2h / (min(dh) / 1e3) / 1e9,
                "engine_upload_gbs": in_bytes / (up_ms / 1e3) / 1e9 if up_ms > 0 else None,
                "engine_download_gbs": d2h / (down_ms / 1e3) / 1e9 if down_ms > 0 else None,
                "bytes_h2d": int(src.numel()), "bytes_d2h": int(d2h),
                "note": "copy test: one pinned-host<->device copy of the job's input and output "
                        "bytes, best of 3; engine: its upload and download phases for one job "
                        "from host buffers (copies in pieces of about a sixteenth of the job, 2-64 MiB)"}
        del src, dst, back

    cpu_res = None
    if cpu and args.cpu_seconds > 0:
        try:
            cpu_res = cpu_baseline(job, args.cpu_seconds)
        except Exception as ex:  # the baseline is reported, never required
            cpu_res = {"error": str(ex)}
    del dev_in, pinned
    torch.cuda.empty_cache()

    total_ms = float(sum(ms_steps))
    alg = alg_bytes(stats_r, in_bytes)
    r = stats_r
    return {
        "workload": WORKLOADS[name][2], "input_mib": in_bytes / MiB,
        "output_mib": r.bytes_out / MiB, "entries_in": r.entries_in, "entries_out": r.entries_out,
        "output_files": len(r.files), "steps": steps,
        "value": steps * in_bytes / MiB / (total_ms / 1e3), "unit": UNIT,
        "ms_per_step": total_ms / steps,
        "latency_ms": {"p50": _pct(ms_steps, 50), "p99": _pct(ms_steps, 99)},
        "phase_pass_ms_per_step": float(np.mean(ph_ms)),
        "phase_ms": mean_ph,
        "alg_bytes": alg,
        "per_kernel_gbs": {k: alg[k] / (mean_ph[k] / 1e3) / 1e9 for k in alg if mean_ph.get(k, 0) > 0},
        "e2e": {"value": steps * in_bytes / MiB / (e2e_total / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_total / steps, "jobs_in_flight": depth,
                "sequential_ms_per_step": float(np.mean(seq_ms)),
                "sequential_value": in_bytes / MiB / (float(np.mean(seq_ms)) / 1e3)},
        "pcie": link,
        "parity": parity,
        "gpu_launches": launches,
        "cpu_baseline": cpu_res,
        "_total_ms": total_ms, "_e2e_total_ms": e2e_total, "_in_bytes": in_bytes,
    }


def roofline_of(leg, name, scale):
    """The slowest of decode / merge / encode_blocks against the HBM peak."""
    peak, peak_kind = measured_peak()
    ph, alg = leg["phase_ms"], leg["alg_bytes"]
    cands = [k for k in ("decode", "merge", "encode_blocks") if ph.get(k, 0) > 0]
    dom = max(cands, key=lambda k: ph[k])
    achieved = alg[dom] / (ph[dom] / 1e3) / 1e9
    traffic = NCU_TRAFFIC.get((name, dom)) if scale == 1.0 else None
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch "
                              "(profiles/)",
            "algorithmic_bytes": alg[dom],
            "whole_job": {"bytes": leg["_in_bytes"] + leg["output_mib"] * MiB,
                          "achieved": (leg["_in_bytes"] + leg["output_mib"] * MiB) /
                          (leg["ms_per_step"] / 1e3) / 1e9,
                          "frac": (leg["_in_bytes"] + leg["output_mib"] * MiB) /
                          (leg["ms_per_step"] / 1e3) / 1e9 / peak},
            "per_kernel_frac": {k: v / peak for k, v in leg["per_kernel_gbs"].items()}}


def _pin(tables, torch):
    keep = []
    for f in tables:
        t = torch.empty(max(1, len(f.data)), dtype=torch.uint8).pin_memory()
        t[:len(f.data)].copy_(torch.frombuffer(bytearray(f.data), dtype=torch.uint8))
        keep.append(t)
        f.data = t[:len(f.data)].numpy()
    return keep


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


def batched_cpu_baseline(jobs, bound_s):
    """The reference's DoCompactionWork over the same jobs: one after another
    on one core (per-job completion latency from the common start), and all
    jobs spread over one thread per host core (one DB per thread)."""
    import concurrent.futures as cf
    import oracle
    if not oracle.has_ref():
        return {"error": "reference CPU build (oracle/_ref) not present"}
    total = sum(j.input_bytes() for j in jobs) / MiB
    lat, t = [], 0.0
    for j in jobs:
        _, s = oracle.ref_compact_timed(j)
        t += s
        lat.append(t * 1e3)
        if t > 4 * bound_s:
            return {"error": f"sequential pass beyond {4 * bound_s:.0f} s"}
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(cores) as ex:
        list(ex.map(lambda j: oracle.ref_compact_timed(j)[1], jobs))
    par = time.perf_counter() - t0
    return {"kind": "reference", "unit": UNIT,
            "sequential_1core": {"value": total / t, "cores": 1, "p50_ms": _pct(lat, 50),
                                 "p99_ms": _pct(lat, 99)},
            "parallel": {"value": total / par, "cores": cores,
                         "note": "one thread per host core, one in-memory DB per job"},
            "sample": f"all {len(jobs)} jobs ({total:.0f} MiB) once"}


def batched_leg(eng, args, rank, flush, torch, cpu_ok=True):
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
    cpu = batched_cpu_baseline(jobs, args.cpu_seconds) if (rank == 0 and args.cpu_seconds > 0
                                                          and cpu_ok) else None
    return {
        "workload": "batched_64 (log-uniform 1-64 MiB per job, 2-12 tables, 16 B keys, 100 B values)",
        "jobs": len(jobs), "input_mib": total_in / MiB,
        "job_mib_min": min(in_bytes) / MiB, "job_mib_max": max(in_bytes) / MiB,
        "steps": steps, "tuning": tuning, **out,
        "speedup_batched_vs_plain": out["batched"]["value"] / out["plain"]["value"],
        "speedup_batched_vs_plain_e2e": out["batched_e2e"]["value"] / out["plain_e2e"]["value"],
        "cpu_baseline": cpu,
        "note": "device-resident inputs and outputs for plain/batched; host pinned buffers for *_e2e; "
                "all jobs start together, latency = completion time from the common start",
    }



class _RefResult:
    def __init__(self, outs):
        self.files = [type("F", (), {"data": memoryview(d), "smallest": s, "largest": l})
                      for d, s, l in outs]
        self.bytes_out = sum(len(d) for d, _, _ in outs)
        self.device_ptr = None
        self.file_offsets = None

    def release(self):
        pass

    def file_bytes(self):
        return [bytes(f.data) for f in self.files]


class _RefPending:
    def __init__(self, job):
        self.job, self.res, self.h = job, None, object()

    def wait(self, timeout_s=-1.0):
        return self.res


class RefLoopEngine:
    """The reference's CPU compaction as the served loop's engine, on one
    thread: a submitted job runs when the loop waits for a completion, the
    oldest first, so the loop behaves like LevelDB's single background
    compaction thread serving many databases."""

    def __init__(self):
        self.pending = []

    def prepare(self, job, device_tables=None, outputs_on_device=0, keep_decoded=False,
                decoded=None):
        # the loop drops its references to the input buffers after this call
        assert device_tables is None
        return job, [(f, f.data) for f in job.input_tables()]

    def submit_prepared(self, prepared):
        h = _RefPending(prepared)
        self.pending.append(h)
        return h

    def wait_any(self, jobs, timeout_s=-1.0):
        import oracle
        for h in self.pending:
            if h.res is None and h in jobs:
                job, inputs = h.job
                for f, data in inputs:
                    f.data = data
                h.res = _RefResult(oracle.compact(job, "ref"))
                for f, _ in inputs:
                    f.data = None
                self.pending.remove(h)
                return jobs.index(h)
        return None


def served_cpu_baseline(flushes, bound_s):
    """The served traces through a one-thread loop whose compactions are the
    reference's CPU DoCompactionWork (closed loop: every flush available at
    once): MiB/s and p50/p99 job latency."""
    import oracle
    from luda_b200 import served
    if not oracle.has_ref():
        return {"error": "reference CPU build (oracle/_ref) not present"}
    fl = [[f for f in db] for db in flushes]
    srv = served.Server(RefLoopEngine(), len(fl), mode="plain")
    st = srv.run(served.schedule(fl, None))
    srv.close()
    s = st.summary()
    return {"kind": "reference", "cores": 1, "value": s["value"], "unit": UNIT,
            "p50_ms": s["p50_ms"], "p99_ms": s["p99_ms"], "jobs": s["jobs"],
            "input_mib": s["input_mib"], "makespan_s": s["makespan_s"],
            "sample": "the served leg's flush traces once, closed loop, one compaction thread"}


def served_leg(args, local, rank, torch, cpu_ok=True):
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
    cpu = served_cpu_baseline(flushes, args.cpu_seconds) if (rank == 0 and args.cpu_seconds > 0
                                                            and cpu_ok) else None
    n_flushes = sum(len(f) for f in flushes)
    return {
        "workload": f"served ({args.served_dbs} databases x {args.served_flushes} flushes of 4 MiB, "
                    "random fill, 16 B keys uniform over 2^26, 100 B values)",
        "flushes": n_flushes, "flush_mib": n_flushes * 4.0,
        "capacity": {"served": cap, "plain": plain_cap,
                     "speedup_served_vs_plain": cap["value"] / plain_cap["value"]},
        "loads": loads,
        "cpu_baseline": cpu,
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

    def barrier():
        if dist is not None:
            dist.barrier()

    eng = Engine(local, max_inflight=4, graphs=not args.no_graphs)
    eng_ph = Engine(local, max_inflight=1, phase_timing=True, graphs=not args.no_graphs)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    cpu_ok = world == 1
    clocks = ClockSampler(local)
    with clocks:
        barrier()
        head = job_leg(HEADLINE, args, eng, eng_ph, flush, torch, args.steps, args.warmup,
                       clocks=clocks, pcie=True, cpu=cpu_ok and rank == 0)
    barrier()
    legs = {}
    for name in args.legs:
        legs[name] = job_leg(name, args, eng, eng_ph, flush, torch,
                             max(1, min(args.steps, args.leg_steps)), args.warmup,
                             cpu=cpu_ok and rank == 0)
    eng_ph.close()
    batched = None
    if args.batch_steps > 0:
        batched = batched_leg(eng, args, rank, flush, torch, cpu_ok)
    served_res = None
    if args.served_flushes > 0:
        served_res = served_leg(args, local, rank, torch, cpu_ok)

    total_ms, e2e_total, all_in = reduce_over_ranks(dist, "cuda", head["_total_ms"],
                                                    head["_e2e_total_ms"], head["_in_bytes"])
    value = args.steps * all_in / MiB / (total_ms / 1e3)
    e2e = dict(head["e2e"])
    e2e["value"] = args.steps * all_in / MiB / (e2e_total / 1e3)
    roofline = roofline_of(head, HEADLINE, args.scale)
    for name, leg in legs.items():
        leg["roofline"] = roofline_of(leg, name, args.scale)
        for k in ("_total_ms", "_e2e_total_ms", "_in_bytes"):
            leg.pop(k)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": WORKLOADS[HEADLINE][2], "input_mib": head["input_mib"],
                       "output_mib": head["output_mib"], "entries_in": head["entries_in"],
                       "entries_out": head["entries_out"], "output_files": head["output_files"],
                       "parallelism": f"replicas{world}",
                       "l2": "input (1 GiB at scale 1) larger than L2; L2 also flushed "
                             "(256 MiB write) between steps", "scale": args.scale},
            "latency_ms": head["latency_ms"],
            "parity": head["parity"],
            "e2e": e2e,
            "pcie": head["pcie"],
            "roofline": roofline,
            "phase_ms": head["phase_ms"],
            "phase_pass_ms_per_step": head["phase_pass_ms_per_step"],
            "per_kernel_gbs": head["per_kernel_gbs"],
            "legs": legs,
            "batched": batched,
            "served": served_res,
            "cpu_baseline": head["cpu_baseline"],
            "clocks": clocks.summary(),
            "gpu_launches": head["gpu_launches"],
            "host": {"cpus": os.cpu_count()},
        }
        print(json.dumps(line))
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
