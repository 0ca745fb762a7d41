"""Generates tests/golden/golden.json from the reference itself.

For every case (the seeded workloads at the sizes the tests use, and the edge
cases of tests/edge_jobs.py) the input tables are built with the reference's
own TableBuilder and compacted with the reference's own CPU
DBImpl::DoCompactionWork (both from oracle/_ref/libluda_ref.so, compiled from
the reference sources by oracle/Makefile).  The fixture records the SHA-256 of
every input table and every output file, with each output's size and
smallest/largest internal keys, so that the GPU tests can check byte identity
on a machine where the reference sources are absent.

Run from the repository root:  python tests/golden/make_golden.py
(``--large`` re-records only the 1 GiB cases, keeping the others.)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from luda_b200 import workloads  # noqa: E402
import edge_jobs  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "golden.json")

# (case name, generator, kwargs): generators are in luda_b200.workloads
WORKLOAD_CASES = [
    ("plain_l0_l1", "plain_l0_l1", {"seed": 0, "scale": 1.0}),
    ("plain_l0_l1_small", "plain_l0_l1", {"seed": 3, "scale": 0.1}),
    ("l1_l2_at_size", "l1_l2_at_size", {"seed": 1, "scale": 1.0}),
    ("l1_l2_quarter", "l1_l2_at_size", {"seed": 2, "scale": 0.25}),
    ("large_A_small", "large_l2_l3", {"run": "A", "seed": 4, "scale": 0.05}),
    ("large_B_small", "large_l2_l3", {"run": "B", "seed": 4, "scale": 0.05}),
] + [(f"batched_{i}", "batched_job", {"seed": i, "scale": 0.1}) for i in range(4)]

# The 1 GiB L2->L3 compactions at size (1 + 15 tables of 64 MiB): run A with
# 8-byte keys and 1 KiB values, run B with 24-byte keys and 32-byte values.
LARGE_CASES = [
    ("large_A", "large_l2_l3", {"run": "A", "seed": 4, "scale": 1.0}),
    ("large_B", "large_l2_l3", {"run": "B", "seed": 4, "scale": 1.0}),
]


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def make_job(gen: str, kwargs: dict):
    return getattr(workloads, gen)(**kwargs)


def record(name, job, spec, large=False):
    job.materialize(lambda e, o: oracle.build_table(e, o, "ref"))
    # the restatement's builder must agree with the reference's
    for f in job.files:
        if f.entries is not None:
            assert oracle.build_table(f.entries, job.options, "oracle") == f.data, name
    outs, secs = oracle.ref_compact_timed(job)
    full = oracle.compact(job, "ref")
    rec = {
        "name": name,
        "spec": spec,
        "input_bytes": job.input_bytes(),
        "inputs": [sha(f.data) for f in job.input_tables()],
        "outputs": [{"sha256": sha(d), "size": len(d), "smallest": s.hex(), "largest": l.hex()}
                    for (d, s, l) in full],
        "ref_seconds": secs,
    }
    if large:
        rec["large"] = True
    print(f"{name:28s} in={job.input_bytes():>10d} files={len(full):3d} ref={secs * 1e3:8.1f} ms",
          flush=True)
    return rec


def main(argv):
    if not oracle.has_ref():
        oracle.build(ref=True)
    cases = []
    if "--large" in argv:
        with open(OUT) as f:
            cases = [c for c in json.load(f)["cases"] if not c.get("large")]
    else:
        for name, gen, kw in WORKLOAD_CASES:
            cases.append(record(name, make_job(gen, kw), {"workload": gen, "kwargs": kw}))
        for job in edge_jobs.all_cases():
            cases.append(record(job.name, job, {"edge": job.name}))
    for name, gen, kw in LARGE_CASES:
        cases.append(record(name, make_job(gen, kw), {"workload": gen, "kwargs": kw}, large=True))
    with open(OUT, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "reference": "xpsair/luda CPU DoCompactionWork (GPU_ACCELERATE 0)",
                   "cases": cases}, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main(sys.argv[1:])
