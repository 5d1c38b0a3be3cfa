"""Benchmark: plain presolve + postsolve of the 25M-nnz synthetic LP on B200.

One step = gpu_preprocessor::preprocess (presolve) + postprocess (postsolve
of a fixed reduced solution) of the single-GPU scale LP: the seeded random
family at m = 2,000,000, n = 5,000,000 with 2,000 hub rows (~29.8M nnz).  The
inputs stay resident in HBM for `value`; `e2e` repeats the step through the
C ABI with the LP loaded from pinned host memory every step (A as CSR and the
vectors cross PCIe; gpp_lp_from_host builds A^T on the GPU) and the solution
read back into host memory.  The LP (~1 GB of arrays) is larger than the 126 MB L2, so no
flush is needed between steps.

--impl reference times the reference's own CPU implementation of the path,
its bundled PSLP presolver (built from the reference sources into
oracle/_ref/pslp_driver), on the same workload.

Multi-GPU: the plain path does not shard (every presolve round couples all
rows and columns), so --gpus N runs N independent replicas, one per rank;
the value is the max-over-ranks step time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-preprocessor-ijoc_b200"))

WORKLOAD = "scale"
WORKLOAD_DESC = "random LP m=2,000,000 n=5,000,000 + 2,000 hub rows (500-5000 nnz), seed 0"


def workload_desc(name):
    return WORKLOAD_DESC if name == WORKLOAD else f"{name} (lpgen.workload), seed 0"
METRIC = "presolve ms, HBM GB/s @25M nnz (presolve+postsolve ms per LP)"
RULES = ["infeasible_and_fixed_variables", "empty_columns", "empty_rows", "singleton_rows",
         "singleton_columns", "bound_strengthening", "infeasible_and_redundant_rows", "dual_fix",
         "parallel_rows", "parallel_columns", "doubleton_equations"]


# Kernel -> the source files whose text fixes its code; a DRAM traffic
# figure measured by ncu is used only while these files are unchanged.
KERNEL_SOURCES = {
    "activity_kernel<false>": ["csrc/live.cu", "csrc/live_visit.cuh", "csrc/common.cuh"],
    "activity_kernel<true>": ["csrc/live.cu", "csrc/live_visit.cuh", "csrc/common.cuh"],
    "candidates_entries": ["csrc/rules_bound.cu", "csrc/common.cuh"],
    "compact_tiles<true>": ["csrc/compact.cu", "csrc/common.cuh"],
}


def source_digest(files):
    import hashlib
    h = hashlib.sha256()
    for f in files:
        with open(os.path.join(ROOT, "gpu-preprocessor-ijoc_b200", f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def measured_traffic(kernel):
    """DRAM read + write bytes per full-size launch of `kernel` from the ncu
    records under profiles/ (lines 'traffic-record: kernel=... digest=...
    dram_bytes_per_launch=... file=...'), used only when the digest of the
    kernel's sources matches the one recorded with the capture.  Returns
    (bytes or None, the record's file or a reason)."""
    import glob
    files = KERNEL_SOURCES.get(kernel)
    if not files:
        return None, "no ncu record for this kernel"
    digest = source_digest(files)
    stale = None
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        for line in open(path):
            if not line.startswith("traffic-record:"):
                continue
            rec = dict(kv.split("=", 1) for kv in line.split()[1:])
            if rec.get("kernel") != kernel:
                continue
            if rec.get("digest") == digest:
                return float(rec["dram_bytes_per_launch"]), os.path.relpath(path, ROOT)
            stale = os.path.relpath(path, ROOT)
    return None, (f"ncu record {stale} predates the kernel's current sources" if stale
                  else "no ncu record for this kernel")


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.proc = None
        self.file = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.file.flush()
        self.file.seek(0)
        sm, mx, reasons = [], None, set()
        for line in self.file.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                                 parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons)}


BATCH_DESC = ("config-0-style LPs, m log-uniform in [1,000, 200,000], n = 2.5m, seeds 1000+k "
              "(the batched-form workload)")


def batch_jobs(count):
    """(m, seed) of every LP of the batched workload."""
    import numpy as np
    rng = np.random.default_rng(7)
    ms = np.exp(rng.uniform(np.log(1000.0), np.log(200000.0), size=count)).astype(int)
    return [(int(m), 1000 + k) for k, m in enumerate(ms)]


def make_batch_lp(job):
    """Generates one LP of the batched workload (runs in a spawned worker process)."""
    from gpp_b200 import lpgen
    m, seed = job
    lp = lpgen.random_lp(m, int(2.5 * m), seed=seed)
    lp.ensure_transpose()
    return lp


LEARNED_SEEDS = (1, 2, 3)


def make_scale_lp(job):
    """One draw of a named workload (runs in a spawned worker process)."""
    from gpp_b200 import lpgen
    name, seed = job
    return lpgen.workload(name, seed=seed)


def batch_nnz_estimate(job):
    """Expected nnz of one batched-workload LP (n = 2.5 m columns of 1 +
    Poisson(4) entries): the weight of the greedy partition across ranks,
    known before any LP is generated."""
    m, _ = job
    return int(12.5 * m)


def run_batched(indices, lps, params, max_workers, rank=0, world=1, group=None):
    """Batched form against looping the plain form over the same LPs, inputs
    resident on the GPU.  With world > 1 every rank runs its share (`indices`,
    `lps`) of the batch on its own GPU; the per-LP records are gathered to
    rank 0 over `group` (gloo) and the times are the max over ranks.

    Returns the JSON object of the batched measurement on rank 0."""
    import numpy as np
    import torch
    from gpp_b200 import capi, device, shard
    dlps = [device.DeviceLp(lp) for lp in lps]
    torch.cuda.synchronize()

    def zeros(s):
        return (torch.zeros(s.reduced_cols, dtype=torch.float64, device="cuda"),
                torch.zeros(s.reduced_rows, dtype=torch.float64, device="cuda"),
                torch.zeros(s.reduced_cols, dtype=torch.float64, device="cuda"))

    def key(s):
        return (s.reduced_rows, s.reduced_cols, s.reduced_nnz, s.iterations, s.has_infeasible, s.has_unbounded,
                s.obj_constant_delta)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier(group=group)
        torch.cuda.synchronize()

    # Looping the plain form: presolve + postsolve of one LP after another.
    lib = capi.load()
    lib.gpp_kernel_launches(1)
    lib.gpp_host_syncs(1)
    barrier()
    t0 = time.perf_counter()
    plain_keys, plain_lat = [], []
    for d in dlps:
        s = device.preprocess(d, params)
        device.postprocess(*zeros(s), s, d)
        plain_keys.append(key(s))
        plain_lat.append(s.preprocessing_seconds)
        device.free_summary(s)
    torch.cuda.synchronize()
    t_loop = time.perf_counter() - t0
    launches, syncs = lib.gpp_kernel_launches(0), lib.gpp_host_syncs(0)

    workers, curve = device.batch_autotune(dlps, params, max_workers=max_workers) if dlps else (1, {})
    barrier()
    t0 = time.perf_counter()
    sums = []
    if dlps:
        sums, _ = device.preprocess_batch(dlps, params, workers=workers)
        reds = [zeros(s) for s in sums]
        device.postprocess_batch([r[0] for r in reds], [r[1] for r in reds], [r[2] for r in reds], sums, dlps,
                                 workers=workers)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    records = {k: {"match": key(s) == pk, "lat": s.preprocessing_seconds, "plain_lat": pl, "nnz": lp.nnz}
               for k, s, pk, pl, lp in zip(indices, sums, plain_keys, plain_lat, lps)}
    for s in sums:
        device.free_summary(s)
    times = [t_loop, t_batch, float(launches), float(syncs)]
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor(times[:2], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        c = torch.tensor(times[2:], dtype=torch.float64)
        dist.all_reduce(c, op=dist.ReduceOp.SUM, group=group)
        times = t.tolist() + c.tolist()
    recs = shard.gather_records(records, rank, world, group)
    if rank != 0:
        return None
    t_loop, t_batch, launches, syncs = times
    count = len(recs)
    lat = [r["lat"] for r in recs]
    plain_lat = [r["plain_lat"] for r in recs]
    match = sum(r["match"] for r in recs)
    pct = lambda v, q: round(1e3 * float(np.percentile(v, q)), 3)
    return {"lps": count, "nnz_total": int(sum(r["nnz"] for r in recs)), "workload": BATCH_DESC,
            "workers": workers, "autotune_sample_lps_per_s": curve,
            "looped_per_lp": {"launches": round(launches / count, 1), "host_syncs": round(syncs / count, 1)},
            "lps_per_s": round(count / t_batch, 2), "looped_lps_per_s": round(count / t_loop, 2),
            "speedup_vs_looped": round(t_loop / t_batch, 2), "batch_s": round(t_batch, 3),
            "looped_s": round(t_loop, 3),
            "latency_ms": {"p50": pct(lat, 50), "p99": pct(lat, 99), "looped_p50": pct(plain_lat, 50),
                           "looped_p99": pct(plain_lat, 99),
                           "definition": "per-LP presolve wall time (preprocessing_seconds) inside each run"},
            "match_plain": f"{match}/{count}",
            "sharding": ("one GPU" if world == 1 else
                         f"{world} ranks, greedy expected-nnz partition, no device collective; per-LP records "
                         f"gathered on the host (gloo); times are the max over ranks"),
            "timing": "wall clock around presolve + postsolve of all LPs, device inputs resident, "
                      "reduced solutions all-zero"}


def reference_gpu(lp, point, steps, warmup, presolve_ms, postsolve_ms):
    """The reference GPU library (built from its sources into
    oracle/_ref/ref_driver) on the same LP, B200 and parameters: `warmup` +
    `steps` presolves (device sync before and after each; the mean over the
    timed ones), then one postprocess of the same reduced point."""
    from gpp_b200 import lpgen
    from gpp_b200.capi import RULE_FLAGS
    driver = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if not os.path.exists(driver):
        return {"unavailable": "oracle/_ref/ref_driver was not built (needs the reference sources at build time)"}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "lp.bin")
        lpgen.save_lp(path, lp)
        files = []
        for name, v in zip(("x", "y", "z"), point):
            files.append(os.path.join(d, name))
            v.astype("float64").tofile(files[-1])
        args = [driver, path, d, "enable_folding=1"]
        args += [f"{f}={1 if f[len('enable_'):] in RULES else 0}" for f in RULE_FLAGS]
        args += ["--repeat", str(warmup + steps), "--postsolve", *files]
        r = subprocess.run(args, capture_output=True, text=True)
        if r.returncode != 0:
            return {"unavailable": "ref_driver failed: " + (r.stderr.strip().splitlines() or ["?"])[-1]}
        meta = {}
        for line in open(os.path.join(d, "meta.txt")):
            k, *v = line.split()
            meta[k] = v
    wall = [float(v) for v in meta["wall_seconds"]][warmup:]
    ref_pre = 1e3 * statistics.mean(wall)
    ref_post = 1e3 * float(meta["postsolve_seconds"][0])
    return {"presolve_ms": round(ref_pre, 3), "postsolve_ms": round(ref_post, 3),
            "preprocessing_seconds_last": float(meta["preprocessing_seconds"][0]),
            "reduced": {"rows": int(meta["reduced_rows"][0]), "cols": int(meta["reduced_cols"][0]),
                        "nnz": int(meta["reduced_nnz"][0]), "iterations": int(meta["iterations"][0])},
            "presolve_speedup": round(ref_pre / presolve_ms, 2),
            "postsolve_speedup": round(ref_post / postsolve_ms, 2),
            "timing": f"wall time of gpu_preprocessor::preprocess with device syncs, mean of {len(wall)} after "
                      f"{warmup} warm-up; one postprocess (host outputs, first call) of the bench's reduced point; "
                      f"this engine's postsolve_ms is device outputs",
            "build": "reference library compiled from its sources with nvcc 12.9 -O3 for sm_100 (oracle/ref.mk)"}


def optional(measure):
    """Runs one of the bench line's optional measurements; a failure there
    becomes {"error": ...} in the line instead of losing the line."""
    try:
        return measure()
    except Exception as e:  # reported, not hidden: the line carries the message
        return {"error": f"{type(e).__name__}: {e}"}


def bind_to_gpu_cpus(device_index):
    """Restrict this process to the host cores NVML reports as closest to
    the GPU (its NUMA node), so page-locked host buffers are allocated next
    to the GPU's PCIe root and launches come from a near core.  Changes only
    this process's CPU affinity; returns the cores used or None."""
    try:
        import pynvml
        import torch
        props = torch.cuda.get_device_properties(device_index)
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(props.uuid))
            words = (os.cpu_count() + 63) // 64
            mask = pynvml.nvmlDeviceGetCpuAffinity(h, words)
        finally:
            pynvml.nvmlShutdown()
        cpus = {64 * w + b for w, m in enumerate(mask) for b in range(64) if (int(m) >> b) & 1}
        cpus &= os.sched_getaffinity(0)
        if not cpus:
            return None
        os.sched_setaffinity(0, cpus)
        return sorted(cpus)
    except Exception:
        return None


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args, world, rank):
    """The reference's CPU path (bundled PSLP) on rank 0 only."""
    if rank != 0:
        return
    from gpp_b200 import lpgen
    driver = os.path.join(ROOT, "oracle", "_ref", "pslp_driver")
    if not os.path.exists(driver):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/pslp_driver was not built "
                          "(needs the reference sources at build time)"}))
        return
    lp = lpgen.workload(args.workload, seed=0)
    desc = workload_desc(args.workload)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "lp.bin")
        lpgen.save_lp(path, lp)
        runs = args.steps
        warm = min(args.warmup, 1)
        out = subprocess.run([driver, path, str(warm + runs)], capture_output=True, text=True, check=True).stdout
    lines = [l for l in out.splitlines() if l.startswith("pslp run=")]
    wall = [float(l.split("wall_s=")[1].split()[0]) for l in lines][warm:]
    post = [float(l.split("postsolve_s=")[1].split()[0]) for l in lines][warm:]
    core = [float(l.split("presolve_s=")[1].split()[0]) for l in lines][warm:]
    ms = 1e3 * (statistics.mean(wall) + statistics.mean(post))
    sample = (f"PSLP 0.0.11 (reference third_party/pslp, gcc -O3) default settings, full {desc}, "
              f"{len(wall)} timed runs after {warm} warm-up; each run presolve + postsolve of a reduced point "
              f"(presolve {1e3*statistics.mean(wall):.0f} ms incl. PSLP core {1e3*statistics.mean(core):.0f} ms, "
              f"postsolve {1e3*statistics.mean(post):.1f} ms)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": world,
        "steps": len(wall), "warmup": warm, "ms_per_step": round(ms, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "nnz": lp.nnz, "parallelism": "cpu, 1 thread"},
        "cpu_baseline": {"value": round(ms, 3), "unit": "ms", "cores": 1, "kind": "reference", "sample": sample},
        "e2e": {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffers) loop")
    ap.add_argument("--batch", type=int, default=512,
                    help="LPs in the batched-form measurement (0 skips it); sharded over the ranks when N > 1")
    ap.add_argument("--batch-max-workers", type=int, default=32)
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-schedule measurement")
    ap.add_argument("--no-qap", action="store_true", help="skip the QAP N=30 measurement")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference GPU library on the same LP")
    ap.add_argument("--kernel-table-out", default=None,
                    help="write every kernel's launches, ms and bytes per step to this CSV file")
    ap.add_argument("--no-kernel-table", action="store_true",
                    help="skip the extra pass that times every kernel with CUDA events")
    ap.add_argument("--source-digests", action="store_true",
                    help="print the source digest of every kernel that has ncu traffic records, then exit")
    args = ap.parse_args()
    if args.source_digests:
        for k, files in KERNEL_SOURCES.items():
            print(k, source_digest(files))
        return
    world, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import ctypes as C
    import numpy as np
    import torch
    import torch.distributed as dist
    from gpp_b200 import capi, device, lpgen
    from gpp_b200.capi import params_with_rules

    torch.cuda.set_device(local)
    near_cpus = bind_to_gpu_cpus(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    lib = capi.load()
    lp = lpgen.workload(args.workload, seed=0)
    params = params_with_rules(RULES, enable_folding=1)
    dlp = device.DeviceLp(lp)
    stream = torch.cuda.current_stream()

    # Warm-up: also fixes the reduced solution the postsolve step replays.
    red = None
    for _ in range(max(args.warmup, 3)):
        s = device.preprocess(dlp, params)
        if red is None:
            res = device.Result(s, copy_lp=True, copy_tape=False)
            x0 = np.clip(np.zeros(s.reduced_cols), res.l, res.u)
            red = (torch.from_numpy(x0).cuda(), torch.zeros(s.reduced_rows, dtype=torch.float64, device="cuda"),
                   torch.zeros(s.reduced_cols, dtype=torch.float64, device="cuda"))
            reduced = (s.reduced_rows, s.reduced_cols, s.reduced_nnz, s.iterations)
            folded = s.folding_applied
        device.postprocess(*red, s, dlp)
        device.free_summary(s)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # Device-resident timed region.
    out = (torch.empty(lp.n, dtype=torch.float64, device="cuda"), torch.empty(lp.m, dtype=torch.float64, device="cuda"),
           torch.empty(lp.n, dtype=torch.float64, device="cuda"))

    post_events = []

    def device_steps(k):
        pre = []
        for _ in range(k):
            s = device.preprocess(dlp, params)
            pre.append(1e3 * s.elapsed_seconds)
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record(stream)
            device.postsolve_device(*red, s, dlp, out)
            ev[1].record(stream)
            post_events.append(ev)
            device.free_summary(s)
        return pre

    clocks = Clocks(local)
    lib.gpp_kernel_launches(1)
    lib.gpp_host_syncs(1)
    barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    pre_ms = device_steps(args.steps)
    t1.record(stream)
    barrier()
    clk = clocks.stop()
    step_ms = t0.elapsed_time(t1) / args.steps
    post_ms = statistics.mean(a.elapsed_time(b) for a, b in post_events)
    launches = int(lib.gpp_kernel_launches(0)) // args.steps
    syncs = int(lib.gpp_host_syncs(0)) // args.steps
    # Per-kernel table for the roofline: the same steps again with every
    # launch bracketed by CUDA events (kept out of the timed region above).
    prof = []
    if not args.no_kernel_table:
        lib.gpp_profile_enable(1)
        barrier()
        device_steps(args.steps)
        barrier()
        prof = capi.profile_read()
        lib.gpp_profile_enable(0)
        if args.kernel_table_out and rank == 0:
            with open(args.kernel_table_out, "w") as f:
                f.write("kernel,launches_per_step,ms_per_step,bytes_per_step\n")
                for n, l, m, b in sorted(prof, key=lambda r: -r[2]):
                    f.write(f"{n},{l / args.steps:.1f},{m / args.steps:.4f},{b / args.steps:.0f}\n")

    # End to end through the C ABI from pinned host memory: gpp_lp_from_host
    # loads A (CSR) and the vectors and builds A^T on the GPU, then presolve
    # and a postsolve into host outputs.
    host = {k: v.cpu().pin_memory() for k, v in dlp.t.items() if not k.startswith("AT_")}
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    d2h = 8 * (lp.n + lp.m + lp.n)
    # Page-locked host outputs for the recovered solution (allocated once).
    host_out = tuple(torch.empty(k, dtype=torch.float64).pin_memory() for k in (lp.n, lp.m, lp.n))
    e2e_ms = None
    if not args.no_e2e:
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            dlp.load_from_host(host)
            s = device.preprocess(dlp, params)
            device.postprocess(*red, s, dlp, out=host_out)
            device.free_summary(s)
        e1.record(stream)
        barrier()
        e2e_ms = e0.elapsed_time(e1) / args.steps

    # The batched workload is generated by spawned processes (after the timed
    # loops, so they do not compete with them for host cores; they overlap the
    # single-core CPU baseline instead).
    learned_pool = learned_result = None
    from gpp_b200 import schedule as _schedule
    if rank == 0 and not args.no_learned and os.path.exists(_schedule.MODEL_FILE):
        import multiprocessing as mp
        learned_pool = mp.get_context("spawn").Pool(len(LEARNED_SEEDS))
        learned_result = learned_pool.map_async(make_scale_lp, [(args.workload, sd) for sd in LEARNED_SEEDS],
                                                chunksize=1)
    batch_pool = batch_result = None
    batch_mine = []
    if args.batch > 0:
        import multiprocessing as mp
        from gpp_b200 import shard
        jobs = batch_jobs(args.batch)
        batch_mine = shard.greedy_nnz_partition([batch_nnz_estimate(j) for j in jobs], world)[rank]
        procs = max(1, min(32, ((os.cpu_count() or 2) - 2) // world))
        batch_pool = mp.get_context("spawn").Pool(procs)
        batch_result = batch_pool.map_async(make_batch_lp, [jobs[k] for k in batch_mine], chunksize=1)

    if world > 1:
        t = torch.tensor([step_ms, e2e_ms or 0.0], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms, e2e_ms = float(t[0]), (float(t[1]) if e2e_ms is not None else None)

    peak, peak_kind = peaks()
    top = max(prof, key=lambda r: r[2]) if prof else None
    roofline = None
    if top:
        name, nl, ms, by = top
        bytes_top = [r for r in prof if r[3] > 0]
        best = max(bytes_top, key=lambda r: r[2]) if bytes_top else None
        if best:
            name, nl, ms, by = best
            achieved = (by / 1e9) / (ms / 1e3)
            roofline = {"kernel": name, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                        "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                        "launches_per_step": nl // args.steps, "avg_launch_us": round(1e3 * ms / nl, 2),
                        "bytes_per_launch": int(by / nl)}
            traffic, source = measured_traffic(name)
            roofline["traffic"] = traffic
            roofline["traffic_source"] = source
    kernels = sorted((r for r in prof if not r[0].startswith("sync:")), key=lambda r: -r[2])[:8]
    # End-to-end algorithmic bandwidth: every launch's algorithmic bytes in
    # one step over the step's device time.
    step_bytes = sum(r[3] for r in prof) / args.steps if prof else 0
    algorithmic = None
    if prof:
        algorithmic = {"kernels_counted": sorted({r[0] for r in prof if r[3] > 0}),
                       "bytes_per_step": int(step_bytes),
                       "gbs_per_step": round(step_bytes / 1e9 / (step_ms / 1e3), 1),
                       "frac_of_peak": round(step_bytes / 1e9 / (step_ms / 1e3) / peak, 4),
                       "kernel_ms_per_step": round(sum(r[2] for r in prof if not r[0].startswith("sync:"))
                                                   / args.steps, 3)}
    ref_gpu = None
    if rank == 0 and not args.no_reference_gpu:
        ref_gpu = optional(lambda: reference_gpu(lp, [t.cpu().numpy() for t in red], args.steps, max(args.warmup, 3),
                                                 statistics.mean(pre_ms), post_ms))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        driver = os.path.join(ROOT, "oracle", "_ref", "pslp_driver")
        if os.path.exists(driver):
            with tempfile.TemporaryDirectory() as d:
                path = os.path.join(d, "lp.bin")
                lpgen.save_lp(path, lp)
                out = subprocess.run([driver, path, "1"], capture_output=True, text=True).stdout
            runs = [l for l in out.splitlines() if l.startswith("pslp run=")]
            if runs:
                wall = float(runs[0].split("wall_s=")[1].split()[0])
                post = float(runs[0].split("postsolve_s=")[1].split()[0])
                cpu = {"value": round(1e3 * (wall + post), 1), "unit": "ms", "cores": 1, "kind": "reference",
                       "sample": f"one PSLP 0.0.11 presolve ({1e3 * wall:.0f} ms) + postsolve ({1e3 * post:.1f} ms) "
                                 f"of the full workload ({workload_desc(args.workload)}) on 1 host core"}
    # Learned round schedule on held-out draws of the scale workload (the
    # schedule is trained on LPs of at most 500,000 rows; seeds 1-3 here, the
    # timed LP above is seed 0): presolve time against the plain loop on the
    # same LP, and the share of the plain run's nnz removal it keeps.
    learned = None
    if learned_result is not None:
        from gpp_b200 import schedule
        try:
            w_sched, skip_below, stop_above = schedule.load_model()
        except ValueError as e:   # a model trained for another feature layout
            learned = {"unavailable": str(e)}
            learned_result = None
            learned_pool.terminate()
    def learned_measurement():
        reps = max(3, min(args.steps, 5))
        per_lp = []
        with schedule.Model(w_sched, skip_below, stop_above) as model:
            for seed, hlp in zip(LEARNED_SEEDS, learned_result.get()):
                hd = device.DeviceLp(hlp)
                run = lambda: device.preprocess(hd, params)
                sched = lambda: schedule.scheduled_preprocess(hd, params, model)
                res = {}
                for kind, fn in (("plain", run), ("scheduled", sched)):
                    times = []
                    for it in range(2 + reps):
                        s = fn()
                        if it >= 2:
                            times.append(1e3 * s.elapsed_seconds)
                        res[kind] = (s.reduced_nnz, s.iterations)
                        device.free_summary(s)
                    res[kind + "_ms"] = statistics.mean(times)
                removed_plain = hlp.nnz - res["plain"][0]
                per_lp.append({"seed": seed, "nnz": hlp.nnz, "plain_presolve_ms": round(res["plain_ms"], 3),
                               "presolve_ms": round(res["scheduled_ms"], 3),
                               "time_ratio": round(res["scheduled_ms"] / res["plain_ms"], 4),
                               "rounds": res["scheduled"][1], "plain_rounds": res["plain"][1],
                               "nnz_removal_kept": round((hlp.nnz - res["scheduled"][0]) / removed_plain, 5)
                               if removed_plain else 1.0})
                del hd, hlp
        ratios = [r["time_ratio"] for r in per_lp]
        kept = [r["nnz_removal_kept"] for r in per_lp]
        return {"time_ratio_mean": round(statistics.mean(ratios), 4), "time_ratio_max": max(ratios),
                   "speedup_mean": round(1.0 / statistics.mean(ratios), 3),
                   "nnz_removal_kept_min": min(kept), "held_out": per_lp,
                   "skip_below": skip_below, "stop_above": stop_above,
                   "workload": f"held-out draws of the scale workload (seeds {list(LEARNED_SEEDS)})",
                   "timing": f"presolve elapsed_seconds, mean of {reps} runs after 2 warm-up, per LP",
                   "model": "2x64 FP32 MLP, trained on plain-loop traces"}

    if learned_result is not None:
        learned = optional(learned_measurement)
        learned_pool.close()
        learned_pool.join()

    # QAP N = 30 (Adams-Johnson linearisation, 1,674,960 rows x 810,900
    # columns): the structured workload of the parallel row / column rules and
    # of folding.  Presolve time, whether folding applies and the sizes, with
    # the reference GPU library on the same LP beside it.
    def qap_measurement():
        qlp = lpgen.workload("qap30", seed=0)
        qd = device.DeviceLp(qlp)
        reps = max(3, min(args.steps, 5))
        times = []
        for it in range(2 + reps):
            s = device.preprocess(qd, params)
            if it >= 2:
                times.append(1e3 * s.elapsed_seconds)
            if it == 0:
                res = device.Result(s, copy_lp=True, copy_tape=False)
                point = [np.clip(np.zeros(s.reduced_cols), res.l, res.u), np.zeros(s.reduced_rows),
                         np.zeros(s.reduced_cols)]
                info = {"folding_applied": bool(s.folding_applied), "folded": [s.folded_rows, s.folded_cols],
                        "reduced": {"rows": s.reduced_rows, "cols": s.reduced_cols, "nnz": s.reduced_nnz,
                                    "iterations": s.iterations}}
            device.free_summary(s)
        pre = statistics.mean(times)
        out = {"workload": "QAP N=30, Adams-Johnson linearisation (lpgen.qap_lp), seed 0", "rows": qlp.m,
               "cols": qlp.n, "nnz": qlp.nnz, "presolve_ms": round(pre, 3), **info,
               "timing": f"presolve elapsed_seconds, mean of {reps} runs after 2 warm-up"}
        if not args.no_reference_gpu:
            ref = reference_gpu(qlp, point, reps, 2, pre, 1.0)
            out["reference_gpu"] = {k: ref[k] for k in ("presolve_ms", "reduced", "presolve_speedup", "unavailable")
                                    if k in ref}
        return out

    qap = optional(qap_measurement) if rank == 0 and not args.no_qap else None

    batched = None
    if batch_result is not None:
        gloo = dist.new_group(backend="gloo") if world > 1 else None
        batched = optional(lambda: run_batched(batch_mine, batch_result.get(), params, args.batch_max_workers, rank,
                                               world, gloo))
        batch_pool.close()
        batch_pool.join()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": round(step_ms, 3), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": round(step_ms, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_desc(args.workload), "rows": lp.m, "cols": lp.n, "nnz": lp.nnz,
                       "rules": RULES, "folding": True, "folding_applied": bool(folded),
                       "reduced": {"rows": reduced[0], "cols": reduced[1], "nnz": reduced[2], "iterations": reduced[3]},
                       "presolve_ms": round(statistics.mean(pre_ms), 3),
                       "postsolve_ms": round(post_ms, 3),
                       "l2": "inputs (~1 GB) larger than L2; no flush",
                       "host_cpus": (f"{len(near_cpus)} cores of the GPU's NUMA node" if near_cpus
                                     else "unbound (no NVML CPU affinity)"),
                       "parallelism": "replicas" if world > 1 else "1 GPU"},
            "gpu_launches": launches,
            "host_syncs_per_step": syncs,
            "e2e": None if e2e_ms is None else {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": h2d,
                                                "d2h_bytes_per_step": d2h,
                                                "path": "gpp_lp_from_host (A as CSR + vectors; A^T built on "
                                                        "the GPU) -> gpp_preprocess -> gpp_postprocess (host x, y, z)"},
            "roofline": roofline,
            "algorithmic": algorithmic,
            "reference_gpu": ref_gpu,
            "kernels": [{"name": n, "launches_per_step": l // args.steps, "ms_per_step": round(m / args.steps, 3)}
                        for n, l, m, b in kernels],
            "cpu_baseline": cpu,
            "batched": batched,
            "learned_schedule": learned,
            "qap30": qap,
            "clocks": clk,
        }))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
