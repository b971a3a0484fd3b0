#!/usr/bin/env python
"""Benchmark of the thrustrtc_b200 hot path on B200.

Default workload: stable Sort_By_Key of 2^28 uint32 keys (uniform over the 32-bit range,
SplitMix64 seed 0) with uint32 values = index, ascending -- the reference's headline case.
Other workloads (--workload): inclusive scan of 2^28 int32 in [-1000, 1000], reduce of 2^28
float32 in [0, 1); the mixed-type cases c1_sort_by_key_2e20, c3a_sort_f32,
c3b_sort_by_key_i64_zipf, c3c_copy_if_functor, c3d_scan_by_key_f32 and a13_unique_i32; the rows after the
hot path, f1_reduce_by_key_f32 (Reduce_By_Key) and f2_lower_bound_u32 (Lower_Bound_V); the batched form
segmented_c4 (100,000 lognormal segments sorted and scanned in one launch, beside one plain
call pair per segment); and serving_c5 (the request server against one plain call per
request).

One JSON line on rank 0:
  value        whole-job throughput with inputs resident in HBM (device-timed with CUDA
               events on the launching stream; max over ranks)
  e2e          the same metric through the drop-in C ABI (n_dvvector_create from pinned host
               memory, n_sort_by_key / n_inclusive_scan / n_reduce, n_dvvector_to_host)
  roofline     the dominant kernel's algorithmic bytes per launch / its average device time
               (per-launch CUDA events recorded by the library over the timed region)
  cpu_baseline the oracle's host sort / scan / reduce on a bounded sample, all host threads
  configs      (default run) the same record for the inclusive scan of 2^28 int32 and the
               reduce of 2^28 float32, and the serving form: both paths' capacity and their
               p50 / p99 latency on one grid of offered request rates

`--impl reference` times the reference algorithm's CPU restatement (the reference itself has
no CPU path and does not build here) on the same workload definition.

Multi-GPU (torchrun, one process per GPU): every rank runs the same workload on its own GPU
(replicas, weak scaling); there is no collective on the data path.
"""
import argparse
import ctypes
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0
L2_BYTES = 126 * 1024 * 1024

# ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of the dominant kernel,
# per unit processed (bytes per pair / element), from captures of smaller cases above L2
# scaled by the units processed (traffic grows in proportion).  Source summaries:
# profiles/<kernel>_<workload>.md
NCU_TRAFFIC_PER_UNIT = {
    "sort_by_key_u32": 15.02,   # radix_pass_kernel, 2^25 pairs: (269.9 + 234.2) MB / 2^25
    "inclusive_scan_i32": 7.31,  # scan2_kernel, 2^26 elements: (282.8 + 207.9) MB / 2^26
    "reduce_f32": 4.07,          # reduce_kernel, 2^26 elements: (268.5 + 4.9) MB / 2^26
}

WORKLOADS = {
    # name: (default n, dominant kernel, algorithmic bytes per unit per dominant launch,
    #        algorithmic bytes per unit for the whole operation, metric, unit)
    "sort_by_key_u32": (1 << 28, "radix_pass_kernel", 16, 68,
                        "Gkeys/s sort 2^28 u32 pairs, % HBM roofline", "Gkeys/s"),
    "inclusive_scan_i32": (1 << 28, "scan_kernel", 8, 8, "GB/s inclusive scan 2^28 i32, % HBM roofline", "GB/s"),
    "reduce_f32": (1 << 28, "reduce_kernel", 4, 4, "GB/s reduce 2^28 f32, % HBM roofline", "GB/s"),
    # batched form: 100,000 lognormal segments (~2^26 pairs), each sorted then exclusive-scanned
    "segmented_c4": (100_000, "seg_sort_scan_kernel", 20, 20,
                     "Gkeys/s batched segmented sort+scan, 100k lognormal segments", "Gkeys/s"),
    # plain mixed types and distributions (run_mixed)
    "c1_sort_by_key_2e20": (1 << 20, "radix_pass_kernel", 16, 68, "Gkeys/s Sort_By_Key 2^20 u32 pairs", "Gkeys/s"),
    "c3a_sort_f32": (1 << 27, "radix_pass_kernel", 8, 36,
                     "Gkeys/s Sort 2^27 f32 N(0,1) with -0.0, NaN, duplicates", "Gkeys/s"),
    "c3b_sort_by_key_i64_zipf": (1 << 27, "radix_pass_kernel", 24, 80,
                                 "Gkeys/s Sort_By_Key 2^27 i64 Zipf keys + i32 payload", "Gkeys/s"),
    "c3c_copy_if_functor": (1 << 28, "jit:trtc::compact2_kernel", 6, 6,
                            "GB/s Copy_If 2^28 i32 with a user Functor (x & 1) != 0", "GB/s"),
    "c3d_scan_by_key_f32": (1 << 28, "scan_by_key_kernel", 12, 12,
                            "GB/s inclusive Scan_By_Key 2^28 f32 values, geometric runs", "GB/s"),
    # the rows after the hot path: by-key reduction (k-means step) and vectorised search
    # (histogram demo); algorithmic bytes: keys + values read, one key + one sum per run
    # written (runs of mean 32); queries read, results written (the searched vector's reads
    # are random and not counted)
    "a13_unique_i32": (1 << 28, "compact_kernel", 4.125, 4.125,
                       "GB/s Unique (copy) 2^28 i32 in geometric runs of mean 32", "GB/s"),
    "f1_reduce_by_key_f32": (1 << 28, None, None, 8.25,
                             "GB/s Reduce_By_Key 2^28 i32 keys (geometric runs) / f32 values", "GB/s"),
    "f2_lower_bound_u32": (1 << 26, "jit:trtc::search_v_kernel", 8, 8,
                           "Gqueries/s Lower_Bound_V 2^26 u32 queries into 2^26 sorted u32", "Gqueries/s"),
    # serving form: a Poisson stream of mixed requests (bounded sample of the 200,000)
    "serving_c5": (1000, None, None, None,
                   "requests/s serving mix 60% sort_by_key 25% scan 15% reduce, sizes 2^10..2^24", "requests/s"),
}

M64 = (1 << 64) - 1
GAMMA = 0x9E3779B97F4A7C15


def _mix64(z):
    """SplitMix64 output function (Steele, Lea & Flood 2014) on a numpy uint64 array."""
    z = z ^ (z >> np.uint64(30))
    z = z * np.uint64(0xBF58476D1CE4E5B9)
    z = z ^ (z >> np.uint64(27))
    z = z * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def splitmix64(seed, stream, n, start=0, chunk=1 << 24):
    """Counter-based SplitMix64: element i is the (i+1)-th output of SplitMix64 started at
    state base = mix(seed << 8 | stream), i.e. mix(base + (i + 1) * GAMMA)."""
    base = int(_mix64(np.array([((seed << 8) | stream) & M64], np.uint64))[0])
    out = np.empty(n, np.uint64)
    with np.errstate(over="ignore"):
        for a in range(0, n, chunk):
            b = min(n, a + chunk)
            i = np.arange(start + a + 1, start + b + 1, dtype=np.uint64)
            out[a:b] = _mix64(np.uint64(base) + i * np.uint64(GAMMA))
    return out


def gen_inputs(workload, n):
    """Host inputs of a workload (identical bytes for the GPU runs, the oracle and the
    reference arm)."""
    if workload == "sort_by_key_u32":
        keys = (splitmix64(0, 0, n) >> np.uint64(32)).astype(np.uint32)
        vals = np.arange(n, dtype=np.uint32)
        return keys, vals
    if workload == "inclusive_scan_i32":
        h = splitmix64(0, 0, n)
        return ((h % np.uint64(2001)).astype(np.int64) - 1000).astype(np.int32), None
    if workload == "reduce_f32":
        h = splitmix64(0, 0, n)
        return ((h >> np.uint64(40)).astype(np.float64) * 2.0 ** -24).astype(np.float32), None
    raise ValueError(workload)


# ---------------------------------------------------------------- clocks during the timed region
_REASONS = [(0x4, "sw_power_cap"), (0x8, "hw_slowdown"), (0x20, "sw_thermal_slowdown"),
            (0x40, "hw_thermal_slowdown"), (0x80, "hw_power_brake_slowdown"), (0x2, "applications_clocks_setting"),
            (0x10, "sync_boost"), (0x100, "display_clock_setting")]


class ClockSampler:
    """Reads SM clock and clock-event reasons through NVML every `period` s (read-only)."""

    def __init__(self, torch_dev, period=0.01):
        self.samples, self.reasons, self.ok = [], set(), False
        self.period = period
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            import torch
            p = torch.cuda.get_device_properties(torch_dev)
            bus = "%08x:%02x:%02x.0" % (getattr(p, "pci_domain_id", 0), p.pci_bus_id, p.pci_device_id)
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception as e:  # noqa: BLE001  (no NVML: report clocks as unavailable)
            self.err = str(e)

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in _REASONS:
                    if r & bit:
                        self.reasons.add(name)
            except Exception:  # noqa: BLE001
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.ok:
            self._stop = threading.Event()
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": "NVML unavailable"}
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------- helpers
def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "of measured"
    except (OSError, KeyError, ValueError):
        return HBM_FALLBACK_GBS, "of fallback"


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def reduce_max(x, world, device):
    """The maximum of x over all ranks (every rank gets it): the whole job's time is the
    slowest replica's.  device: where the process group's collectives run (cuda for NCCL,
    cpu for gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, world, secs_max):
    """Whole-job throughput of N independent replicas (weak scaling): all ranks' units over
    the slowest rank's time."""
    return units_per_rank * world / secs_max


def cpu_threads():
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_run(workload, sample_n, threads):
    """One timed oracle run on the host over the first `sample_n` units; returns (seconds,
    threads used): the pair sort runs on `threads` threads, the scan and reduce on one."""
    from oracle import oracle as O
    if workload == "segmented_c4":
        # sample_n segments spread over the batch, one oracle sort + scan per segment,
        # segments spread over `threads` host threads
        import concurrent.futures as cf
        keys, vals, off = gen_segmented(WORKLOADS["segmented_c4"][0])
        idx = np.linspace(0, len(off) - 2, sample_n).astype(np.int64)

        def one(i):
            a, b = int(off[i]), int(off[i + 1])
            kk, vv = O.sort_pairs32(keys[a:b], vals[a:b], False, 1)
            np.cumsum(vv, dtype=np.uint32)
            return b - a

        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(threads) as ex:
            pairs = sum(ex.map(one, idx))
        return time.perf_counter() - t0, threads, pairs
    if workload == "serving_c5":
        # the first sample_n requests of the mix, served one after another by the oracle
        reqs = serving_requests(WORKLOADS["serving_c5"][0])[:sample_n]
        rng = np.random.default_rng(0)
        data = []
        for kind, t, n in reqs:
            if t == 8:
                data.append(rng.standard_normal(n).astype(np.float32))
            else:
                data.append(rng.integers(0, 2**31, n).astype(np.uint32 if t == 5 else np.int64))
        t0 = time.perf_counter()
        for (kind, t, n), x in zip(reqs, data):
            if kind == 0:
                if x.dtype.itemsize == 4:
                    O.sort_pairs32(x, np.arange(n, dtype=np.uint32), False, threads)
                else:
                    O.sort_by_key(x, np.arange(n, dtype=np.uint32))
            elif kind == 1:
                O.scan(x, exclusive=True, init=0)
            else:
                O.reduce(x)
        return time.perf_counter() - t0, threads, sample_n
    x, v = gen_inputs(workload, sample_n)
    t0 = time.perf_counter()
    if workload == "sort_by_key_u32":
        O.sort_pairs32(x, v, False, threads)
    elif workload == "inclusive_scan_i32":
        O.scan(x)
    else:
        O.reduce(x)
    return time.perf_counter() - t0, (threads if workload == "sort_by_key_u32" else 1), sample_n


def units_per_s_to_metric(workload, units, seconds):
    """Throughput in the metric's unit: Gkeys/s for sorts, GB/s of algorithmic bytes otherwise."""
    if workload in ("sort_by_key_u32", "segmented_c4"):
        return units / seconds / 1e9
    if workload == "serving_c5":
        return units / seconds
    return units * WORKLOADS[workload][3] / seconds / 1e9


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    wl = args.workload
    n, _, _, _, metric, unit = WORKLOADS[wl]
    threads = cpu_threads()
    sample = args.cpu_sample or {"sort_by_key_u32": 1 << 25, "segmented_c4": 20000, "serving_c5": 16}.get(wl, 1 << 27)
    from oracle import oracle as O
    O.build()
    for _ in range(args.warmup):
        cpu_run(wl, sample, threads)
    ts = [cpu_run(wl, sample, threads) for _ in range(args.steps)]
    tot = sum(t for t, _, _ in ts)
    threads = ts[0][1]
    units = sum(u for _, _, u in ts)
    value = units_per_s_to_metric(wl, units, tot)
    if wl == "serving_c5":
        desc = ("the first %d requests of the mix per step, one after another, oracle restatement, sorts of "
                "4-byte keys on %d host threads" % (sample, threads))
    elif wl == "segmented_c4":
        desc = ("%d of the %d segments per step, spread over the batch; oracle sort + exclusive scan per "
                "segment, %d host threads" % (sample, n, threads))
    else:
        desc = ("first %d units of the %s workload (n=%d); oracle restatement of the reference's "
                "algorithm, %d host threads" % (sample, wl, n, threads))
    line = {"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": _dtype(wl),
            "data": "synthetic (SplitMix64 seed 0)", "config": _config(wl, n, world),
            "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference (fynv/ThrustRTC) has no CPU path (every kernel is an NVRTC string run on "
                    "the GPU); the arm times the oracle's host restatement of its algorithm on the host cores",
            "thrustrtc_same_gpu": _thrustrtc_gpu(wl, n)}
    print(json.dumps(line), flush=True)
    return 0


# The reference itself on this box's GPU, for the record beside the host arm: its library as
# built from its sources by oracle/build_ref.py (present when the repository was built where
# the reference tree is), run through its own Python package in a child process.
_REF_CALLS = {
    "sort_by_key_u32": "T.Sort_By_Key(a[0], a[1])",
    "inclusive_scan_i32": "T.Inclusive_Scan(a[0], a[1])",
    "reduce_f32": "T.Reduce(a[0])",
}


def _thrustrtc_gpu(wl, n):
    if wl not in _REF_CALLS:
        return {"skipped": "timed for the plain sort, scan and reduce workloads only"}
    try:
        from oracle import build_ref
    except ImportError as e:
        return {"unavailable": "oracle/build_ref.py not importable: %s" % e}
    pkg = build_ref.package_dir(False)
    if pkg is None:
        return {"unavailable": "oracle/_ref was not built (the reference tree was absent where the repository was built)"}
    env = dict(os.environ)
    cl = build_ref.cuda_lib_dir()
    if cl:
        env["LD_LIBRARY_PATH"] = cl + (":" + env["LD_LIBRARY_PATH"] if env.get("LD_LIBRARY_PATH") else "")
    env["PYTHONPATH"] = pkg + ":" + ROOT + (":" + env["PYTHONPATH"] if env.get("PYTHONPATH") else "")
    import subprocess
    try:
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--thrustrtc-child", wl, "--n", str(n)],
                           env=env, capture_output=True, text=True, timeout=600)
    except subprocess.TimeoutExpired:
        return {"unavailable": "the reference's run exceeded 600 s"}
    ls = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not ls:
        return {"unavailable": "the reference's run failed (rc %d): %s" % (r.returncode, (r.stderr or r.stdout)[-300:])}
    return json.loads(ls[-1])


def _thrustrtc_child(wl, n):
    """Times one call of the reference's own API on the workload's inputs, already on the
    device: one warm-up call on a 4,096-element slice compiles its kernels (NVRTC), then three
    calls, each bracketed by Wait() and timed by the host clock."""
    import ThrustRTC as T
    keys_h, vals_h = gen_inputs(wl, n)
    def inputs(m):
        if wl == "sort_by_key_u32":
            return [T.device_vector_from_numpy(keys_h[:m]), T.device_vector_from_numpy(vals_h[:m])]
        if wl == "inclusive_scan_i32":
            return [T.device_vector_from_numpy(keys_h[:m]), T.device_vector("int32_t", m)]
        return [T.device_vector_from_numpy(keys_h[:m])]
    call = _REF_CALLS[wl]
    a = inputs(4096)
    eval(call)
    T.Wait()
    ts = []
    for _ in range(3):
        a = inputs(n) if wl == "sort_by_key_u32" or not ts else a
        T.Wait()
        t0 = time.perf_counter()
        eval(call)
        T.Wait()
        ts.append(time.perf_counter() - t0)
    best = min(ts)
    print(json.dumps({"value": units_per_s_to_metric(wl, n, best), "unit": WORKLOADS[wl][5],
                      "ms_per_call": best * 1e3, "ms_all_calls": [t * 1e3 for t in ts],
                      "how": "the reference's library built from its sources (its block-size query answered by "
                             "the CUDA driver, oracle/ref_launch_calc.cpp), its own Python package, inputs on "
                             "the device, best of 3 calls after a warm-up compile; host clock with Wait()"}))


def _dtype(wl):
    return {"sort_by_key_u32": "u32", "inclusive_scan_i32": "int32", "reduce_f32": "f32", "segmented_c4": "u32",
            "serving_c5": "u32/i64/f32"}[wl]


def _config(wl, n, world):
    base = {"workload": wl, "n": n, "parallelism": "replicas x%d" % world,
            "l2": "inputs (%d MiB) exceed the 126 MB L2" % (n * (8 if wl == "sort_by_key_u32" else 4) >> 20)}
    if wl == "sort_by_key_u32":
        base.update({"keys": "uint32 uniform over 32 bits", "values": "uint32 = index", "order": "ascending, stable",
                     "step": "restore the unsorted pairs from a pristine copy (untimed), then one sort (timed)"})
    elif wl == "serving_c5":
        base = {"workload": wl, "requests": n, "mix": "60% Sort_By_Key, 25% exclusive scan, 15% reduce",
                "sizes": "log-uniform 2^10..2^24", "types": "uint32 / int64 / float", "parallelism": "1 GPU"}
    elif wl == "segmented_c4":
        base = {"workload": wl, "segments": n, "lengths": "lognormal median 256 sigma 1.5 clipped [1, 2^20]",
                "keys": "uint32 uniform", "values": "uint32 = index", "parallelism": "replicas x%d" % world}
    elif wl == "inclusive_scan_i32":
        base.update({"values": "int32 uniform in [-1000, 1000]", "op": "Plus"})
    else:
        base.update({"values": "float32 uniform in [0, 1)", "op": "Plus", "accumulation": "fp32"})
    return base


# ---------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: a CUDA device is required (there is no CPU path)")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    import thrustrtc_b200 as trtc
    trtc.init()
    assert args.warmup >= 3 or args.allow_short_warmup, "at least 3 warm-up steps"

    line = _measure_plain(args.workload, args, dev, rank, world, with_e2e=not args.no_e2e,
                          with_cpu=not args.no_cpu)
    if args.workload == "sort_by_key_u32" and not args.no_sub:
        # the other configurations of the headline metric, measured in the same run:
        # C2b scan and C2c reduce (replicas on every rank, max over ranks), and the serving
        # form (rank 0 of a one-GPU run only: the serving loop is a one-GPU measurement)
        sub = {}
        for wl in ("inclusive_scan_i32", "reduce_f32"):
            sub[wl] = _measure_plain(wl, args, dev, rank, world, with_e2e=not args.no_e2e,
                                     with_cpu=not args.no_cpu)
        if world == 1:
            sub["serving_c5"] = _serving_measure(args.sub_requests, dev, shared_grid=True)
        else:
            sub["serving_c5"] = {"skipped": "one-GPU measurement; run with --gpus 1"}
        if line is not None:
            line["configs"] = sub
    if world > 1:
        torch.distributed.barrier()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def _measure_plain(wl, args, dev, rank, world, with_e2e=True, with_cpu=True):
    """One plain workload (sort_by_key_u32 / inclusive_scan_i32 / reduce_f32): warm-up, K
    timed steps on the legacy default stream, correctness check, roofline of the dominant
    kernel, end-to-end line and CPU baseline.  Returns the JSON record on rank 0 (else None)."""
    import torch
    from thrustrtc_b200 import _native as N
    L = N.lib
    n, kname, b_launch, b_unit, metric, unit = WORKLOADS[wl]
    n = (args.n or n) if wl == args.workload else n

    keys_h, vals_h = gen_inputs(wl, n)
    stream = None  # the legacy default stream: torch's current stream and the library's
    if wl == "sort_by_key_u32":
        k0 = torch.from_numpy(keys_h.view(np.int32)).to(dev)
        v0 = torch.from_numpy(vals_h.view(np.int32)).to(dev)
        k, v = torch.empty_like(k0), torch.empty_like(v0)

        def restore():
            k.copy_(k0)
            v.copy_(v0)

        def step():
            if L.trtc_raw_sort_by_key(5, ctypes.c_void_p(k.data_ptr()), ctypes.c_void_p(v.data_ptr()), 4, n, 0,
                                      stream) != 0:
                raise RuntimeError(N.last_error())
    elif wl == "inclusive_scan_i32":
        x = torch.from_numpy(keys_h).to(dev)
        y = torch.empty_like(x)
        flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=dev)

        def restore():
            flush.fill_(1)  # evicts the previous step's lines from L2

        def step():
            if L.trtc_raw_scan(4, 0, 0, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), n, None,
                               stream) != 0:
                raise RuntimeError(N.last_error())
    else:
        x = torch.from_numpy(keys_h).to(dev)
        flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=dev)
        res = ctypes.c_void_p()

        def restore():
            flush.fill_(1)

        def step():
            if L.trtc_raw_reduce_async(8, 0, ctypes.c_void_p(x.data_ptr()), n, None, ctypes.byref(res), stream) != 0:
                raise RuntimeError(N.last_error())

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max(x, world, dev)

    # ---- warm-up
    for _ in range(args.warmup):
        restore()
        step()
    barrier()

    # ---- timed region: K steps, each bracketed by events on the launching stream
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(dev)
    lc0 = N.launch_count()
    N.timing_enable(True)
    with sampler:
        barrier()
        for i in range(args.steps):
            restore()
            ev[i][0].record()
            step()
            ev[i][1].record()
        barrier()
    launches = N.launch_count() - lc0
    recs = N.timing_records()
    N.timing_enable(False)
    if L.trtc_raw_sync(stream) != 0:
        raise RuntimeError(N.last_error())
    step_ms = [a.elapsed_time(b) for a, b in ev]
    tot_ms = max_over_ranks(sum(step_ms))
    value = units_per_s_to_metric(wl, n * world * args.steps, tot_ms / 1e3)

    # ---- correctness of the last step (size-independent properties), loud on failure
    _check(wl, n, locals())

    # ---- dominant kernel roofline from the per-launch events of the timed region
    kt = [ms for name, ms in recs if name == kname]
    peak, peak_src = measured_peak()
    per_launch_ms = statistics.mean(kt) if kt else None
    achieved = (b_launch * n / (per_launch_ms / 1e3) / 1e9) if per_launch_ms else None
    traffic = NCU_TRAFFIC_PER_UNIT.get(wl)
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "peak_source": peak_src,
                "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                "traffic": (traffic * n) if traffic else None, "algorithmic_bytes_per_launch": b_launch * n,
                "launch_ms": per_launch_ms, "launches_timed": len(kt)}
    whole = b_unit * n / (tot_ms / args.steps / 1e3) / 1e9
    kernel_share = {}
    for name, ms in recs:
        kernel_share[name] = kernel_share.get(name, 0.0) + ms

    # ---- end to end through the C ABI with pinned host buffers
    e2e = None
    if with_e2e:
        e2e = _e2e(args, wl, n, keys_h, vals_h, world, max_over_ranks, barrier)

    cpu = None
    if world == 1 and rank == 0 and with_cpu:
        threads = cpu_threads()
        sample = args.cpu_sample or (1 << 25 if wl == "sort_by_key_u32" else 1 << 27)
        sample = min(sample, n)
        secs, threads, _ = cpu_run(wl, sample, threads)
        cpu = {"value": units_per_s_to_metric(wl, sample, secs), "unit": unit, "cores": threads, "kind": "port",
               "sample": "first %d units of the same workload, oracle host restatement, %d threads" % (sample, threads)}
    del keys_h, vals_h
    if rank != 0:
        return None
    return {"metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": _dtype(wl),
            "data": "synthetic (SplitMix64 seed 0, generated on the host)", "config": _config(wl, n, world),
            "roofline": roofline,
            "roofline_whole_op": {"algorithmic_bytes_per_unit": b_unit, "achieved": whole,
                                  "frac": whole / peak, "unit": "GB/s"},
            "kernel_ms_timed_region": {k2: round(v2, 4) for k2, v2 in sorted(kernel_share.items())},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": sampler.summary(), "gpu_launches": launches,
            "step_ms": [round(s, 4) for s in step_ms]}


def _check(wl, n, env):
    import torch
    if wl == "sort_by_key_u32":
        k, v, k0 = env["k"], env["v"], env["k0"]
        ku = k.to(torch.int64) & 0xFFFFFFFF
        if n > 1 and not bool((ku[1:] >= ku[:-1]).all()):
            raise RuntimeError("sort check failed: keys not ascending")
        perm = v.to(torch.int64)
        if not bool((k0[perm] == k).all()):
            raise RuntimeError("sort check failed: values are not the keys' permutation")
        eq = ku[1:] == ku[:-1]
        if n > 1 and not bool((perm[1:][eq] > perm[:-1][eq]).all()):
            raise RuntimeError("sort check failed: not stable")
        if int(torch.bincount(perm, minlength=n).max()) != 1:
            raise RuntimeError("sort check failed: values are not a permutation")
    elif wl == "inclusive_scan_i32":
        x, y = env["x"], env["y"]
        ref = torch.cumsum(x.to(torch.int64), 0)
        if not bool((ref.to(torch.int32) == y).all()):
            raise RuntimeError("scan check failed")
    else:
        x = env["x"]
        import thrustrtc_b200._native as N
        val = ctypes.c_float()
        if N.lib.trtc_raw_reduce(8, 0, ctypes.c_void_p(x.data_ptr()), n, None, ctypes.byref(val), None) != 0:
            raise RuntimeError(N.last_error())
        ref = float(x.to(torch.float64).sum())
        if abs(val.value - ref) > 1e-5 * abs(ref):
            raise RuntimeError("reduce check failed: %r vs %r" % (val.value, ref))


def _e2e(args, wl, n, keys_h, vals_h, world, max_over_ranks, barrier):
    """Per step: H2D of the inputs from pinned host memory into new DVVectors, the call,
    D2H of the result into pinned host memory, all through the n_* C ABI."""
    import torch
    from thrustrtc_b200.api import lib as A, check_i
    kp = torch.from_numpy(keys_h.view(np.int32) if keys_h.dtype == np.uint32 else keys_h).pin_memory()
    vp_ = torch.from_numpy(vals_h.view(np.int32)).pin_memory() if vals_h is not None else None
    ko = torch.empty_like(kp).pin_memory()
    vo = torch.empty_like(vp_).pin_memory() if vp_ is not None else None
    esz = keys_h.dtype.itemsize
    cls = {"sort_by_key_u32": b"uint32_t", "inclusive_scan_i32": b"int32_t", "reduce_f32": b"float"}[wl]
    h2d = n * esz + (n * 4 if vp_ is not None else 0)
    d2h = {"sort_by_key_u32": 2 * n * 4, "inclusive_scan_i32": n * 4, "reduce_f32": 4}[wl]
    steps = max(1, min(args.steps, args.e2e_steps))

    def one():
        dk = A.n_dvvector_create(cls, n, ctypes.c_void_p(kp.data_ptr()))
        if not dk:
            raise RuntimeError("n_dvvector_create failed")
        try:
            if wl == "sort_by_key_u32":
                dv = A.n_dvvector_create(b"uint32_t", n, ctypes.c_void_p(vp_.data_ptr()))
                try:
                    check_i(A.n_sort_by_key(dk, dv, None))
                    A.n_dvvector_to_host(dk, ctypes.c_void_p(ko.data_ptr()), 0, n)
                    A.n_dvvector_to_host(dv, ctypes.c_void_p(vo.data_ptr()), 0, n)
                finally:
                    A.n_dv_destroy(dv)
            elif wl == "inclusive_scan_i32":
                check_i(A.n_inclusive_scan(dk, dk, None))
                A.n_dvvector_to_host(dk, ctypes.c_void_p(ko.data_ptr()), 0, n)
            else:
                r = A.n_reduce(dk, None, None)
                if not r:
                    raise RuntimeError("n_reduce failed")
                A.n_dv_destroy(r)
        finally:
            A.n_dv_destroy(dk)

    for _ in range(max(3, args.warmup)):  # first calls grow the memory pool and load modules
        one()
    barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    barrier()
    secs = max_over_ranks(time.perf_counter() - t0)
    if wl == "sort_by_key_u32":
        kk = ko.numpy().view(np.uint32)
        if n > 1 and not (kk[1:] >= kk[:-1]).all():
            raise RuntimeError("e2e sort check failed")
    return {"value": units_per_s_to_metric(wl, n * world * steps, secs), "unit": WORKLOADS[wl][5],
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": steps,
            "ms_per_step": secs / steps * 1e3,
            "path": "n_dvvector_create(pinned host) -> %s -> n_dvvector_to_host(pinned host)" %
                    {"sort_by_key_u32": "n_sort_by_key", "inclusive_scan_i32": "n_inclusive_scan",
                     "reduce_f32": "n_reduce"}[wl]}


# ---------------------------------------------------------------- batched segmented form
def segment_lengths(nseg, seed=0):
    """Lognormal lengths, median 256, sigma 1.5, clipped to [1, 2^20] (Box-Muller on SplitMix64)."""
    h = splitmix64(seed, 1, 2 * nseg)
    u1 = ((h[0::2] >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
    u2 = ((h[1::2] >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
    z = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    return np.clip(np.round(np.exp(np.log(256.0) + 1.5 * z)), 1, 1 << 20).astype(np.int64)


_SEG_CACHE = {}


def gen_segmented(nseg):
    if nseg in _SEG_CACHE:
        return _SEG_CACHE[nseg]
    _SEG_CACHE[nseg] = _gen_segmented(nseg)
    return _SEG_CACHE[nseg]


def _gen_segmented(nseg):
    lens = segment_lengths(nseg)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    n = int(off[-1])
    keys = (splitmix64(0, 0, n) >> np.uint64(32)).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    return keys, vals, off


def _seg_sigs(L):
    L.trtc_raw_segmented_workspace_bytes.restype = ctypes.c_ulonglong
    L.trtc_raw_segmented_workspace_bytes.argtypes = [ctypes.c_int, ctypes.c_ulonglong, ctypes.c_ulonglong]
    L.trtc_raw_segmented_sort_scan.restype = ctypes.c_int
    L.trtc_raw_segmented_sort_scan.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 4 + \
        [ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_int, ctypes.c_void_p]
    L.trtc_raw_segmented_autotune.restype = ctypes.c_int
    L.trtc_raw_segmented_autotune.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_ulonglong,
                                              ctypes.c_ulonglong, ctypes.c_void_p]
    L.trtc_raw_segmented_tuning_json.restype = ctypes.c_ulonglong
    L.trtc_raw_segmented_tuning_json.argtypes = [ctypes.c_char_p, ctypes.c_ulonglong]


def _seg_tuning(L):
    """The batched kernel's size-class table (versioned JSON), parsed."""
    buf = ctypes.create_string_buffer(8192)
    L.trtc_raw_segmented_tuning_json(buf, 8192)
    return json.loads(buf.value.decode())


def run_segmented(args):
    """100,000 uneven segments sorted and exclusive-scanned in one persistent launch, replayed
    from a CUDA graph; beside it one plain sort + scan call pair per segment on a sample."""
    import torch
    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: a CUDA device is required (there is no CPU path)")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    import thrustrtc_b200 as trtc
    from thrustrtc_b200 import _native as N
    trtc.init()
    L = N.lib
    _seg_sigs(L)
    if args.seg_len:
        # one segment length for the whole batch (cost per pair of one size class)
        nseg = args.n or max(1, (1 << 25) // args.seg_len)
        n = nseg * args.seg_len
        off_h = np.arange(0, n + 1, args.seg_len, dtype=np.int64)
        keys_h = (splitmix64(0, 0, n) >> np.uint64(32)).astype(np.uint32)
        vals_h = np.arange(n, dtype=np.uint32)
        lengths = "all %d keys" % args.seg_len
    else:
        nseg = args.n or WORKLOADS["segmented_c4"][0]
        keys_h, vals_h, off_h = gen_segmented(nseg)
        lengths = "lognormal median 256 sigma 1.5 clipped [1, 2^20]"
        if args.seg_max:
            # the same lengths clipped at seg_max (what the longest segments cost); the keys
            # keep their positions, so the batch is a prefix-preserving cut of each segment
            lens = np.minimum(np.diff(off_h), args.seg_max)
            keep = np.concatenate([np.arange(a, a + m) for a, m in zip(off_h[:-1], lens)])
            keys_h, vals_h = keys_h[keep], np.arange(len(keep), dtype=np.uint32)
            off_h = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
            lengths += ", then clipped at %d" % args.seg_max
    n = len(keys_h)
    k0 = torch.from_numpy(keys_h.view(np.int32)).to(dev)
    v0 = torch.from_numpy(vals_h.view(np.int32)).to(dev)
    k, v, sc = torch.empty_like(k0), torch.empty_like(v0), torch.empty_like(v0)
    off = torch.from_numpy(off_h).to(dev)
    wsb = L.trtc_raw_segmented_workspace_bytes(5, n, nseg)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    if args.seg_items:
        # the shape forced through a tuning table instead of the autotuner
        L.trtc_raw_segmented_tuning_load.restype = ctypes.c_int
        L.trtc_raw_segmented_tuning_load.argtypes = [ctypes.c_char_p]
        table = json.dumps({"format": "thrustrtc_b200.segmented_tuning", "version": 1,
                            "entries": [{"key_type": 5, "items": args.seg_items, "warp_small": 32}]})
        if L.trtc_raw_segmented_tuning_load(table.encode()) != 0:
            raise RuntimeError(N.last_error())
        items = args.seg_items
    else:
        items = L.trtc_raw_segmented_autotune(5, P(off), nseg, n, None)
        if items < 0:
            raise RuntimeError(N.last_error())
    stream = torch.cuda.Stream(device=dev)

    def call():
        rc = L.trtc_raw_segmented_sort_scan(5, P(k), P(v), P(sc), P(off), nseg, n, P(ws), wsb, 0,
                                            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc != 0:
            raise RuntimeError(N.last_error())

    with torch.cuda.stream(stream):
        k.copy_(k0); v.copy_(v0)
        call()  # uncaptured first call: kernel set-up
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        call()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            k.copy_(k0); v.copy_(v0)
            g.replay()
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(dev)
    with sampler, torch.cuda.stream(stream):
        barrier()
        for i in range(args.steps):
            k.copy_(k0); v.copy_(v0)  # restore (untimed)
            ev[i][0].record()
            g.replay()
            ev[i][1].record()
        barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    tot_ms = reduce_max(sum(step_ms), world, dev)
    value = replica_rate(n * args.steps, world, tot_ms / 1e3) / 1e9

    # correctness of the last replay: per-segment sortedness, stability, scan (size-independent
    # properties over the whole batch, on the device)
    seg_id = torch.repeat_interleave(torch.arange(nseg, device=dev), off[1:] - off[:-1])
    ku = k.to(torch.int64) & 0xFFFFFFFF
    same = seg_id[1:] == seg_id[:-1]
    if not bool(((ku[1:] >= ku[:-1]) | ~same).all()):
        raise RuntimeError("segmented check failed: a segment is not sorted")
    perm = v.to(torch.int64) & 0xFFFFFFFF
    if not bool((k0[perm] == k).all()) or not bool((seg_id[perm] == seg_id).all()):
        raise RuntimeError("segmented check failed: values are not the keys' permutation within segments")
    eq = same & (ku[1:] == ku[:-1])
    if not bool((perm[1:][eq] > perm[:-1][eq]).all()):
        raise RuntimeError("segmented check failed: not stable")
    cs = torch.cumsum(perm, 0)
    seg_start_cs = torch.cat([torch.zeros(1, dtype=torch.int64, device=dev), cs])[off[:-1]]
    excl = (cs - perm - seg_start_cs[seg_id]) & 0xFFFFFFFF
    if not bool((excl == (sc.to(torch.int64) & 0xFFFFFFFF)).all()):
        raise RuntimeError("segmented check failed: exclusive scan")

    # dominant kernel time from uncaptured calls with per-launch events
    N.timing_enable(True)
    with torch.cuda.stream(stream):
        for _ in range(3):
            k.copy_(k0); v.copy_(v0)
            call()
    recs = N.timing_records()
    N.timing_enable(False)
    kt = [ms for name, ms in recs if name == "seg_sort_scan_kernel"]
    peak, peak_src = measured_peak()
    per_launch_ms = statistics.mean(kt) if kt else None
    achieved = 20.0 * n / (per_launch_ms / 1e3) / 1e9 if per_launch_ms else None

    # plain path: one trtc_raw_sort_by_key + one exclusive trtc_raw_scan per segment, on a
    # sample of segments spread over the batch, extrapolated by segment count
    plain = None
    if not args.no_plain:
        sample = min(nseg, 1000)
        idx = np.linspace(0, nseg - 1, sample).astype(np.int64)
        zero = np.zeros(1, np.uint32)
        torch.cuda.synchronize()
        k.copy_(k0); v.copy_(v0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in idx:
            a, b = int(off_h[i]), int(off_h[i + 1])
            if L.trtc_raw_sort_by_key(5, ctypes.c_void_p(k.data_ptr() + 4 * a), ctypes.c_void_p(v.data_ptr() + 4 * a),
                                      4, b - a, 0, None) != 0:
                raise RuntimeError(N.last_error())
            if L.trtc_raw_scan(5, 0, 1, ctypes.c_void_p(v.data_ptr() + 4 * a), ctypes.c_void_p(sc.data_ptr() + 4 * a),
                               b - a, zero.ctypes.data_as(ctypes.c_void_p), None) != 0:
                raise RuntimeError(N.last_error())
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        pairs = int((off_h[idx + 1] - off_h[idx]).sum())
        plain = {"value": pairs / secs / 1e9, "unit": "Gkeys/s", "sample_segments": int(sample),
                 "ms_per_segment": secs / sample * 1e3,
                 "ms_all_segments_extrapolated": secs / sample * nseg * 1e3,
                 "path": "trtc_raw_sort_by_key + trtc_raw_scan (exclusive) per segment"}

    e2e = None
    if not args.no_e2e:
        kp = torch.from_numpy(keys_h.view(np.int32)).pin_memory()
        vp_ = torch.from_numpy(vals_h.view(np.int32)).pin_memory()
        op = torch.from_numpy(off_h).pin_memory()
        ko, vo, so = torch.empty_like(kp).pin_memory(), torch.empty_like(vp_).pin_memory(), torch.empty_like(vp_).pin_memory()
        steps = max(1, min(args.steps, args.e2e_steps))

        def e2e_step():
            k.copy_(kp, non_blocking=True); v.copy_(vp_, non_blocking=True); off.copy_(op, non_blocking=True)
            call()
            ko.copy_(k, non_blocking=True); vo.copy_(v, non_blocking=True); so.copy_(sc, non_blocking=True)

        for _ in range(max(3, args.warmup)):
            e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            e2e_step()
        barrier()
        secs = time.perf_counter() - t0
        e2e = {"value": n * world * steps / secs / 1e9, "unit": "Gkeys/s", "h2d_bytes_per_step": 8 * n + 8 * (nseg + 1),
               "d2h_bytes_per_step": 12 * n, "steps": steps, "ms_per_step": secs / steps * 1e3,
               "path": "pinned host -> device, trtc_raw_segmented_sort_scan, device -> pinned host"}

    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu:
        from oracle import oracle as O
        sample = min(nseg, 5000)
        idx = np.linspace(0, nseg - 1, sample).astype(np.int64)
        t0 = time.perf_counter()
        pairs = 0
        for i in idx:
            a, b = int(off_h[i]), int(off_h[i + 1])
            kk, vv = O.sort_pairs32(keys_h[a:b], vals_h[a:b], False, 1)
            np.cumsum(vv, dtype=np.uint32)
            pairs += b - a
        secs = time.perf_counter() - t0
        cpu = {"value": pairs / secs / 1e9, "unit": "Gkeys/s", "cores": 1, "kind": "port",
               "sample": "%d of the %d segments (%d pairs), oracle sort + scan per segment, 1 thread" %
                         (sample, nseg, pairs)}

    if world > 1:
        torch.distributed.barrier()
    if rank == 0:
        line = {"metric": WORKLOADS["segmented_c4"][4], "value": value, "unit": "Gkeys/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic (SplitMix64 seed 0, generated on the host)",
                "config": {"workload": "segmented_c4", "segments": nseg, "n": n,
                           "lengths": lengths,
                           "keys": "uint32 uniform", "values": "uint32 = index",
                           "op": "stable sort by key per segment, then exclusive Plus scan of its values",
                           "launch": "1 persistent launch from a device work queue (+2 queue kernels), CUDA graph replay",
                           ("forced_items_per_thread" if args.seg_items else "autotuned_items_per_thread"): items,
                           "tuning_table": _seg_tuning(L),
                           "parallelism": "replicas x%d" % world,
                           "l2": "inputs (%d MiB) exceed the 126 MB L2" % (8 * n >> 20)},
                "roofline": {"bound": "hbm", "kernel": "seg_sort_scan_kernel", "achieved": achieved, "peak": peak,
                             "peak_source": peak_src, "unit": "GB/s",
                             "frac": (achieved / peak) if achieved else None, "traffic": None,
                             "algorithmic_bytes_per_unit": 20, "launch_ms": per_launch_ms},
                "plain_per_segment": plain, "cpu_baseline": cpu, "e2e": e2e, "clocks": sampler.summary(),
                "gpu_launches": 3 * args.steps, "step_ms": [round(x, 4) for x in step_ms]}
        print(json.dumps(line), flush=True)
    del g
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


# ---------------------------------------------------------------- plain mixed types and distributions
def _uniform01(seed, stream, n):
    return ((splitmix64(seed, stream, n) >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53


def gen_mixed(wl, n):
    """Host inputs of the mixed workloads: (keys, values) arrays."""
    if wl == "c1_sort_by_key_2e20":
        return (splitmix64(0, 0, n) >> np.uint64(32)).astype(np.uint32), np.arange(n, dtype=np.int32)
    if wl == "c3a_sort_f32":
        u1, u2 = _uniform01(0, 10, n), _uniform01(0, 11, n)
        x = (np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)).astype(np.float32)
        h2 = splitmix64(0, 12, n)
        h3 = splitmix64(0, 13, n)
        dup = (h2 % np.uint64(10)) == np.uint64(2)
        x[dup] = x[(h3[dup] % np.uint64(n)).astype(np.int64)]          # 10% duplicated values
        x[(h2 % np.uint64(100)) == np.uint64(0)] = -0.0                 # 1% negative zeros
        xb = x.view(np.uint32)
        xb[(h2 % np.uint64(1000)) == np.uint64(1)] = 0x7FC00000         # 0.1% canonical NaN
        return x, None
    if wl == "c3b_sort_by_key_i64_zipf":
        ranks = np.arange(1, (1 << 20) + 1, dtype=np.float64)
        cdf = np.cumsum(ranks ** -1.1)
        cdf /= cdf[-1]
        r = np.searchsorted(cdf, _uniform01(0, 20, n)).astype(np.int64) + 1
        pi = (r * 0x9E3B1) & ((1 << 20) - 1)
        return (0x0123456700000000 + pi).astype(np.int64), np.arange(n, dtype=np.int32)
    if wl == "c3c_copy_if_functor":
        return (splitmix64(0, 0, n) >> np.uint64(32)).astype(np.uint32).view(np.int32), None
    if wl == "f2_lower_bound_u32":
        # sorted uint32 keys (the searched vector) and uniform uint32 queries, n of each
        keys = np.sort((splitmix64(0, 40, n) >> np.uint64(32)).astype(np.uint32))
        return keys.view(np.int32), (splitmix64(0, 41, n) >> np.uint64(32)).astype(np.uint32).view(np.int32)
    if wl == "a13_unique_i32":
        k, _ = gen_mixed("c3d_scan_by_key_f32", n)
        return k, None
    if wl in ("c3d_scan_by_key_f32", "f1_reduce_by_key_f32"):
        u = _uniform01(0, 30, n)
        heads = u < (1.0 / 32.0)                                         # run lengths ~ Geometric(1/32)
        heads[0] = True
        keys = (np.cumsum(heads) - 1).astype(np.int32)
        vals = ((splitmix64(0, 31, n) >> np.uint64(40)).astype(np.float64) * 2.0 ** -24).astype(np.float32)
        return keys, vals
    raise ValueError(wl)


def run_mixed(args):
    import torch
    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: a CUDA device is required (there is no CPU path)")
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import thrustrtc_b200 as trtc
    from thrustrtc_b200 import _native as N
    trtc.init()
    L = N.lib
    wl = args.workload
    n, kname, b_launch, b_unit, metric, unit = WORKLOADS[wl]
    n = args.n or n
    keys_h, vals_h = gen_mixed(wl, n)
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=dev)
    k0 = torch.from_numpy(keys_h.view(np.int64) if keys_h.dtype.itemsize == 8 else keys_h.view(np.int32)).to(dev)
    v0 = torch.from_numpy(vals_h.view(np.int32)).to(dev) if vals_h is not None else None
    k = torch.empty_like(k0)
    v = torch.empty_like(v0) if v0 is not None else None
    out = {}
    if wl in ("c1_sort_by_key_2e20", "c3b_sort_by_key_i64_zipf"):
        tc = 5 if wl.startswith("c1") else 6

        def restore():
            k.copy_(k0); v.copy_(v0)

        def step():
            if L.trtc_raw_sort_by_key(tc, P(k), P(v), 4, n, 0, None) != 0:
                raise RuntimeError(N.last_error())
    elif wl == "c3a_sort_f32":
        def restore():
            k.copy_(k0)

        def step():
            if L.trtc_raw_sort(8, P(k), n, 0, None) != 0:
                raise RuntimeError(N.last_error())
    elif wl == "c3c_copy_if_functor":
        dst = torch.empty_like(k0)
        vin = trtc.DVVectorAdaptor("int32_t", n, k0.data_ptr())
        vout = trtc.DVVectorAdaptor("int32_t", n, dst.data_ptr())
        odd = trtc.Functor({}, ["x"], "        return (x & 1) != 0;\n")

        def restore():
            flush.fill_(1)

        def step():
            out["count"] = trtc.Copy_If(vin, vout, odd)
    elif wl == "a13_unique_i32":
        dst = torch.empty_like(k0)

        def restore():
            flush.fill_(1)

        def step():
            c = L.trtc_raw_unique_copy(4, P(k0), P(dst), n, None)
            if c == (1 << 64) - 1:
                raise RuntimeError(N.last_error())
            out["count"] = c
    elif wl == "f1_reduce_by_key_f32":
        kout, vout_t = torch.empty_like(k0), torch.empty_like(v0)
        ka, va = trtc.DVVectorAdaptor("int32_t", n, k0.data_ptr()), trtc.DVVectorAdaptor("float", n, v0.data_ptr())
        koa = trtc.DVVectorAdaptor("int32_t", n, kout.data_ptr())
        voa = trtc.DVVectorAdaptor("float", n, vout_t.data_ptr())

        def restore():
            flush.fill_(1)

        def step():
            out["count"] = trtc.Reduce_By_Key(ka, va, koa, voa)
    elif wl == "f2_lower_bound_u32":
        res = torch.empty_like(v0)
        sa, qa = trtc.DVVectorAdaptor("uint32_t", n, k0.data_ptr()), trtc.DVVectorAdaptor("uint32_t", n, v0.data_ptr())
        ra = trtc.DVVectorAdaptor("int32_t", n, res.data_ptr())

        def restore():
            flush.fill_(1)

        def step():
            trtc.Lower_Bound_V(sa, qa, ra)
    else:
        dst = torch.empty_like(v0)

        def restore():
            flush.fill_(1)

        def step():
            if L.trtc_raw_scan_by_key(4, 8, 0, P(k0), P(v0), P(dst), n, None, None) != 0:
                raise RuntimeError(N.last_error())
    for _ in range(max(args.warmup, 3)):
        restore(); step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(dev)
    lc0 = N.launch_count()
    N.timing_enable(True)
    with sampler:
        torch.cuda.synchronize()
        for i in range(args.steps):
            restore()
            ev[i][0].record()
            step()
            ev[i][1].record()
        torch.cuda.synchronize()
    launches = N.launch_count() - lc0
    recs = N.timing_records()
    N.timing_enable(False)
    if L.trtc_raw_sync(None) != 0:
        raise RuntimeError(N.last_error())
    step_ms = [a.elapsed_time(b) for a, b in ev]
    ms = sum(step_ms) / args.steps
    value = n / (ms / 1e3) / 1e9 if unit in ("Gkeys/s", "Gqueries/s") else b_unit * n / (ms / 1e3) / 1e9

    # ---- size-independent checks of the last step
    if wl in ("c1_sort_by_key_2e20", "c3b_sort_by_key_i64_zipf"):
        kk = k.to(torch.int64) & 0xFFFFFFFF if tc == 5 else k
        perm = v.to(torch.int64)
        ok = bool((kk[1:] >= kk[:-1]).all()) and bool((k0[perm] == k).all())
        eq = kk[1:] == kk[:-1]
        ok = ok and bool((perm[1:][eq] > perm[:-1][eq]).all()) and int(torch.bincount(perm, minlength=n).max()) == 1
    elif wl == "c3a_sort_f32":
        # a permutation of the input whose ordered codes are sorted up to one rotation (the
        # reference's NaN rule); the codes map -0.0 and +0.0 to the same value
        b = k.to(torch.int64) & 0xFFFFFFFF
        neg = (b >> 31) == 1
        code = torch.where(neg, (-(b & 0x7FFFFFFF)) & 0xFFFFFFFF, b) ^ 0x80000000
        descents = int((code[1:] < code[:-1]).sum())
        ok = descents <= 1 and torch.equal(torch.sort(k.to(torch.int64))[0], torch.sort(k0.to(torch.int64))[0])
    elif wl == "c3c_copy_if_functor":
        sel = k0[(k0 & 1) != 0]
        ok = out["count"] == sel.numel() and torch.equal(dst[: sel.numel()], sel)
    elif wl == "a13_unique_i32":
        exp = torch.unique_consecutive(k0)
        ok = out["count"] == exp.numel() and torch.equal(dst[: exp.numel()], exp)
    elif wl == "f1_reduce_by_key_f32":
        # one (key, sum) per run, in order; sums against float64 within 1e-5 (values >= 0)
        ukeys, counts = torch.unique_consecutive(k0, return_counts=True)
        m = ukeys.numel()
        ends = torch.cumsum(counts, 0)
        cs = torch.cumsum(v0.view(torch.float32).to(torch.float64), 0)
        ref = cs[ends - 1] - torch.cat([torch.zeros(1, dtype=torch.float64, device=dev), cs[ends[:-1] - 1]])
        got = vout_t[:m].view(torch.float32).to(torch.float64)
        rel = ((got - ref).abs() / ref.abs().clamp_min(1e-30)).max().item() if m else 0.0
        out["runs"] = m
        out["max_rel_err_vs_fp64"] = rel
        ok = out["count"] == m and torch.equal(kout[:m], ukeys) and rel <= 1e-5
    elif wl == "f2_lower_bound_u32":
        mask = 0xFFFFFFFF
        exp = torch.searchsorted(k0.to(torch.int64) & mask, v0.to(torch.int64) & mask, right=False)
        ok = torch.equal(res.to(torch.int64), exp)
    else:
        seg_start = torch.nonzero(torch.cat([torch.ones(1, dtype=torch.bool, device=dev), k0[1:] != k0[:-1]]))[:, 0]
        cs = torch.cumsum(v0.view(torch.float32).to(torch.float64), 0)
        base = torch.cat([torch.zeros(1, dtype=torch.float64, device=dev), cs])[seg_start]
        seg_of = torch.cumsum(torch.cat([torch.ones(1, dtype=torch.int64, device=dev),
                                         (k0[1:] != k0[:-1]).to(torch.int64)]), 0) - 1
        ref = cs - base[seg_of]
        # relative error against FP64; prefixes below 0.01 (where the FP64 reference itself
        # carries ~1e-8 of cancellation noise from the global cumsum) are compared at 0.01
        rel = ((dst.view(torch.float32).to(torch.float64) - ref).abs() / ref.abs().clamp_min(0.01)).max().item()
        out["max_rel_err_vs_fp64"] = rel
        ok = rel <= 1e-5
    if not ok:
        raise RuntimeError("%s: result check failed %s" % (wl, out))

    kt = [t for name, t in recs if name == kname]
    if kt:  # skipped digit passes return at once: average the launches that moved data
        kt = [t for t in kt if t > 0.1 * max(kt)]
    peak, peak_src = measured_peak()
    per_launch_ms = statistics.mean(kt) if kt else None
    achieved = b_launch * n / (per_launch_ms / 1e3) / 1e9 if per_launch_ms else None
    if kname is None:
        # a composed call (Reduce_By_Key: segmented scan + compaction): its algorithmic bytes
        # over the device time of all its kernels per call
        kname = "all kernels of the call"
        kt = [t for _, t in recs]
        per_launch_ms = sum(kt) / args.steps if kt else None
        b_launch = b_unit
        achieved = b_unit * n / (per_launch_ms / 1e3) / 1e9 if per_launch_ms else None
    share = {}
    for name, t in recs:
        share[name] = share.get(name, 0.0) + t
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"c1_sort_by_key_2e20": "u32", "c3a_sort_f32": "f32",
                                           "c3b_sort_by_key_i64_zipf": "int64", "c3c_copy_if_functor": "int32",
                                           "c3d_scan_by_key_f32": "f32", "f1_reduce_by_key_f32": "i32/f32",
                                           "f2_lower_bound_u32": "u32", "a13_unique_i32": "int32"}[wl],
            "data": "synthetic (SplitMix64 seed 0, generated on the host)",
            "config": {"workload": wl, "n": n, "l2": "inputs exceed the 126 MB L2 (flush between steps for "
                                                     "non-destructive ops)" if n > (1 << 24) else
                       "inputs fit in L2; restored from a pristine copy each step"},
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "peak_source": peak_src,
                         "unit": "GB/s", "frac": achieved / peak if achieved else None, "traffic": None,
                         "algorithmic_bytes_per_launch": b_launch * n, "launch_ms": per_launch_ms,
                         "launches_timed": len(kt)},
            "roofline_whole_op": {"algorithmic_bytes_per_unit": b_unit, "achieved": b_unit * n / (ms / 1e3) / 1e9,
                                  "frac": b_unit * n / (ms / 1e3) / 1e9 / peak, "unit": "GB/s"},
            "kernel_ms_timed_region": {a: round(b, 4) for a, b in sorted(share.items())},
            "check": {k2: v2 for k2, v2 in out.items() if k2 != "count"},
            "e2e": None, "cpu_baseline": None, "clocks": sampler.summary(), "gpu_launches": launches,
            "step_ms": [round(x, 4) for x in step_ms]}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- serving form
def serving_requests(count, seed=0):
    """(kind, type, n) per request: kinds 60/25/15 % (Sort_By_Key / exclusive scan / reduce),
    element types uint32 / int64 / float in equal shares, sizes log-uniform on [2^10, 2^24]."""
    h = splitmix64(seed, 2, 3 * count)
    u = (h >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    kind = np.where(u[0::3] < 0.6, 0, np.where(u[0::3] < 0.85, 1, 2))
    types = np.array([5, 6, 8])[np.minimum((u[1::3] * 3).astype(np.int64), 2)]
    n = np.floor(2.0 ** (10 + 14 * u[2::3])).astype(np.int64)
    return list(zip(kind.tolist(), types.tolist(), n.tolist()))


def _srv_sigs(L):
    L.trtc_server_create.restype = ctypes.c_void_p
    L.trtc_server_create.argtypes = [ctypes.c_ulonglong, ctypes.c_int, ctypes.c_ulonglong]
    L.trtc_server_submit.restype = ctypes.c_longlong
    L.trtc_server_submit.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 3 + \
        [ctypes.c_ulonglong]
    L.trtc_server_poll.restype = ctypes.c_int
    L.trtc_server_poll.argtypes = [ctypes.c_void_p]
    L.trtc_server_info.restype = ctypes.c_int
    L.trtc_server_info.argtypes = [ctypes.c_void_p, ctypes.c_longlong] + [ctypes.POINTER(ctypes.c_double)] * 3
    L.trtc_server_now.restype = ctypes.c_double
    L.trtc_server_now.argtypes = [ctypes.c_void_p]
    L.trtc_server_forget_done.argtypes = [ctypes.c_void_p]
    L.trtc_server_destroy.argtypes = [ctypes.c_void_p]


# offered rates as fractions of the plain path's capacity; the grid runs past the served
# path's own capacity (about 4x the plain one), so both paths saturate inside it and the
# highest achieved rate of each is its sustained throughput rather than the top offered rate
SERVING_GRID = (0.25, 0.50, 0.75, 0.90, 1.00, 1.25, 1.50, 2.00, 2.50, 3.00, 3.50, 4.00, 4.50, 5.00)


def run_serving(args):
    """The serving form as its own JSON line (see _serving_measure)."""
    import torch
    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: a CUDA device is required (there is no CPU path)")
    if rank != 0:
        return 0  # one GPU: the serving form is measured on rank 0 only
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    count = args.n or WORKLOADS["serving_c5"][0]
    levels = tuple(float(f) for f in args.levels.split(",")) if args.levels else SERVING_GRID
    rec = _serving_measure(count, dev, shared_grid=True, grid=levels, coalesce=args.coalesce, streams=args.streams)
    line = {"metric": WORKLOADS["serving_c5"][4], "value": rec["capacity_rps"]["served"], "unit": "requests/s",
            "n_gpus": 1, "steps": len(rec["levels"]), "warmup": 1,
            "ms_per_step": 1e3 * 1000 / rec["capacity_rps"]["served"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32/i64/f32",
            "data": "synthetic (SplitMix64 seed 0 request mix; torch generator seed 0 contents)",
            "config": rec["config"], "capacity_rps": rec["capacity_rps"], "sustained_rps": rec["sustained_rps"],
            "levels": rec["levels"],
            "clocks": rec["clocks"], "gpu_launches": rec["gpu_launches"],
            "e2e": None, "cpu_baseline": None, "roofline": None}
    print(json.dumps(line), flush=True)
    return 0


def _serving_measure(count, dev, shared_grid=True, grid=SERVING_GRID, block=1000, coalesce=1 << 16, streams=8):
    """Poisson arrivals of `count` mixed requests into the request server (continuous
    batching: 8 streams, coalescing of requests up to 2^16 elements, 32 GB admission budget)
    beside the plain path (the same requests one call at a time on one stream, no coalescing).

    Capacity: each path's closed-loop throughput on the first block of requests (all
    submitted at once).  Latency: offered rates on one grid for both paths (fractions of the
    plain path's capacity, shared_grid=True) or each path at fractions of its own capacity;
    p50 / p99 of submit-to-done latency over all requests.  Streams longer than `block`
    requests run block after block (inputs restored between blocks, queues drained), so the
    device buffers stay the size of one block."""
    import torch
    import thrustrtc_b200 as trtc
    from thrustrtc_b200 import _native as N
    trtc.init()
    L = N.lib
    _srv_sigs(L)
    reqs = serving_requests(count)
    block = min(block, count)
    blocks = [reqs[i:i + block] for i in range(0, count, block)]
    esz = {5: 4, 6: 8, 8: 4}
    # capacity per element type (and of the value array) for the largest block
    cap_t = {5: 1, 6: 1, 8: 1}
    cap_v = 1
    for b in blocks:
        tot = {5: 0, 6: 0, 8: 0}
        for kind, t, n in b:
            tot[t] += n
        for t in tot:
            cap_t[t] = max(cap_t[t], tot[t])
        cap_v = max(cap_v, sum(n for k, t, n in b if k == 0))
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    pristine = {5: torch.randint(-2**31, 2**31 - 1, (cap_t[5],), dtype=torch.int32, device=dev, generator=g),
                6: torch.randint(-2**62, 2**62, (cap_t[6],), dtype=torch.int64, device=dev, generator=g),
                8: torch.randn(cap_t[8], device=dev, generator=g)}
    work = {t: torch.empty_like(x) for t, x in pristine.items()}
    outs = {t: torch.empty_like(x) for t, x in pristine.items()}
    vals = torch.empty(cap_v + 1, dtype=torch.int32, device=dev)
    vals0 = torch.arange(cap_v + 1, dtype=torch.int32, device=dev)

    def layout(b):
        """Pointers of each request of block b inside the work / value / output buffers."""
        offs, vof = {5: 0, 6: 0, 8: 0}, 0
        ptr = []
        for kind, t, n in b:
            k = ctypes.c_void_p(work[t].data_ptr() + esz[t] * offs[t])
            v = ctypes.c_void_p(vals.data_ptr() + 4 * vof) if kind == 0 else None
            o = ctypes.c_void_p(outs[t].data_ptr() + esz[t] * offs[t]) if kind == 1 else None
            ptr.append((kind, t, n, k, v, o))
            offs[t] += n
            vof += n if kind == 0 else 0
        return ptr

    layouts = [layout(b) for b in blocks]

    def restore():
        for t in work:
            work[t].copy_(pristine[t])
        vals.copy_(vals0)
        torch.cuda.synchronize()

    def run_block(srv, bi, arrivals):
        """Submits request i of block bi at arrivals[i] (seconds from the block's start;
        None = all at once) and polls until all are done; returns (latencies, makespan)."""
        restore()
        ptr = layouts[bi]
        cnt = len(ptr)
        ids = [0] * cnt
        t0 = L.trtc_server_now(srv)
        nxt = 0
        while True:
            now = L.trtc_server_now(srv) - t0
            while nxt < cnt and (arrivals is None or arrivals[nxt] <= now):
                kind, t, n, k, v, o = ptr[nxt]
                ids[nxt] = L.trtc_server_submit(srv, kind, t, k, v, o, n)
                if ids[nxt] <= 0:
                    raise RuntimeError(N.last_error())
                nxt += 1
            left = L.trtc_server_poll(srv)
            if left < 0:
                raise RuntimeError(N.last_error())
            if nxt == cnt and left == 0:
                break
        lat, first, last = [], None, 0.0
        ts, td = ctypes.c_double(), ctypes.c_double()
        for rid in ids:
            st = L.trtc_server_info(srv, rid, ctypes.byref(ts), ctypes.byref(td), None)
            if st != 2:
                raise RuntimeError("request %d not done (state %d)" % (rid, st))
            lat.append(td.value - ts.value)
            first = ts.value if first is None else min(first, ts.value)
            last = max(last, td.value)
        L.trtc_server_forget_done(srv)
        return np.array(lat), last - first

    def capacity(srv):
        run_block(srv, 0, None)  # warm-up (kernel set-up, memory pool)
        _, span = run_block(srv, 0, None)
        return len(blocks[0]) / span

    def at_rate(srv, rate):
        lat, span = [], 0.0
        for bi, b in enumerate(blocks):
            h = splitmix64(1 + bi, 3, len(b))
            u = ((h >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
            arrivals = np.cumsum(-np.log(u) / rate)
            lb, sb = run_block(srv, bi, arrivals)
            lat.append(lb)
            span += sb
        lat = np.concatenate(lat)
        return {"achieved_rps": count / span, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3)}

    budget = 32 << 30
    served = L.trtc_server_create(budget, streams, coalesce)
    plain = L.trtc_server_create(budget, 1, 0)
    if not served or not plain:
        raise RuntimeError(N.last_error())
    lc0 = N.launch_count()
    sampler = ClockSampler(dev)
    try:
        with sampler:
            cap_b = capacity(served)
            cap_p = capacity(plain)
            levels = []
            for f in grid:
                if shared_grid:
                    rate = f * cap_p
                    levels.append({"offered_rps": rate, "fraction_of_plain_capacity": f,
                                   "served": at_rate(served, rate), "plain": at_rate(plain, rate)})
                else:
                    levels.append({"fraction_of_own_capacity": f, "served": at_rate(served, f * cap_b),
                                   "plain": at_rate(plain, f * cap_p)})
    finally:
        L.trtc_server_destroy(served)
        L.trtc_server_destroy(plain)
    launches = N.launch_count() - lc0
    elems = sum(n for _, _, n in reqs)
    # open-loop throughput: the highest request rate each path achieved under Poisson arrivals
    sus_b = max(l["served"]["achieved_rps"] for l in levels)
    sus_p = max(l["plain"]["achieved_rps"] for l in levels)
    return {"capacity_rps": {"served": cap_b, "plain": cap_p, "ratio": cap_b / cap_p},
            "sustained_rps": {"served": sus_b, "plain": sus_p, "ratio": sus_b / sus_p,
                              "how": "highest achieved rate over the offered-rate grid (Poisson arrivals)"},
            "levels": levels, "clocks": sampler.summary(), "gpu_launches": launches,
            "config": {"workload": "serving_c5", "requests": count, "block": block,
                       "sample": ("the full %d-request stream" % count) if count >= 200000 else
                                 ("%d requests per load level (a bounded sample of the 200,000-request stream)"
                                  % count),
                       "mix": "60% Sort_By_Key (+uint32 values), 25% exclusive scan, 15% reduce",
                       "sizes": "log-uniform 2^10..2^24", "types": "uint32 / int64 / float equal shares",
                       "elements": elems, "budget_bytes": budget,
                       "server": "%d streams, coalescing of requests up to %d elements, admission by budget"
                                 % (streams, coalesce),
                       "plain": "same requests, one call at a time on one stream, no coalescing",
                       "grid": ("the same offered rates for both paths, as fractions of the plain path's "
                                "capacity") if shared_grid else "fractions of each path's own capacity",
                       "capacity": "closed loop on the first %d requests, all submitted at once" % len(blocks[0])}}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="sort_by_key_u32")
    ap.add_argument("--n", type=int, default=0, help="override the element count (development only)")
    ap.add_argument("--cpu-sample", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--allow-short-warmup", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="segmented_c4: skip the per-segment plain calls")
    ap.add_argument("--seg-len", type=int, default=0, help="segmented_c4: every segment this long (one size class)")
    ap.add_argument("--seg-max", type=int, default=0, help="segmented_c4: clip the lognormal lengths at this many keys")
    ap.add_argument("--seg-items", type=int, default=0, choices=[0, 8, 16],
                    help="segmented_c4: force this items-per-thread shape instead of autotuning")
    ap.add_argument("--no-sub", action="store_true", help="default run: skip the scan / reduce / serving records")
    ap.add_argument("--sub-requests", type=int, default=1000, help="requests of the serving record")
    ap.add_argument("--levels", default="", help="serving_c5: comma-separated fractions of the plain capacity")
    ap.add_argument("--coalesce", type=int, default=1 << 16, help="serving_c5: largest request the server coalesces")
    ap.add_argument("--streams", type=int, default=8, help="serving_c5: streams of the server")
    ap.add_argument("--thrustrtc-child", default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.thrustrtc_child:
        _thrustrtc_child(args.thrustrtc_child, args.n or WORKLOADS[args.thrustrtc_child][0])
        return 0
    _, world, _ = dist_env()
    if args.gpus != world and not (args.gpus == 1 and world == 1):
        if world == 1:
            raise SystemExit("bench.py: for --gpus N > 1 launch one process per GPU with torchrun")
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "segmented_c4":
        return run_segmented(args)
    if args.workload == "serving_c5":
        return run_serving(args)
    if args.workload.startswith(("c1_", "c3", "f1_", "f2_", "a13_")):
        return run_mixed(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
