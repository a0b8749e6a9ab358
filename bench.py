#!/usr/bin/env python
"""FlashMap B200 backend benchmark: prints ONE JSON line.

Workload (one "step"), the account shape FlashMap<[u8;32],[u8;128]> at load
factor 0.8: with_capacity(2^24), clear, 13,421,773 distinct pairs inserted as
bulk_insert calls of 100,000 (the last one shorter), one bulk_get of 8,000,000
keys (50% present, 50% fresh random keys, shuffled), one bulk_remove of a
random 10% of the present keys.  Keys and values are seeded uniform random
bytes.  with_capacity(10,000,000) as written rounds up to 2^24 slots, where
8,000,000 pairs are load 0.477; that variant is timed too and reported under
"as_written".

  value  = ops of the step x ranks / device time (CUDA events, max over
           ranks), inputs resident in HBM, device-pointer API.
  e2e    = the same step through the host API (fm_bulk_insert/get/remove with
           pinned host buffers: H2D of inputs and D2H of results inside).
  roofline: per kernel set (insert: the round kernels of every call; get: the
           one lookup kernel), algorithmic bytes per op (counted by the CPU
           oracle on the same workload at 1/16 scale) x ops / the set's device
           time, read from the library's per-kernel CUDA events in an extra
           step, against MEASURED_PEAKS.json hbm_gbs.
  cpu_baseline: the sequential CPU oracle on the 1/16-scale sample.
  oracle_check: the same leg replays the whole step the GPU ran on the
           sequential oracle and compares every result and the final table.

`--impl reference` times the reference's CPU algorithm (multithreaded CAS
restatement of src/rayon_cpu.rs, all host threads) on the same full-size
workload.
Multi-GPU (torchrun): every rank runs an independent table (replicas, weak
scaling); no collective on the data path.
"""
import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "flash-map_b200"))

METRIC = "bulk get/insert Mops/s at load 0.8, % HBM roofline; served p50/p99 vs plain"
CALL = 100_000
KB, VB = 32, 128
SAMPLE_DIV = 16  # CPU sample: same load factors and call size at 1/16 scale


class Workload:
    def __init__(self, name, cap_req, pairs, gets, removes):
        self.name, self.cap_req, self.pairs, self.gets, self.removes = name, cap_req, pairs, gets, removes

    @property
    def cap(self):
        c = 1
        while c < self.cap_req:
            c <<= 1
        return c

    @property
    def ops(self):
        return self.pairs + self.gets + self.removes

    def scaled(self, div):
        return Workload(self.name, self.cap_req // div, self.pairs // div, self.gets // div, self.removes // div)

    def desc(self):
        calls = (self.pairs + CALL - 1) // CALL
        return {
            "workload": f"account shape [u8;32]->[u8;128], {self.name}: with_capacity({self.cap_req})="
                        f"{self.cap} slots, clear, {self.pairs} pairs as {calls} bulk_insert calls of <= {CALL}, "
                        f"bulk_get of {self.gets} (50% hits), bulk_remove of {self.removes} present",
            "capacity": self.cap,
            "pairs": self.pairs,
            "insert_calls": f"{calls}x<={CALL}",
            "gets": self.gets,
            "get_hit_rate": 0.5,
            "removes": self.removes,
            "load_after_insert": round(self.pairs / self.cap, 4),
            "l2": "inputs larger than L2 (table 2.9 GB, 256 MB of get keys per call); no flush",
            "api": "device-pointer API (fm_*_device), stream-ordered",
        }


LOAD08 = Workload("load 0.8", 1 << 24, 13_421_773, 8_000_000, 1_342_177)
AS_WRITTEN = Workload("as written (load 0.477)", 10_000_000, 8_000_000, 8_000_000, 800_000)


def read_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU sample (oracle / reference restatement): 1/16 scale, same load factors
# ---------------------------------------------------------------------------
def cpu_sample_inputs(w, seed=3):
    rng = np.random.default_rng(seed)
    n = w.pairs
    keys = rng.integers(0, 256, (n, KB), dtype=np.uint8)
    vals = rng.integers(0, 256, (n, VB), dtype=np.uint8)
    ng = w.gets
    q = np.concatenate([keys[rng.choice(n, ng // 2, replace=False)],
                        rng.integers(0, 256, (ng - ng // 2, KB), dtype=np.uint8)])
    q = q[rng.permutation(len(q))]
    rem = keys[rng.choice(n, w.removes, replace=False)]
    return keys, vals, q, rem


def cpu_step(O, w, inp, threads=None, traffic=False):
    """One sample step on the oracle (threads=None: sequential) -> seconds."""
    keys, vals, q, rem = inp
    m = O.OracleMap(w.cap, KB, VB)
    if traffic:
        m.traffic(True)
    t0 = time.perf_counter()
    for b in range(0, len(keys), CALL):
        if threads:
            m.mt_bulk_insert(keys[b:b + CALL], vals[b:b + CALL], threads)
        else:
            m.bulk_insert(keys[b:b + CALL], vals[b:b + CALL])
    if threads:
        m.mt_bulk_get(q, threads)
        m.mt_bulk_remove(rem, threads)
    else:
        m.bulk_get(q)
        m.bulk_remove(rem)
    dt = time.perf_counter() - t0
    tr = None
    if traffic:
        tr = {k: m.traffic_get(k) for k in ("insert", "get", "remove")}
    return dt, tr


def oracle_replay_check(run):
    """Part of the CPU-baseline leg: the sequential oracle replays the step
    the GPU just ran (same inputs, same call sizes) and every result is
    compared: each insert call's new-key count summed, every get's found flag
    and value bytes, the remove count, len, and the whole final table
    (metadata word of every slot, key and value bytes of every occupied slot)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    w, m = run.w, run.m
    t0 = time.perf_counter()
    keys, vals = run.keys.cpu().numpy(), run.vals.cpu().numpy()
    q, rem = run.q.cpu().numpy(), run.rem.cpu().numpy()
    # the GPU's results of its last step: outputs, then the final table
    gv, gf = run.out_v.cpu().numpy(), run.out_f.cpu().numpy().astype(bool)
    gsnap = m.snapshot()
    o = O.OracleMap(w.cap, KB, VB)
    added = sum(o.bulk_insert(keys[b:b + CALL], vals[b:b + CALL]) for b in range(0, w.pairs, CALL))
    ov, of = o.bulk_get(q)
    removed = o.bulk_remove(rem)
    osnap = o.snapshot()
    ok = {
        "inserts_new_keys": added == w.pairs,
        "gets_found": bool(np.array_equal(gf, of)),
        "gets_values": bool(np.array_equal(gv, ov)),
        "removes": removed == w.removes,
        "len": m.len() == len(o),
        "table": all(bool(np.array_equal(a, b)) for a, b in zip(gsnap, osnap)),
    }
    return {"replayed": f"the whole step on the sequential CPU oracle ({w.pairs} inserts in calls of {CALL}, "
                        f"{w.gets} gets, {w.removes} removes)",
            "identical": all(ok.values()), "checks": ok, "seconds": round(time.perf_counter() - t0, 1)}


def bytes_per_op(tr):
    out = {}
    for k, v in tr.items():
        b = (v["table_sectors_read"] + v["table_sectors_written"]) * 32 + v["stream_bytes_in"] + v["stream_bytes_out"]
        out[k] = b / max(v["ops"], 1)
    return out


def cpu_baseline_leg(w):
    """Sequential oracle timed on the 1/16-scale sample of workload w, and the
    algorithmic bytes per op it counts on the same sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    ws = w.scaled(SAMPLE_DIV)
    inp = cpu_sample_inputs(ws)
    reps, total = 0, 0.0
    while reps < 64 and (total < 8.0 or reps < 2):  # ~10 s of CPU work
        dt, _ = cpu_step(O, ws, inp)
        total += dt
        reps += 1
    _, tr = cpu_step(O, ws, inp, traffic=True)
    return {
        "value": round(ws.ops * reps / total / 1e6, 3),
        "unit": "Mops/s",
        "cores": 1,
        "kind": "port",
        "sample": f"the same step at 1/{SAMPLE_DIV} scale ({ws.cap} slots, {ws.pairs} pairs in calls of {CALL}, "
                  f"{ws.gets} gets, {ws.removes} removes; same load factors), sequential C oracle, "
                  f"{reps} reps in {total:.1f} s",
    }, bytes_per_op(tr)


def reference_arm(args, w):
    """The reference's CPU algorithm on the host cores, on the same workload
    as the GPU arm (full size: every step is one clear + the step's inserts,
    gets and removes)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    threads = os.cpu_count() or 1
    inp = cpu_sample_inputs(w)
    for _ in range(args.warmup):
        cpu_step(O, w, inp, threads=threads)
    times = [cpu_step(O, w, inp, threads=threads)[0] for _ in range(args.steps)]
    total = sum(times)
    v = w.ops * len(times) / total / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "Mops/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total / len(times) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": dict(w.desc(), parallelism="host threads"),
        "cpu_baseline": {"value": round(v, 3), "unit": "Mops/s", "cores": threads, "kind": "port",
                         "sample": f"the whole step ({w.cap} slots, {w.pairs} pairs in calls of {CALL}, "
                                   f"{w.gets} gets, {w.removes} removes), {threads} threads; multithreaded CAS "
                                   "restatement of src/rayon_cpu.rs (the reference's Rust crate cannot be "
                                   "built here)"},
        "e2e": {"value": round(v, 3), "unit": "Mops/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
class Clocks:
    def __init__(self, gpu_index):
        self.path = f"/tmp/fm_clocks_{os.getpid()}.csv"
        self.proc = None
        self.gpu = gpu_index

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}",
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "20"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        try:
            self.fh.close()
        except Exception:
            pass

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, val in zip(names, r[5:9]):
                if "Active" in val and "Not" not in val:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(rows)}


def gpu_inputs(torch, dev, w, seed=3):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    keys = torch.randint(0, 256, (w.pairs, KB), dtype=torch.uint8, device=dev, generator=g)
    vals = torch.randint(0, 256, (w.pairs, VB), dtype=torch.uint8, device=dev, generator=g)
    hit = torch.randperm(w.pairs, device=dev, generator=g)[: w.gets // 2]
    fresh = torch.randint(0, 256, (w.gets - w.gets // 2, KB), dtype=torch.uint8, device=dev, generator=g)
    q = torch.cat([keys[hit], fresh])
    q = q[torch.randperm(w.gets, device=dev, generator=g)].contiguous()
    rem = keys[torch.randperm(w.pairs, device=dev, generator=g)[:w.removes]].contiguous()
    return keys, vals, q, rem


def max_over_ranks(value, dist, device):
    """The largest of every rank's value (all ranks call it; identity without
    a process group)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


INSERT_KERNELS = ("ins_find", "ins_flow", "ins_exec", "ins_warp", "k_ins_tail", "k_ins_serial")
REMOVE_KERNELS = ("k_rem_p1", "k_rem_p2", "k_rem_p3", "k_rem_tail", "rem_group")

# DRAM traffic (ncu dram__bytes_read.sum + dram__bytes_write.sum) per op of
# each kernel set, from captures of the same kernels on a 2^22-slot table at
# the same load factor and call size (the traffic summary under
# profiles/ gives the command and the per-kernel figures); traffic grows with
# the ops processed.
NCU_TRAFFIC_PER_OP = {"insert": 2446.0, "get": 334.7, "remove": 515.2}


class DeviceRun:
    """Times one workload's step on one GPU through the device-pointer API."""

    def __init__(self, torch, F, dev, stream, w, local):
        self.torch, self.w, self.stream = torch, w, stream
        self.keys, self.vals, self.q, self.rem = gpu_inputs(torch, dev, w)
        self.out_v = torch.empty((w.gets, VB), dtype=torch.uint8, device=dev)
        self.out_f = torch.empty((w.gets,), dtype=torch.uint8, device=dev)
        self.m = F.FlashMap(w.cap_req, KB, VB, F.HashStrategy.Identity, local)

    def step(self, ev=None):
        w, m, s = self.w, self.m, self.stream
        m.clear()
        for b in range(0, w.pairs, CALL):
            n = min(CALL, w.pairs - b)
            m.bulk_insert_device(self.keys[b:b + n], self.vals[b:b + n], n, s)
        if ev:
            ev[0].record(s)
        m.bulk_get_device(self.q, w.gets, self.out_v, self.out_f, s)
        if ev:
            ev[1].record(s)
        m.bulk_remove_device(self.rem, w.removes, s)

    def check(self):
        assert self.m.len() == self.w.pairs - self.w.removes, self.m.len()
        assert int(self.out_f.sum().item()) == self.w.gets // 2

    def timed(self, steps, barrier, native):
        torch, s = self.torch, self.stream
        Ev = torch.cuda.Event
        phase = [(Ev(enable_timing=True), Ev(enable_timing=True)) for _ in range(steps)]
        starts = [Ev(enable_timing=True) for _ in range(steps)]
        ends = [Ev(enable_timing=True) for _ in range(steps)]
        t0, t1 = Ev(enable_timing=True), Ev(enable_timing=True)
        l0 = native.launch_count()
        barrier()
        torch.cuda.synchronize()
        t0.record(s)
        for k in range(steps):
            starts[k].record(s)
            self.step(phase[k])
            ends[k].record(s)
        t1.record(s)
        torch.cuda.synchronize()
        barrier()
        return {
            "total_ms": t0.elapsed_time(t1),
            "launches": native.launch_count() - l0,
            "ins_ms": statistics.median(starts[k].elapsed_time(phase[k][0]) for k in range(steps)),
            "get_ms": statistics.median(phase[k][0].elapsed_time(phase[k][1]) for k in range(steps)),
            "rem_ms": statistics.median(phase[k][1].elapsed_time(ends[k]) for k in range(steps)),
        }

    def kernel_pass(self, nvtx=False):
        """One more step with the library's per-kernel CUDA events on.  With
        nvtx, the step sits in the NVTX range "step", and within it the last
        full insert call (the highest load) and the bulk_get in "insert_call"
        and "get_call" (for ncu --nvtx-include)."""
        self.m.kernel_timing(True, reset=True)
        if nvtx:
            w, m, s, nv = self.w, self.m, self.stream, self.torch.cuda.nvtx
            self.torch.cuda.synchronize()
            nv.range_push("step")
            m.clear()
            mid = (w.pairs // CALL - 1) * CALL
            for b in range(0, w.pairs, CALL):
                n = min(CALL, w.pairs - b)
                if b == mid:
                    nv.range_push("insert_call")
                m.bulk_insert_device(self.keys[b:b + n], self.vals[b:b + n], n, s)
                if b == mid:
                    self.torch.cuda.synchronize()
                    nv.range_pop()
            nv.range_push("get_call")
            m.bulk_get_device(self.q, w.gets, self.out_v, self.out_f, s)
            self.torch.cuda.synchronize()
            nv.range_pop()
            m.bulk_remove_device(self.rem, w.removes, s)
            self.torch.cuda.synchronize()
            nv.range_pop()
        else:
            self.step()
        self.torch.cuda.synchronize()
        kt = self.m.kernel_times()
        self.m.kernel_timing(False)
        return kt

    def ops(self, t):
        w = self.w
        return {"insert_mops": round(w.pairs / t["ins_ms"] / 1e3, 3), "get_mops": round(w.gets / t["get_ms"] / 1e3, 3),
                "remove_mops": round(w.removes / t["rem_ms"] / 1e3, 3), "insert_ms": round(t["ins_ms"], 3),
                "get_ms": round(t["get_ms"], 3), "remove_ms": round(t["rem_ms"], 3)}

    def e2e(self, steps, barrier, dist, world):
        torch, w, m = self.torch, self.w, self.m
        hk = self.keys.cpu().pin_memory().numpy()
        hv = self.vals.cpu().pin_memory().numpy()
        hq = self.q.cpu().pin_memory().numpy()
        hr = self.rem.cpu().pin_memory().numpy()
        ho = torch.empty((w.gets, VB), dtype=torch.uint8).pin_memory().numpy()
        hf = torch.empty((w.gets,), dtype=torch.uint8).pin_memory().numpy()

        def step_host():
            m.clear()
            for b in range(0, w.pairs, CALL):
                m.bulk_insert(hk[b:b + CALL], hv[b:b + CALL])
            m.bulk_get(hq, out_values=ho, out_found=hf)
            m.bulk_remove(hr)

        step_host()
        assert int(hf.sum()) == w.gets // 2
        n = max(1, min(steps, 3))
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(n):
            step_host()
        torch.cuda.synchronize()
        e2e_s = max_over_ranks((time.perf_counter() - t0) / n, dist, self.q.device)
        calls = (w.pairs + CALL - 1) // CALL
        # the link these copies cross: pinned 256 MB copies each way
        hb = torch.empty(1 << 28, dtype=torch.uint8).pin_memory()
        db = torch.empty(1 << 28, dtype=torch.uint8, device=self.q.device)
        Ev = torch.cuda.Event
        bw = {}
        for name, dst, src in (("h2d_gbs", db, hb), ("d2h_gbs", hb, db)):
            dst.copy_(src, non_blocking=True)
            a, b = Ev(enable_timing=True), Ev(enable_timing=True)
            a.record()
            for _ in range(3):
                dst.copy_(src, non_blocking=True)
            b.record()
            torch.cuda.synchronize()
            bw[name] = round(3 * (1 << 28) / (a.elapsed_time(b) / 1e3) / 1e9, 1)
        h2d = w.pairs * (KB + VB) + w.gets * KB + w.removes * KB
        d2h = w.gets * (VB + 1) + 8 * (calls + 1)
        return {"value": round(w.ops * world / e2e_s / 1e6, 3), "unit": "Mops/s",
                "link_gbs": bw,
                "copy_bound_ms": round((h2d / bw["h2d_gbs"] + d2h / bw["d2h_gbs"]) / 1e6, 3),
                "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "ms_per_step": round(e2e_s * 1e3, 3)}


def kernel_summary(kt, w):
    total = sum(v[0] for v in kt.values()) or 1.0
    return {k: {"ms": round(v[0], 3), "launches": v[1], "share": round(v[0] / total, 4)}
            for k, v in sorted(kt.items(), key=lambda kv: -kv[1][0])}


def get_kernel_label():
    from flash_map import _native

    lanes, bps = _native.tuned_get_config(KB, VB, 0.8)
    name = "k_get_thread<32,128>" if lanes == 1 else f"k_get<32,128,{lanes}>"
    return f"{name} ({lanes} lane(s) per query, {bps} blocks per SM; one launch of all gets)"


def roofline_for(kt, names, nops, bpo, peak, kind, label, traffic_per_op):
    ms = sum(kt[k][0] for k in names if k in kt)
    launches = sum(kt[k][1] for k in names if k in kt)
    if ms <= 0:
        return None
    achieved = bpo * nops / (ms / 1e3) / 1e9
    return {"kernel": label, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": kind,
            "algorithmic_bytes_per_op": round(bpo, 2), "ops": nops, "kernel_ms": round(ms, 3),
            "launches": launches,
            "traffic": None if traffic_per_op is None else round(traffic_per_op * nops / max(launches, 1)),
            "traffic_per_op": traffic_per_op,
            "traffic_unit": "bytes per launch (ncu dram bytes per op, small case, x ops per launch)"}


# ---------------------------------------------------------------------------
# Batched form: 512 queued bulk ops over 64 independent tables
# ---------------------------------------------------------------------------
BATCH_TABLES, BATCH_OPS = 64, 512


def batched_leg(torch, F, native, dev, steps, warmup, scale=1, clip=False):
    """The batching workload: 64 tables (capacities log-uniform 2^14..2^24,
    alternating u64->u64 and [u8;32]->[u8;128], prefilled to loads uniform in
    0.5..0.9) and 512 queued ops (40% get / 40% insert / 20% remove, sizes
    log-uniform 256..4M, gets and removes half present keys), seed 5, as
    specified: inserts larger than their table's free space fail with
    TableFull, the others run whatever load they reach.  With clip, an insert
    that fits but would take its table past 95% load (by a conservative
    count) is clipped to end there (the variant reported beside it).  Timed
    from the same prefilled state (restored on the device before every run)
    as the plain per-call path (fm_*_device calls in queue order) and as one
    batch replayed from a CUDA graph; both must give the same results."""
    rng = np.random.default_rng(5)
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    stream = torch.cuda.Stream(dev)
    tables, backups, known = [], [], []
    for i in range(BATCH_TABLES):
        ks, vs = (8, 8) if i % 2 == 0 else (KB, VB)
        cap = max(int(2 ** rng.uniform(14, 24)) // scale, 256)
        m = F.FlashMap(cap, ks, vs, F.HashStrategy.Identity, dev.index or 0)
        n = int(m.capacity() * rng.uniform(0.5, 0.9))
        k = torch.randint(0, 256, (n, ks), dtype=torch.uint8, device=dev, generator=g)
        v = torch.randint(0, 256, (n, vs), dtype=torch.uint8, device=dev, generator=g)
        m.bulk_insert_device(k, v, n, stream)
        bk = F.FlashMap(cap, ks, vs, F.HashStrategy.Identity, dev.index or 0)
        bk.copy_from(m, stream)
        tables.append(m)
        backups.append(bk)
        known.append(k)
    ops, outs = [], [[], []]
    level = [m.len() for m in tables]  # keys present, tracked conservatively (removes not subtracted)
    clipped = 0
    for i in range(BATCH_OPS):
        ti = int(rng.integers(BATCH_TABLES))
        m = tables[ti]
        kind = int(rng.choice([0, 1, 2], p=[0.4, 0.4, 0.2]))
        n = max(int(np.exp(rng.uniform(np.log(256), np.log(4_000_000)))) // scale, 1)
        ks, vs = m.key_size, m.value_size
        if kind == 1 and clip:
            cap = m.capacity()
            if level[ti] + n <= cap and level[ti] + n > 0.95 * cap:
                # fits, but would fill the table past 95%: clipped (see docstring)
                n = int(0.95 * cap) - level[ti]
                clipped += 1
                if n < 1:
                    n = cap  # an oversized insert instead: TableFull
        if kind == 1:
            if level[ti] + n <= m.capacity():
                level[ti] += n
        if kind == 1:
            k = torch.randint(0, 256, (n, ks), dtype=torch.uint8, device=dev, generator=g)
            v = torch.randint(0, 256, (n, vs), dtype=torch.uint8, device=dev, generator=g)
        else:
            kn = known[ti]
            half = n // 2
            idx = torch.randint(0, len(kn), (half,), device=dev, generator=g)
            k = torch.cat([kn[idx], torch.randint(0, 256, (n - half, ks), dtype=torch.uint8, device=dev, generator=g)])
            v = None
        ops.append((ti, kind, n, k, v))
        for arm in range(2):
            outs[arm].append((torch.empty((n, vs), dtype=torch.uint8, device=dev),
                              torch.empty((n,), dtype=torch.uint8, device=dev)) if kind == 0 else None)
    torch.cuda.synchronize()

    def restore():
        for m, bk in zip(tables, backups):
            m.copy_from(bk, stream)
        stream.synchronize()

    def plain(arm):
        res = []
        for (ti, kind, n, k, v), o in zip(ops, outs[arm]):
            m = tables[ti]
            if kind == 0:
                m.bulk_get_device(k, n, o[0], o[1], stream)
                res.append((0, 0))
            elif kind == 1:
                try:
                    res.append((m.bulk_insert_device(k, v, n, stream), 0))
                except F.TableFull:
                    res.append((0, 5))
            else:
                res.append((m.bulk_remove_device(k, n, stream), 0))
        return res

    Ev = torch.cuda.Event
    times = []
    for rep in range(warmup + steps):
        restore()
        a, b = Ev(enable_timing=True), Ev(enable_timing=True)
        a.record(stream)
        res_plain = plain(0)
        b.record(stream)
        stream.synchronize()
        if rep >= warmup:
            times.append(a.elapsed_time(b))
    plain_ms = statistics.median(times)
    probe_plain = [m.bulk_get(np.asarray(kn[:4096].cpu()))[0] for m, kn in zip(tables, known)]

    bops = [F.BatchOp(kind, tables[ti], n, k, v, o[0] if o else None, o[1] if o else None)
            for (ti, kind, n, k, v), o in zip(ops, outs[1])]
    restore()  # the batch is planned from the tables' counts at creation: the start state
    batch = F.FlashMapBatch(bops)
    restore()
    batch.run(stream)  # eager run: records each wave's grid rounds for the capture
    res_eager = batch.wait()
    restore()
    batch.capture(stream)
    times = []
    l0 = native.launch_count()
    for rep in range(warmup + steps):
        restore()
        a, b = Ev(enable_timing=True), Ev(enable_timing=True)
        a.record(stream)
        batch.run(stream)
        b.record(stream)
        res_batch = batch.wait()
        if rep >= warmup:
            times.append(a.elapsed_time(b))
    launches = (native.launch_count() - l0) // (warmup + steps)
    batched_ms = statistics.median(times)
    probe_batch = [m.bulk_get(np.asarray(kn[:4096].cpu()))[0] for m, kn in zip(tables, known)]
    same = res_plain == res_batch == res_eager and all(np.array_equal(x, y) for x, y in zip(probe_plain, probe_batch))
    for (ti, kind, n, k, v), o0, o1 in zip(ops, outs[0], outs[1]):
        if kind == 0:
            same = same and torch.equal(o0[0], o1[0]) and torch.equal(o0[1], o1[1])
    executed = sum(n for (ti, kind, n, k, v), r in zip(ops, res_batch) if r[1] == 0)
    waves = batch.waves
    batch.close()
    for m in tables + backups:
        m.close()
    return {
        "workload": f"{BATCH_OPS} queued ops (40% get / 40% insert / 20% remove, sizes log-uniform "
                    f"256..4M{'/' + str(scale) if scale > 1 else ''}) over {BATCH_TABLES} tables (capacities "
                    "log-uniform 2^14..2^24, u64->u64 and [u8;32]->[u8;128] alternating, loads 0.5..0.9), seed 5",
        "keys_executed": executed, "rejected_table_full": sum(1 for r in res_batch if r[1] == 5),
        "inserts_clipped_at_load_0_95": clipped,
        "plain_ms": round(plain_ms, 3), "batched_ms": round(batched_ms, 3),
        "plain_mops": round(executed / plain_ms / 1e3, 3), "batched_mops": round(executed / batched_ms / 1e3, 3),
        "speedup": round(plain_ms / batched_ms, 3), "waves": waves, "cuda_graph": True,
        "gpu_launches_per_batch": int(launches), "identical_results": bool(same),
    }


# ---------------------------------------------------------------------------
# Served form: Poisson request stream against a device-resident table
# ---------------------------------------------------------------------------
SERVE_RATE, SERVE_REQS, SERVE_SAT_REQS = 2000.0, 10000, 2000
SERVE_INSERT_POOL = 16_000_000  # fresh insert keys, taken in turn (later passes update)


def served_leg(torch, F, dev, scale=1):
    """The serving workload: FlashMap<[u8;32],[u8;128]> with_capacity(50M)
    (2^26 slots) prefilled with 30M random entries; requests arrive as a
    Poisson stream at 2,000/s, each insert / get / remove with probability
    0.3 / 0.6 / 0.1 and a size log-uniform in 64..1M keys, get and remove keys
    80% present (Zipf s=0.9 over a 4M-key sample of the present keys); 20 GB
    staging budget (admitted against free HBM).  10,000 requests (five seconds
    of arrivals) are served in real time with continuous batching and, from
    the same start state (a device copy), by the plain one-call-per-request
    server through AsyncFlashMap; then the first 2,000 requests arrive all at
    once (saturation) for both, which gives each form's throughput.  Request
    inputs are slices of pinned host pools (inserts: a pool of 16M fresh keys
    taken in turn, so later passes update; gets/removes: the skewed mix); get
    results land in one shared pinned buffer (timing only; the results
    compared between the forms are the per-request counts and statuses)."""
    from flash_map.serve import AsyncPlainServer, FlashMapServer, Request, latency_summary

    # earlier legs' buffers and the allocator's cached blocks go first: under
    # memory pressure one staging allocation can stall the host for 100 ms
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    rng = np.random.default_rng(6)
    g = torch.Generator(device=dev)
    g.manual_seed(6)
    cap_req, prefill = 50_000_000 // scale, 30_000_000 // scale
    m = F.FlashMap(cap_req, KB, VB, F.HashStrategy.Identity, dev.index or 0)
    pk = torch.randint(0, 256, (prefill, KB), dtype=torch.uint8, device=dev, generator=g)
    pv = torch.randint(0, 256, (prefill, VB), dtype=torch.uint8, device=dev, generator=g)
    for b in range(0, prefill, 4_000_000):
        n = min(4_000_000, prefill - b)
        m.bulk_insert_device(pk[b:b + n], pv[b:b + n], n)
    backup = F.FlashMap(cap_req, KB, VB, F.HashStrategy.Identity, dev.index or 0)
    backup.copy_from(m)
    sample = pk[: min(4_000_000, prefill)].cpu().numpy()
    del pk, pv
    n_req = SERVE_REQS
    kinds = rng.choice([1, 0, 2], size=n_req, p=[0.3, 0.6, 0.1])
    sizes = np.exp(rng.uniform(np.log(64), np.log(1_000_000 // scale), n_req)).astype(np.int64)
    arrivals = np.cumsum(rng.exponential(1.0 / SERVE_RATE, n_req))
    pool_i = SERVE_INSERT_POOL // scale
    ins_k = torch.randint(0, 256, (pool_i, KB), dtype=torch.uint8).pin_memory().numpy()
    ins_v = torch.randint(0, 256, (pool_i, VB), dtype=torch.uint8).pin_memory().numpy()
    # lookup pool: 80% present with Zipf(0.9) ranks (inverse CDF of r^-0.9), 20% fresh
    pool_n = 24_000_000 // scale
    ranks = np.minimum((rng.random(pool_n) ** 10 * len(sample)).astype(np.int64), len(sample) - 1)
    look = sample[ranks]
    fresh = rng.random(pool_n) < 0.2
    look[fresh] = rng.integers(0, 256, (int(fresh.sum()), KB), dtype=np.uint8)
    look = torch.from_numpy(look).pin_memory().numpy()
    out_v = torch.empty((1_000_000 // scale + 1, VB), dtype=torch.uint8).pin_memory()
    out_f = torch.empty((1_000_000 // scale + 1,), dtype=torch.uint8).pin_memory()

    def requests(count, at_once):
        reqs, io, lo = [], 0, 0
        for i in range(count):
            n = int(sizes[i])
            t = 0.0 if at_once else float(arrivals[i])
            if kinds[i] == 1:
                if io + n > pool_i:
                    io = 0
                reqs.append(Request(1, ins_k[io:io + n], ins_v[io:io + n], t))
                io += n
            else:
                if lo + n > pool_n:
                    lo = 0
                reqs.append(Request(int(kinds[i]), look[lo:lo + n], None, t))
                lo += n
        return reqs

    def quiet(serve, reqs, realtime):
        # no garbage collection while requests are timed: freeing another
        # leg's pinned buffers can stall the host for a long time
        gc.collect()
        torch.cuda.synchronize()
        gc.disable()
        try:
            return serve(reqs, realtime=realtime)
        finally:
            gc.enable()

    def restore():
        m.copy_from(backup)
        torch.cuda.synchronize()
        gc.collect()

    torch.cuda.synchronize()
    out = {"workload": f"{n_req} requests, Poisson {SERVE_RATE:.0f}/s, insert/get/remove 0.3/0.6/0.1, sizes "
                       f"log-uniform 64..{1_000_000 // scale}, 80% present Zipf(0.9) on get/remove, table "
                       f"with_capacity({cap_req}) prefilled with {prefill}, 20 GB staging budget against free "
                       f"HBM; saturation: the first {SERVE_SAT_REQS} requests all at t=0",
           "keys": int(sizes.sum()), "keys_saturated": int(sizes[:SERVE_SAT_REQS].sum())}
    srv = FlashMapServer(m, budget=20 << 30, out_pool=lambda n, v: (out_v[:n], out_f[:n]))
    out["staging_bytes"] = srv.staging_bytes
    srv.warmup()  # first-use costs outside the timing (the plain path's kernels ran in earlier legs)
    runs = {}
    for name, count, at_once in (("realtime", n_req, False), ("saturated", SERVE_SAT_REQS, True)):
        restore()
        srv.batches = 0
        rs = requests(count, at_once)
        wall = quiet(srv.serve, rs, not at_once)
        keys = int(sizes[:count].sum())
        served = dict(latency_summary(rs), mops=round(keys / wall / 1e6, 3), wall_s=round(wall, 3),
                      batches=srv.batches, mean_requests_per_batch=round(count / max(srv.batches, 1), 2))
        runs[name] = (rs, served)
    del srv  # its staging buffer goes before the plain server runs
    gc.collect()
    torch.cuda.empty_cache()
    plain = AsyncPlainServer(m, out_pool=lambda n, v: (out_v[:n].numpy(), out_f[:n].numpy()))
    for name, count, at_once in (("realtime", n_req, False), ("saturated", SERVE_SAT_REQS, True)):
        restore()
        rp = requests(count, at_once)
        wall_p = quiet(plain.serve, rp, not at_once)
        keys = int(sizes[:count].sum())
        rs, served = runs[name]
        out[name] = {
            "served": served,
            "plain_async": dict(latency_summary(rp), mops=round(keys / wall_p / 1e6, 3), wall_s=round(wall_p, 3)),
            "served_vs_plain_mops": round(served["mops"] / (keys / wall_p / 1e6), 3),
            "identical_results": all((a.result, a.status) == (b.result, b.status) for a, b in zip(rs, rp)),
        }
    m.close()
    backup.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-as-written", action="store_true", help="skip the load-0.477 variant")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-form workload")
    ap.add_argument("--no-served", action="store_true", help="skip the served-form workload")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default lookup kernel configuration")
    ap.add_argument("--no-oracle-check", action="store_true",
                    help="skip the oracle replay of the step (part of the CPU-baseline leg)")
    ap.add_argument("--nvtx", action="store_true",
                    help="mark one insert call and the bulk_get of the kernel-timing step with NVTX ranges")
    ap.add_argument("--scale", type=int, default=1,
                    help="divide the table and batch counts by this power of two (same call size and load "
                         "factors; for profiling captures on a small case)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    main_w, alt_w = LOAD08, AS_WRITTEN
    if args.scale > 1:
        main_w, alt_w = main_w.scaled(args.scale), alt_w.scaled(args.scale)
    if args.impl == "reference":
        return reference_arm(args, main_w)

    import torch

    import flash_map as F
    from flash_map import _native

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    if not args.no_autotune:
        _native.autotune(local)  # lookup kernel configuration per record shape and load
    stream = torch.cuda.current_stream(dev)
    run = DeviceRun(torch, F, dev, stream, main_w, local)
    with Clocks(local) as clk:  # sampled from the warm-up on, through the timed steps
        for _ in range(args.warmup):
            run.step()
        torch.cuda.synchronize()
        run.check()  # correctness guard on the timed workload (not a parity test)
        t = run.timed(args.steps, barrier, _native)
    total_ms = max_over_ranks(t["total_ms"], dist, dev)
    ms_step = total_ms / args.steps
    value = main_w.ops * world / (ms_step / 1e3) / 1e6
    kt = run.kernel_pass(args.nvtx)
    check = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.no_oracle_check:
        check = oracle_replay_check(run)
    e2e = None if args.no_e2e else run.e2e(args.steps, barrier, dist, world)

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mops/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded uniform random bytes)",
        "config": dict(main_w.desc(), parallelism=f"replicas x{world}" if world > 1 else "single GPU"),
        "ops": run.ops(t),
        "gpu_launches": int(t["launches"]),
        "lookup_config": {"lanes_per_query_and_blocks_per_sm": _native.tuned_get_config(KB, VB, 0.8),
                          "autotuned": not args.no_autotune},
        "kernels": kernel_summary(kt, main_w),
    }
    if check:
        line["oracle_check"] = check
    if e2e:
        line["e2e"] = e2e
    clk_sum = clk.summary()
    if clk_sum:
        line["clocks"] = clk_sum
    run.m.close()
    del run
    torch.cuda.empty_cache()

    if not args.no_as_written:
        alt = DeviceRun(torch, F, dev, stream, alt_w, local)
        for _ in range(args.warmup):
            alt.step()
        torch.cuda.synchronize()
        alt.check()
        ta = alt.timed(args.steps, barrier, _native)
        line["as_written"] = {"config": alt_w.desc(),
                              "value": round(alt_w.ops * world / (ta["total_ms"] / args.steps / 1e3) / 1e6, 3),
                              "ms_per_step": round(ta["total_ms"] / args.steps, 4), "ops": alt.ops(ta)}
        alt.m.close()
        del alt

    if not args.no_batched:
        line["batched"] = batched_leg(torch, F, _native, dev, max(1, min(args.steps, 3)), 1, args.scale)
        line["batched"]["clipped_variant"] = {
            k: v for k, v in batched_leg(torch, F, _native, dev, 1, 1, args.scale, clip=True).items()
            if k in ("keys_executed", "rejected_table_full", "inserts_clipped_at_load_0_95", "plain_ms",
                     "batched_ms", "plain_mops", "batched_mops", "speedup", "gpu_launches_per_batch",
                     "identical_results")}
        line["batched"]["autotuned_get"] = {"u64": _native.tuned_get_config(8, 8, 0.7),
                                            "account": _native.tuned_get_config(KB, VB, 0.7)}

    if not args.no_served:
        line["served"] = served_leg(torch, F, dev, args.scale)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, bpo = cpu_baseline_leg(main_w)
        line["cpu_baseline"] = cb
        peak, kind = read_peak()
        line["roofline"] = roofline_for(
            kt, INSERT_KERNELS, main_w.pairs, bpo["insert"], peak, kind,
            "bulk_insert kernel set (k_dx_find, k_dx_flow, k_dx_exec, k_dx_warp, every call of the step; the step's "
            "largest device-time share)", NCU_TRAFFIC_PER_OP["insert"])
        line["roofline_get"] = roofline_for(
            kt, ("k_get",), main_w.gets, bpo["get"], peak, kind, get_kernel_label(),
            NCU_TRAFFIC_PER_OP["get"])
        line["roofline_remove"] = roofline_for(
            kt, REMOVE_KERNELS, main_w.removes, bpo["remove"], peak, kind, "bulk_remove kernel set",
            NCU_TRAFFIC_PER_OP["remove"])
        line["algorithmic_bytes_per_op"] = {k: round(v, 2) for k, v in bpo.items()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
