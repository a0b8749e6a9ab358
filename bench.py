#!/usr/bin/env python
"""FlashMap B200 backend benchmark: prints ONE JSON line.

Workload (one "step"), the account shape FlashMap<[u8;32],[u8;128]>:
  with_capacity(10,000,000) (2^24 slots), clear, 8,000,000 distinct pairs
  inserted as 80 bulk_insert calls of 100,000, one bulk_get of 8,000,000 keys
  (50% present, 50% fresh random keys, shuffled), one bulk_remove of a random
  800,000 present keys.  Keys and values are seeded uniform random bytes.

  value  = ops of the step (16.8M) x ranks / device time (CUDA events, max
           over ranks), inputs resident in HBM, device-pointer API.
  e2e    = the same step through the host API (fm_bulk_insert/get/remove with
           pinned host buffers: H2D of inputs and D2H of results inside).
  roofline: the bulk_get kernel, algorithmic bytes per query (counted by the
           CPU oracle on the same workload at 1/16 scale) x queries / launch
           time, against MEASURED_PEAKS.json hbm_gbs.
  cpu_baseline: the sequential CPU oracle on the 1/16-scale sample.

`--impl reference` times the reference's CPU algorithm (multithreaded CAS
restatement of src/rayon_cpu.rs, all host threads) on the 1/16-scale sample.
Multi-GPU (torchrun): every rank runs an independent table (replicas, weak
scaling); no collective on the data path.
"""
import argparse
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
CAP_REQ = 10_000_000
N_PAIRS = 8_000_000
CALL = 100_000
N_GET = 8_000_000
N_REM = 800_000
KB, VB = 32, 128
SAMPLE_DIV = 16  # CPU sample: same load factors and call size at 1/16 scale


def workload_desc():
    return {
        "workload": "account shape [u8;32]->[u8;128], with_capacity(10M)=2^24 slots: clear, 8M pairs as "
                    "80 bulk_insert calls of 100K, bulk_get of 8M (50% hits), bulk_remove of 800K present",
        "capacity": 1 << 24,
        "pairs": N_PAIRS,
        "insert_calls": f"80x{CALL}",
        "gets": N_GET,
        "get_hit_rate": 0.5,
        "removes": N_REM,
        "load_after_insert": round(N_PAIRS / (1 << 24), 4),
        "l2": "inputs larger than L2 (table 2.9 GB, 256 MB of get keys per call); no flush",
        "api": "device-pointer API (fm_*_device), stream-ordered",
    }


def read_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU sample (oracle / reference restatement): 1/16 scale, same load factors
# ---------------------------------------------------------------------------
def cpu_sample_inputs(seed=3):
    rng = np.random.default_rng(seed)
    n = N_PAIRS // SAMPLE_DIV
    keys = rng.integers(0, 256, (n, KB), dtype=np.uint8)
    vals = rng.integers(0, 256, (n, VB), dtype=np.uint8)
    ng = N_GET // SAMPLE_DIV
    q = np.concatenate([keys[rng.choice(n, ng // 2, replace=False)],
                        rng.integers(0, 256, (ng - ng // 2, KB), dtype=np.uint8)])
    q = q[rng.permutation(len(q))]
    rem = keys[rng.choice(n, N_REM // SAMPLE_DIV, replace=False)]
    return keys, vals, q, rem


def cpu_step(O, inp, threads=None, traffic=False):
    """One sample step on the oracle (threads=None: sequential) -> seconds."""
    keys, vals, q, rem = inp
    m = O.OracleMap((1 << 24) // SAMPLE_DIV, KB, VB)
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


def sample_ops():
    return (N_PAIRS + N_GET + N_REM) // SAMPLE_DIV


def bytes_per_op(tr):
    out = {}
    for k, v in tr.items():
        b = (v["table_sectors_read"] + v["table_sectors_written"]) * 32 + v["stream_bytes_in"] + v["stream_bytes_out"]
        out[k] = b / max(v["ops"], 1)
    return out


def cpu_baseline_leg():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    inp = cpu_sample_inputs()
    reps, total = 0, 0.0
    while reps < 64 and (total < 8.0 or reps < 2):  # ~10 s of CPU work
        dt, _ = cpu_step(O, inp)
        total += dt
        reps += 1
    _, tr = cpu_step(O, inp, traffic=True)
    return {
        "value": round(sample_ops() * reps / total / 1e6, 3),
        "unit": "Mops/s",
        "cores": 1,
        "kind": "port",
        "sample": f"the same step at 1/{SAMPLE_DIV} scale (2^20 slots, 500K pairs in 5x100K inserts, 500K gets, "
                  f"50K removes; same load factors), sequential C oracle, {reps} reps in {total:.1f} s",
    }, bytes_per_op(tr)


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    threads = os.cpu_count() or 1
    inp = cpu_sample_inputs()
    for _ in range(args.warmup):
        cpu_step(O, inp, threads=threads)
    times = [cpu_step(O, inp, threads=threads)[0] for _ in range(args.steps)]
    total = sum(times)
    v = sample_ops() * len(times) / total / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "Mops/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total / len(times) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": dict(workload_desc(), parallelism="host threads"),
        "cpu_baseline": {"value": round(v, 3), "unit": "Mops/s", "cores": threads, "kind": "port",
                         "sample": f"the step at 1/{SAMPLE_DIV} scale; multithreaded CAS restatement of "
                                   "src/rayon_cpu.rs (the reference's Rust crate cannot be built here)"},
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


def gpu_inputs(torch, dev, seed=3):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    keys = torch.randint(0, 256, (N_PAIRS, KB), dtype=torch.uint8, device=dev, generator=g)
    vals = torch.randint(0, 256, (N_PAIRS, VB), dtype=torch.uint8, device=dev, generator=g)
    hit = torch.randperm(N_PAIRS, device=dev, generator=g)[: N_GET // 2]
    fresh = torch.randint(0, 256, (N_GET - N_GET // 2, KB), dtype=torch.uint8, device=dev, generator=g)
    q = torch.cat([keys[hit], fresh])
    q = q[torch.randperm(N_GET, device=dev, generator=g)].contiguous()
    rem = keys[torch.randperm(N_PAIRS, device=dev, generator=g)[:N_REM]].contiguous()
    return keys, vals, q, rem


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--scale", type=int, default=1,
                    help="divide the table and batch counts by this power of two (same call size and load "
                         "factors; for profiling captures on a small case)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.scale > 1:
        global CAP_REQ, N_PAIRS, N_GET, N_REM
        CAP_REQ //= args.scale
        N_PAIRS //= args.scale
        N_GET //= args.scale
        N_REM //= args.scale
    if args.impl == "reference":
        return reference_arm(args)

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

    keys, vals, q, rem = gpu_inputs(torch, dev)
    out_v = torch.empty((N_GET, VB), dtype=torch.uint8, device=dev)
    out_f = torch.empty((N_GET,), dtype=torch.uint8, device=dev)
    m = F.FlashMap(CAP_REQ, KB, VB, F.HashStrategy.Identity, local)
    stream = torch.cuda.current_stream(dev)
    Ev = torch.cuda.Event

    def step(ev=None):
        m.clear()
        for b in range(0, N_PAIRS, CALL):
            m.bulk_insert_device(keys[b:b + CALL], vals[b:b + CALL], CALL, stream)
        if ev:
            ev[0].record(stream)
        m.bulk_get_device(q, N_GET, out_v, out_f, stream)
        if ev:
            ev[1].record(stream)
        m.bulk_remove_device(rem, N_REM, stream)

    phase = [(Ev(enable_timing=True), Ev(enable_timing=True)) for _ in range(args.steps)]
    starts = [Ev(enable_timing=True) for _ in range(args.steps)]
    ends = [Ev(enable_timing=True) for _ in range(args.steps)]
    t_all0, t_all1 = Ev(enable_timing=True), Ev(enable_timing=True)
    with Clocks(local) as clk:  # sampled from the warm-up on, through the timed steps
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        # correctness guard on the timed workload (not a parity test)
        assert m.len() == N_PAIRS - N_REM, m.len()
        assert int(out_f.sum().item()) == N_GET // 2
        l0 = _native.launch_count()
        barrier()
        torch.cuda.synchronize()
        t_all0.record(stream)
        for k in range(args.steps):
            starts[k].record(stream)
            step(phase[k])
            ends[k].record(stream)
        t_all1.record(stream)
        torch.cuda.synchronize()
        barrier()
    launches = _native.launch_count() - l0
    total_ms = t_all0.elapsed_time(t_all1)
    ins_ms = statistics.median(starts[k].elapsed_time(phase[k][0]) for k in range(args.steps))
    get_ms = statistics.median(phase[k][0].elapsed_time(phase[k][1]) for k in range(args.steps))
    rem_ms = statistics.median(phase[k][1].elapsed_time(ends[k]) for k in range(args.steps))
    if dist is not None:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ops_step = N_PAIRS + N_GET + N_REM
    ms_step = total_ms / args.steps
    value = ops_step * world / (ms_step / 1e3) / 1e6

    # ---- end to end through the host API (pinned host buffers) ----------
    def run_e2e():
        hk = keys.cpu().pin_memory().numpy()
        hv = vals.cpu().pin_memory().numpy()
        hq = q.cpu().pin_memory().numpy()
        hr = rem.cpu().pin_memory().numpy()
        ho = torch.empty((N_GET, VB), dtype=torch.uint8).pin_memory().numpy()
        hf = torch.empty((N_GET,), dtype=torch.uint8).pin_memory().numpy()

        def step_host():
            m.clear()
            for b in range(0, N_PAIRS, CALL):
                m.bulk_insert(hk[b:b + CALL], hv[b:b + CALL])
            m.bulk_get(hq, out_values=ho, out_found=hf)
            m.bulk_remove(hr)

        for _ in range(1):
            step_host()
        assert int(hf.sum()) == N_GET // 2
        e2e_steps = max(1, min(args.steps, 3))
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            step_host()
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        if dist is not None:
            t = torch.tensor([e2e_s], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": round(ops_step * world / e2e_s / 1e6, 3), "unit": "Mops/s",
               "h2d_bytes_per_step": N_PAIRS * (KB + VB) + N_GET * KB + N_REM * KB,
               "d2h_bytes_per_step": N_GET * (VB + 1) + 8 * (N_PAIRS // CALL + 1),
               "ms_per_step": round(e2e_s * 1e3, 3)}
        return e2e

    e2e = None if args.no_e2e else run_e2e()

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mops/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded uniform random bytes)",
        "config": dict(workload_desc(), parallelism=f"replicas x{world}" if world > 1 else "single GPU"),
        "ops": {"insert_mops": round(N_PAIRS / ins_ms / 1e3, 3), "get_mops": round(N_GET / get_ms / 1e3, 3),
                "remove_mops": round(N_REM / rem_ms / 1e3, 3), "insert_ms": round(ins_ms, 3),
                "get_ms": round(get_ms, 3), "remove_ms": round(rem_ms, 3)},
        "gpu_launches": int(launches),
    }
    if e2e:
        line["e2e"] = e2e
    clk_sum = clk.summary()
    if clk_sum:
        line["clocks"] = clk_sum
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, bpo = cpu_baseline_leg()
        line["cpu_baseline"] = cb
        peak, kind = read_peak()
        achieved = bpo["get"] * N_GET / (get_ms / 1e3) / 1e9
        line["roofline"] = {"kernel": "k_get<32,128,8> (bulk_get, one launch of 8M queries)", "bound": "hbm",
                            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                            "frac": round(achieved / peak, 4), "peak_kind": kind,
                            "algorithmic_bytes_per_query": round(bpo["get"], 2), "traffic": None}
        line["algorithmic_bytes_per_op"] = {k: round(v, 2) for k, v in bpo.items()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    m.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
