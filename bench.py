"""Benchmark: random-walk expander decomposition throughput on one B200 per rank.

Workload: 3D 7-point grid 128^3 (n = 2,097,152 vertices, m = 6,242,304
undirected edges), seed 6582, sweep threshold 0.3, potential threshold 1e-4 -
the plain-method GPU configuration of the reference's benchmark set.  One
step is one whole decomposition: initialise the device state from the CSR and
run rounds until every cluster is certified.  The metric is decomposition
throughput in undirected edges per second (m / step time), summed over ranks.

* value: CSR resident in HBM before the timed region; per step
  pxr_initialize_device + pxr_decompose; CUDA events on the library's stream;
  L2 flushed (256 MiB write) before every step, outside the events.
* e2e: the public API with host buffers: pxr_initialize from pinned host
  memory (host-to-device copy inside the timed region), pxr_decompose and
  pxr_final_partition (device-to-host copy of the n cluster ids).
* roofline: one extra decomposition with per-phase CUDA events (stream
  driver); the dominant kernel's algorithmic bytes over its summed device time,
  against the measured HBM copy peak.
* cpu_baseline: the reference's own single-threaded CPU decomposition
  (oracle/_ref/ref_cpu, built from the reference sources) on the same graph.

Multi-GPU: the decomposition of one graph does not shard, so every rank runs
its own replica ("scaling": "weak"); the 512-instance batch is split over the
ranks by expected edges instead (each rank decomposes its shard; the job's
edges are the shards' sum, "scaling": "strong").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "decomp edges/s"
UNIT = "edges/s"
SEED, SC, RW = 6582, 0.3, 1e-4
SIDE = 128
L2_FLUSH_BYTES = 256 << 20


WORKLOADS = {
    "grid128": "3D 7-point grid 128^3 (2,097,152 vertices, 6,242,304 edges)",
    "sbm16k": "planted partition n=16,384, 16 blocks, intra degree 12, inter degree 0.5, seed 6582",
    "rmat22": "R-MAT scale 22, edge factor 16, (a,b,c)=(0.57,0.19,0.19), seed 1, built on the GPU",
    "rmat24": "R-MAT scale 24, edge factor 16, (a,b,c)=(0.57,0.19,0.19), seed 1, built on the GPU",
    "regular22": "random 8-regular graph on 2^22 vertices, seed 1 (the no-split case)",
    "batch512": ("512 planted-partition instances in one batched decomposition: n log-uniform in [1e3, 1e6], "
                 "blocks U{2..64}, intra degree U[4, 32], inter degree U[0.1, 2], int64 offsets, built on the GPU"),
}


def load_workload(name, dev=None, rank=0, world=1):
    """(CSRGraph or None, device offsets, device cols, n, m, instance starts or
    None) for a named workload.  The instance batch is split over the ranks
    (this rank's shard); the other workloads are replicated."""
    from parex_b200 import graphs as G
    if name.startswith("rmat"):
        from parex_b200 import gpu_build as B
        off_d, cols_d, n, m = B.rmat(int(name[4:]), 16, seed=1, device=dev.index or 0)
        return None, off_d, cols_d, n, m, None
    if name == "batch512":
        import torch
        from parex_b200 import gpu_build as B
        shard = None if world == 1 else B.shard_instances(B.sbm_batch_params(512, seed=1), world)[rank]
        off_d, cols_d, n, m, starts = B.sbm_batch(512, seed=1, device=dev.index or 0, instances=shard)
        return None, off_d.to(torch.int64), cols_d, n, m, starts
    g = {"grid128": lambda: G.grid3d(SIDE), "sbm16k": lambda: G.sbm_graph(),
         "regular22": lambda: G.random_regular(1 << 22, 8, seed=1)}[name]()
    return g, None, None, g.n, g.m, None



def workload_config(g, extra=None, name="grid128"):
    n, m = (g.n, g.m) if hasattr(g, "n") else g
    cfg = {
        "workload": f"{name}: {WORKLOADS[name]}, seed {SEED}, sc {SC}, rw {RW}",
        "n": n, "m": m, "seed": SEED, "sc_threshold": SC, "rw_threshold": RW,
        "l2": "flushed before every step (256 MiB write)",
        "parallelism": "replicas",
    }
    if extra:
        cfg.update(extra)
    return cfg


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def run_reference_cpu(g, reps: int, warm_graph=None, warmups: int = 0):
    """The reference's single-threaded CPU decomposition (oracle/_ref/ref_cpu)."""
    from parex_b200 import graphs as G
    binary = os.path.join(ROOT, "oracle", "_ref", "ref_cpu")
    with tempfile.TemporaryDirectory() as td:
        if os.path.exists(binary):
            if warm_graph is not None and warmups:
                wp = os.path.join(td, "warm.pxg")
                G.write_pxg(wp, warm_graph)
                subprocess.run([binary, "decomp", wp, str(SEED), str(SC), str(RW), str(warmups), "-"],
                               check=True, capture_output=True, text=True)
            gp = os.path.join(td, "g.pxg")
            G.write_pxg(gp, g)
            out = subprocess.run([binary, "decomp", gp, str(SEED), str(SC), str(RW), str(reps), "-"],
                                 check=True, capture_output=True, text=True).stdout
            runs = [json.loads(l) for l in out.splitlines() if l.startswith("{")]
            secs = [r["ms"] / 1e3 for r in runs]
            return {"kind": "reference", "secs": secs, "clusters": runs[0]["clusters"],
                    "cut_edges": runs[0]["cut_edges"]}
    # the reference binary was not built: time the oracle port of the same algorithm
    from oracle import oracle as O
    secs = []
    for _ in range(reps):
        x0 = O.initial_potentials(g.offsets, SEED)
        orc = O.Oracle(g.offsets, g.cols, O.MODE_REF, SC, RW)
        orc.set_potentials(x0.astype(np.float64))
        t = time.perf_counter()
        orc.decompose()
        secs.append(time.perf_counter() - t)
    return {"kind": "port", "secs": secs}


def reference_arm(args, rank):
    from parex_b200 import graphs as G
    if rank != 0:
        return 0
    g = G.grid3d(SIDE)
    res = run_reference_cpu(g, args.steps, warm_graph=G.grid3d(32), warmups=args.warmup)
    total = sum(res["secs"])
    value = g.m * len(res["secs"]) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(res["secs"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(g, {"runner": "reference CPU decomposition, single thread"}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": res["kind"],
                         "sample": f"{len(res['secs'])} full decompositions of the {SIDE}^3 grid "
                                   f"(the reference code has no threads)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(values, world, device):
    """Each value's maximum over the ranks (every rank gets it): the job's
    time is its slowest replica's."""
    if world == 1:
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def sum_over_ranks(values, world, device):
    """Each value's sum over the ranks (every rank gets it)."""
    if world == 1:
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.tolist()


def job_rate(m, world, steps, ms):
    """Whole-job edges/s: every rank decomposes its own replica of the m-edge
    graph each step, so the job processes m x world x steps edges in ms."""
    return m * world * steps / (ms / 1e3)


def product_arm(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import parex_b200 as P
    from parex_b200 import graphs as G

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    g, off_d, cols_d, n, m, starts = load_workload(args.workload, dev, rank, world)
    sharded = starts is not None and world > 1   # instances split over the ranks, not replicated
    off64 = off_d is not None and off_d.dtype == torch.int64
    stream = torch.cuda.Stream(device=dev)
    if g is not None:
        off_d = torch.from_numpy(g.offsets.view(np.int32)).to(dev)
        cols_d = torch.from_numpy(g.cols.view(np.int32)).to(dev)
        off_h = torch.from_numpy(g.offsets.view(np.int32)).pin_memory()
        cols_h = torch.from_numpy(g.cols.view(np.int32)).pin_memory()
    else:
        off_h = off_d.cpu().pin_memory()
        cols_h = cols_d.cpu().pin_memory()
    off_hn = off_h.numpy().view(np.uint64 if off64 else np.uint32)
    ids_h = torch.empty(n, dtype=torch.int32).pin_memory()   # the final ids land in page-locked memory
    ids_hn = ids_h.numpy()
    cols_hn = cols_h.numpy().view(np.uint32)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)

    model = None
    if args.schedule == "learned":
        from parex_b200 import learn
        model = learn.Model.load()

    def manager(driver):
        dmx = P.CudaDeviceManager(seed=SEED, sc_threshold=SC, rw_threshold=RW, device=local_rank, driver=driver)
        if args.row_plan:
            dmx.set_row_plan(*[int(t) for t in args.row_plan.split(",")])
        if model is not None:
            dmx.set_schedule(P._lib.SCHEDULE_LEARNED, model.weights, model.norm, safety=0.25, max_skip=16)
        return dmx

    dm = manager(P.DRIVER_GRAPH)
    dm.set_stream(stream.cuda_stream)

    def barrier():
        if world > 1:
            dist.barrier()

    def init_device(dmx):
        if starts is not None:
            dmx.initialize_batched_device(n, m, off_d.data_ptr(), off64, cols_d.data_ptr(), starts)
        else:
            dmx.initialize_device(n, m, off_d.data_ptr(), off64, cols_d.data_ptr())

    def init_host(dmx):
        if starts is not None:
            dmx.initialize_batched((off_hn, cols_hn), starts)
        else:
            dmx.initialize((off_hn, cols_hn))

    def device_step():
        init_device(dm)
        return dm.expanderDecomposition()

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            device_step()
        torch.cuda.synchronize(dev)
        launches0 = dm.stats()["kernel_launches"]
        total_ms, rounds = 0.0, 0
        with ClockSampler(local_rank) as clocks:
            for _ in range(args.steps):
                flush.zero_()
                barrier()
                torch.cuda.synchronize(dev)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                rounds = device_step()
                e1.record(stream)
                torch.cuda.synchronize(dev)
                barrier()
                total_ms += e0.elapsed_time(e1)
        launches = dm.stats()["kernel_launches"] - launches0
        fp = dm.getFinalPartition()
        clusters = fp.numClusters
        device_cut = dm.getNumCutEdges()

        # end to end through the public API with host buffers (one untimed
        # step first: the first transfer from the pinned buffers is slower)
        init_host(dm)
        dm.expanderDecomposition()
        dm.getFinalPartition(out=ids_hn)
        e2e_ms = 0.0
        for _ in range(args.steps):
            flush.zero_()
            barrier()
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            init_host(dm)
            dm.expanderDecomposition()
            fp_e2e = dm.getFinalPartition(out=ids_hn)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            barrier()
            e2e_ms += e0.elapsed_time(e1)
        assert fp_e2e.numClusters == clusters

        # per-phase device times with the stream driver (roofline)
        prof = manager(P.DRIVER_STREAM)
        prof.set_stream(stream.cuda_stream)
        init_device(prof)
        prof.set_profiling(True)
        prof.expanderDecomposition()
        phases = prof.phase_stats()
        pst = prof.stats()
        prof_labels_equal = bool(np.array_equal(prof.getFinalPartition().clusterIds, fp.clusterIds))

    total_ms, e2e_ms = max_over_ranks([total_ms, e2e_ms], world, dev)
    # edges per step of the whole job: each replica's m, or the shards' sum
    job_m = int(sum_over_ranks([m], world, dev)[0]) if sharded else m * world

    if rank != 0:
        return 0
    value = job_rate(job_m, 1, args.steps, total_ms)
    e2e_value = job_rate(job_m, 1, args.steps, e2e_ms)
    h2d = (n + 1) * (8 if off64 else 4) + 2 * m * 4
    d2h = n * 4 + 4

    # roofline of the dominant phase among those with algorithmic byte counts;
    # per launch: the sort counts its active digit passes, the walk one launch per round
    peak, peak_kind = measured_peaks()
    by = {p["name"]: p for p in phases}
    walk_bytes = 28 * pst["walk_vertices"] + 4 * pst["walk_slots"] + 4 * pst["walk_gathers"]
    sort_bytes = 24 * pst["sort_items"]
    cands = {"walk": (walk_bytes, max(1, pst["rounds"])), "sort": (sort_bytes, max(1, pst["sort_passes"]))}
    dom = max(cands, key=lambda k: by[k]["ms"])
    alg_total, units = cands[dom]
    ach = alg_total / (by[dom]["ms"] / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        if dom == "sort" and "sort" in tj:
            traffic = tj["sort"]["dram_bytes_per_item_pass"] * pst["sort_items"] / units
        elif dom == "walk" and "walk" in tj:
            traffic = tj["walk"]["dram_over_algorithmic"] * alg_total / units
    total_phase = sum(p["ms"] for p in phases)
    roofline = {
        "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "traffic": traffic,
        "kernel": {"walk": "k_walk (+ warp/CTA long-row kernels)",
                   "sort": "sweep sort: sort_pass_kernel<u64> passes and k_chunk_sort (time includes histogram, plan)"}[dom],
        "algorithmic_bytes_per_launch": alg_total / units, "launches": units,
        "device_ms": by[dom]["ms"], "device_us_per_launch": 1e3 * by[dom]["ms"] / units,
        "traffic_source": "profiles/traffic.json: ncu DRAM bytes of full-size round-1 launches, scaled by items",
        "peak_source": f"{peak_kind} HBM copy peak",
        "phase_share": {p["name"]: round(p["ms"] / total_phase, 4) for p in phases if p["ms"] > 0},
        "prof_run_identical": prof_labels_equal,
    }

    cpu = None
    if world == 1 and not args.no_cpu_baseline and args.workload in ("grid128", "sbm16k"):
        res = run_reference_cpu(g, 1)
        cpu = {"value": m / res["secs"][0], "unit": UNIT, "cores": 1, "kind": res["kind"],
               "sample": f"one full decomposition of {args.workload} ({res['secs'][0]:.1f} s, single thread)"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if sharded else "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config((n, m), {"driver": "cuda graph, device-driven round loop", "rounds": rounds,
                                           "clusters": clusters, "cut_edges_device": device_cut,
                                           "sweep_schedule": args.schedule, "row_plan": dm.row_plan(),
                                           "instances": None if starts is None else int(len(starts) - 1),
                                           "parallelism": (f"{world} ranks, instances split by expected edges"
                                                           if sharded else "replicas"),
                                           "job_edges_per_step": job_m},
                                  args.workload),
        "clocks": clocks.summary(),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms / args.steps},
        "gpu_launches": launches,
        "roofline": roofline,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="grid128", choices=sorted(WORKLOADS))
    ap.add_argument("--schedule", default="plain", choices=["plain", "learned"])
    ap.add_argument("--row-plan", default=None, help="force lanes_per_row,light_max,wide_max (default: autotuned)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        return product_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
