"""Benchmark: random-walk expander decomposition throughput on one B200 per rank.

Default workload: R-MAT scale 24 (16,777,216 vertices, edge factor 16,
(a,b,c) = (0.57,0.19,0.19), symmetrised, deduplicated, no self-loops: about
260 M undirected edges), graph seed 1, walk seed 6582, sweep threshold 0.3,
potential threshold 1e-4 - the learned-schedule configuration of the
reference's benchmark set.  One step is one whole decomposition: initialise
the device state from the CSR and run rounds until every cluster is
certified.  The metric is decomposition throughput in undirected edges per
second (m / step time) of the batched+learned form, measured in the same run
as the plain form on the same graph; the line carries both, their ratio, the
cut edges of both and whether every cluster of both passed the certificate
check (parex_b200/certificate.py).

* value: CSR resident in HBM before the timed region; per step
  pxr_initialize_device + pxr_decompose; CUDA events on the library's stream;
  L2 flushed (256 MiB write) before every step, outside the events.
* e2e: the public API with host buffers, learned form: pxr_initialize from
  pinned host memory (host-to-device copy inside the timed region),
  pxr_decompose and pxr_final_partition (device-to-host copy of the n ids).
* roofline: one extra decomposition with per-phase CUDA events (stream
  driver): the walk step's algorithmic bytes per launch over its mean device
  time per launch, against the measured HBM copy peak; every phase with
  algorithmic byte counts gets its own fraction.
* cpu_baseline: the reference's own single-threaded CPU decomposition
  (oracle/_ref/ref_cpu, built from the reference sources) on a bounded
  sample (see cpu_sample()).

Multi-GPU: the decomposition of one graph does not shard, so every rank runs
its own replica ("scaling": "weak"); the 512-instance batch is split over the
ranks by expected edges instead (each rank decomposes its shard; the job's
edges are the shards' sum, "scaling": "strong").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload NAME] [--schedule both|plain|learned]
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
WALK_SEED, GRAPH_SEED, SC, RW = 6582, 1, 0.3, 1e-4
L2_FLUSH_BYTES = 256 << 20
SAFETY, MAX_SKIP, CUT_GATE, DUE_PERIOD = 0.25, 32, 0.01, 8


WORKLOADS = {
    "rmat24": "R-MAT scale 24, edge factor 16, (a,b,c)=(0.57,0.19,0.19), built on the GPU",
    "rmat22": "R-MAT scale 22, edge factor 16, (a,b,c)=(0.57,0.19,0.19), built on the GPU",
    "regular22": "random 8-regular graph on 2^22 vertices (the no-split case)",
    "grid128": "3D 7-point grid 128^3 (2,097,152 vertices, 6,242,304 edges)",
    "sbm16k": "planted partition n=16,384, 16 blocks, intra degree 12, inter degree 0.5",
    "batch512": ("512 planted-partition instances in one batched decomposition: n log-uniform in [1e3, 1e6], "
                 "blocks U{2..64}, intra degree U[4, 32], inter degree U[0.1, 2], int64 offsets, built on the GPU"),
}
GRAPH_SEEDS = {"rmat24": 1, "rmat22": 1, "regular22": 1, "grid128": None, "sbm16k": 6582, "batch512": 1}


def load_workload(name, dev=None, rank=0, world=1):
    """(CSRGraph or None, device offsets, device cols, n, m, instance starts or
    None, shard instances or None) for a named workload.  The instance batch
    is split over the ranks (this rank's shard); the other workloads are
    replicated."""
    from parex_b200 import graphs as G
    if name.startswith("rmat"):
        from parex_b200 import gpu_build as B
        off_d, cols_d, n, m = B.rmat(int(name[4:]), 16, seed=GRAPH_SEEDS[name], device=dev.index or 0)
        return None, off_d, cols_d, n, m, None, None
    if name == "batch512":
        import torch
        from parex_b200 import gpu_build as B
        shard = None if world == 1 else B.shard_instances(B.sbm_batch_params(512, seed=1), world)[rank]
        off_d, cols_d, n, m, starts = B.sbm_batch(512, seed=1, device=dev.index or 0, instances=shard)
        return None, off_d.to(torch.int64), cols_d, n, m, starts, shard
    g = {"grid128": lambda: G.grid3d(128), "sbm16k": lambda: G.sbm_graph(),
         "regular22": lambda: G.random_regular(1 << 22, 8, seed=1)}[name]()
    return g, None, None, g.n, g.m, None, None


def workload_config(n, m, name, extra=None):
    cfg = {
        "workload": f"{name}: {WORKLOADS[name]}, graph seed {GRAPH_SEEDS[name]}, walk seed {WALK_SEED}, "
                    f"sc {SC}, rw {RW}",
        "n": n, "m": m, "graph_seed": GRAPH_SEEDS[name], "walk_seed": WALK_SEED, "sc_threshold": SC,
        "rw_threshold": RW, "l2": "flushed before every step (256 MiB write)", "parallelism": "replicas",
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


def host_cpu():
    """CPU model and core count of this host."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


# ----------------------------------------------------------------------------
# reference CPU decomposition (oracle/_ref/ref_cpu)


def _write_pxg(path, offsets, cols):
    from parex_b200 import graphs as G
    n = offsets.shape[0] - 1
    off = offsets.astype(np.uint32) if cols.shape[0] < 2**32 else offsets.astype(np.uint64)
    G.write_pxg(path, G.CSRGraph(off, cols.astype(np.uint32, copy=False), "bench"))


def run_reference_cpu(offsets, cols, reps: int, warm=None, warmups: int = 0, timeout=None):
    """The reference's single-threaded CPU decomposition (oracle/_ref/ref_cpu)
    of the CSR (offsets, cols), reps times; warm = (offsets, cols) of a graph
    decomposed warmups times first."""
    binary = os.path.join(ROOT, "oracle", "_ref", "ref_cpu")
    with tempfile.TemporaryDirectory() as td:
        if os.path.exists(binary):
            if warm is not None and warmups:
                wp = os.path.join(td, "warm.pxg")
                _write_pxg(wp, *warm)
                subprocess.run([binary, "decomp", wp, str(WALK_SEED), str(SC), str(RW), str(warmups), "-"],
                               check=True, capture_output=True, text=True, timeout=timeout)
            gp = os.path.join(td, "g.pxg")
            _write_pxg(gp, offsets, cols)
            out = subprocess.run([binary, "decomp", gp, str(WALK_SEED), str(SC), str(RW), str(reps), "-"],
                                 check=True, capture_output=True, text=True, timeout=timeout).stdout
            runs = [json.loads(l) for l in out.splitlines() if l.startswith("{")]
            return {"kind": "reference", "secs": [r["ms"] / 1e3 for r in runs], "clusters": runs[0]["clusters"],
                    "cut_edges": runs[0]["cut_edges"]}
    # the reference binary was not built: time the oracle port of the same algorithm
    from oracle import oracle as O
    secs = []
    for _ in range(reps):
        x0 = O.initial_potentials(offsets, WALK_SEED)
        orc = O.Oracle(offsets, cols, O.MODE_REF, SC, RW)
        orc.set_potentials(x0.astype(np.float64))
        t = time.perf_counter()
        orc.decompose()
        secs.append(time.perf_counter() - t)
    return {"kind": "port", "secs": secs}


def run_reference_gpu(offsets, cols, off64, timeout=900):
    """The reference's own GPU decomposition of the same graph on the same
    B200 (oracle/_ref/ref_gpu, built from the reference's cuda/ sources with
    its own flags): CudaDeviceManager::expanderDecomposition timed with CUDA
    events, one run, for context beside the product's numbers."""
    binary = os.path.join(ROOT, "oracle", "_ref", "ref_gpu")
    if not os.path.exists(binary):
        return {"unavailable": "oracle/_ref/ref_gpu not built"}
    if off64:
        return {"unavailable": "the reference's EdgeIx is 32-bit"}
    with tempfile.TemporaryDirectory() as td:
        gp = os.path.join(td, "g.pxg")
        _write_pxg(gp, np.asarray(offsets), np.asarray(cols))
        try:
            out = subprocess.run([binary, "time", gp, str(WALK_SEED), str(SC), str(RW), "1"], capture_output=True,
                                 text=True, timeout=timeout).stdout
        except subprocess.TimeoutExpired:
            return {"unavailable": f"did not finish within {timeout} s"}
    runs = [json.loads(l) for l in out.splitlines() if l.startswith("{")]
    if not runs:
        return {"unavailable": "no timing printed"}
    r = runs[0]
    return {"loop_ms": r["loop_ms"], "e2e_ms": r["e2e_ms"], "clusters": r["num_clusters_fp"],
            "edges_per_s": r["m"] / (r["loop_ms"] / 1e3)}


def host_graph(name):
    """The workload's CSR on the host, built without the product library
    (the R-MAT graphs by the oracle's C builder, the same edges as the device
    generator); None for the device-built instance batch."""
    from parex_b200 import graphs as G
    if name.startswith("rmat"):
        from oracle import oracle as O
        return O.rmat_csr(int(name[4:]), 16, seed=GRAPH_SEEDS[name])
    if name == "batch512":
        return None
    g = {"grid128": lambda: G.grid3d(128), "sbm16k": lambda: G.sbm_graph(),
         "regular22": lambda: G.random_regular(1 << 22, 8, seed=1)}[name]()
    return g.offsets, g.cols


def cpu_sample(name):
    """A bounded sample of the workload for the product line's CPU baseline
    (tens of seconds of the reference's single-threaded CPU decomposition):
    the whole graph where that fits, else the same R-MAT generator at scale
    20 (1/16 of the vertices)."""
    if name in ("grid128", "sbm16k"):
        return host_graph(name), f"one full decomposition of {name}"
    if name.startswith("rmat"):
        from oracle import oracle as O
        return O.rmat_csr(20, 16, seed=GRAPH_SEEDS[name]), \
            "one full decomposition of R-MAT scale 20 (same generator and seed, 1/16 of the vertices)"
    return None, None


def reference_arm(args, rank):
    """The reference's own CPU decomposition on the workload's graph, rank 0
    only.  Where one decomposition takes minutes (R-MAT scale 24: about ten),
    a single decomposition is the whole sample: --steps and --warmup apply to
    the graphs whose decomposition takes seconds."""
    if rank != 0:
        return 0
    name = args.workload
    hg = host_graph(name)
    if hg is None:
        print(json.dumps({"impl": "reference", "unavailable": "the 512-instance batch is built on the GPU only"}))
        return 0
    off, cols = hg
    n, m = off.shape[0] - 1, cols.shape[0] // 2
    long_run = name in ("rmat24", "rmat22", "regular22")
    reps = 1 if long_run else args.steps
    res = run_reference_cpu(off, cols, reps, warm=None if long_run else hg, warmups=0 if long_run else args.warmup)
    total = sum(res["secs"])
    value = m * len(res["secs"]) / total
    sample = (f"{len(res['secs'])} full decomposition(s) of {name} "
              + ("(one decomposition is the whole sample: --steps/--warmup do not apply)" if long_run
                 else f"after {args.warmup} warm-up decompositions"))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(res["secs"]), "warmup": 0 if long_run else args.warmup,
        "ms_per_step": 1e3 * total / len(res["secs"]), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(n, m, name, {"runner": "reference CPU decomposition, single thread",
                                               "graph_built_by": "oracle C builder (same edges as the device "
                                                                 "generator)",
                                               "clusters": res.get("clusters"), "cut_edges": res.get("cut_edges")}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": res["kind"], "sample": sample,
                         **host_cpu()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# ranks


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


# ----------------------------------------------------------------------------
# per-phase roofline


def phase_roofline(phases, pst, peak, form):
    """Per phase: device ms, share, and - where the phase's algorithmic bytes
    are known - GB/s and fraction of the HBM peak.  Walk step: 28 nA + 4 EA +
    4 Ev bytes (ids, two offsets, x, internal degree, x' and x/d writes;
    column slots; one x/d gather per valid slot), counted by the walk kernels
    themselves; edge differences (plain form: the same rows as the walk):
    24 nA + 4 EA + 4 Ev; sweep sort: 24 B per item and digit pass; sweep
    scan: 20 B per swept vertex."""
    walk_b = 28 * pst["walk_vertices"] + 4 * pst["walk_slots"] + 4 * pst["walk_gathers"]
    alg = {"walk": walk_b, "sort": 24 * pst["sort_items"], "sweep_scan": 20 * pst["swept_items"]}
    if form == "plain":
        alg["nodediff"] = 24 * pst["walk_vertices"] + 4 * pst["walk_slots"] + 4 * pst["walk_gathers"]
    total = sum(p["ms"] for p in phases)
    out = {}
    for p in phases:
        if p["ms"] <= 0:
            continue
        e = {"ms": round(p["ms"], 3), "share": round(p["ms"] / total, 4), "launches": p["launches"]}
        if p["name"] in alg:
            gbs = alg[p["name"]] / (p["ms"] / 1e3) / 1e9
            e.update({"alg_bytes": alg[p["name"]], "gbs": round(gbs, 1), "frac": round(gbs / peak, 4)})
        out[p["name"]] = e
    return out


def measured_traffic(name):
    """DRAM bytes per walk step measured by ncu on this workload
    (profiles/traffic.json), or None."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None, None
    with open(path) as f:
        tj = json.load(f)
    w = tj.get("workloads", {}).get(name, {}).get("walk")
    if not w:
        return None, None
    return w["dram_bytes_per_step"], w["source"]


# ----------------------------------------------------------------------------
# product arm


def product_arm(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import parex_b200 as P
    from parex_b200 import certificate as CERT

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    g, off_d, cols_d, n, m, starts, shard = load_workload(args.workload, dev, rank, world)
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

    forms = ["plain", "learned"] if args.schedule == "both" else [args.schedule]
    model = None
    if "learned" in forms:
        from parex_b200 import learn
        model = learn.Model.load()

    def manager(driver, form):
        dmx = P.CudaDeviceManager(seed=WALK_SEED, sc_threshold=SC, rw_threshold=RW, device=local_rank,
                                  driver=driver)
        if args.row_plan:
            dmx.set_row_plan(*[int(t) for t in args.row_plan.split(",")])
        if form == "learned":
            dmx.set_schedule(P._lib.SCHEDULE_LEARNED, model.weights, model.norm, safety=SAFETY, max_skip=args.max_skip,
                             cut_gate=args.cut_gate, due_period=args.due_period)
        dmx.set_stream(stream.cuda_stream)
        return dmx

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

    res = {}
    with torch.cuda.stream(stream):
        for form in forms:
            dm = manager(P.DRIVER_GRAPH, form)
            for _ in range(args.warmup):
                init_device(dm)
                dm.expanderDecomposition()
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
                    init_device(dm)
                    rounds = dm.expanderDecomposition()
                    e1.record(stream)
                    torch.cuda.synchronize(dev)
                    barrier()
                    total_ms += e0.elapsed_time(e1)
            st = dm.stats()
            fp = dm.getFinalPartition()
            r = {"dm": dm, "ms": total_ms, "rounds": rounds, "clusters": fp.numClusters, "ids": fp.clusterIds,
                 "cut_edges": dm.countCutEdges(), "cut_edges_device_reference_count": dm.getNumCutEdges(),
                 "launches": st["kernel_launches"] - launches0, "clocks": clocks.summary(),
                 "swept_items": st["swept_items"], "skipped_sweeps": st["skipped_sweeps"]}
            # every output cluster certified (outside the timed region)
            cert = CERT.check(off_d, cols_d.to(torch.int64) & 0xFFFFFFFF, torch.from_numpy(fp.clusterIds).to(dev),
                              torch.from_numpy(dm.readRandomWalkValues()).to(dev),
                              torch.from_numpy(dm.downloadCertificates().view(np.int32)).to(dev), SC, RW,
                              device=dev, connectivity=args.connectivity, degrees=None)
            r["certificate"] = {k: cert[k] for k in ("ok", "clusters", "uncertified_vertices",
                                                       "threshold_violations", "sweep_checked", "sweep_violations",
                                                       "min_sweep_sparsity", "disconnected", "potential_ties")}
            if not args.connectivity:
                r["certificate"]["disconnected"] = "not checked (--no-connectivity)"
            res[form] = r
        head = "learned" if "learned" in forms else forms[0]
        dm = res[head]["dm"]

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
        assert fp_e2e.numClusters == res[head]["clusters"]
        assert np.array_equal(ids_hn, res[head]["ids"]), "ids written to page-locked memory differ"

        # per-phase device times with the stream driver (roofline), every form
        peak, peak_kind = measured_peaks()
        for form in forms:
            prof = manager(P.DRIVER_STREAM, form)
            init_device(prof)
            prof.set_profiling(True)
            prof.expanderDecomposition()
            pst = prof.stats()
            res[form]["phases"] = phase_roofline(prof.phase_stats(), pst, peak, form)
            res[form]["prof_stats"] = pst
            res[form]["prof_identical"] = bool(np.array_equal(prof.getFinalPartition().clusterIds,
                                                              res[form]["ids"]))
            prof.close()

    times = max_over_ranks([res[f]["ms"] for f in forms] + [e2e_ms], world, dev)
    for f, t in zip(forms, times):
        res[f]["ms"] = t
    e2e_ms = times[-1]
    # edges per step of the whole job: each replica's m, or the shards' sum
    job_m = int(sum_over_ranks([m], world, dev)[0]) if sharded else m * world

    if rank != 0:
        return 0
    hr = res[head]
    value = job_rate(job_m, 1, args.steps, hr["ms"])
    e2e_value = job_rate(job_m, 1, args.steps, e2e_ms)
    h2d = (n + 1) * (8 if off64 else 4) + 2 * m * 4
    d2h = n * 4 + 4

    # roofline: the walk step, the kernel the metric names (one launch = one
    # walk step: the light-row kernel and the warp / CTA long-row kernels)
    pst = hr["prof_stats"]
    walk = hr["phases"]["walk"]
    steps_walked = max(1, pst["rounds"])
    alg_walk = walk["alg_bytes"] / steps_walked
    us_walk = 1e3 * walk["ms"] / steps_walked
    ach = alg_walk / (us_walk / 1e6) / 1e9
    traffic, tsrc = measured_traffic(args.workload)
    roofline = {
        "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "traffic": traffic,
        "kernel": "walk step: k_walk (light rows) + k_walk_long (warp / CTA per long row), one step per round",
        "algorithmic_bytes_per_launch": alg_walk, "launches": steps_walked, "device_us_per_launch": us_walk,
        "traffic_source": tsrc, "peak_source": f"{peak_kind} HBM copy peak", "form": head,
    }

    forms_out = {}
    for f in forms:
        r = res[f]
        forms_out[f] = {
            "value": job_rate(job_m, 1, args.steps, r["ms"]), "ms_per_step": r["ms"] / args.steps,
            "rounds": r["rounds"], "clusters": r["clusters"], "cut_edges": r["cut_edges"],
            "cut_edges_device_reference_count": r["cut_edges_device_reference_count"],
            "swept_vertices": r["swept_items"], "skipped_cluster_sweeps": r["skipped_sweeps"],
            "gpu_launches": r["launches"], "clocks": r["clocks"], "certificate": r["certificate"],
            "phases": r["phases"], "profiled_run_identical": r["prof_identical"],
        }
    extra = {"driver": "cuda graph, device-driven round loop", "schedule": head, "forms": forms_out,
             "row_plan": dm.row_plan(), "instances": None if starts is None else int(len(starts) - 1),
             "parallelism": (f"{world} ranks, instances split by expected edges" if sharded else "replicas"),
             "job_edges_per_step": job_m}
    if model is not None:
        extra["learned_schedule"] = {"safety": SAFETY, "max_skip": args.max_skip, "cut_gate": args.cut_gate,
                                     "due_period": args.due_period,
                                     "model": "parex_b200/data/stop_predictor.npz"}
    if sharded:
        extra["shard_instances"] = len(shard)
    if len(forms) == 2:
        p, l = res["plain"], res["learned"]
        extra["learned_vs_plain"] = p["ms"] / l["ms"]
        extra["cut_edges_learned_over_plain"] = l["cut_edges"] / max(p["cut_edges"], 1)
        extra["every_cluster_certified"] = bool(p["certificate"]["ok"] and l["certificate"]["ok"])

    if world == 1 and not args.no_reference_gpu:
        extra["reference_gpu"] = run_reference_gpu(off_hn, cols_hn, off64)

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        sample, what = cpu_sample(args.workload)
        if sample is not None:
            rc = run_reference_cpu(sample[0], sample[1], 1)
            ms = sample[1].shape[0] // 2
            cpu = {"value": ms / rc["secs"][0], "unit": UNIT, "cores": 1, "kind": rc["kind"],
                   "sample": f"{what} ({rc['secs'][0]:.1f} s, single thread)", **host_cpu()}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": hr["ms"] / args.steps, "higher_is_better": True,
        "scaling": "strong" if sharded else "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(n, m, args.workload, extra),
        "clocks": hr["clocks"],
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms / args.steps, "form": head},
        "gpu_launches": hr["launches"],
        "roofline": roofline,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU decomposition of the graph")
    ap.add_argument("--workload", default="rmat24", choices=sorted(WORKLOADS))
    ap.add_argument("--schedule", default="both", choices=["both", "plain", "learned"])
    ap.add_argument("--no-connectivity", dest="connectivity", action="store_false",
                    help="skip the connectivity part of the certificate check")
    ap.add_argument("--max-skip", type=int, default=MAX_SKIP, help="learned form: cap on consecutive skipped sweeps")
    ap.add_argument("--cut-gate", type=float, default=CUT_GATE,
                    help="learned form: after a round that cut more than this fraction of its clusters, sweep all")
    ap.add_argument("--due-period", type=int, default=DUE_PERIOD,
                    help="learned form: clusters come due only in rounds whose index is a multiple of this")
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
