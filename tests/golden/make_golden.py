"""Generate the golden fixtures from the reference's own binaries.

Two phases:

``--run OUT``   (on a machine with a B200 and the binaries built by
                oracle/ref/Makefile) writes the fixture graphs, runs the
                reference GPU decomposition in its ``trace`` mode (every stage's
                device state per round) and ``decomp`` mode, and the reference
                CPU decomposition, into OUT.
``--pack OUT``  packs selected rounds of those traces into the compressed
                fixtures in this directory.

The graphs are the seeded generators of parex_b200.graphs; each fixture also
stores its CSR so it does not depend on the generator's version.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from parex_b200 import graphs as G  # noqa: E402

SEED = 6582
SC = 0.3
RW = 1e-4
LNODE = np.dtype([("nix", "<u4"), ("label", "<i4")])
NODE_DATA = np.dtype([("nix", "<u4"), ("prefix_volume", "<u4"), ("prefix_edge_diff", "<i4"), ("offset", "<u4")])
SWEEP_CUT = np.dtype([("label", "<i4"), ("sparsity", "<f4"), ("offset", "<u4")])
CLUSTER_DATA = np.dtype([("sum", "<f4"), ("max", "<f4"), ("min", "<f4"), ("count", "<u4")])

# name -> (generator, rounds to keep in the fixture)
TRACED = {
    "sbm2k": (lambda: G.sbm_graph(2048, 8, 10.0, 0.5, 7), [1, 3, 4, 6, 12, 18]),
    "grid16": (lambda: G.grid3d(16), [1, 2, 5, 11, 20, 35]),
}
DECOMPOSED = {
    "sbm16k": lambda: G.sbm_graph(),
    "grid32": lambda: G.grid3d(32),
}


def _run(cmd, out_path):
    with open(out_path, "w") as f:
        subprocess.run(cmd, check=True, stdout=f, stderr=subprocess.STDOUT)


def run(out: str) -> None:
    ref_gpu = os.path.join(ROOT, "oracle", "_ref", "ref_gpu")
    ref_cpu = os.path.join(ROOT, "oracle", "_ref", "ref_cpu")
    os.makedirs(out, exist_ok=True)
    for name, (gen, rounds) in TRACED.items():
        g = gen()
        gpath = os.path.join(out, f"{name}.pxg")
        G.write_pxg(gpath, g)
        tdir = os.path.join(out, f"trace_{name}")
        os.makedirs(tdir, exist_ok=True)
        _run([ref_gpu, "trace", gpath, str(SEED), str(SC), str(RW), str(max(rounds)), tdir],
             os.path.join(out, f"trace_{name}.log"))
        _run([ref_cpu, "decomp", gpath, str(SEED), str(SC), str(RW), "1", os.path.join(out, f"cpu_{name}.i32")],
             os.path.join(out, f"cpu_{name}.log"))
    for name, gen in DECOMPOSED.items():
        g = gen()
        gpath = os.path.join(out, f"{name}.pxg")
        G.write_pxg(gpath, g)
        ddir = os.path.join(out, f"dec_{name}")
        os.makedirs(ddir, exist_ok=True)
        _run([ref_gpu, "decomp", gpath, str(SEED), str(SC), str(RW), ddir], os.path.join(out, f"dec_{name}.log"))
        _run([ref_cpu, "decomp", gpath, str(SEED), str(SC), str(RW), "1", os.path.join(out, f"cpu_{name}.i32")],
             os.path.join(out, f"cpu_{name}.log"))


def _json_lines(path):
    rows = []
    for line in open(path):
        line = line.strip()
        if line.startswith("{"):
            rows.append(json.loads(line))
        elif line.startswith("iterations:"):
            rows.append({"iterations": int(line.split(":")[1])})
    return rows


def _valid_bits(cols):
    return np.packbits(cols != 0xFFFFFFFF)


def pack(out: str) -> None:
    summary = {"seed": SEED, "sc_threshold": SC, "rw_threshold": RW, "graphs": {}}
    for name, (gen, rounds) in TRACED.items():
        g = G.read_pxg(os.path.join(out, f"{name}.pxg"))
        tdir = os.path.join(out, f"trace_{name}")
        meta = [json.loads(l) for l in open(os.path.join(tdir, "meta.jsonl"))]
        arrays = {
            "offsets": g.offsets.astype(np.uint32), "cols": g.cols,
            "x0": np.fromfile(os.path.join(tdir, "x0.f64")).astype(np.float32),
            "final_ids": np.fromfile(os.path.join(tdir, "final_ids.i32"), dtype=np.int32),
            "final_labels": np.fromfile(os.path.join(tdir, "final_labels.i32"), dtype=np.int32),
            "final_valid": _valid_bits(np.fromfile(os.path.join(tdir, "final_cols.u32"), dtype=np.uint32)),
        }
        for r in rounds:
            p = os.path.join(tdir, f"r{r}_")
            rd = lambda n, dt: np.fromfile(p + n, dtype=dt)  # noqa: E731
            arrays.update({
                f"r{r}_act_pre": rd("act_pre.ln", LNODE), f"r{r}_lab_pre": rd("lab_pre.i32", np.int32),
                f"r{r}_x_pre": rd("x_pre.f64", np.float64), f"r{r}_deg_pre": rd("deg_pre.u32", np.uint32),
                f"r{r}_valid_pre": _valid_bits(rd("cols_pre.u32", np.uint32)),
                f"r{r}_x_walk": rd("x_walk.f64", np.float64), f"r{r}_sorted": rd("sorted.nd", NODE_DATA),
                f"r{r}_allcuts": rd("allcuts.scd", SWEEP_CUT), f"r{r}_lab_cut": rd("lab_cut.i32", np.int32),
                f"r{r}_lab_cc": rd("lab_cc.i32", np.int32), f"r{r}_clabels": rd("clabels.i32", np.int32),
                f"r{r}_cdata": rd("cdata.cd", CLUSTER_DATA), f"r{r}_lab_final": rd("lab_final.i32", np.int32),
                f"r{r}_x_final": rd("x_final.f64", np.float64), f"r{r}_deg_final": rd("deg_final.u32", np.uint32),
                f"r{r}_valid_final": _valid_bits(rd("cols_final.u32", np.uint32)),
            })
        np.savez_compressed(os.path.join(HERE, f"ref_trace_{name}.npz"), **arrays)
        trace_log = _json_lines(os.path.join(out, f"trace_{name}.log"))
        summary["graphs"][name] = {
            "n": g.n, "m": g.m, "rounds_kept": rounds,
            "meta": {str(m["round"]): m for m in meta},
            "reference_gpu": [r for r in trace_log if r.get("mode") == "trace"][0],
            "reference_cpu": _json_lines(os.path.join(out, f"cpu_{name}.log"))[0],
        }
    for name in DECOMPOSED:
        rows = _json_lines(os.path.join(out, f"dec_{name}.log"))
        its = [r["iterations"] for r in rows if "iterations" in r]
        gpu = [r for r in rows if r.get("mode") == "decomp"][0]
        gpu["iterations_printed"] = its[0] if its else None
        summary["graphs"][name] = {
            "reference_gpu": gpu,
            "reference_cpu": _json_lines(os.path.join(out, f"cpu_{name}.log"))[0],
        }
        ids = np.fromfile(os.path.join(out, f"dec_{name}", "final_ids.i32"), dtype=np.int32)
        np.savez_compressed(os.path.join(HERE, f"ref_final_{name}.npz"), final_ids=ids)
    with open(os.path.join(HERE, "reference_summary.json"), "w") as f:
        json.dump(summary, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--run", metavar="OUT")
    ap.add_argument("--pack", metavar="OUT")
    a = ap.parse_args()
    if a.run:
        run(a.run)
    if a.pack:
        pack(a.pack)
