"""Seeded synthetic graph generators and the binary CSR file format.

Every generator returns an undirected, unweighted, simple graph as CSR arrays
``(offsets, cols)``: ``offsets`` has n+1 entries (uint32, or uint64 once the
slot count reaches 2**32) and ``cols`` holds the 2m neighbour ids (uint32),
each row sorted ascending.  That is the layout ``DynamicGraph::finalize``
produces in the reference (lib/core/graph.h:147-184): both directions of
every edge, rows ordered by neighbour id.

The generators stand in for the reference's Matrix Market inputs, which are
not distributed with it; they follow the graph families the decomposition is
measured on (planted partition, 3D grid, R-MAT, random regular, batches of
planted partitions).
"""
from __future__ import annotations

import dataclasses
import math
import os
import struct

import numpy as np

MAGIC = b"PXCSR001"


@dataclasses.dataclass
class CSRGraph:
    """CSR graph: ``offsets`` (n+1), ``cols`` (2m, uint32)."""

    offsets: np.ndarray
    cols: np.ndarray
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.offsets.shape[0] - 1)

    @property
    def m(self) -> int:
        return int(self.cols.shape[0] // 2)

    def degrees(self) -> np.ndarray:
        return np.diff(self.offsets.astype(np.int64)).astype(np.uint32)


def csr_from_edges(u: np.ndarray, v: np.ndarray, n: int, name: str = "") -> CSRGraph:
    """Build the symmetric CSR of the undirected edge list (u, v).

    Self-loops are dropped and duplicate edges merged, as the reference's
    inputs are simple graphs.
    """
    u = np.asarray(u, dtype=np.uint64)
    v = np.asarray(v, dtype=np.uint64)
    keep = u != v
    u, v = u[keep], v[keep]
    lo = np.minimum(u, v)
    hi = np.maximum(u, v)
    key = np.unique((lo << np.uint64(32)) | hi)
    lo = (key >> np.uint64(32)).astype(np.uint32)
    hi = (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    del key
    src = np.concatenate([lo, hi])
    dst = np.concatenate([hi, lo])
    del lo, hi
    full = (src.astype(np.uint64) << np.uint64(32)) | dst.astype(np.uint64)
    del dst
    full.sort()
    cols = (full & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    deg = np.bincount(src, minlength=n).astype(np.int64)
    del full, src
    off_dtype = np.uint32 if cols.shape[0] < 2**32 else np.uint64
    offsets = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(deg, out=offsets[1:])
    return CSRGraph(offsets.astype(off_dtype), cols, name)


# ----------------------------------------------------------------------------
# counter-based randomness: splitmix64 over (seed, stream, index)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    x = x + np.uint64(0x9E3779B97F4A7C15)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def _hash_stream(seed: int, stream: int, count: int, start: int = 0) -> np.ndarray:
    base = np.uint64((seed * 0x100000001B3 + stream * 0x9E3779B1) & 0xFFFFFFFFFFFFFFFF)
    with np.errstate(over="ignore"):
        idx = np.arange(start, start + count, dtype=np.uint64)
        return _splitmix64(_splitmix64(idx ^ base) + base)


# ----------------------------------------------------------------------------
# generators


def grid3d(side: int = 128) -> CSRGraph:
    """3D 7-point grid side^3: vertex (x, y, z) has id x + side*(y + side*z)."""
    n = side**3
    ids = np.arange(n, dtype=np.int64).reshape(side, side, side)  # [z, y, x]
    us, vs = [], []
    us.append(ids[:, :, :-1].ravel()); vs.append(ids[:, :, 1:].ravel())
    us.append(ids[:, :-1, :].ravel()); vs.append(ids[:, 1:, :].ravel())
    us.append(ids[:-1, :, :].ravel()); vs.append(ids[1:, :, :].ravel())
    return csr_from_edges(np.concatenate(us), np.concatenate(vs), n, f"grid3d_{side}")


def _sample_pairs(rng: np.random.Generator, total: int, p: float) -> np.ndarray:
    """Bernoulli(p) subset of [0, total), drawn as Binomial count + distinct indices."""
    if total <= 0 or p <= 0:
        return np.zeros(0, dtype=np.int64)
    k = int(rng.binomial(total, min(p, 1.0)))
    if k == 0:
        return np.zeros(0, dtype=np.int64)
    if k > total // 4:
        return np.nonzero(rng.random(total) < p)[0].astype(np.int64)
    out = np.unique(rng.integers(0, total, size=k, dtype=np.int64))
    while out.shape[0] < k:
        extra = rng.integers(0, total, size=k - out.shape[0], dtype=np.int64)
        out = np.unique(np.concatenate([out, extra]))
    return out


def _tri_unrank(idx: np.ndarray, size: int):
    """Map pair index in [0, size*(size-1)/2) to (a, b), a < b (row-major upper triangle)."""
    # a = largest row with start(a) <= idx, start(a) = a*size - a*(a+1)/2
    idx = idx.astype(np.float64)
    s = float(size)
    a = np.floor((2 * s - 1 - np.sqrt((2 * s - 1) ** 2 - 8 * idx)) / 2).astype(np.int64)
    a = np.clip(a, 0, size - 2)
    start = a * size - a * (a + 1) // 2
    fix = start > idx
    a[fix] -= 1
    start = a * size - a * (a + 1) // 2
    nxt = (a + 1) * size - (a + 1) * (a + 2) // 2
    fix = nxt <= idx
    a[fix] += 1
    start = a * size - a * (a + 1) // 2
    b = (idx.astype(np.int64) - start) + a + 1
    return a, b


def sbm(n: int = 16384, blocks: int = 16, d_in: float = 12.0, d_out: float = 0.5,
        seed: int = 6582, offset: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Planted partition edge list: equal blocks, Bernoulli pairs.

    Expected intra-block degree d_in and inter-block degree d_out, so
    p_in = d_in / (b - 1) and p_out = d_out / (n - b) with block size b.
    Returns (u, v) with vertex ids shifted by ``offset``.
    """
    rng = np.random.default_rng(seed)
    bsz = n // blocks
    sizes = [bsz] * blocks
    sizes[-1] += n - bsz * blocks
    starts = np.concatenate([[0], np.cumsum(sizes)])
    p_in = d_in / max(bsz - 1, 1)
    p_out = d_out / max(n - bsz, 1)
    us, vs = [], []
    for i in range(blocks):
        s = sizes[i]
        idx = _sample_pairs(rng, s * (s - 1) // 2, p_in)
        if idx.size:
            a, b = _tri_unrank(idx, s)
            us.append(a + starts[i]); vs.append(b + starts[i])
        for j in range(i + 1, blocks):
            t = sizes[j]
            idx = _sample_pairs(rng, s * t, p_out)
            if idx.size:
                us.append(idx // t + starts[i]); vs.append(idx % t + starts[j])
    if not us:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    return np.concatenate(us) + offset, np.concatenate(vs) + offset


def sbm_graph(n: int = 16384, blocks: int = 16, d_in: float = 12.0, d_out: float = 0.5,
              seed: int = 6582) -> CSRGraph:
    u, v = sbm(n, blocks, d_in, d_out, seed)
    return csr_from_edges(u, v, n, f"sbm_{n}_{blocks}_{seed}")


def rmat(scale: int = 22, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
         c: float = 0.19, seed: int = 1) -> CSRGraph:
    """R-MAT: edge_factor * 2^scale samples, symmetrised, deduplicated, no self-loops.

    Each sample picks one quadrant per bit level from a 16-bit uniform drawn
    from a counter-based hash of (seed, sample, level), so the graph depends
    only on the arguments.
    """
    n = 1 << scale
    samples = edge_factor * n
    ta = int(round(a * 65536))
    tab = int(round((a + b) * 65536))
    tabc = int(round((a + b + c) * 65536))
    chunk = 1 << 24
    us, vs = [], []
    for start in range(0, samples, chunk):
        cnt = min(chunk, samples - start)
        u = np.zeros(cnt, dtype=np.uint32)
        v = np.zeros(cnt, dtype=np.uint32)
        h = None
        for lvl in range(scale):
            if lvl % 4 == 0:
                h = _hash_stream(seed, 1000 + lvl // 4, cnt, start)
            r = ((h >> np.uint64(16 * (lvl % 4))) & np.uint64(0xFFFF)).astype(np.int32)
            ubit = r >= tab
            vbit = ((r >= ta) & (r < tab)) | (r >= tabc)
            bit = np.uint32(1 << (scale - 1 - lvl))
            u |= np.where(ubit, bit, np.uint32(0))
            v |= np.where(vbit, bit, np.uint32(0))
        us.append(u); vs.append(v)
    return csr_from_edges(np.concatenate(us), np.concatenate(vs), n, f"rmat_{scale}_{seed}")


def random_regular(n: int = 1 << 22, d: int = 8, seed: int = 1, max_rounds: int = 200) -> CSRGraph:
    """Simple d-regular graph by the pairing model with repair of bad pairs.

    Stubs are shuffled and paired; pairs that form self-loops or duplicates
    are released and re-paired with a fresh shuffle until none remain.
    """
    assert (n * d) % 2 == 0
    rng = np.random.default_rng(seed)
    stubs = np.repeat(np.arange(n, dtype=np.int64), d)
    rng.shuffle(stubs)
    u = stubs[0::2].copy()
    v = stubs[1::2].copy()
    for _ in range(max_rounds):
        lo = np.minimum(u, v)
        hi = np.maximum(u, v)
        key = lo * n + hi
        order = np.argsort(key, kind="stable")
        ks = key[order]
        dup = np.zeros(ks.shape[0], dtype=bool)
        dup[1:] = ks[1:] == ks[:-1]
        bad = np.zeros(u.shape[0], dtype=bool)
        bad[order[dup]] = True
        bad |= u == v
        nbad = int(bad.sum())
        if nbad == 0:
            return csr_from_edges(u, v, n, f"regular_{d}_{n}_{seed}")
        # release the bad pairs plus an equal number of random good pairs and re-pair
        good_idx = np.nonzero(~bad)[0]
        extra = rng.choice(good_idx, size=min(good_idx.shape[0], max(nbad, 64)), replace=False)
        release = np.concatenate([np.nonzero(bad)[0], extra])
        pool = np.concatenate([u[release], v[release]])
        rng.shuffle(pool)
        u[release] = pool[0::2]
        v[release] = pool[1::2]
    raise RuntimeError("random_regular: pairing repair did not converge")


def sbm_batch(count: int = 512, seed: int = 1, n_lo: float = 1e3, n_hi: float = 1e6,
              scale: float = 1.0) -> tuple[CSRGraph, np.ndarray]:
    """Disjoint union of ``count`` planted-partition instances.

    Instance i draws n ~ log-uniform[n_lo, n_hi] (times ``scale``), blocks ~
    U{2..64}, d_in ~ U[4, 32], d_out ~ U[0.1, 2] from a generator keyed by
    (seed, i).  Returns the concatenated CSR and the vertex offset of every
    instance (count+1 entries).
    """
    us, vs, starts = [], [], [0]
    for i in range(count):
        rng = np.random.default_rng([seed, i])
        n = max(4, int(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi))) * scale))
        blocks = int(rng.integers(2, 65))
        blocks = min(blocks, max(1, n // 2))
        d_in = float(rng.uniform(4, 32))
        d_out = float(rng.uniform(0.1, 2))
        u, v = sbm(n, blocks, d_in, d_out, seed=int(rng.integers(1 << 31)), offset=starts[-1])
        us.append(u); vs.append(v)
        starts.append(starts[-1] + n)
    g = csr_from_edges(np.concatenate(us), np.concatenate(vs), starts[-1], f"sbm_batch_{count}_{seed}")
    return g, np.asarray(starts, dtype=np.int64)


# ----------------------------------------------------------------------------
# binary CSR file


def write_pxg(path: str | os.PathLike, g: CSRGraph) -> None:
    off_bytes = g.offsets.dtype.itemsize
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<QQQ", g.n, g.m, off_bytes))
        f.write(np.ascontiguousarray(g.offsets).tobytes())
        f.write(np.ascontiguousarray(g.cols, dtype=np.uint32).tobytes())


def read_pxg(path: str | os.PathLike) -> CSRGraph:
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path}: not a PXCSR001 file")
        n, m, off_bytes = struct.unpack("<QQQ", f.read(24))
        odt = np.uint32 if off_bytes == 4 else np.uint64
        offsets = np.frombuffer(f.read((n + 1) * off_bytes), dtype=odt).copy()
        cols = np.frombuffer(f.read(2 * m * 4), dtype=np.uint32).copy()
    return CSRGraph(offsets, cols, os.path.basename(str(path)))


def write_mtx(path: str | os.PathLike, g: CSRGraph) -> None:
    """Matrix Market coordinate file, each undirected edge once, 1-based ids:
    the input format of the reference's readDynGraph (lib/utils/graph_io.h:49-84)."""
    src = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(g.offsets.astype(np.int64)))
    keep = src < g.cols
    u, v = src[keep] + 1, g.cols[keep].astype(np.int64) + 1
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern symmetric\n")
        f.write(f"{g.n} {g.n} {u.shape[0]}\n")
        np.savetxt(f, np.stack([u, v], axis=1), fmt="%d")


def by_name(name: str) -> CSRGraph:
    """Named workloads: ``sbm16k``, ``grid<side>``, ``rmat<scale>``, ``regular<log2n>``."""
    if name == "sbm16k":
        return sbm_graph()
    if name.startswith("grid"):
        return grid3d(int(name[4:]))
    if name.startswith("rmat"):
        return rmat(int(name[4:]))
    if name.startswith("regular"):
        return random_regular(1 << int(name[7:]))
    raise KeyError(name)
