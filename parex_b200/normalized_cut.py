"""Normalized cut over the expander hierarchy (NormalizedCut,
lib/algorithms/normalized_cut.h:12-141), on a hierarchy built on the GPU
(parex_b200/hierarchy.py).

The reference's algorithm is a greedy walk over the hierarchy tree and stays
on the host: k times, for every current root (a tree node that heads one
output cluster), find the tree node below it whose separation raises the
normalized cut objective least (edgePenalty, :43-51), take the best over all
roots relative to the root's own term (:117-131), make that node a root and
move its volume and cut up its ancestor path (split, :84-99).  Vertices are
labelled by the index of the root they hang under, in the order the reference
keeps its roots (std::set of (level, index)), during the last search - as the
reference does.  Arithmetic in float32 (frac_t); ties keep the first
candidate in the traversal order (children of a tree node in increasing
index order here; the reference follows its partition's vertex order).
"""
from __future__ import annotations

import numpy as np

from .hierarchy import Level

F32 = np.float32


class NormalizedCut:
    def __init__(self, levels: list[Level], n_vertices: int):
        if not levels:
            raise ValueError("empty hierarchy")
        self.levels = levels
        self.volumes = [lvl.volumes.astype(np.int64).copy() for lvl in levels]
        self.cuts = [lvl.cut_sizes.astype(np.int64).copy() for lvl in levels]
        # children of cluster c of level l: the vertices of level l's graph whose parent is c
        self.children = []
        for lvl in levels:
            order = np.argsort(lvl.parents, kind="stable")
            bounds = np.searchsorted(lvl.parents[order], np.arange(lvl.clusters + 1))
            self.children.append((order, bounds))
        self.labels = np.zeros(n_vertices, dtype=np.int64)
        self.roots: set[tuple[int, int]] = set()

    def _kids(self, level: int, nix: int) -> np.ndarray:
        order, bounds = self.children[level]
        return order[bounds[nix]:bounds[nix + 1]]

    def _edge_penalty(self, level: int, nix: int, cluster_cut: int, cluster_vol: int) -> np.float32:
        cut_a = self.cuts[level][nix]
        vol_a = self.volumes[level][nix]
        cut_b = cluster_cut + cut_a
        vol_b = cluster_vol - vol_a
        return F32(F32(cut_a) / F32(vol_a)) + F32(F32(cut_b) / F32(vol_b))

    def _candidate(self, level: int, nix: int, label: int, cluster_cut: int, cluster_vol: int):
        """getCandidate (:57-82): the best tree node below (level, nix), labelling its vertices."""
        best = ((0, 0), F32(100000))

        # depth-first in the reference's order: children in order, each child's subtree right after it
        def visit(lv, nx):
            nonlocal best
            for cv in self._kids(lv, nx):
                if lv == 0:
                    self.labels[cv] = label
                    continue
                child = (lv - 1, int(cv))
                if child in self.roots:
                    continue
                if self.volumes[lv - 1][cv] < cluster_vol:
                    pen = self._edge_penalty(lv - 1, int(cv), cluster_cut, cluster_vol)
                    if pen < best[1]:
                        best = (child, pen)
                visit(lv - 1, int(cv))

        visit(level, nix)
        return best

    def _split(self, level: int, nix: int) -> None:
        vol_a = self.volumes[level][nix]
        cut_a = self.cuts[level][nix]
        child = nix
        lv = level
        while lv + 1 < len(self.levels):
            lv += 1
            parent = self._parent(lv, child)
            self.volumes[lv][parent] -= vol_a
            self.cuts[lv][parent] += cut_a
            child = parent

    def _parent(self, lv: int, child: int) -> int:
        """Cluster at level lv of vertex `child` of level lv's graph (a cluster of level lv - 1)."""
        return int(self.levels[lv].parents[child])

    def compute(self, k: int) -> np.ndarray:
        """Labels of the input graph's vertices after k greedy splits (:109-141)."""
        top = len(self.levels) - 1
        self.volumes = [lvl.volumes.astype(np.int64).copy() for lvl in self.levels]
        self.cuts = [lvl.cut_sizes.astype(np.int64).copy() for lvl in self.levels]
        self.labels[:] = 0
        self.roots = {(top, 0)}
        for _ in range(k):
            best_cand = ((0, 0), F32(1000))
            best_delta = F32(100000)
            for root_ix, root in enumerate(sorted(self.roots)):
                vol = self.volumes[root[0]][root[1]]
                cut = self.cuts[root[0]][root[1]]
                cand = self._candidate(root[0], root[1], root_ix, int(cut), int(vol))
                delta = F32(cand[1] - F32(F32(cut) / F32(vol)))
                if delta < best_delta:
                    best_delta = delta
                    best_cand = cand
            tn = best_cand[0]
            self._split(*tn)
            self.roots.add(tn)
        return self.labels.copy()
