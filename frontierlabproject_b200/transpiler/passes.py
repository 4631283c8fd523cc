"""Lazy Qubit Reordering (LQR): flat time-space tiling of a circuit into tiles.

Restates the algorithms of qgpusim/transpiler/passes.py so that the schedule
(the ``Tile`` list) is identical to the reference's for the same gate order:

* ``tile_construction``   -- Alg. 2, passes.py:89-128
* ``greedy_qubit_mapping`` -- Alg. 3, passes.py:131-176
* ``flat_tiling``          -- Alg. 1 with the forced single-gate tile, passes.py:182-243
* ``extract_tiles`` / ``summarize_tiling`` / ``build_tiling_plan`` -- passes.py:247-357
* ``run``                  -- depth computation and stable depth sort, passes.py:359-420

The gate list is handled as integer indices with a "removed" mask instead of the
reference's per-gate list rebuild, so tiling a 4,500-gate circuit is linear per
tile rather than quadratic.  ``run`` hands Alg. 1-3 and the tile extraction to the
native library (``qs_lqr_flat_tiling``, the same algorithms on 64-bit qubit masks) when
it loads and the circuit has at most 64 qubits; ``flat_tiling`` here is the Python
statement of the same steps.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Set, Tuple

from ..circuit import DAGCircuit, DAGOpNode


@dataclass
class Tile:
    tile_idx: int
    # global qubit ids local to this tile, sorted (Q_L)
    logical_qubits: List[int]
    # global qubit -> local bit index 0..|Q_L|-1
    global_to_local_map: Dict[int, int]
    # layout[pos] = global qubit at bit position pos
    layout: List[int]
    # gate nodes of the tile, in schedule order
    gates: list


def _build_tile_layout(logical_qubits: Sequence[int], num_qubits: int) -> List[int]:
    """Tile qubits at the lowest bit positions, the others after them in ascending order."""
    local = set(logical_qubits)
    return list(logical_qubits) + [q for q in range(num_qubits) if q not in local]


_NATIVE_OK: Optional[bool] = None


def _native_available() -> bool:
    global _NATIVE_OK
    if _NATIVE_OK is None:
        try:
            from .. import _native
            _native.lib()
            _NATIVE_OK = True
        except Exception:  # library not built: the Python statement of the algorithms runs
            _NATIVE_OK = False
    return _NATIVE_OK


class LazyQubitReordering:
    """LQR pass.  ``run(dag)`` stores the tile plan in ``property_set["flat_tiling_plan"]``.
    ``native``: None = the C++ tiler when the library loads, True / False = force it on / off."""

    def __init__(self, nL: int, native: Optional[bool] = None):
        if nL < 1:
            raise ValueError("nL must be >= 1")
        self.nL = nL
        self.native = native
        self.property_set: dict = {}

    # ---- Alg. 2 -------------------------------------------------------------------
    @staticmethod
    def _scan_tile(QL: Set[int], order: List[int], targets: List[frozenset]) -> List[int]:
        avail = set(QL)
        picked: List[int] = []
        for g in order:
            t = targets[g]
            if t <= avail:
                picked.append(g)
            else:
                avail -= t
                if not avail:
                    break
        return picked

    def tile_construction(self, QL: Set[int], Cremain: List, T_map: Dict) -> List:
        avail = set(QL)
        G = []
        for U in Cremain:
            t = T_map[U]
            if t <= avail:
                G.append(U)
            else:
                avail -= t
                if not avail:
                    break
        return G

    # ---- Alg. 3 -------------------------------------------------------------------
    @staticmethod
    def _scan_mapping(Q: Set[int], order: List[int], targets: List[frozenset], nL: int) -> Set[int]:
        avail = set(Q)
        chosen: Set[int] = set()
        for g in order:
            t = targets[g]
            if t <= avail and len(chosen | t) <= nL:
                chosen |= t
            else:
                avail -= t
                if not avail:
                    break
        if not chosen:
            return set()
        for q in sorted(Q - chosen):
            if len(chosen) >= nL:
                break
            chosen.add(q)
        return chosen

    def greedy_qubit_mapping(self, Q: Set[int], Cremain: List, T_map: Dict, nL: int) -> Set[int]:
        order = list(range(len(Cremain)))
        targets = [frozenset(T_map[U]) for U in Cremain]
        return self._scan_mapping(set(Q), order, targets, nL)

    qubit_mapping = greedy_qubit_mapping

    # ---- Alg. 1 -------------------------------------------------------------------
    def flat_tiling(self, Q: Set[int], C: List, T_map: Dict, nL: int) -> Tuple[List, Dict]:
        nodes = list(C)
        targets = [frozenset(T_map[U]) for U in nodes]
        remaining = list(range(len(nodes)))
        QL: Set[int] = set(range(min(nL, len(Q))))
        schedule: List = []
        M: Dict = {}
        while remaining:
            picked = self._scan_tile(QL, remaining, targets)
            if not picked:
                # forced tile: the first remaining gate alone, Q_L = its qubits + lowest others
                first = remaining[0]
                QL = set(targets[first])
                if len(QL) < nL:
                    for q in sorted(set(Q) - QL):
                        if len(QL) >= nL:
                            break
                        QL.add(q)
                picked = [first]
            ql_copy = frozenset(QL)
            for g in picked:
                schedule.append(nodes[g])
                M[nodes[g]] = set(ql_copy)
            taken = set(picked)
            remaining = [g for g in remaining if g not in taken]
            if remaining:
                QL = self._scan_mapping(set(Q), remaining, targets, nL)
        return schedule, M

    @staticmethod
    def flat_tiling_native(n: int, C: List, T_map: Dict, nL: int, tiles_out: Optional[list] = None
                           ) -> Tuple[List, Dict]:
        """``flat_tiling`` by the native library (qubit sets as 64-bit masks, n <= 64).  The
        gates of one tile share one qubit set in M; tiles_out (optional) receives the
        (qubit set, gates) pairs of ``extract_tiles``."""
        import numpy as np
        from .. import _native as N
        nodes = list(C)
        ng = len(nodes)
        masks = np.fromiter((sum(1 << q for q in T_map[nd]) for nd in nodes), dtype=np.uint64, count=ng)
        order = np.empty(max(ng, 1), np.int32)
        tile_of = np.empty(max(ng, 1), np.int32)
        tmasks = np.empty(max(ng, 1), np.uint64)
        nt = ctypes.c_int()
        N.call("qs_lqr_flat_tiling", n, nL, masks.ctypes.data, ng, order.ctypes.data, tile_of.ctypes.data,
               tmasks.ctypes.data, ctypes.byref(nt))
        sets = [{q for q in range(n) if (int(m) >> q) & 1} for m in tmasks[:nt.value]]
        schedule = [nodes[i] for i in order[:ng].tolist()]
        tl = tile_of[:ng].tolist()
        M = {nd: sets[t] for nd, t in zip(schedule, tl)}
        if tiles_out is not None:
            tiles_out.extend((s, []) for s in sets)
            for nd, t in zip(schedule, tl):
                tiles_out[t][1].append(nd)
        return schedule, M

    # ---- helpers ------------------------------------------------------------------
    @staticmethod
    def extract_tiles(g_schedule: List, M: Dict) -> List[Tuple[Set[int], List]]:
        tiles: List[Tuple[Set[int], List]] = []
        for node in g_schedule:
            if tiles and M[node] == tiles[-1][0]:
                tiles[-1][1].append(node)
            else:
                tiles.append((M[node], [node]))
        return tiles

    @staticmethod
    def summarize_tiling(g_schedule: List, M: Dict) -> dict:
        tiles = LazyQubitReordering.extract_tiles(g_schedule, M)
        if not tiles:
            return {"num_tiles": 0, "avg_tile_size": 0.0, "max_tile_size": 0,
                    "avg_Q_L_size": 0.0, "max_Q_L_size": 0}
        sizes = [len(g) for _, g in tiles]
        qls = [len(q) for q, _ in tiles]
        return {"num_tiles": len(tiles), "avg_tile_size": sum(sizes) / len(tiles),
                "max_tile_size": max(sizes), "avg_Q_L_size": sum(qls) / len(tiles),
                "max_Q_L_size": max(qls)}

    @staticmethod
    def build_tiling_plan(g_schedule: List, M: Dict, num_qubits: int, tiles: Optional[list] = None) -> List[Tile]:
        plan: List[Tile] = []
        if tiles is None:
            tiles = LazyQubitReordering.extract_tiles(g_schedule, M)
        for idx, (ql_set, gates) in enumerate(tiles):
            ql = sorted(ql_set)
            plan.append(Tile(tile_idx=idx, logical_qubits=ql,
                             global_to_local_map={gq: i for i, gq in enumerate(ql)},
                             layout=_build_tile_layout(ql, num_qubits), gates=gates))
        return plan

    # ---- pass entry -----------------------------------------------------------------
    def run(self, dag: DAGCircuit) -> DAGCircuit:
        n = len(dag.qubits)
        qindex = {q: i for i, q in enumerate(dag.qubits)}
        nodes = list(dag.topological_op_nodes())
        last = [-1] * n
        depth: Dict = {}
        for node in nodes:
            qi = [qindex[q] for q in node.qargs]
            d = (max(last[i] for i in qi) + 1) if qi else 0
            depth[node] = d
            for i in qi:
                last[i] = d
        nodes.sort(key=lambda nd: depth[nd])  # stable, as list.sort is
        T_map = {node: {qindex[q] for q in node.qargs} for node in nodes}
        native = self.native if self.native is not None else _native_available()
        tiles = None
        if native and n <= 64:
            tiles = []
            schedule, M = self.flat_tiling_native(n, nodes, T_map, self.nL, tiles)
        else:
            schedule, M = self.flat_tiling(set(range(n)), nodes, T_map, self.nL)
        self.property_set["flat_tiling_schedule"] = schedule
        self.property_set["flat_tiling_mapping"] = M
        self.property_set["flat_tiling_plan"] = self.build_tiling_plan(schedule, M, n, tiles)
        out = dag.copy_empty_like()
        for node in schedule:
            out.apply_operation_back(node.op, qargs=node.qargs, cargs=node.cargs)
        return out
