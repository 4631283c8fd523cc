"""Host tile executor: the drop-in ``run_custom_backend`` of the qgpusim custom backend.

Mirrors qgpusim/backends/custom/backend.py:

* ``GATE_CACHE`` / ``get_gate_matrix_host`` / ``clear_gate_cache``: LRU cache (512) of
  gate matrices keyed by ``(name, params)`` (backend.py:16-85).  Matrices stay on the
  host; the executor copies them into its own device program, so there is no borrowed
  device pointer.
* ``fuse_tile_ops``: same-qubit 1q runs and same-ordered-pair 2q runs, ``U_new = U @ U_prev``
  (backend.py:88-200).
* ``run_custom_backend(qc, tile_plan, task, shots=None, use_float32=False,
  use_cuda_graphs=True, tile_mode="cooperative", enable_fusion=True)`` -> (statevector,
  metrics) with the reference's metric keys (backend.py:336-522).  The statevector is in
  the physical layout of the last tile, as the reference returns it; ``logical_order=True``
  returns it in logical qubit order instead.
"""
from __future__ import annotations

import time
from collections import OrderedDict
from typing import List, Optional

import numpy as np

from ctypes import byref, c_int

from . import _native as N
from .qgpusim_cuda import Statevector, StatevectorF32, _OpBatch

MAX_CACHE_SIZE = 512
GATE_CACHE: "OrderedDict[tuple, dict]" = OrderedDict()
KERNEL_LAUNCH_OVERHEAD_US = 10.0


def _evict_cache_if_needed() -> None:
    while len(GATE_CACHE) > MAX_CACHE_SIZE:
        GATE_CACHE.popitem(last=False)


def _gate_key(op):
    try:
        params = tuple(float(p) for p in getattr(op, "params", []))
    except (TypeError, ValueError):
        return None  # matrix-valued parameters: not cacheable by value
    return (op.name, params)


def get_gate_matrix_host(op, dtype=np.complex128) -> np.ndarray:
    key = _gate_key(op)
    dt = np.dtype(dtype)
    if key is None or getattr(op, "_matrix", None) is not None:
        return np.ascontiguousarray(op.to_matrix(), dtype=dt)
    item = GATE_CACHE.get(key)
    if item is None:
        _evict_cache_if_needed()
        item = {}
        GATE_CACHE[key] = item
    else:
        GATE_CACHE.move_to_end(key)
    m = item.get(dt.str)
    if m is None:
        m = np.ascontiguousarray(op.to_matrix(), dtype=dt)
        item[dt.str] = m
    return m


def clear_gate_cache() -> None:
    GATE_CACHE.clear()


def _touches(op, qs) -> bool:
    if op[0] == "1q":
        return op[1] in qs
    return op[1] in qs or op[2] in qs


def fuse_tile_ops(tile_ops: list, cp_dtype=None) -> list:
    """Fuse consecutive gates on the same qubit / same ordered qubit pair (backend.py:88-200)."""
    if len(tile_ops) <= 1:
        return tile_ops
    result: list = []
    last_gate_idx: dict = {}
    for op in tile_ops:
        if op[0] == "1q":
            q, U = op[1], op[2]
            idx = last_gate_idx.get(q)
            if idx is not None:
                prev = result[idx]
                if prev[0] == "1q" and prev[1] == q and not any(_touches(o, (q,)) for o in result[idx + 1:]):
                    result[idx] = ("1q", q, np.asarray(U) @ np.asarray(prev[2]))
                    last_gate_idx[q] = idx
                    continue
            last_gate_idx[q] = len(result)
            result.append(("1q", q, U))
        else:
            q0, q1, U = op[1], op[2], op[3]
            prev_idx = None
            for i in range(len(result) - 1, -1, -1):
                o = result[i]
                if o[0] == "2q" and o[1] == q0 and o[2] == q1:
                    prev_idx = i
                    break
                if _touches(o, (q0, q1)):
                    break
            if prev_idx is not None and not any(_touches(o, (q0, q1)) for o in result[prev_idx + 1:]):
                result[prev_idx] = ("2q", q0, q1, np.asarray(U) @ np.asarray(result[prev_idx][3]))
                last_gate_idx[q0] = prev_idx
                last_gate_idx[q1] = prev_idx
                continue
            last_gate_idx[q0] = len(result)
            last_gate_idx[q1] = len(result)
            result.append(("2q", q0, q1, U))
    return result


def tile_ops_for(tile, qubit_map: dict, np_dtype) -> list:
    """('1q', local, U) / ('2q', l0, l1, U) for the unitary nodes of a tile (backend.py:432-451)."""
    ops = []
    g2l = tile.global_to_local_map
    for node in tile.gates:
        op = node.op
        if not hasattr(op, "to_matrix"):
            continue
        qs = [g2l[qubit_map[q]] for q in node.qargs]
        U = get_gate_matrix_host(op, np_dtype)
        if len(qs) == 1:
            ops.append(("1q", qs[0], U))
        elif len(qs) == 2:
            ops.append(("2q", qs[0], qs[1], U))
        else:
            raise RuntimeError(f"gate {op.name} on {len(qs)} qubits is not supported (1- and 2-qubit gates only)")
    return ops


def _apply_on_columns(M: np.ndarray, G: np.ndarray, slots) -> None:
    """M <- G M, G acting on block index bits ``slots`` (1 or 2 of them; G's index
    b_slot0 + 2 b_slot1), every column of M a state of the block's qubits."""
    dim = M.shape[0]
    m = dim.bit_length() - 1
    T = M.reshape((2,) * m + (dim,))  # axis m-1-j holds index bit j
    if len(slots) == 1:
        ax = m - 1 - slots[0]
        Tm = np.moveaxis(T, ax, 0)
        Tm[...] = np.tensordot(G, Tm, axes=(1, 0))
    else:
        a0, a1 = m - 1 - slots[0], m - 1 - slots[1]
        Tm = np.moveaxis(T, (a1, a0), (0, 1))  # index (b_slot1, b_slot0) = G's row/col / 2, % 2
        Tm[...] = np.tensordot(G.reshape(2, 2, 2, 2), Tm, axes=((2, 3), (0, 1)))


def plan_dense_blocks(ops: list, k: int) -> list:
    """Group an op list (('1q', q, U) / ('2q', q0, q1, U) in execution order) into blocks of at
    most k qubits, run in creation order.  Every gate must stay after the earlier gates on its
    qubits and may only move across gates on other qubits; with last[q] the block holding the
    latest gate on q:

    * a one-qubit gate waits on its qubit and is placed just before the next two-qubit gate on
      that qubit, in that gate's block (or, at the end, in last[q]);
    * a gate joins the later of its qubits' last blocks when the qubit union stays within k (the
      blocks in between do not touch its other qubit, since that qubit's last block is earlier);
    * when its qubits' last blocks b1 < b2 are both still the latest blocks of all their qubits
      and fit together in k qubits, b1 moves into b2 (nothing between them touches b1's qubits)
      and the gate joins the merged block;
    * a gate on qubits no block has met joins the most recent block with room; otherwise a new
      block opens.

    Returns [(qubits, U)], U the 2^m x 2^m product of the block's gates (m <= k), row/column
    index sum_j b_{qubits[j]} 2^j."""
    if not 1 <= k <= 6:
        raise ValueError("dense blocks hold 1 to 6 qubits")
    qsets: list = []   # qubits of each block (first-touch order)
    gates: list = []
    alive: list = []
    last: dict = {}
    pending: dict = {}

    def add(b, op, qs):
        for q in qs:
            if q not in qsets[b]:
                qsets[b].append(q)
            last[q] = b
        gates[b].append(op)

    def latest(b):
        return all(last.get(q) == b for q in qsets[b])

    def newest_with_room(qs):
        for c in range(len(qsets) - 1, -1, -1):
            if alive[c]:
                return c if len(set(qsets[c]) | set(qs)) <= k else None
        return None

    def open_block():
        qsets.append([])
        gates.append([])
        alive.append(True)
        return len(qsets) - 1

    for op in ops:
        if op[0] == "1q":
            pending.setdefault(op[1], []).append(op)
            continue
        qs = [op[1], op[2]]
        owners = sorted({last.get(q) for q in qs} - {None})
        b = None
        if len(owners) == 2:
            b1, b2 = owners
            if len(set(qsets[b1]) | set(qsets[b2])) <= k and latest(b1) and latest(b2):
                gates[b2] = gates[b1] + gates[b2]
                for q in qsets[b1]:
                    qsets[b2].append(q)
                    last[q] = b2
                alive[b1], gates[b1], qsets[b1] = False, [], []
                b = b2
        if b is None and owners and len(set(qsets[owners[-1]]) | set(qs)) <= k:
            b = owners[-1]
        if b is None and not owners:
            b = newest_with_room(qs)
        if b is None:
            b = open_block()
        for q in qs:
            for g in pending.pop(q, []):
                add(b, g, [q])
        add(b, op, qs)
    for q in list(pending):
        b = last.get(q)
        if b is None:
            b = newest_with_room([q])
        if b is None:
            b = open_block()
        for g in pending.pop(q):
            add(b, g, [q])
    out = []
    for b in range(len(qsets)):
        if not alive[b] or not gates[b]:
            continue
        qubits = qsets[b]
        d = 1 << len(qubits)
        M = np.eye(d, dtype=np.complex128)
        slot = {q: j for j, q in enumerate(qubits)}
        for op in gates[b]:
            if op[0] == "1q":
                _apply_on_columns(M, np.asarray(op[2], dtype=np.complex128), [slot[op[1]]])
            else:
                _apply_on_columns(M, np.asarray(op[3], dtype=np.complex128), [slot[op[1]], slot[op[2]]])
        out.append((list(qubits), M))
    return out


_NO_PARAMS = (0.0, 0.0, 0.0)


def prepare_tile_ops(tile, qubit_map: dict, dtype_code: int, fuse: bool = True):
    """The tile's unitary nodes as a packed ``qs_op`` batch in one native call
    (``qs_prepare_ops``: matrices of the named gates built natively, equal entry for entry to
    ``gates.gate_matrix``; other gates through ``get_gate_matrix_host``; fused as
    ``fuse_tile_ops`` when ``fuse``).  Returns (batch, number of gates before fusion)."""
    g2l = tile.global_to_local_map
    ids, q0, q1, prm = [], [], [], []
    custom = {}
    gate_ids = N.GATE_IDS
    for node in tile.gates:
        op = node.op
        if not hasattr(op, "to_matrix"):
            continue
        qa = node.qargs
        if len(qa) == 1:
            q0.append(g2l[qubit_map[qa[0]]])
            q1.append(-1)
        elif len(qa) == 2:
            q0.append(g2l[qubit_map[qa[0]]])
            q1.append(g2l[qubit_map[qa[1]]])
        else:
            raise RuntimeError(f"gate {op.name} on {len(qa)} qubits is not supported (1- and 2-qubit gates only)")
        gid = gate_ids.get(op.name) if getattr(op, "_matrix", None) is None else None
        ps = getattr(op, "params", ())
        pv = None
        if gid is not None and len(ps) <= 3:
            try:
                pv = (float(ps[0]) if len(ps) > 0 else 0.0, float(ps[1]) if len(ps) > 1 else 0.0,
                      float(ps[2]) if len(ps) > 2 else 0.0)
            except (TypeError, ValueError):
                pv = None  # symbolic parameters: the gate's own matrix
        if pv is None:
            custom[len(ids)] = get_gate_matrix_host(op, np.complex128)
            ids.append(N.QS_GATE_MATRIX)
            prm.append(_NO_PARAMS)
        else:
            ids.append(gid)
            prm.append(pv)
    n = len(ids)
    batch = _OpBatch([], dtype_code)
    if n == 0:
        return batch, 0
    cust = None
    if custom:
        cust = np.zeros((n, 32), dtype=np.float64)
        for i, m in custom.items():
            flat = np.ascontiguousarray(m, dtype=np.complex128).reshape(-1).view(np.float64)
            cust[i, :flat.size] = flat
    ida = np.asarray(ids, dtype=np.int32)
    q0a = np.asarray(q0, dtype=np.int32)
    q1a = np.asarray(q1, dtype=np.int32)
    pa = np.asarray(prm, dtype=np.float64)
    out = np.zeros(n, dtype=N.OP_DTYPE)
    mats = np.empty(16 * n, dtype=np.complex64 if dtype_code == N.QS_C64 else np.complex128)
    nout = c_int()
    N.call("qs_prepare_ops", dtype_code, n, ida.ctypes.data, pa.ctypes.data, q0a.ctypes.data, q1a.ctypes.data,
           cust.ctypes.data if cust is not None else None, 1 if fuse else 0, out.ctypes.data, mats.ctypes.data,
           byref(nout))
    batch.arr = out[:nout.value]
    batch._keep = [mats]
    return batch, n


def run_custom_backend(qc, tile_plan, task: str = "statevector", shots: Optional[int] = None,
                       use_float32: bool = False, use_cuda_graphs: bool = True, tile_mode: str = "cooperative",
                       enable_fusion: bool = True, logical_order: bool = False, sv=None, out: np.ndarray = None,
                       native_fusion: bool = False, native_prep: bool = True, dense_fusion: int = 0):
    """Simulate ``qc`` along ``tile_plan``; returns (statevector ndarray, metrics).

    ``sv`` may be an existing Statevector/StatevectorF32 of the right size, reset to
    |0...0> here (avoids re-allocating HBM between runs); ``out`` an existing host array
    (e.g. pinned) that receives the result.  ``native_prep`` (default) prepares each tile's op
    list in one native call (gate matrices, fusion and packing, ``prepare_tile_ops``); with
    ``native_prep=False`` the per-gate Python path of the reference runs (``tile_ops_for``,
    ``GATE_CACHE``, ``fuse_tile_ops``), and ``native_fusion`` then fuses its packed ops natively.
    ``dense_fusion=k`` (1..6; complex64, >= 13 qubits) groups each tile's gates into blocks of at
    most k qubits (``plan_dense_blocks``) and applies every block as one dense unitary on the
    tensor cores (``apply_dense_block``: one sweep per block) instead of the pass executor.
    """
    if tile_mode not in ("cooperative", "graphed", "sequential"):
        raise ValueError(f"unknown tile_mode: {tile_mode}")
    num_qubits = qc.num_qubits
    np_dtype = np.complex64 if use_float32 else np.complex128
    qubit_map = {q: qc.find_bit(q).index for q in qc.qubits}
    t_start = time.perf_counter()
    num_tiles = len(tile_plan)
    num_reorders = num_gates = num_fused_ops = 0
    num_kernel_launches = num_graph_replays = num_dense_blocks = 0
    if dense_fusion and not use_float32:
        raise RuntimeError("dense_fusion runs complex64 states (use_float32=True)")
    t_perm = t_apply = 0.0

    if sv is None:
        sv = StatevectorF32(num_qubits) if use_float32 else Statevector(num_qubits)
    else:
        if sv.num_qubits != num_qubits or sv._np_dtype != np_dtype:
            raise RuntimeError("sv does not match the circuit size / precision")
        sv.reset()
    sv.reset_stats()
    layout = list(range(num_qubits))
    for tile in tile_plan:
        if list(tile.layout) != layout:
            t0 = time.perf_counter()
            sv.permute(layout, tile.layout)
            t_perm += time.perf_counter() - t0
            num_reorders += 1
            layout = list(tile.layout)
        t0 = time.perf_counter()
        if dense_fusion:
            ops = tile_ops_for(tile, qubit_map, np.complex128)
            num_gates += len(ops)
            blocks = plan_dense_blocks(ops, dense_fusion)
            num_fused_ops += len(blocks)
            num_dense_blocks += len(blocks)
            for qs, U in blocks:
                sv.apply_dense_block(qs, U)
            num_kernel_launches += len(blocks)
            t_apply += time.perf_counter() - t0
            continue
        if native_prep:
            ops, ng = prepare_tile_ops(tile, qubit_map, 0 if np_dtype == np.complex64 else 1, enable_fusion)
            num_gates += ng
        else:
            ops = tile_ops_for(tile, qubit_map, np_dtype)
            num_gates += len(ops)
            if ops:
                if enable_fusion and native_fusion and all(isinstance(o[-1], np.ndarray) for o in ops):
                    ops = _OpBatch(ops, 0 if np_dtype == np.complex64 else 1).fused()
                elif enable_fusion:
                    ops = fuse_tile_ops(ops)
        if len(ops):
            num_fused_ops += len(ops)
            if tile_mode == "cooperative":
                sv.apply_tile_cooperative(ops)
                num_kernel_launches += 1
            elif tile_mode == "graphed":
                sv.apply_tile_graphed(ops)
                num_graph_replays += 1
            else:
                sv.apply_tile_dev(ops)
                num_kernel_launches += len(ops)
        t_apply += time.perf_counter() - t0
    if logical_order:
        sv.permute(layout, list(range(num_qubits)))
    t0 = time.perf_counter()
    sv.synchronize()
    t_sync = time.perf_counter() - t0
    counts = None
    t_sample = 0.0
    if task == "sampling" and shots:
        # the runner's sampling task (runner.py:25-27, 74); the reference's custom backend
        # ignores it.  Device sampler; indices mapped from layout positions to circuit qubits.
        t0 = time.perf_counter()
        idx = sv.sample(int(shots))
        order = layout if not logical_order else list(range(num_qubits))
        logical = np.zeros_like(idx)
        for pos, q in enumerate(order):
            logical |= ((idx >> np.uint64(pos)) & np.uint64(1)) << np.uint64(q)
        vals, cnt = np.unique(logical, return_counts=True)
        counts = {format(int(v), f"0{num_qubits}b"): int(c) for v, c in zip(vals, cnt)}
        t_sample = time.perf_counter() - t0
    if out is not None:
        result = sv.copy_to(out)
    else:
        result = sv.to_numpy()
    st = sv.stats()
    t_total = time.perf_counter() - t_start
    fusion_ratio = num_gates / max(1, num_fused_ops) if enable_fusion else 1.0
    if tile_mode == "graphed":
        avoided = num_fused_ops - num_graph_replays
    elif tile_mode == "cooperative":
        avoided = num_fused_ops - num_tiles
    else:
        avoided = 0
    elem = 8 if use_float32 else 16
    sweep_bytes = 2 * (1 << num_qubits) * elem
    metrics = {
        "num_tiles": num_tiles,
        "num_gates": num_gates,
        "num_fused_ops": num_fused_ops,
        "fusion_ratio": fusion_ratio,
        "num_reorders": num_reorders,
        "num_kernel_launches": num_kernel_launches,
        "num_graph_replays": num_graph_replays,
        "avoided_launches": avoided,
        "t_perm_s": t_perm,
        "t_apply_s": t_apply,
        "t_sync_s": t_sync,
        "t_total_s": t_total,
        "t_launch_overhead_saved_us": avoided * KERNEL_LAUNCH_OVERHEAD_US,
        "tile_mode": tile_mode,
        # executor-side counts (not in the reference)
        "sweeps": st["sweeps"] + st["gate_sweeps"],
        "perm_sweeps": st["perm_sweeps"],
        "device_launches": st["launches"],
        "graph_builds": st["graph_builds"],
        "hbm_bytes_alg": (num_tiles + num_reorders + 1) * sweep_bytes,
        "hbm_bytes_executed": (st["sweeps"] + st["gate_sweeps"]) * sweep_bytes,
        "t_sample_s": t_sample,
        "counts": counts,
        "dense_blocks": num_dense_blocks,
    }
    return result, metrics
