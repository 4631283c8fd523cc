"""Batched variational workload: energies and full adjoint gradients of many circuits of
uneven qubit count in one persistent launch per batch, with a tile-shape autotuner.

Each instance is a ``ParamCircuit`` (parameterised rotations R(theta) = exp(-i theta G/2),
fixed gates), its parameters and an observable H = sum_i a_i Z_i Z_{i+1} + b_i X_i.  Small
instances (n <= ``small_max``) run wholly in shared memory; larger ones stream their states
from an HBM arena in planned passes of 2^m staged amplitudes (``m``), ``chunk`` groups per
work item.  ``autotune`` times candidate shapes on the batch itself and keeps the fastest
(cached by the batch's size signature, in the process and in a JSON file).

The device code is libqsim_b200's ``batch_kernel`` (C ABI ``qs_batch_*``); ``emulate`` runs
the same program on the host (FP64) for tests.
"""
from __future__ import annotations

import ctypes
import itertools
import json
import os
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .adjoint import ADJ_OP, GEN, ParamCircuit


class QsBatchInstance(ctypes.Structure):
    _fields_ = [("num_qubits", ctypes.c_int), ("ops", ctypes.c_void_p), ("nops", ctypes.c_int),
                ("nparams", ctypes.c_int), ("a", ctypes.c_void_p), ("b", ctypes.c_void_p)]


class QsBatchConfig(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int), ("small_max", ctypes.c_int), ("chunk", ctypes.c_int),
                ("threads", ctypes.c_int), ("blocks_per_sm", ctypes.c_int), ("pad", ctypes.c_int),
                ("wait_limit_ns", ctypes.c_ulonglong)]


@dataclass
class Instance:
    circuit: ParamCircuit
    theta: np.ndarray
    a: np.ndarray
    b: np.ndarray


@dataclass(frozen=True)
class BatchShape:
    m: int = 13
    small_max: int = 13
    chunk: int = 4
    threads: int = 256
    blocks_per_sm: int = 0
    wait_limit_ns: int = 0   # dependency waits of the kernel (0: the library default, 10 s)

    def c(self) -> QsBatchConfig:
        return QsBatchConfig(self.m, self.small_max, self.chunk, self.threads, self.blocks_per_sm, 0,
                             self.wait_limit_ns)


def hea_batch(count: int, n_range=(12, 22), l_range=(4, 16), seed: int = 0) -> List[Instance]:
    """``count`` hardware-efficient-ansatz instances with n ~ U{n_range}, L ~ U{l_range},
    theta ~ U[-pi, pi), a, b ~ N(0, 1) (each instance its own)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        L = int(rng.integers(l_range[0], l_range[1] + 1))
        pc = ParamCircuit.hea(n, L)
        out.append(Instance(pc, rng.uniform(-np.pi, np.pi, pc.num_params), rng.standard_normal(n),
                            rng.standard_normal(n)))
    return out


class _Packed:
    """C descriptors of a list of instances (keeps the buffers alive)."""

    def __init__(self, insts: Sequence[Instance]):
        self.keep = []
        self.arr = (QsBatchInstance * len(insts))()
        for i, inst in enumerate(insts):
            pc = inst.circuit
            mats = pc.matrices(inst.theta)
            ops = np.zeros(len(pc.gates), dtype=ADJ_OP)
            for k, (g, U) in enumerate(zip(pc.gates, mats)):
                U = np.ascontiguousarray(U, dtype=np.complex128)
                self.keep.append(U)
                ops[k]["kind"] = len(g.qubits)
                ops[k]["q0"] = g.qubits[0]
                ops[k]["q1"] = g.qubits[1] if len(g.qubits) > 1 else -1
                if g.param is not None:
                    ops[k]["gen"] = GEN[g.name]
                    ops[k]["grad_index"] = g.param
                ops[k]["U"] = U.ctypes.data
            a = np.ascontiguousarray(inst.a, dtype=np.float64)
            b = np.ascontiguousarray(inst.b, dtype=np.float64)
            if a.size != pc.num_qubits or b.size != pc.num_qubits:
                raise ValueError("observable coefficients must have num_qubits entries")
            self.keep += [ops, a, b]
            self.arr[i] = QsBatchInstance(pc.num_qubits, ops.ctypes.data, len(ops), pc.num_params, a.ctypes.data,
                                          b.ctypes.data)
        self.nparams = [inst.circuit.num_params for inst in insts]

    def split(self, flat: np.ndarray) -> List[np.ndarray]:
        out, k = [], 0
        for p in self.nparams:
            out.append(flat[k:k + p].copy())
            k += p
        return out


def emulate(insts: Sequence[Instance], shape: BatchShape = BatchShape()) -> Tuple[np.ndarray, List[np.ndarray]]:
    """Host (FP64) run of the batch's device program: energies and gradients."""
    P = _Packed(insts)
    E = np.zeros(len(insts))
    G = np.zeros(sum(P.nparams))
    cfg = shape.c()
    N.call("qs_batch_emulate", ctypes.cast(P.arr, ctypes.c_void_p), len(insts), ctypes.byref(cfg),
           E.ctypes.data, G.ctypes.data)
    return E, P.split(G)


def describe(insts: Sequence[Instance], shape: BatchShape = BatchShape()) -> List[Dict[str, int]]:
    """Host-side plan of the batch, per instance: passes, passes run in register phases,
    register phases, gates and work items (no device work)."""
    P = _Packed(insts)
    S = np.zeros(5 * len(insts), dtype=np.int32)
    cfg = shape.c()
    N.call("qs_batch_describe", ctypes.cast(P.arr, ctypes.c_void_p), len(insts), ctypes.byref(cfg), S.ctypes.data)
    keys = ("passes", "register_passes", "phases", "gates", "items")
    return [dict(zip(keys, map(int, S[5 * i:5 * i + 5]))) for i in range(len(insts))]


class BatchedAdjoint:
    """One device batch: ``run`` launches the persistent kernel, ``results`` waits and returns
    (energies, per-instance gradients); ``update`` sets new parameters / observables."""

    def __init__(self, insts: Sequence[Instance], shape: Optional[BatchShape] = None):
        self.insts = list(insts)
        self.shape = shape or BatchShape()
        self._packed = _Packed(self.insts)
        h = ctypes.c_void_p()
        cfg = self.shape.c()
        N.call("qs_batch_create", ctypes.cast(self._packed.arr, ctypes.c_void_p), len(self.insts), ctypes.byref(cfg),
               ctypes.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                N.lib().qs_batch_destroy(h)
            except Exception:  # interpreter shutdown: the library may already be unloaded
                pass
            self._h = None

    def update(self, insts: Sequence[Instance]) -> None:
        self.insts = list(insts)
        self._packed = _Packed(self.insts)
        N.call("qs_batch_set_params", self._h, ctypes.cast(self._packed.arr, ctypes.c_void_p), len(self.insts))

    def run(self, stream: int = 0, timed: bool = False) -> Optional[float]:
        """Launch on ``stream`` (0: legacy default); timed: wait and return device ms."""
        ms = ctypes.c_float()
        N.call("qs_batch_run", self._h, ctypes.c_void_p(stream or None), ctypes.byref(ms) if timed else None)
        return ms.value if timed else None

    def results(self) -> Tuple[np.ndarray, List[np.ndarray]]:
        E = np.zeros(len(self.insts))
        G = np.zeros(sum(self._packed.nparams))
        N.call("qs_batch_results", self._h, E.ctypes.data, G.ctypes.data)
        return E, self._packed.split(G)

    def info(self) -> Dict[str, int]:
        ni, npar, grid = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ab = ctypes.c_longlong()
        N.call("qs_batch_info", self._h, ctypes.byref(ni), ctypes.byref(npar), ctypes.byref(ab), ctypes.byref(grid))
        return {"items": ni.value, "params": npar.value, "arena_bytes": ab.value, "grid": grid.value}

    def energies_and_grads(self) -> Tuple[np.ndarray, List[np.ndarray]]:
        self.run()
        return self.results()


# ---- autotuner ---------------------------------------------------------------------------
_TUNED: Dict[tuple, BatchShape] = {}


def autotune_cache_path() -> str:
    """JSON file of tuned shapes: $QSIM_AUTOTUNE_CACHE, else ~/.cache/qsim_b200/autotune.json."""
    p = os.environ.get("QSIM_AUTOTUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "qsim_b200", "autotune.json")


def _device_tag() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(torch.cuda.current_device())
    except Exception:
        pass
    return "unknown-device"


def _cache_key(sig: tuple) -> str:
    return _device_tag() + "|" + json.dumps([[list(k), v] for k, v in sig])


def _load_cache(path: str) -> Dict[str, dict]:
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def _store_cache(path: str, key: str, shape: BatchShape) -> None:
    d = _load_cache(path)
    d[key] = {"m": shape.m, "small_max": shape.small_max, "chunk": shape.chunk, "threads": shape.threads,
              "blocks_per_sm": shape.blocks_per_sm}
    try:
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # an unwritable cache only costs a re-tune in the next process


def _signature(insts: Sequence[Instance]) -> tuple:
    """Size signature of a batch: count of instances per (qubits, gates) bucket."""
    hist: Dict[tuple, int] = {}
    for inst in insts:
        key = (inst.circuit.num_qubits, len(inst.circuit.gates) // 64)
        hist[key] = hist.get(key, 0) + 1
    return tuple(sorted(hist.items()))


def candidate_shapes(max_qubits: int) -> List[BatchShape]:
    shapes = []
    for m, small, chunk, threads in itertools.product((12, 13), (12, 13), (2, 4, 8), (256, 512)):
        if max_qubits - m > 14:
            continue
        shapes.append(BatchShape(m=m, small_max=small, chunk=chunk, threads=threads))
    return shapes


def autotune(insts: Sequence[Instance], shapes: Optional[Sequence[BatchShape]] = None, reps: int = 2,
             verbose: bool = False, cache_path: Optional[str] = None, persist: bool = True) -> BatchShape:
    """Time each candidate shape on this batch (device time of the launch, best of ``reps``)
    and return the fastest.  Results are cached by the batch's size signature and the device
    name, in this process and (``persist``) in the JSON file ``cache_path`` (default
    ``autotune_cache_path()``), so a later process with a batch of the same sizes skips the
    timing runs."""
    sig = _signature(insts)
    if sig in _TUNED:
        return _TUNED[sig]
    path = cache_path or autotune_cache_path()
    key = _cache_key(sig)
    if persist:
        hit = _load_cache(path).get(key)
        if hit is not None:
            try:
                shape = BatchShape(**{k: int(hit[k]) for k in ("m", "small_max", "chunk", "threads",
                                                                "blocks_per_sm")})
                _TUNED[sig] = shape
                return shape
            except (KeyError, TypeError, ValueError):
                pass
    nmax = max(inst.circuit.num_qubits for inst in insts)
    best, best_ms = None, float("inf")
    for shape in (shapes or candidate_shapes(nmax)):
        try:
            b = BatchedAdjoint(insts, shape)
        except RuntimeError:
            continue
        b.run(timed=True)  # warm-up
        ms = min(b.run(timed=True) for _ in range(reps))
        b.results()
        if verbose:
            print(f"autotune {shape}: {ms:.3f} ms")
        if ms < best_ms:
            best, best_ms = shape, ms
        del b
    if best is None:
        raise RuntimeError("autotune: no candidate shape runs this batch")
    _TUNED[sig] = best
    if persist:
        _store_cache(path, key, best)
    return best
