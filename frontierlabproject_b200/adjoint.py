"""Adjoint gradients of an expectation value on the GPU, with a torch.autograd.Function.

E(theta) = <psi(theta)| H |psi(theta)>, psi(theta) = U_G(theta) ... U_1(theta) |0...0>,
H = sum_i a_i Z_i Z_{i+1} + b_i X_i (periodic).  For R(theta) = exp(-i theta G / 2):
dE/dtheta_k = Im <lam_k| G |psi_k>, with psi_k the state after gate k and
lam_k = U_{k+1}^dagger ... U_G^dagger H psi.  The reverse sweep uncomputes psi and lam
gate by gate (no stored intermediate states) and accumulates the inner products in FP64.

* ``ParamCircuit``: gates with parameter slots (``hea`` builds the hardware-efficient ansatz:
  per layer RY, RZ on every qubit, then a CZ ring).
* ``AdjointEngine``: two device states (psi, lam) reused across evaluations; ``energy``,
  ``energy_and_grad``, and ``param_shift_grad`` (two energy evaluations per parameter, the
  comparison method).
* ``AdjointExpectation``: torch.autograd.Function returning E with dE/dtheta in backward.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .gates import gate_matrix
from .qgpusim_cuda import Statevector, StatevectorF32, _OpBatch

ADJ_OP = np.dtype({"names": ["kind", "q0", "q1", "gen", "grad_index", "pad", "U"],
                   "formats": ["<i4", "<i4", "<i4", "<i4", "<i4", "<i4", "<u8"],
                   "offsets": [0, 4, 8, 12, 16, 20, 24], "itemsize": 32})
GEN = {"rx": 1, "ry": 2, "rz": 3}


class AdjOps:
    """The ``qs_adj_op`` table of a ParamCircuit (complex128 matrices in one buffer).  ``update``
    rewrites the rotations' matrices for new parameters in place (numpy over all gates of a
    generator at once); fixed gates are computed once.  The table points into this object's
    buffer: keep the object alive while the table is in use."""

    def __init__(self, pc: "ParamCircuit"):
        G = len(pc.gates)
        self.ops = np.zeros(G, dtype=ADJ_OP)
        sizes = np.array([4 if len(g.qubits) == 1 else 16 for g in pc.gates], dtype=np.int64)
        off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.buf = np.zeros(int(off[-1]), dtype=np.complex128)
        base = self.buf.ctypes.data
        rot = {1: ([], []), 2: ([], []), 3: ([], [])}
        for i, g in enumerate(pc.gates):
            o = self.ops[i]
            o["kind"] = len(g.qubits)
            o["q0"] = g.qubits[0]
            o["q1"] = g.qubits[1] if len(g.qubits) > 1 else -1
            o["U"] = base + 16 * int(off[i])
            if g.param is not None:
                if g.name not in GEN:
                    raise ValueError(f"parameterised gate {g.name!r} is not a single-qubit rotation")
                o["gen"] = GEN[g.name]
                o["grad_index"] = g.param
                rot[GEN[g.name]][0].append(int(off[i]))
                rot[GEN[g.name]][1].append(g.param)
            else:
                self.buf[off[i]:off[i + 1]] = np.asarray(gate_matrix(g.name, g.fixed), dtype=np.complex128).reshape(-1)
        self.rot = {k: (np.array(v[0], dtype=np.int64), np.array(v[1], dtype=np.int64)) for k, v in rot.items() if v[0]}

    def update(self, theta) -> np.ndarray:
        th = np.asarray(theta, dtype=np.float64)
        for gen, (offs, slots) in self.rot.items():
            h = 0.5 * th[slots]
            c, s = np.cos(h), np.sin(h)
            if gen == 1:
                M = np.stack([c, -1j * s, -1j * s, c], axis=1)
            elif gen == 2:
                M = np.stack([c, -s, s, c], axis=1).astype(np.complex128)
            else:
                z = np.zeros_like(c)
                M = np.stack([np.exp(-1j * h), z, z, np.exp(1j * h)], axis=1)
            self.buf[offs[:, None] + np.arange(4)] = M
        return self.ops


@dataclass
class ParamGate:
    name: str
    qubits: Tuple[int, ...]
    param: Optional[int] = None     # index into theta, for rx/ry/rz
    fixed: Tuple[float, ...] = ()   # parameters of non-trainable gates


@dataclass
class ParamCircuit:
    num_qubits: int
    gates: List[ParamGate] = field(default_factory=list)
    num_params: int = 0

    @staticmethod
    def hea(n: int, layers: int) -> "ParamCircuit":
        pc = ParamCircuit(n)
        k = 0
        for _ in range(layers):
            for q in range(n):
                pc.gates.append(ParamGate("ry", (q,), k)); k += 1
            for q in range(n):
                pc.gates.append(ParamGate("rz", (q,), k)); k += 1
            if n == 2:
                pc.gates.append(ParamGate("cz", (0, 1)))
            elif n > 2:
                for q in range(n):
                    pc.gates.append(ParamGate("cz", (q, (q + 1) % n)))
        pc.num_params = k
        return pc

    def matrices(self, theta) -> List[np.ndarray]:
        th = np.asarray(theta, dtype=np.float64)
        out = []
        for g in self.gates:
            p = (float(th[g.param]),) if g.param is not None else g.fixed
            out.append(gate_matrix(g.name, p))
        return out

    def to_circuit(self, theta):
        from .circuit import QuantumCircuit
        qc = QuantumCircuit(self.num_qubits)
        for g, U in zip(self.gates, self.matrices(theta)):
            qc.unitary(U, g.qubits, label=g.name)
        return qc


class AdjointEngine:
    """Energy and gradient of ``ParamCircuit`` expectations on one GPU."""

    def __init__(self, num_qubits: int, f32: bool = True, mode: str = "graphed", method: str = "auto"):
        """method: "jit" (complex64, 10..33 qubits: the forward tile and ONE reverse program over
        the stacked state psi (+) H psi, both with the plan-time specialised kernels),
        "fused" (complex64: the whole gradient in one persistent launch of the batched kernel,
        planned passes over psi and lam), "per_gate" (one reverse kernel per gate over the two
        states), "auto" (jit for complex64 with 14..33 qubits when NVRTC is available, fused
        for 2..13, per_gate otherwise)."""
        cls = StatevectorF32 if f32 else Statevector
        self.n = num_qubits
        self.f32 = f32
        self.mode = mode
        if method not in ("auto", "jit", "fused", "per_gate"):
            raise ValueError(f"unknown method: {method}")
        if method in ("fused", "jit") and not f32:
            raise ValueError(f"the {method} gradient runs complex64 states")
        if method == "jit" and not 10 <= num_qubits <= 33:
            raise ValueError("the jit gradient needs 10..33 qubits")
        if method == "auto":
            if f32 and 14 <= num_qubits <= 33 and _jit_available():
                method = "jit"
            elif f32 and 2 <= num_qubits <= 26:
                method = "fused"
            else:
                method = "per_gate"
        self.method = method
        self.psi = None if method == "jit" else cls(num_qubits)
        self.lam = None if method == "jit" else cls(num_qubits)
        self._np_dtype = np.complex64 if f32 else np.complex128
        self._fused = None      # (structure key, BatchedAdjoint)
        self._grad = None       # (structure key, qs_grad handle, AdjOps)
        self._grad_cfg = None   # plan knobs of the jit method

    def __del__(self):
        g = getattr(self, "_grad", None)
        if g is not None:
            try:
                N.lib().qs_grad_destroy(g[1])
            except Exception:  # interpreter shutdown: the library may already be unloaded
                pass
            self._grad = None

    def set_config(self, **kw) -> None:
        """Executor knobs (``StatevectorF32.set_config``); the jit method takes ``m``, ``k``,
        ``hill_iters`` and ``jit_lr`` (5 or 6) for its plans (applied to the next handle)."""
        if self.method == "jit":
            allowed = {"m", "k", "hill_iters", "jit_lr"}
            if set(kw) - allowed:
                raise ValueError(f"the jit gradient takes only {sorted(allowed)}")
            self._grad_cfg = dict(self._grad_cfg or {}, **kw)
            if self._grad is not None:
                N.lib().qs_grad_destroy(self._grad[1])
                self._grad = None
            return
        self.psi.set_config(**kw)
        self.lam.set_config(**kw)

    def _forward(self, pc: ParamCircuit, theta) -> List[np.ndarray]:
        if pc.num_qubits != self.n:
            raise ValueError("circuit size differs from the engine's")
        mats = pc.matrices(theta)
        ops = []
        for g, U in zip(pc.gates, mats):
            if len(g.qubits) == 1:
                ops.append(("1q", g.qubits[0], U))
            else:
                ops.append(("2q", g.qubits[0], g.qubits[1], U))
        self.psi.reset()
        batch = _OpBatch(ops, 0 if self.f32 else 1)
        {"graphed": self.psi.apply_tile_graphed, "cooperative": self.psi.apply_tile_cooperative,
         "sequential": self.psi.apply_tile_dev}[self.mode](batch)
        return mats

    def energy(self, pc: ParamCircuit, theta, a, b) -> float:
        if self.method == "jit":
            return self._jit_energy_and_grad(pc, theta, a, b, grad=False)[0]
        self._forward(pc, theta)
        return self._expect(a, b)

    def _expect(self, a, b) -> float:
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        if a.size != self.n or b.size != self.n:
            raise ValueError("observable coefficients must have num_qubits entries")
        e = ctypes.c_double()
        N.call("qs_expect_zz_x", self.psi._h, self.lam._h, a.ctypes.data, b.ctypes.data, ctypes.byref(e))
        return e.value

    def energy_and_grad(self, pc: ParamCircuit, theta, a, b) -> Tuple[float, np.ndarray]:
        if self.method == "jit":
            return self._jit_energy_and_grad(pc, theta, a, b)
        if self.method == "fused":
            return self._fused_energy_and_grad(pc, theta, a, b)
        return self._per_gate_energy_and_grad(pc, theta, a, b)

    def _jit_energy_and_grad(self, pc: ParamCircuit, theta, a, b, grad: bool = True) -> Tuple[float, np.ndarray]:
        if pc.num_qubits != self.n:
            raise ValueError("circuit size differs from the engine's")
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        if a.size != self.n or b.size != self.n:
            raise ValueError("observable coefficients must have num_qubits entries")
        key = (tuple((g.name, g.qubits, g.param, g.fixed) for g in pc.gates), pc.num_params)
        if self._grad is None or self._grad[0] != key:
            if self._grad is not None:
                N.lib().qs_grad_destroy(self._grad[1])
                self._grad = None
            tab = AdjOps(pc)
            ops = tab.update(theta)
            h = ctypes.c_void_p()
            cfg = None
            if self._grad_cfg:
                c = N.QsConfig(13, 3, 16, 0, 1, 5, 2, 0)
                for name, v in self._grad_cfg.items():
                    setattr(c, name, int(v))
                cfg = ctypes.byref(c)
            N.call("qs_grad_create", self.n, ops.ctypes.data, len(ops), pc.num_params, cfg, ctypes.byref(h))
            self._grad = (key, h, tab)
        h, tab = self._grad[1], self._grad[2]
        ops = tab.update(theta)
        E = ctypes.c_double()
        G = np.zeros(pc.num_params, dtype=np.float64)
        N.call("qs_grad_run", h, ops.ctypes.data, len(ops), a.ctypes.data, b.ctypes.data, ctypes.byref(E),
               G.ctypes.data if grad else None)
        return float(E.value), G

    def info(self) -> dict:
        """jit method: sweeps of the last forward run and of the reverse program, register phases
        of the reverse program, gradient terms, and the handle's execution counters."""
        if self._grad is None:
            return {}
        fs, rs, ph, nt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        N.call("qs_grad_info", self._grad[1], ctypes.byref(fs), ctypes.byref(rs), ctypes.byref(ph), ctypes.byref(nt))
        st = N.QsStats()
        N.call("qs_grad_stats", self._grad[1], ctypes.byref(st))
        return {"forward_sweeps": fs.value, "reverse_sweeps": rs.value, "reverse_phases": ph.value,
                "terms": nt.value, **st.as_dict()}

    def _fused_energy_and_grad(self, pc: ParamCircuit, theta, a, b) -> Tuple[float, np.ndarray]:
        from .batch import BatchedAdjoint, BatchShape, Instance
        if pc.num_qubits != self.n:
            raise ValueError("circuit size differs from the engine's")
        inst = Instance(pc, np.asarray(theta, dtype=np.float64), np.asarray(a, dtype=np.float64),
                        np.asarray(b, dtype=np.float64))
        key = (tuple((g.name, g.qubits, g.param) for g in pc.gates), pc.num_params)
        if self._fused is None or self._fused[0] != key:
            # 12 staged bits: two blocks per SM (measured faster than 13 for one instance)
            self._fused = (key, BatchedAdjoint([inst], BatchShape(m=12, small_max=12, chunk=1, threads=256)))
        else:
            self._fused[1].update([inst])
        E, G = self._fused[1].energies_and_grads()
        return float(E[0]), G[0]

    def _per_gate_energy_and_grad(self, pc: ParamCircuit, theta, a, b) -> Tuple[float, np.ndarray]:
        mats = self._forward(pc, theta)
        E = self._expect(a, b)
        ops = np.zeros(len(pc.gates), dtype=ADJ_OP)
        store = [np.ascontiguousarray(U, dtype=np.complex128) for U in mats]
        for i, (g, U) in enumerate(zip(pc.gates, store)):
            ops[i]["kind"] = len(g.qubits)
            ops[i]["q0"] = g.qubits[0]
            ops[i]["q1"] = g.qubits[1] if len(g.qubits) > 1 else -1
            if g.param is not None:
                ops[i]["gen"] = GEN[g.name]
                ops[i]["grad_index"] = g.param
            ops[i]["U"] = U.ctypes.data
        grads = np.zeros(pc.num_params, dtype=np.float64)
        N.call("qs_adjoint_sweep", self.psi._h, self.lam._h, ops.ctypes.data, len(ops), grads.ctypes.data,
               pc.num_params)
        return E, grads

    def param_shift_grad(self, pc: ParamCircuit, theta, a, b, params: Optional[Sequence[int]] = None) -> np.ndarray:
        """dE/dtheta_k = (E(theta + pi/2 e_k) - E(theta - pi/2 e_k)) / 2 for the listed slots."""
        th = np.array(theta, dtype=np.float64)
        ks = range(pc.num_params) if params is None else params
        out = np.zeros(len(list(ks)) if params is not None else pc.num_params)
        for j, k in enumerate(ks):
            tp, tm = th.copy(), th.copy()
            tp[k] += math.pi / 2
            tm[k] -= math.pi / 2
            out[j] = 0.5 * (self.energy(pc, tp, a, b) - self.energy(pc, tm, a, b))
        return out


def _jit_available() -> bool:
    """NVRTC (the specialised kernels' compiler) can be loaded."""
    import ctypes.util
    for name in ("libnvrtc.so.12", "libnvrtc.so"):
        try:
            ctypes.CDLL(name)
            return True
        except OSError:
            continue
    return os.path.exists("/usr/local/cuda/lib64/libnvrtc.so.12")


def grad_emulate(pc: ParamCircuit, theta, psi: np.ndarray, lam: np.ndarray) -> np.ndarray:
    """Host interpretation of the jit method's reverse program (CPU tests): gradients from the
    final state psi = U|0> and lam = H psi (complex64)."""
    tab = AdjOps(pc)
    ops = tab.update(theta)
    psi = np.ascontiguousarray(psi, dtype=np.complex64)
    lam = np.ascontiguousarray(lam, dtype=np.complex64)
    G = np.zeros(pc.num_params, dtype=np.float64)
    N.call("qs_grad_emulate", pc.num_qubits, ops.ctypes.data, len(ops), pc.num_params, None, psi.ctypes.data,
           lam.ctypes.data, G.ctypes.data)
    return G


def _torch_function():
    import torch

    class AdjointExpectation(torch.autograd.Function):
        """E = <psi(theta)|H|psi(theta)>; backward multiplies the adjoint gradient."""

        @staticmethod
        def forward(ctx, theta, engine: AdjointEngine, pc: ParamCircuit, a, b):
            th = theta.detach().to("cpu", torch.float64).numpy()
            E, g = engine.energy_and_grad(pc, th, a, b)
            ctx.save_for_backward(torch.as_tensor(g, dtype=theta.dtype, device=theta.device))
            return torch.tensor(E, dtype=theta.dtype, device=theta.device)

        @staticmethod
        def backward(ctx, gout):
            (g,) = ctx.saved_tensors
            return gout * g, None, None, None, None

    return AdjointExpectation


def expectation(theta, engine: AdjointEngine, pc: ParamCircuit, a, b):
    """Differentiable E(theta) (torch tensor in, scalar tensor out)."""
    return _torch_function().apply(theta, engine, pc, a, b)
