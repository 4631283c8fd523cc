"""Drop-in replacement of the reference's native module ``qgpusim_cuda``.

Same classes, methods, argument names and error messages as the pybind11 module of
qgpusim/backends/custom/qgpusim_cuda/src/bindings.cpp:1004-1092:

* ``Statevector(num_qubits)`` (complex128) and ``StatevectorF32(num_qubits)`` (complex64)
  with ``apply_tile_cooperative / apply_tile_graphed / apply_tile_dev``, ``permute``,
  ``to_numpy``, ``reset``, ``synchronize``, ``num_qubits``, ``dim`` and, for both
  precisions, ``from_numpy``, ``apply_1q/2q(_dev)`` and ``apply_diagonal_1q``;
* ``apply_1q_gate(psi, U, target_qubit, num_qubits)`` and
  ``apply_2q_gate(psi, U, q0, q1, num_qubits)`` on a device array.

Tile ops are ``('1q', q0, U)`` or ``('2q', q0, q1, U)``; ``U`` may be a host array
(numpy) or a device array exposing ``__cuda_array_interface__`` (torch CUDA tensors,
CuPy).  Matrices are copied when the call returns, so the caller may free or reuse them.
All compute runs in libqsim_b200 (sm_100a); there is no CPU path.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_double, c_int, c_ulonglong, c_void_p
from typing import Iterable, List, Sequence

import numpy as np

from . import _native as N


def _host_matrix(U, dtype, shape, what: str) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(U), dtype=dtype)
    if a.shape != shape:
        raise RuntimeError(f"U must be a {shape[0]}x{shape[1]} matrix")
    return a


def _dev_info(U):
    iface = getattr(U, "__cuda_array_interface__", None)
    if iface is None:
        return None
    ptr = int(iface["data"][0])
    if ptr == 0:
        raise RuntimeError("CuPy array has null device pointer")
    return ptr, tuple(iface["shape"]), iface["typestr"], iface.get("strides")


_TYPESTR = {N.QS_C64: ("<c8", np.complex64), N.QS_C128: ("<c16", np.complex128)}


class _OpBatch:
    """Packs a Python op list into the C ``qs_op`` array, keeping host matrices alive."""

    def __init__(self, ops: Sequence, dtype_code: int):
        typestr, npdt = _TYPESTR[dtype_code]
        n = len(ops)
        self._code = dtype_code
        self.arr = np.zeros(n, dtype=N.OP_DTYPE)
        self._keep: List[np.ndarray] = []
        kinds: List[int] = []
        q0s: List[int] = []
        q1s: List[int] = []
        devs: List[int] = []
        ptrs: List[int] = []
        host_mats = []
        host_idx = []
        item = np.dtype(npdt).itemsize
        for i, op in enumerate(ops):
            t = tuple(op)
            if len(t) < 1:
                raise RuntimeError("apply_tile_dev: empty tuple op descriptor")
            kind = t[0]
            if kind == "1q":
                if len(t) != 3:
                    raise RuntimeError("apply_tile_dev: 1q expects ('1q', q0, U_dev)")
                kinds.append(N.QS_OP_1Q)
                q0s.append(int(t[1]))
                q1s.append(-1)
                U, shape = t[2], (2, 2)
            elif kind == "2q":
                if len(t) != 4:
                    raise RuntimeError("apply_tile_dev: 2q expects ('2q', q0, q1, U_dev)")
                kinds.append(N.QS_OP_2Q)
                q0s.append(int(t[1]))
                q1s.append(int(t[2]))
                U, shape = t[3], (4, 4)
            else:
                raise RuntimeError(f"apply_tile_dev: unknown op kind: {kind}")
            dev = _dev_info(U)
            if dev is not None:
                ptr, dshape, dts, strides = dev
                if dts != typestr:
                    raise RuntimeError(f"apply_tile_dev: device matrix must have typestr {typestr}, got {dts}")
                if dshape != shape or strides not in (None, (shape[1] * item, item)):
                    raise RuntimeError(f"U must be a contiguous {shape[0]}x{shape[1]} matrix")
                devs.append(1)
                ptrs.append(ptr)
                self._keep.append(U)
            else:
                host_mats.append(_host_matrix(U, npdt, shape, kind).reshape(-1))
                host_idx.append(i)
                devs.append(0)
                ptrs.append(0)
        if n:
            self.arr["kind"] = kinds
            self.arr["q0"] = q0s
            self.arr["q1"] = q1s
            self.arr["dev"] = devs
            self.arr["U"] = ptrs
        if host_mats:
            # one buffer for all host matrices; each op points at its entries
            buf = np.concatenate(host_mats)
            sizes = np.fromiter((m.size for m in host_mats), dtype=np.uint64, count=len(host_mats))
            offs = np.cumsum(sizes) - sizes  # entry offset of each matrix in buf
            self.arr["U"][np.asarray(host_idx)] = np.uint64(buf.ctypes.data) + offs * np.uint64(item)
            self._keep.append(buf)

    def fused(self) -> "_OpBatch":
        """The ops fused natively (``qs_fuse_ops``: consecutive gates on the same qubit / ordered
        pair multiplied, as ``backend.fuse_tile_ops``); host matrices only."""
        out = _OpBatch.__new__(_OpBatch)
        n = len(self.arr)
        out.arr = np.zeros(n, dtype=N.OP_DTYPE)
        mats = np.empty(16 * max(n, 1), dtype=np.complex64 if self._code == N.QS_C64 else np.complex128)
        nout = c_int()
        N.call("qs_fuse_ops", self._code, self.ptr, n, out.arr.ctypes.data, mats.ctypes.data, byref(nout))
        out.arr = out.arr[:nout.value]
        out._keep = [mats]
        out._code = self._code
        return out

    @property
    def ptr(self) -> int:
        return self.arr.ctypes.data

    def __len__(self) -> int:
        return len(self.arr)


class _StatevectorBase:
    _dtype_code = N.QS_C128
    _np_dtype = np.complex128

    def __init__(self, num_qubits: int):
        h = c_void_p()
        N.call("qs_create", int(num_qubits), self._dtype_code, byref(h))
        self._h = h

    # -- lifetime ------------------------------------------------------------------
    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                N.lib().qs_destroy(h)
            except Exception:
                pass
            self._h = None

    def close(self) -> None:
        self.__del__()

    # -- properties ------------------------------------------------------------------
    @property
    def num_qubits(self) -> int:
        v = c_int()
        N.call("qs_num_qubits", self._h, byref(v))
        return v.value

    @property
    def dim(self) -> int:
        v = c_ulonglong()
        N.call("qs_dim", self._h, byref(v))
        return v.value

    # -- state I/O ---------------------------------------------------------------------
    def to_numpy(self) -> np.ndarray:
        out = np.empty(self.dim, dtype=self._np_dtype)
        N.call("qs_copy_to_host", self._h, out.ctypes.data, out.nbytes)
        return out

    def copy_to(self, out: np.ndarray) -> np.ndarray:
        """Copy the state into an existing C-contiguous array (e.g. pinned host memory)."""
        if out.dtype != self._np_dtype or out.size != self.dim or not out.flags.c_contiguous:
            raise RuntimeError("output array must be C-contiguous with size 2^num_qubits and the state's dtype")
        N.call("qs_copy_to_host", self._h, out.ctypes.data, out.nbytes)
        return out

    def from_numpy(self, psi) -> None:
        a = np.ascontiguousarray(np.asarray(psi), dtype=self._np_dtype)
        if a.ndim != 1 or a.size != self.dim:
            raise RuntimeError("Input array must have size 2^num_qubits")
        N.call("qs_copy_from_host", self._h, a.ctypes.data, a.nbytes)

    def reset(self) -> None:
        N.call("qs_reset", self._h)

    # -- checkpoint / resume (the reference has only to_numpy / from_numpy, bindings.cpp:547-574) --
    def save(self, path: str, layout: Sequence[int] = None) -> None:
        """Write the amplitudes (current layout, the state's precision) and ``layout``
        (layout[p] = circuit qubit at bit position p; default identity) to ``path`` (.npz), so a
        run can resume from the same tile of its schedule."""
        n = self.num_qubits
        lay = np.arange(n, dtype=np.int32) if layout is None else np.asarray(layout, dtype=np.int32)
        if lay.shape != (n,) or sorted(lay.tolist()) != list(range(n)):
            raise RuntimeError("layout must be a permutation of range(num_qubits)")
        np.savez(path, psi=self.to_numpy(), layout=lay, num_qubits=np.int32(n),
                 dtype=np.array(np.dtype(self._np_dtype).str))

    def restore(self, path: str) -> List[int]:
        """Load a checkpoint written by ``save`` into this state (same size and precision);
        returns its layout."""
        with np.load(path) as z:
            psi, lay, n = z["psi"], z["layout"], int(z["num_qubits"])
            dt = str(z["dtype"])
        if n != self.num_qubits or np.dtype(dt) != np.dtype(self._np_dtype):
            raise RuntimeError("checkpoint does not match the state's size / precision")
        self.from_numpy(psi)
        return [int(x) for x in lay]

    @classmethod
    def load(cls, path: str):
        """A new state of this class from a checkpoint: (state, layout)."""
        with np.load(path) as z:
            n = int(z["num_qubits"])
        sv = cls(n)
        return sv, sv.restore(path)

    def synchronize(self) -> None:
        N.call("qs_synchronize", self._h)

    def flush(self) -> None:
        """Launch queued ops now (asynchronous)."""
        N.call("qs_flush", self._h)

    def materialize(self) -> None:
        """Launch queued ops and the data movement to the current layout (asynchronous)."""
        N.call("qs_materialize", self._h)

    def sample(self, shots: int, seed: int = 0) -> np.ndarray:
        """``shots`` basis indices drawn from |psi|^2 on the device (ascending, uint64; bit p of
        an index = layout position p).  Same seed and state give the same indices."""
        shots = int(shots)
        if shots < 0:
            raise RuntimeError("shots must be >= 0")
        out = np.zeros(shots, dtype=np.uint64)
        N.call("qs_sample", self._h, shots, int(seed) & 0xFFFFFFFFFFFFFFFF, out.ctypes.data if shots else None)
        return out

    def sample_counts(self, shots: int, seed: int = 0) -> dict:
        """Counts per outcome bitstring (qubit 0 rightmost, as Aer's ``get_counts``)."""
        idx = self.sample(shots, seed)
        vals, cnt = np.unique(idx, return_counts=True)
        n = self.num_qubits
        return {format(int(v), f"0{n}b"): int(c) for v, c in zip(vals, cnt)}

    def apply_dense(self, U, qubits: Sequence[int] = (0, 1, 2, 3, 4, 5)) -> None:
        """Dense 64x64 unitary on six layout positions in one tensor-core sweep (complex64,
        >= 13 qubits); row/column index sum_j b_{qubits[j]} 2^j.  Other positions are first
        relabelled onto 0..5 (and back), which costs in-place permutation sweeps."""
        U = np.ascontiguousarray(U, dtype=np.complex128)
        if U.shape != (64, 64):
            raise RuntimeError("U must be a 64x64 matrix")
        q = [int(x) for x in qubits]
        n = self.num_qubits
        if len(q) != 6 or len(set(q)) != 6 or any(x < 0 or x >= n for x in q):
            raise RuntimeError("apply_dense: six distinct qubit positions required")
        if q == list(range(6)):
            N.call("qs_apply_dense6", self._h, U.ctypes.data)
            return
        # label each position by itself; the new layout lists q first (positions 0..5)
        ident = list(range(n))
        moved = q + [p for p in range(n) if p not in q]
        self.permute(ident, moved)
        N.call("qs_apply_dense6", self._h, U.ctypes.data)
        self.permute(moved, ident)

    def apply_dense_block(self, qubits: Sequence[int], U) -> None:
        """Dense 2^k x 2^k unitary (k = len(qubits) <= 6) on layout positions ``qubits`` in one
        tensor-core sweep (complex64, >= 13 qubits); row/column index sum_j b_{qubits[j]} 2^j.
        No data moves to another layout (the kernel gathers the block's bits in place)."""
        q = np.ascontiguousarray([int(x) for x in qubits], dtype=np.int32)
        k = q.size
        U = np.ascontiguousarray(U, dtype=np.complex128)
        if U.shape != (1 << k, 1 << k):
            raise RuntimeError(f"U must be a {1 << k}x{1 << k} matrix")
        N.call("qs_apply_dense", self._h, int(k), q.ctypes.data, U.ctypes.data)

    # -- layout ------------------------------------------------------------------------
    def permute(self, layout_old: Sequence[int], layout_new: Sequence[int]) -> None:
        n = self.num_qubits
        if len(layout_old) != n or len(layout_new) != n:
            raise RuntimeError("layout_old/layout_new must have length num_qubits")
        a = np.ascontiguousarray(layout_old, dtype=np.int32)
        b = np.ascontiguousarray(layout_new, dtype=np.int32)
        N.call("qs_permute", self._h, a.ctypes.data, b.ctypes.data, n)

    def pos2bit(self) -> List[int]:
        n = self.num_qubits
        out = np.empty(n, dtype=np.int32)
        N.call("qs_get_pos2bit", self._h, out.ctypes.data, n)
        return out.tolist()

    # -- tiles -------------------------------------------------------------------------
    def _tile(self, ops, mode: int) -> None:
        batch = ops if isinstance(ops, _OpBatch) else _OpBatch(list(ops), self._dtype_code)
        if len(batch) == 0:
            return
        N.call("qs_apply_tile", self._h, batch.ptr, len(batch), mode)

    def apply_tile_dev(self, ops) -> None:
        self._tile(ops, N.MODES["sequential"])

    def apply_tile_graphed(self, ops) -> None:
        self._tile(ops, N.MODES["graphed"])

    def apply_tile_cooperative(self, ops) -> None:
        self._tile(ops, N.MODES["cooperative"])

    # -- single gates ------------------------------------------------------------------
    def apply_1q(self, target_qubit: int, U) -> None:
        m = _host_matrix(U, self._np_dtype, (2, 2), "1q")
        N.call("qs_apply_1q", self._h, int(target_qubit), m.ctypes.data, 0)

    def apply_2q(self, q0: int, q1: int, U) -> None:
        m = _host_matrix(U, self._np_dtype, (4, 4), "2q")
        N.call("qs_apply_2q", self._h, int(q0), int(q1), m.ctypes.data, 0)

    def apply_1q_dev(self, target_qubit: int, U_dev) -> None:
        self._tile([("1q", int(target_qubit), U_dev)], N.MODES["sequential"])

    def apply_2q_dev(self, q0: int, q1: int, U_dev) -> None:
        self._tile([("2q", int(q0), int(q1), U_dev)], N.MODES["sequential"])

    def apply_diagonal_1q(self, target_qubit: int, phase0, phase1) -> None:
        p0 = np.array([complex(phase0).real, complex(phase0).imag], dtype=np.float64)
        p1 = np.array([complex(phase1).real, complex(phase1).imag], dtype=np.float64)
        N.call("qs_apply_diagonal_1q", self._h, int(target_qubit), p0.ctypes.data, p1.ctypes.data)

    # -- extras (not in the reference) -------------------------------------------------
    def norm_squared(self) -> float:
        v = c_double()
        N.call("qs_norm_squared", self._h, byref(v))
        return v.value

    def inner(self, other: "_StatevectorBase") -> complex:
        re, im = c_double(), c_double()
        N.call("qs_inner_product", self._h, other._h, byref(re), byref(im))
        return complex(re.value, im.value)

    def stats(self) -> dict:
        st = N.QsStats()
        N.call("qs_get_stats", self._h, byref(st))
        return st.as_dict()

    def reset_stats(self) -> None:
        N.call("qs_reset_stats", self._h)

    def set_config(self, m: int = None, k: int = None, hill_iters: int = None, grid_mult: int = None,
                   jit: int = None, jit_lr: int = None, jit_blocks: int = None, jit_packed: int = None,
                   wait_limit_ns: int = None, jit_async: int = None) -> None:
        """Executor knobs: staged bits per sweep ``m``, always-staged low bits ``k``, planner
        effort ``hill_iters``, blocks per SM ``grid_mult``, specialised kernels ``jit``
        (0 auto, 1 always, -1 never) with ``jit_lr`` register bits per thread,
        ``jit_blocks`` geometry (1 double-buffered block per SM, 2 single-buffered blocks per
        SM, 3 one block of two teams over three buffers), ``jit_packed`` FP32x2 arithmetic and
        ``wait_limit_ns``, the limit of the kernels' bounded device waits (0: 20 s), and
        ``jit_async`` (1: the generic kernel runs while a new structure's specialised kernels
        compile in the background)."""
        c = N.QsConfig()
        N.call("qs_get_config", self._h, byref(c))
        if jit_async is not None:
            c.jit_async = int(jit_async)
        if wait_limit_ns is not None:
            c.wait_limit_ns = int(wait_limit_ns)
        if jit is not None:
            c.jit = jit
        if jit_lr is not None:
            c.jit_lr = jit_lr
        if jit_blocks is not None:
            c.jit_blocks = jit_blocks
        if jit_packed is not None:
            c.jit_packed = jit_packed
        if m is not None:
            c.m = m
        if k is not None:
            c.k = k
        if hill_iters is not None:
            c.hill_iters = hill_iters
        if grid_mult is not None:
            c.grid_mult = grid_mult
        N.call("qs_set_config", self._h, byref(c))

    def get_config(self) -> dict:
        c = N.QsConfig()
        N.call("qs_get_config", self._h, byref(c))
        return {"m": c.m, "k": c.k, "hill_iters": c.hill_iters, "grid_mult": c.grid_mult, "jit": c.jit,
                "jit_lr": c.jit_lr, "jit_blocks": c.jit_blocks, "jit_packed": c.jit_packed,
                "wait_limit_ns": int(c.wait_limit_ns), "jit_async": c.jit_async}

    @staticmethod
    def jit_wait() -> None:
        """Wait for every background compile of specialised kernels (``jit_async``)."""
        N.call("qs_jit_wait")

    def device_ptr(self) -> int:
        p = c_void_p()
        N.call("qs_device_ptr", self._h, byref(p))
        return int(p.value)

    @property
    def stream(self) -> int:
        p = c_void_p()
        N.call("qs_get_stream", self._h, byref(p))
        return int(p.value or 0)

    def set_stream(self, stream: int) -> None:
        N.call("qs_set_stream", self._h, c_void_p(int(stream) if stream else None))

    @property
    def __cuda_array_interface__(self) -> dict:
        ptr = self.device_ptr()
        return {"shape": (self.dim,), "typestr": _TYPESTR[self._dtype_code][0], "data": (ptr, False),
                "version": 3, "strides": None}

    def torch_view(self):
        """Zero-copy torch view of the amplitudes (current layout); valid until the next call."""
        import torch
        return torch.as_tensor(self, device="cuda")


class Statevector(_StatevectorBase):
    """complex128 statevector initialised to |0...0> (bindings.cpp:90-637)."""
    _dtype_code = N.QS_C128
    _np_dtype = np.complex128


class StatevectorF32(_StatevectorBase):
    """complex64 statevector initialised to |0...0> (bindings.cpp:643-927)."""
    _dtype_code = N.QS_C64
    _np_dtype = np.complex64


def _raw_gate(psi, U, qubits, num_qubits: int, shape) -> None:
    dev = _dev_info(psi)
    if dev is None:
        raise RuntimeError("psi must be a device array exposing __cuda_array_interface__")
    ptr, dshape, dts, _ = dev
    code = {"<c8": N.QS_C64, "<c16": N.QS_C128}.get(dts)
    if code is None:
        raise RuntimeError(f"psi must be complex64 or complex128, got {dts}")
    if dshape != (1 << num_qubits,):
        raise RuntimeError("psi must have 2^num_qubits entries")
    m = _host_matrix(np.asarray(U), _TYPESTR[code][1], shape, "gate")
    stream = _torch_current_stream()
    if len(qubits) == 1:
        N.call("qs_apply_1q_gate", ptr, code, m.ctypes.data, int(qubits[0]), int(num_qubits), stream)
    else:
        N.call("qs_apply_2q_gate", ptr, code, m.ctypes.data, int(qubits[0]), int(qubits[1]), int(num_qubits),
               stream)


def _torch_current_stream():
    try:
        import torch
        if torch.cuda.is_available():
            return c_void_p(torch.cuda.current_stream().cuda_stream)
    except Exception:
        pass
    return c_void_p(None)


def apply_1q_gate(psi, U, target_qubit: int, num_qubits: int) -> None:
    """Module function of bindings.cpp:931-962 (psi: device array, U: host 2x2)."""
    _raw_gate(psi, U, (target_qubit,), num_qubits, (2, 2))


def apply_2q_gate(psi, U, q0: int, q1: int, num_qubits: int) -> None:
    """Module function of bindings.cpp:965-1001 (psi: device array, U: host 4x4)."""
    _raw_gate(psi, U, (q0, q1), num_qubits, (4, 4))


def permute_scatter(psi_in, psi_out, map_old_to_new: Sequence[int]) -> None:
    """Reference permute kernel on device arrays: out[sum_p bit_p(i) << map[p]] = in[i]."""
    a, b = _dev_info(psi_in), _dev_info(psi_out)
    if a is None or b is None:
        raise RuntimeError("psi_in and psi_out must be device arrays")
    code = {"<c8": N.QS_C64, "<c16": N.QS_C128}.get(a[2])
    if code is None or a[2] != b[2] or a[1] != b[1]:
        raise RuntimeError("psi_in/psi_out must be equal-size complex64 or complex128 arrays")
    n = int(a[1][0]).bit_length() - 1
    mp = np.ascontiguousarray(map_old_to_new, dtype=np.int32)
    if mp.size != n:
        raise RuntimeError("map must have length num_qubits")
    N.call("qs_permute_scatter", a[0], b[0], code, n, mp.ctypes.data, _torch_current_stream())


__all__ = ["Statevector", "StatevectorF32", "apply_1q_gate", "apply_2q_gate", "permute_scatter"]
