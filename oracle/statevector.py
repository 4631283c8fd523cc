"""CPU oracle for the tile executor -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may use this module, and only as the checker.  The product path never imports it.

Restates, in numpy FP64 (or FP32), the reference's per-gate arithmetic and tile
loop on the CPU:

* 1-qubit gate on pair (i0, i0 + 2^q)           -- qgpusim_cuda/src/kernels.cu:10-50
* 2-qubit gate, index b_q0 + 2 b_q1             -- kernels.cu:56-137
* diagonal 1-qubit gate                          -- kernels.cu:142-160
* permute: map building + scatter out[j] = in[i] -- bindings.cpp:434-464, kernels.cu:165-185
* tile loop: permute when the layout changes, then the tile's (fused) ops at
  local bit positions                            -- qgpusim/backends/custom/backend.py:416-482
* same-qubit fusion U_new = U @ U_prev           -- backend.py:88-200
* normalised overlap                             -- qgpusim/metrics/correctness.py:22-38

Pinned against ``tests/golden`` (fixtures produced by the reference's own Python
executor, see tests/golden/make_golden.py).
"""
from __future__ import annotations

import numpy as np


# ------------------------------------------------------------------------------------
# per-gate kernels
# ------------------------------------------------------------------------------------
def apply_1q(psi: np.ndarray, U: np.ndarray, q: int) -> None:
    """psi[i0], psi[i1] <- U @ (psi[i0], psi[i1]) for every i0 with bit q clear, i1 = i0 | 2^q."""
    n = psi.size.bit_length() - 1
    v = psi.reshape(1 << (n - q - 1), 2, 1 << q)
    a0 = v[:, 0, :].copy()
    a1 = v[:, 1, :].copy()
    U = np.asarray(U, dtype=psi.dtype)
    v[:, 0, :] = U[0, 0] * a0 + U[0, 1] * a1
    v[:, 1, :] = U[1, 0] * a0 + U[1, 1] * a1


def apply_2q(psi: np.ndarray, U: np.ndarray, q0: int, q1: int) -> None:
    """4x4 U on the quadruple of (q0, q1); matrix index = b_q0 + 2*b_q1."""
    if q0 == q1:
        raise ValueError("q0 and q1 must be different")
    n = psi.size.bit_length() - 1
    lo, hi = min(q0, q1), max(q0, q1)
    v = psi.reshape(1 << (n - hi - 1), 2, 1 << (hi - lo - 1), 2, 1 << lo)
    # v[a, b_hi, c, b_lo, d]
    amp = {}
    for bh in (0, 1):
        for bl in (0, 1):
            b_q0 = bl if q0 == lo else bh
            b_q1 = bh if q0 == lo else bl
            amp[b_q0 + 2 * b_q1] = (bh, bl, v[:, bh, :, bl, :].copy())
    U = np.asarray(U, dtype=psi.dtype)
    for r in range(4):
        bh, bl, _ = amp[r]
        acc = U[r, 0] * amp[0][2]
        for c in range(1, 4):
            acc = acc + U[r, c] * amp[c][2]
        v[:, bh, :, bl, :] = acc


def apply_diagonal_1q(psi: np.ndarray, phase0, phase1, q: int) -> None:
    n = psi.size.bit_length() - 1
    v = psi.reshape(1 << (n - q - 1), 2, 1 << q)
    v[:, 0, :] *= phase0
    v[:, 1, :] *= phase1


def permute_map(layout_old, layout_new) -> list:
    """map_old_to_new[p_old] = position of layout_old[p_old] in layout_new, with the
    reference's validation and messages (bindings.cpp:434-464)."""
    n = len(layout_new)
    if len(layout_old) != n:
        raise RuntimeError("layout_old/layout_new must have length num_qubits")
    new_pos = [-1] * n
    for p, gq in enumerate(layout_new):
        if gq < 0 or gq >= n:
            raise RuntimeError("layout_new contains invalid qubit id")
        if new_pos[gq] != -1:
            raise RuntimeError("layout_new is not a permutation")
        new_pos[gq] = p
    out = []
    for gq in layout_old:
        if gq < 0 or gq >= n:
            raise RuntimeError("layout_old contains invalid qubit id")
        out.append(new_pos[gq])
    return out


def permute_scatter(psi: np.ndarray, layout_old, layout_new) -> np.ndarray:
    """out[j] = in[i], j = sum_p bit_p(i) << map_old_to_new[p]."""
    n = psi.size.bit_length() - 1
    mp = permute_map(list(layout_old), list(layout_new))
    i = np.arange(1 << n, dtype=np.uint64)
    j = np.zeros_like(i)
    for p in range(n):
        j |= ((i >> np.uint64(p)) & np.uint64(1)) << np.uint64(mp[p])
    out = np.empty_like(psi)
    out[j] = psi
    return out


# ------------------------------------------------------------------------------------
# fusion and the tile loop
# ------------------------------------------------------------------------------------
def _touches(op, qs) -> bool:
    if op[0] == "1q":
        return op[1] in qs
    return op[1] in qs or op[2] in qs


def fuse_ops(ops: list) -> list:
    """Same-qubit 1q runs and same-ordered-pair 2q runs, U_new = U @ U_prev."""
    if len(ops) <= 1:
        return list(ops)
    out: list = []
    last: dict = {}
    for op in ops:
        if op[0] == "1q":
            q, U = op[1], op[2]
            idx = last.get(q)
            if idx is not None and out[idx][0] == "1q" and out[idx][1] == q and \
                    not any(_touches(o, (q,)) for o in out[idx + 1:]):
                out[idx] = ("1q", q, np.asarray(U) @ np.asarray(out[idx][2]))
                continue
            last[q] = len(out)
            out.append(("1q", q, U))
        else:
            q0, q1, U = op[1], op[2], op[3]
            prev = None
            for i in range(len(out) - 1, -1, -1):
                o = out[i]
                if o[0] == "2q" and o[1] == q0 and o[2] == q1:
                    prev = i
                    break
                if _touches(o, (q0, q1)):
                    break
            if prev is not None and not any(_touches(o, (q0, q1)) for o in out[prev + 1:]):
                out[prev] = ("2q", q0, q1, np.asarray(U) @ np.asarray(out[prev][3]))
                last[q0] = prev
                last[q1] = prev
                continue
            last[q0] = len(out)
            last[q1] = len(out)
            out.append(("2q", q0, q1, U))
    return out


def tile_ops_from_tile(tile, qubit_index, dtype=np.complex128) -> list:
    """('1q', local, U) / ('2q', l0, l1, U) for the unitary nodes of a tile (backend.py:432-451)."""
    ops = []
    for node in tile.gates:
        op = node.op
        if not hasattr(op, "to_matrix"):
            continue
        U = np.asarray(op.to_matrix(), dtype=dtype)
        loc = [tile.global_to_local_map[qubit_index[q]] for q in node.qargs]
        if len(loc) == 1:
            ops.append(("1q", loc[0], U))
        elif len(loc) == 2:
            ops.append(("2q", loc[0], loc[1], U))
    return ops


def run_tile_plan(qc, tile_plan, dtype=np.complex128, fuse: bool = True):
    """The reference's native executor loop on the CPU.  Returns (psi, final layout)."""
    n = qc.num_qubits
    qindex = {q: qc.find_bit(q).index for q in qc.qubits}
    psi = np.zeros(1 << n, dtype=dtype)
    psi[0] = 1.0
    layout = list(range(n))
    for tile in tile_plan:
        if list(tile.layout) != layout:
            psi = permute_scatter(psi, layout, tile.layout)
            layout = list(tile.layout)
        ops = tile_ops_from_tile(tile, qindex, dtype)
        if fuse:
            ops = fuse_ops(ops)
        for op in ops:
            if op[0] == "1q":
                apply_1q(psi, op[2], op[1])
            else:
                apply_2q(psi, op[3], op[1], op[2])
    return psi, layout


def simulate(qc, dtype=np.complex128, psi0=None) -> np.ndarray:
    """Plain gate-by-gate simulation in logical qubit order (identity layout)."""
    n = qc.num_qubits
    qindex = {q: qc.find_bit(q).index for q in qc.qubits}
    if psi0 is None:
        psi = np.zeros(1 << n, dtype=dtype)
        psi[0] = 1.0
    else:
        psi = np.array(psi0, dtype=dtype)
    for ins in qc.data:
        op = ins.operation
        if not hasattr(op, "to_matrix"):
            continue
        qs = [qindex[q] for q in ins.qubits]
        U = np.asarray(op.to_matrix(), dtype=dtype)
        if len(qs) == 1:
            apply_1q(psi, U, qs[0])
        elif len(qs) == 2:
            apply_2q(psi, U, qs[0], qs[1])
        else:
            raise ValueError(f"oracle handles 1- and 2-qubit gates, got {len(qs)}")
    return psi


def to_layout(psi: np.ndarray, layout) -> np.ndarray:
    """Logical-order state -> physical layout ``layout`` (layout[pos] = qubit at bit pos)."""
    n = len(layout)
    return permute_scatter(psi, list(range(n)), list(layout))


# ------------------------------------------------------------------------------------
# metrics
# ------------------------------------------------------------------------------------
def statevector_overlap(a, b):
    """Normalised |<a|b>| and the l2 norm of the difference (correctness.py:22-38)."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    a = a / np.linalg.norm(a)
    b = b / np.linalg.norm(b)
    return float(abs(np.vdot(a, b))), float(np.linalg.norm(a - b))


def infidelity(ref, psi) -> float:
    """1 - |<ref|psi>|^2 for normalised vectors, accumulated in FP64."""
    ov, _ = statevector_overlap(ref, psi)
    return max(0.0, 1.0 - ov * ov)


# ------------------------------------------------------------------------------------
# observable and adjoint gradient (FP64) for the hardware-efficient ansatz
# ------------------------------------------------------------------------------------
def zz_x_apply(psi: np.ndarray, a, b) -> np.ndarray:
    """H psi for H = sum_i a_i Z_i Z_{i+1} + b_i X_i, periodic (i+1 mod n)."""
    n = psi.size.bit_length() - 1
    idx = np.arange(psi.size, dtype=np.int64)
    diag = np.zeros(psi.size, dtype=np.float64)
    for i in range(n):
        zp = 1 - 2 * ((idx >> i) & 1)
        zq = 1 - 2 * ((idx >> ((i + 1) % n)) & 1)
        diag += a[i] * zp * zq
    out = diag * psi
    for i in range(n):
        out += b[i] * psi[idx ^ (1 << i)]
    return out


def energy(psi, a, b) -> float:
    return float(np.real(np.vdot(psi, zz_x_apply(psi, a, b))))


def adjoint_gradient(qc, a, b):
    """dE/dtheta for every rx/ry/rz gate of ``qc`` in circuit order, FP64 adjoint method."""
    qindex = {q: qc.find_bit(q).index for q in qc.qubits}
    psi = simulate(qc, np.complex128)
    lam = zz_x_apply(psi, a, b)
    E = float(np.real(np.vdot(psi, lam)))
    paulis = {"x": np.array([[0, 1], [1, 0]], dtype=np.complex128),
              "y": np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
              "z": np.array([[1, 0], [0, -1]], dtype=np.complex128)}
    grads = []
    for ins in reversed(qc.data):
        op = ins.operation
        if not hasattr(op, "to_matrix"):
            continue
        qs = [qindex[q] for q in ins.qubits]
        U = op.to_matrix()
        if op.name in ("rx", "ry", "rz"):
            g = psi.copy()
            apply_1q(g, paulis[op.name[1]], qs[0])
            # dE/dtheta = 2 Re <lam| dU/dtheta |psi_prev> = Im <lam| G |psi_k>
            grads.append(float(np.imag(np.vdot(lam, g))))
        Ud = U.conj().T
        if len(qs) == 1:
            apply_1q(psi, Ud, qs[0]); apply_1q(lam, Ud, qs[0])
        else:
            apply_2q(psi, Ud, qs[0], qs[1]); apply_2q(lam, Ud, qs[0], qs[1])
    return E, np.array(grads[::-1])


# ------------------------------------------------------------------------------------
# the same gate-by-gate simulation through the C/OpenMP restatement (oracle/cpu_kernels.c)
# ------------------------------------------------------------------------------------
def simulate_c(qc, dtype=np.complex128, psi0=None) -> np.ndarray:
    """``simulate`` run by the C/OpenMP kernels (one pass per gate, all host cores): the FP64
    checker for states too large for the numpy loop."""
    import ctypes
    from . import build as _build
    lib = ctypes.CDLL(_build.build())
    suf = "c128" if np.dtype(dtype) == np.complex128 else "c64"
    real = np.float64 if suf == "c128" else np.float32
    run = getattr(lib, f"qo_run_ops_{suf}")
    run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                    ctypes.c_void_p, ctypes.c_void_p]
    n = qc.num_qubits
    qindex = {q: qc.find_bit(q).index for q in qc.qubits}
    kinds, q0s, q1s, mats = [], [], [], []
    for ins in qc.data:
        op = ins.operation
        if not hasattr(op, "to_matrix"):
            continue
        qs = [qindex[q] for q in ins.qubits]
        U = np.zeros(16, dtype=np.complex128)
        M = np.asarray(op.to_matrix(), dtype=np.complex128).reshape(-1)
        U[:M.size] = M
        if len(qs) == 1:
            kinds.append(1); q0s.append(qs[0]); q1s.append(-1)
        elif len(qs) == 2:
            kinds.append(2); q0s.append(qs[0]); q1s.append(qs[1])
        else:
            raise ValueError(f"oracle handles 1- and 2-qubit gates, got {len(qs)}")
        mats.append(U)
    if psi0 is None:
        psi = np.zeros(1 << n, dtype=dtype)
        psi[0] = 1.0
    else:
        psi = np.array(psi0, dtype=dtype)
    if not kinds:
        return psi
    k = np.asarray(kinds, dtype=np.int32)
    a = np.asarray(q0s, dtype=np.int32)
    b = np.asarray(q1s, dtype=np.int32)
    Us = np.ascontiguousarray(np.stack(mats).view(np.float64).astype(real))  # 32 reals per op
    run(psi.ctypes.data, n, len(kinds), k.ctypes.data, a.ctypes.data, b.ctypes.data, Us.ctypes.data)
    return psi
