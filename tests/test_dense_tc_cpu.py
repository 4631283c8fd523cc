"""Tensor-core operand of the dense 6-qubit unitary, checked on the host: decode the canonical
layout, emulate D = X_hi W_hi^T + X_hi W_lo^T + X_lo W_hi^T with the kernel's BF16 split of X, and
compare with U x."""
import ctypes

import numpy as np

from frontierlabproject_b200 import _native as N


def _bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> nearest-even BF16, returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32)


def _decode(buf: np.ndarray) -> np.ndarray:
    """(128, 128) float32 matrix from one canonical K-major BF16 operand (32 KiB)."""
    b16 = buf.view(np.uint16)
    out = np.zeros((128, 128), np.float32)
    for n in range(128):
        for kc in range(16):
            off = ((n >> 3) * 2048 + kc * 128 + (n & 7) * 16) // 2
            out[n, 8 * kc:8 * kc + 8] = (b16[off:off + 8].astype(np.uint32) << 16).view(np.float32)
    return out


def _unitary(rng, d=64):
    q, r = np.linalg.qr(rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d)))
    return q * (np.diag(r) / np.abs(np.diag(r)))


def test_dense6_operand_and_split_arithmetic(native_lib):
    rng = np.random.default_rng(0)
    U = _unitary(rng)
    w = np.zeros(65536, np.uint8)
    N.call("qs_dense6_weights", np.ascontiguousarray(U).ctypes.data, w.ctypes.data)
    w_hi, w_lo = _decode(w[:32768]), _decode(w[32768:])
    # real form: row 2r+q, column 2s+p
    W = np.zeros((128, 128))
    W[0::2, 0::2], W[0::2, 1::2] = U.real, -U.imag
    W[1::2, 0::2], W[1::2, 1::2] = U.imag, U.real
    assert np.max(np.abs(w_hi + w_lo - W)) < 1e-5
    # 128 columns of 64 amplitudes, memory order (re, im interleaved)
    X = (rng.standard_normal((128, 64)) + 1j * rng.standard_normal((128, 64))).astype(np.complex64)
    X /= np.linalg.norm(X, axis=1, keepdims=True)
    xr = X.view(np.float32).reshape(128, 128)
    x_hi = _bf16_round(xr)
    x_lo = _bf16_round(xr - x_hi)
    D = x_hi.astype(np.float64) @ w_hi.T + x_hi.astype(np.float64) @ w_lo.T + x_lo.astype(np.float64) @ w_hi.T
    Y = D.astype(np.float32).view(np.complex64).reshape(128, 64)
    ref = X.astype(np.complex128) @ U.T
    err = np.max(np.abs(Y - ref))
    assert err < 3e-5, err
    # normalised overlap per column (as the reference's statevector_overlap); norms within 1e-5
    yn = np.linalg.norm(Y, axis=1)
    assert np.max(np.abs(yn - 1)) < 1e-5
    fid = np.abs(np.sum(np.conj(ref) * Y, axis=1) / yn) ** 2
    # three BF16 products (about 16 significant bits per operand): infidelity ~1e-7 per application
    assert np.min(fid) > 1 - 1e-6
