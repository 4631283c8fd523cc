"""Small workloads, one per device kernel of the library, for profiling (ncu) and timing.

    python -m frontierlabproject_b200.kernel_cases <case> [--n N] [--reps R]

Each case sets up its inputs, runs the kernel once to warm up, then ``reps`` more launches
on the same stream, and prints one JSON line with the CUDA-event time per launch and the
algorithmic bytes per launch (the unit of the kernel's roofline).  States default to 2^26
amplitudes (512 MiB complex64: larger than the 126 MB L2, a few GB on the device at most).

Cases and the kernels they launch:
  pass      qp_<key>_<p>        specialised pass kernels (random circuit, graphed mode)
  perm      pass_kernel<float>  in-place permutation passes (a random layout materialised)
  gate      gate1/gate2_kernel  one sweep per gate (sequential mode: the plain method)
  adjoint   adjoint_gate1/2, zz_x_kernel   per-gate adjoint sweep (method="per_gate")
  gradient  qp_<key>_<p>        the jit gradient of one ansatz (n qubits, 20 layers): forward tile,
                                zz_x stack kernel, reverse program over the stacked state
  gradient_batch  batch_kernel  the same gradient as one persistent batched launch (method="fused")
  batch     batch_kernel        one persistent launch of a batched variational workload
  sample    sample_* kernels    measurement sampling
  dense6    dense6_tc_pipe_kernel    tensor-core 64x64 unitary on positions 0..5
  dense     dense6_tc_gather_kernel  tensor-core block on arbitrary positions
  reduce    norm2 / inner kernels    FP64 reductions
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def _timed(stream, fn, reps):
    import torch
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / max(1, reps) / 1e3


def case_pass(n, reps):
    import torch
    from . import circuits as C
    from .backend import prepare_tile_ops
    from .qgpusim_cuda import StatevectorF32
    from .transpiler import tile_circuit
    qc = C.random_layered(n, 40, 0)
    _, plan = tile_circuit(qc, min(20, n - 4))
    qmap = {q: qc.find_bit(q).index for q in qc.qubits}
    tiles = [(list(t.layout), prepare_tile_ops(t, qmap, 0, True)[0]) for t in plan]
    sv = StatevectorF32(n)
    sv.set_config(jit=1)
    stream = torch.cuda.ExternalStream(sv.stream)

    def run():
        sv.reset()
        lay = list(range(n))
        for l2, b in tiles:
            if l2 != lay:
                sv.permute(lay, l2)
                lay = l2
            if len(b):
                sv.apply_tile_graphed(b)
        sv.flush()

    run()
    sv.synchronize()
    sv.reset_stats()
    t = _timed(stream, run, reps)
    sweeps = sv.stats()["sweeps"] / (reps + 1)
    return {"kernel": "qp_<key>_<pass>", "seconds_per_launch": t / sweeps, "launches_per_run": sweeps,
            "bytes_per_launch": 2 * (1 << n) * 8}


def case_perm(n, reps):
    import torch
    from .qgpusim_cuda import StatevectorF32
    sv = StatevectorF32(n)
    stream = torch.cuda.ExternalStream(sv.stream)
    rng = np.random.default_rng(1)
    layouts = [list(rng.permutation(n)) for _ in range(reps + 1)]
    cur = [list(range(n))]

    def run():
        new = layouts[len(cur) % len(layouts)]
        sv.permute(cur[-1], new)
        cur.append(new)
        sv.materialize()

    sv.reset_stats()
    t = _timed(stream, run, reps)
    sweeps = sv.stats()["perm_sweeps"] / (reps + 1)
    return {"kernel": "pass_kernel<float,5> (store permutation)", "seconds_per_launch": t / sweeps,
            "launches_per_run": sweeps, "bytes_per_launch": 2 * (1 << n) * 8}


def case_gate(n, reps):
    import torch
    from .qgpusim_cuda import StatevectorF32
    sv = StatevectorF32(n)
    stream = torch.cuda.ExternalStream(sv.stream)
    H = np.array([[1, 1], [1, -1]]) / np.sqrt(2)
    CX = np.eye(4)[[0, 3, 2, 1]]
    ops = [("1q", q, H) for q in range(0, n, 3)] + [("2q", q, (q + 7) % n, CX) for q in range(0, n, 5)]
    t = _timed(stream, lambda: sv.apply_tile_dev(ops), reps)
    return {"kernel": "gate1_kernel / gate2_kernel", "seconds_per_launch": t / len(ops), "launches_per_run": len(ops),
            "bytes_per_launch": 2 * (1 << n) * 8}


def case_adjoint(n, reps):
    import torch
    from . import circuits as C
    from .adjoint import AdjointEngine, ParamCircuit
    pc = ParamCircuit.hea(n, 2)
    th = np.random.default_rng(0).uniform(-np.pi, np.pi, pc.num_params)
    a, b = C.hea_observable(n, 1)
    eng = AdjointEngine(n, f32=True, method="per_gate")
    stream = torch.cuda.ExternalStream(eng.psi.stream)
    t = _timed(stream, lambda: eng.energy_and_grad(pc, th, a, b), reps)
    return {"kernel": "adjoint_gate1 / adjoint_gate2 / zz_x_kernel", "seconds_per_run": t,
            "reverse_launches_per_run": len(pc.gates), "bytes_per_reverse_launch": 4 * (1 << n) * 8}


def _gradient(n, reps, method):
    import torch
    from . import circuits as C
    from .adjoint import AdjointEngine, ParamCircuit
    pc = ParamCircuit.hea(n, 20)
    th = np.random.default_rng(0).uniform(-np.pi, np.pi, pc.num_params)
    a, b = C.hea_observable(n, 1)
    eng = AdjointEngine(n, f32=True, method=method)
    eng.energy_and_grad(pc, th, a, b)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        eng.energy_and_grad(pc, th, a, b)
    torch.cuda.synchronize()
    out = {"seconds_per_gradient_wall": (time.perf_counter() - t0) / reps, "parameters": pc.num_params,
           "gates": len(pc.gates)}
    if method == "jit":
        out["engine"] = eng.info()
    return out


def case_gradient(n, reps):
    out = _gradient(n, reps, "jit")
    out["kernel"] = "qp_<key>_<p> (forward tile and reverse program), zz_x_kernel<float2,true>"
    return out


def case_gradient_batch(n, reps):
    out = _gradient(n, reps, "fused")
    out["kernel"] = "batch_kernel<256> (one instance)"
    return out


def case_batch(n, reps):
    from .batch import BatchedAdjoint, BatchShape, hea_batch
    insts = hea_batch(48, n_range=(12, min(n, 20)), l_range=(4, 8), seed=0)
    b = BatchedAdjoint(insts, BatchShape())
    ms = [b.run(timed=True) for _ in range(reps + 1)]
    b.results()
    return {"kernel": "batch_kernel<256>", "seconds_per_launch": min(ms) / 1e3, "instances": len(insts)}


def case_sample(n, reps):
    from .qgpusim_cuda import StatevectorF32
    sv = StatevectorF32(n)
    sv.apply_tile_cooperative([("1q", q, np.array([[1, 1], [1, -1]]) / np.sqrt(2)) for q in range(n)])
    sv.synchronize()
    t0 = time.perf_counter()
    for i in range(reps + 1):
        sv.sample(1 << 20, seed=i)
    return {"kernel": "sample kernels", "seconds_per_call_wall": (time.perf_counter() - t0) / (reps + 1),
            "shots": 1 << 20, "bytes_per_call": 2 * (1 << n) * 8}


def _dense(n, reps, qubits):
    import torch
    from .qgpusim_cuda import StatevectorF32
    rng = np.random.default_rng(0)
    d = 1 << len(qubits)
    q, r = np.linalg.qr(rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d)))
    U = q * (np.diag(r) / np.abs(np.diag(r)))
    sv = StatevectorF32(n)
    stream = torch.cuda.ExternalStream(sv.stream)
    t = _timed(stream, lambda: sv.apply_dense_block(qubits, U), reps)
    return {"seconds_per_launch": t, "bytes_per_launch": 2 * (1 << n) * 8, "qubits": list(qubits)}


def case_dense6(n, reps):
    out = _dense(n, reps, [0, 1, 2, 3, 4, 5])
    out["kernel"] = "dense6_tc_pipe_kernel"
    return out


def case_dense(n, reps):
    out = _dense(n, reps, [3, 9, 14, 7, 20 % n, 11])
    out["kernel"] = "dense6_tc_gather_kernel"
    return out


def case_reduce(n, reps):
    import torch
    from .qgpusim_cuda import StatevectorF32
    a, b = StatevectorF32(n), StatevectorF32(n)
    stream = torch.cuda.ExternalStream(a.stream)
    t = _timed(stream, lambda: a.inner(b), reps)
    return {"kernel": "inner_kernel", "seconds_per_call": t, "bytes_per_call": 2 * (1 << n) * 8}


CASES = {"pass": case_pass, "perm": case_perm, "gate": case_gate, "adjoint": case_adjoint, "gradient": case_gradient,
         "gradient_batch": case_gradient_batch,
         "batch": case_batch,
         "sample": case_sample, "dense6": case_dense6, "dense": case_dense, "reduce": case_reduce}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--n", type=int, default=26)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    from . import build
    build.build()
    out = CASES[args.case](args.n, args.reps)
    out.update(case=args.case, n=args.n)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
