#!/usr/bin/env python
"""Benchmark of the statevector tile executor.

Workload (one step): the seeded random circuit n=30, depth 100 (per layer one gate per
qubit from {H, X, SX, RX, RZ}, then CX on a random perfect matching), complex64, run from
|0...0> along the reference LQR tile schedule at nL=20, ending with the state in the last
tile's layout (the reference executor's output).

Metric: algorithmic HBM throughput of a circuit, B_alg / t, with
B_alg = (tiles + reorders + 1) * 2 * 2^n * 8 bytes (one read+write sweep of the state per
tile, per reorder and for the final read-out, as the reference schedule executes it).
``circuit_time_s`` is t itself.  ``value`` is device-timed (CUDA events on the executor's
stream, inputs resident); ``e2e`` is the same metric through ``run_custom_backend`` with a
pinned host result (8 GiB device->host per step) and the host-side op preparation.
``fidelity_err_vs_fp64`` = 1 - |<psi64|psi32>|^2 of the timed circuit against the complex128
executor on the same GPU; ``n33`` times the same circuit family at n=33 (64 GiB state);
``first_call_s`` is the cold start of the first step (planning, kernel compiles, graph capture).

``--impl reference`` times the CPU implementation of the reference algorithm (one full-state
pass per gate, out-of-place scatter per reorder: the C/OpenMP restatement of the reference's
kernels in oracle/) on the host cores; each step runs a sample of the schedule's work units
(fused gates and reorders, spread over the whole schedule) on the full state, and the value is
the sampled units' share of B_alg divided by their measured time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "n=30 circuit time & HBM GB/s vs peak; adjoint gradients/s at ≤1e-5 rel err"


def peaks():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) >= 9:
                for nm, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_workload(n, depth, nl, seed):
    from frontierlabproject_b200 import circuits as C
    from frontierlabproject_b200.transpiler import tile_circuit
    qc = C.random_layered(n, depth, seed)
    _, plan = tile_circuit(qc, nl)
    layouts = [list(range(n))] + [list(t.layout) for t in plan]
    reorders = sum(1 for a, b in zip(layouts[:-1], layouts[1:]) if a != b)
    return qc, plan, reorders


def prepared_tiles(qc, plan, np_dtype):
    """Per tile: (layout, fused op batch) -- the executor inputs, built once, as
    run_custom_backend builds them (native preparation)."""
    from frontierlabproject_b200.backend import prepare_tile_ops
    qmap = {q: qc.find_bit(q).index for q in qc.qubits}
    code = 0 if np_dtype == np.complex64 else 1
    out = []
    for t in plan:
        batch, _ = prepare_tile_ops(t, qmap, code, True)
        out.append((list(t.layout), batch if len(batch) else None))
    return out


class CpuReference:
    """The reference algorithm on the host cores (oracle/cpu_kernels.c, C/OpenMP): one full-state
    pass per fused gate, an out-of-place scatter per reorder.  Loads no library of the package.
    Work units are the schedule's fused gates and reorders in execution order."""

    def __init__(self, qc, plan, n_cpu: int):
        import ctypes
        from oracle import build as ob
        from oracle import statevector as O
        self.ct = ctypes
        lib = ctypes.CDLL(ob.build())
        lib.qo_apply_1q_c64.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        lib.qo_apply_2q_c64.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        lib.qo_permute_scatter_c64.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        lib.qo_max_threads.restype = ctypes.c_int
        self.lib = lib
        self.threads = lib.qo_max_threads()
        self.n = qc.num_qubits
        self.n_cpu = n_cpu
        qindex = {q: qc.find_bit(q).index for q in qc.qubits}
        units = []
        layout = list(range(self.n))
        for t in plan:
            if list(t.layout) != layout:
                units.append(("perm", layout, list(t.layout)))
                layout = list(t.layout)
            for op in O.fuse_ops(O.tile_ops_from_tile(t, qindex, np.complex64)):
                units.append(op)
        self.units = units
        self.gates = sum(1 for u in units if u[0] != "perm")
        self.reorders = len(units) - self.gates
        self.psi = np.zeros(1 << n_cpu, dtype=np.complex64)
        self.psi[0] = 1
        self.tmp = np.empty_like(self.psi)

    def run_unit(self, u) -> None:
        n = self.n_cpu
        fold = lambda q: q if q < n else n - 1 - (q - n) % n  # only when the sample state is smaller
        if u[0] == "perm":
            new_pos = {q: p for p, q in enumerate(u[2])}
            mp = [new_pos[u[1][p]] for p in range(self.n)]
            if n < self.n:
                mp = list(np.random.default_rng(len(self.units)).permutation(n))
            mp = np.asarray(mp[:n], dtype=np.int32)
            self.lib.qo_permute_scatter_c64(self.psi.ctypes.data, self.tmp.ctypes.data, n, mp.ctypes.data)
            self.psi, self.tmp = self.tmp, self.psi
        elif u[0] == "1q":
            U = np.ascontiguousarray(u[2], np.complex64)
            self.lib.qo_apply_1q_c64(self.psi.ctypes.data, n, fold(u[1]), U.ctypes.data)
        else:
            U = np.ascontiguousarray(u[3], np.complex64)
            q0, q1 = fold(u[1]), fold(u[2])
            if q1 == q0:
                q1 = (q0 + 1) % n
            self.lib.qo_apply_2q_c64(self.psi.ctypes.data, n, q0, q1, U.ctypes.data)

    def sample(self, k: int, step: int):
        """k work units spread over the whole schedule (offset by step): (seconds, units run)."""
        U = len(self.units)
        off = (step * 0.6180339887498949) % 1.0
        idx = sorted({min(U - 1, int((j + off) * U / k)) for j in range(k)})
        t0 = time.perf_counter()
        for i in idx:
            self.run_unit(self.units[i])
        return time.perf_counter() - t0, len(idx)

    def describe(self, units_run: int, steps: int) -> str:
        st = (f"{units_run} work units ({steps} samples spread over the schedule's {self.gates} fused gates "
              f"+ {self.reorders} reorders) on the full {self.n_cpu}-qubit complex64 state")
        if self.n_cpu != self.n:
            st += f" (host memory limited the sample state to {self.n_cpu} of {self.n} qubits)"
        return st


def cpu_rate(ref: "CpuReference", b_alg_n: float, t: float, units: int) -> float:
    """GB/s of algorithmic bytes: the sampled units' share of B_alg over their time."""
    return (units / len(ref.units)) * b_alg_n / t / 1e9


def run_reference_arm(args, rank, world):
    from frontierlabproject_b200 import circuits as C
    from frontierlabproject_b200.transpiler import tile_circuit
    qc = C.random_layered(args.n, args.depth, args.seed)
    _, plan = tile_circuit(qc, args.nl, native=False)  # the Python restatement of the LQR pass
    layouts = [list(range(args.n))] + [list(t.layout) for t in plan]
    R = sum(1 for a, b in zip(layouts[:-1], layouts[1:]) if a != b)
    n_cpu = choose_cpu_n(args.n)
    ref = CpuReference(qc, plan, n_cpu)
    b_alg = (len(plan) + R + 1) * 2 * (1 << n_cpu) * 8
    for i in range(args.warmup):
        ref.sample(args.ref_units, i)
    times, units = [], 0
    for i in range(args.steps):
        t, k = ref.sample(args.ref_units, args.warmup + i)
        times.append(t)
        units += k
    t_tot = float(np.sum(times))
    v = cpu_rate(ref, b_alg, t_tot, units)
    t_circuit = t_tot / units * len(ref.units) * (1 << (args.n - n_cpu))
    sample = ref.describe(units, args.steps)
    line = {"metric": METRIC, "value": v, "unit": "GB/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_tot / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": config_of(args, plan, R, world),
            "circuit_time_s_extrapolated": t_circuit,
            "cpu_baseline": {"value": v, "unit": "GB/s", "cores": ref.threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def adjoint_bench(n: int = 24, layers: int = 20, reps: int = 10, seed: int = 0) -> dict:
    """Adjoint gradients of the hardware-efficient ansatz (RY, RZ per qubit + CZ ring per
    layer; theta ~ U[-pi, pi), H = sum a_i Z_i Z_{i+1} + b_i X_i, a, b ~ N(0, 1)), complex64
    states with FP64 accumulation; error against the complex128 adjoint on the same GPU;
    parameter-shift throughput (two energies per parameter) with the pass executor and with
    the plain per-gate executor, timed on a sample of energies."""
    import torch
    from frontierlabproject_b200 import circuits as C
    from frontierlabproject_b200.adjoint import AdjointEngine, ParamCircuit
    rng = np.random.default_rng(seed)
    pc = ParamCircuit.hea(n, layers)
    th = rng.uniform(-np.pi, np.pi, pc.num_params)
    a, b = C.hea_observable(n, seed + 1)
    eng = AdjointEngine(n, f32=True)
    # first call of the structure: plans and kernel compiles (the bench's private kernel cache
    # starts empty), then a warm call
    t0 = time.perf_counter()
    eng.energy_and_grad(pc, th, a, b)
    t_first = time.perf_counter() - t0
    eng.energy_and_grad(pc, th, a, b)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        E, g = eng.energy_and_grad(pc, th, a, b)
    t_adj = (time.perf_counter() - t0) / reps
    info = eng.info() if eng.method == "jit" else {}
    # the same gradient as one persistent launch of the batched kernel, for comparison
    fu = AdjointEngine(n, f32=True, method="fused")
    fu.energy_and_grad(pc, th, a, b)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        fu.energy_and_grad(pc, th, a, b)
    t_fused = (time.perf_counter() - t0) / reps
    del fu
    ref = AdjointEngine(n, f32=False)
    E64, g64 = ref.energy_and_grad(pc, th, a, b)
    rel = float(np.linalg.norm(g - g64) / np.linalg.norm(g64))
    # the per-gate reverse sweep (one kernel per gate over both states), for comparison
    pg = AdjointEngine(n, f32=True, method="per_gate")
    pg.energy_and_grad(pc, th, a, b)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pg.energy_and_grad(pc, th, a, b)
    t_pg = time.perf_counter() - t0
    del pg
    # parameter shift with the pass executor
    for _ in range(2):
        eng.energy(pc, th, a, b)
    k = 10
    t0 = time.perf_counter()
    for _ in range(k):
        eng.energy(pc, th, a, b)
    t_e = (time.perf_counter() - t0) / k
    plain = AdjointEngine(n, f32=True, mode="sequential", method="per_gate")
    plain.energy(pc, th, a, b)
    t0 = time.perf_counter()
    plain.energy(pc, th, a, b)
    t_plain = time.perf_counter() - t0
    ps_fast = 1.0 / (2 * pc.num_params * t_e)
    ps_plain = 1.0 / (2 * pc.num_params * t_plain)
    return {"workload": f"hardware-efficient ansatz n={n} L={layers} ({pc.num_params} parameters, "
                        f"{len(pc.gates)} gates), complex64 states, FP64 accumulation",
            "gradients_per_s": 1.0 / t_adj, "seconds_per_gradient": t_adj, "first_call_s": t_first, "energy": E,
            "method": eng.method, "fused_gradients_per_s": 1.0 / t_fused,
            "forward_sweeps": info.get("forward_sweeps"), "reverse_sweeps": info.get("reverse_sweeps"),
            "reverse_phases": info.get("reverse_phases"), "per_gate_gradients_per_s": 1.0 / t_pg,
            "rel_err_vs_fp64_adjoint": rel, "energy_abs_err_vs_fp64": abs(E - E64),
            "param_shift_gradients_per_s": ps_fast, "param_shift_plain_gradients_per_s": ps_plain,
            "speedup_vs_param_shift": (1.0 / t_adj) / ps_fast,
            "speedup_vs_plain_param_shift": (1.0 / t_adj) / ps_plain,
            "param_shift_sample": f"{k} energies with the pass executor, 1 with the per-gate executor, "
                                  f"x {2 * pc.num_params} per gradient"}


def batch_bench(count: int = 512, seed: int = 0, reps: int = 3) -> dict:
    """Batched variational workload: ``count`` hardware-efficient-ansatz instances (n ~
    U{12..22}, L ~ U{4..16}, own theta and observable each), energy and full gradient of every
    instance in one persistent launch, shape chosen by the autotuner; errors against the FP64
    oracle on a sample of instances; per-instance adjoint engine (one launch per gate) timed on
    a sample as the comparison."""
    from frontierlabproject_b200 import circuits as C
    from frontierlabproject_b200.adjoint import AdjointEngine
    from frontierlabproject_b200.batch import BatchedAdjoint, BatchShape, autotune, hea_batch
    from oracle import statevector as O
    insts = hea_batch(count, seed=seed)
    t0 = time.perf_counter()
    shape = autotune(insts, shapes=[BatchShape(13, 13, 4, 256), BatchShape(13, 13, 8, 256),
                                    BatchShape(12, 12, 4, 256), BatchShape(13, 13, 4, 512)], reps=1)
    t_tune = time.perf_counter() - t0
    b = BatchedAdjoint(insts, shape)
    b.run(timed=True)
    ms = min(b.run(timed=True) for _ in range(reps))
    E, G = b.results()
    # FP64 oracle on the smallest instances
    order = sorted(range(count), key=lambda i: (insts[i].circuit.num_qubits, len(insts[i].circuit.gates)))[:4]
    rel = []
    for i in order:
        pc = insts[i].circuit
        L = sum(1 for g in pc.gates if g.name == "ry") // pc.num_qubits
        E_ref, g_ref = O.adjoint_gradient(C.hea_ansatz(pc.num_qubits, L, insts[i].theta), insts[i].a, insts[i].b)
        rel.append(float(np.linalg.norm(G[i] - g_ref) / np.linalg.norm(g_ref)))
    # per-instance engine on a sample (largest and a middle instance), extrapolated by gate count x 2^n
    sample = [max(range(count), key=lambda i: insts[i].circuit.num_qubits), order[-1]]
    cost = lambda i: len(insts[i].circuit.gates) * (1 << insts[i].circuit.num_qubits)
    t_s, c_s = 0.0, 0
    for i in sample:
        inst = insts[i]
        eng = AdjointEngine(inst.circuit.num_qubits, f32=True)
        eng.energy_and_grad(inst.circuit, inst.theta, inst.a, inst.b)
        s = time.perf_counter()
        eng.energy_and_grad(inst.circuit, inst.theta, inst.a, inst.b)
        t_s += time.perf_counter() - s
        c_s += cost(i)
    t_per_inst = t_s * sum(cost(i) for i in range(count)) / c_s
    info = b.info()
    nparams = sum(inst.circuit.num_params for inst in insts)
    return {"workload": f"{count} hardware-efficient-ansatz instances, n ~ U{{12..22}}, L ~ U{{4..16}}, "
                        f"{nparams} parameters in total, complex64 states, FP64 energies and gradients",
            "batch_ms": ms, "instances_per_s": count / (ms / 1e3), "parameters_per_s": nparams / (ms / 1e3),
            "shape": {"m": shape.m, "small_max": shape.small_max, "chunk": shape.chunk, "threads": shape.threads},
            "autotune_s": t_tune, "work_items": info["items"], "grid": info["grid"],
            "arena_bytes": info["arena_bytes"], "launches_per_batch": 1,
            "max_rel_err_vs_fp64_oracle": max(rel), "oracle_sample": [insts[i].circuit.num_qubits for i in order],
            "per_instance_engine_s_extrapolated": t_per_inst,
            "speedup_vs_per_instance_engine": t_per_inst / (ms / 1e3)}


def dense_bench(n: int = 30, reps: int = 10, seed: int = 0) -> dict:
    """Dense 64x64 unitary (a fused 6-qubit block) on the six lowest qubits of an n-qubit
    complex64 state, one tensor-core sweep per application (tcgen05, 3 BF16 products, FP32
    accumulation): device time per sweep, HBM roofline fraction and tensor throughput;
    infidelity against FP64 on an n=18 state."""
    import torch
    from frontierlabproject_b200.qgpusim_cuda import StatevectorF32
    rng = np.random.default_rng(seed)
    q, r = np.linalg.qr(rng.standard_normal((64, 64)) + 1j * rng.standard_normal((64, 64)))
    U = q * (np.diag(r) / np.abs(np.diag(r)))
    sv = StatevectorF32(n)
    stream = torch.cuda.ExternalStream(sv.stream)
    for _ in range(3):
        sv.apply_dense(U)
    sv.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    for _ in range(reps):
        sv.apply_dense(U)
    ev[1].record(stream)
    sv.synchronize()
    t = ev[0].elapsed_time(ev[1]) / reps / 1e3
    hbm_peak, _ = peaks()
    sweep = 2 * (1 << n) * 8
    flops_exec = 3 * 2 * 128 * 128 * 128 * ((1 << n) // 8192)    # three BF16 products per 128-column tile
    flops_useful = 8 * 64 * (1 << n)                              # complex 64x64 matrix-vector per column
    # accuracy on a smaller state
    m = 18
    psi = rng.standard_normal(1 << m) + 1j * rng.standard_normal(1 << m)
    psi = (psi / np.linalg.norm(psi)).astype(np.complex64)
    small = StatevectorF32(m)
    small.from_numpy(psi)
    small.apply_dense(U)
    out = small.to_numpy().astype(np.complex128)
    ref = (psi.astype(np.complex128).reshape(-1, 64) @ U.T).reshape(-1)
    fid = abs(np.vdot(ref / np.linalg.norm(ref), out / np.linalg.norm(out))) ** 2
    return {"workload": f"dense 64x64 complex unitary on qubits 0-5 of a {n}-qubit complex64 state",
            "seconds_per_sweep": t, "achieved_gbs": sweep / t / 1e9, "hbm_frac": sweep / t / 1e9 / hbm_peak,
            "tensor_tflops_executed": flops_exec / t / 1e12, "complex_tflops_useful": flops_useful / t / 1e12,
            "infidelity_vs_fp64_n18": 1.0 - fid, "precision": "BF16 high+low split, 3 products, FP32 accumulation"}


def dense_fusion_bench(qc, plan, k, sv64, hbm_peak) -> dict:
    """The timed circuit as fused k-qubit blocks on the tensor cores (run_custom_backend's
    dense_fusion path: each tile's gates grouped by plan_dense_blocks, one tcgen05 sweep per
    block): device time per circuit, per-sweep bandwidth, FP64 fidelity against sv64."""
    import torch
    from frontierlabproject_b200.backend import plan_dense_blocks, tile_ops_for
    from frontierlabproject_b200.qgpusim_cuda import StatevectorF32
    n = qc.num_qubits
    qmap = {q: qc.find_bit(q).index for q in qc.qubits}
    t0 = time.perf_counter()
    work = []
    ngates = 0
    for t in plan:
        ops = tile_ops_for(t, qmap, np.complex128)
        ngates += len(ops)
        work.append((list(t.layout), plan_dense_blocks(ops, k)))
    t_plan = time.perf_counter() - t0
    nblocks = sum(len(b) for _, b in work)
    sv = StatevectorF32(n)
    stream = torch.cuda.ExternalStream(sv.stream)

    def run():
        sv.reset()
        layout = list(range(n))
        for lay, blocks in work:
            if lay != layout:
                sv.permute(layout, lay)
                layout = lay
            for qs, U in blocks:
                sv.apply_dense_block(qs, U)
        sv.materialize()

    run()
    sv.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    run()
    ev[1].record(stream)
    sv.synchronize()
    t = ev[0].elapsed_time(ev[1]) / 1e3
    ov = sv64.inner(sv)
    fid = max(0.0, 1.0 - abs(ov) ** 2 / (sv.norm_squared() * sv64.norm_squared()))
    sv.close()
    sweep = 2 * (1 << n) * 8
    per = t / max(1, nblocks)
    return {"k": k, "blocks_per_circuit": nblocks, "gates_per_block": ngates / nblocks if nblocks else None,
            "circuit_time_s": t, "seconds_per_block_sweep": per, "block_sweep_gbs": sweep / per / 1e9,
            "hbm_frac_per_sweep": sweep / per / 1e9 / hbm_peak, "fidelity_err_vs_fp64": fid,
            "host_planning_s": t_plan,
            "note": "same circuit and schedule as the headline; each fused block is one tensor-core sweep "
                    "(3 BF16 products, FP32 accumulation) and covers far fewer gates than a pass of the pass "
                    "executor, which stays the timed path"}


def cold_start_async_bench(args) -> dict:
    """First call of a circuit structure this process has not compiled (the same family, next
    seed) with jit_async: the generic pass kernel runs it while the specialised kernels compile in
    the background; then the wait for the compile and the first specialised run."""
    from frontierlabproject_b200.backend import run_custom_backend
    from frontierlabproject_b200.qgpusim_cuda import StatevectorF32
    qc, plan, _ = build_workload(args.n, args.depth, args.nl, args.seed + 1)
    sv = StatevectorF32(args.n)
    sv.set_config(jit_async=1)
    out = np.empty(1 << args.n, dtype=np.complex64)
    t0 = time.perf_counter()
    run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode="graphed", sv=sv, out=out)
    t_first = time.perf_counter() - t0
    pending = sv.stats()["jit_pending_flushes"]
    t0 = time.perf_counter()
    StatevectorF32.jit_wait()
    t_wait = time.perf_counter() - t0
    t0 = time.perf_counter()
    run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode="graphed", sv=sv, out=out)
    t_second = time.perf_counter() - t0
    st = sv.stats()
    sv.close()
    return {"workload": f"random circuit n={args.n} depth={args.depth} seed {args.seed + 1} (a new structure), "
                        "end to end through run_custom_backend",
            "first_call_s": t_first, "generic_flushes": pending, "compile_wait_after_first_s": t_wait,
            "second_call_s": t_second, "second_call_specialised_modules": st["jit_modules"]}


def n33_bench(args, hbm_peak) -> dict:
    """The same circuit family at n=33 (64 GiB complex64 state), depth 100, the reference
    schedule at nL=20: device time per circuit (CUDA events), B_alg / t and the sweep count."""
    import torch
    from frontierlabproject_b200.qgpusim_cuda import StatevectorF32
    n = 33
    qc, plan, R = build_workload(n, args.depth, args.nl, args.seed)
    tiles = prepared_tiles(qc, plan, np.complex64)
    sv = StatevectorF32(n)
    sv.set_config(m=args.m, k=args.k, jit=args.jit, jit_lr=args.jit_lr, jit_blocks=args.jit_blocks,
                  jit_packed=args.jit_packed)
    stream = torch.cuda.ExternalStream(sv.stream)

    def run():
        sv.reset()
        layout = list(range(n))
        for lay, batch in tiles:
            if lay != layout:
                sv.permute(layout, lay)
                layout = lay
            if batch is not None:
                sv.apply_tile_graphed(batch)
        sv.materialize()

    t0 = time.perf_counter()
    run()
    sv.synchronize()
    first = time.perf_counter() - t0
    sv.reset_stats()
    reps = 2
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    for _ in range(reps):
        run()
    ev[1].record(stream)
    sv.synchronize()
    t = ev[0].elapsed_time(ev[1]) / reps / 1e3
    st = sv.stats()
    sweep = 2 * (1 << n) * 8
    b_alg = (len(plan) + R + 1) * sweep
    sv.close()
    return {"workload": f"random circuit n={n} depth={args.depth} complex64, reference LQR schedule nL={args.nl} "
                        f"({len(plan)} tiles, {R} reorders), seed {args.seed}",
            "circuit_time_s": t, "value_gbs": b_alg / t / 1e9, "hbm_frac_alg": b_alg / t / 1e9 / hbm_peak,
            "sweeps_per_circuit": (st["sweeps"] + st["gate_sweeps"]) / reps,
            "reference_sweeps_per_circuit": len(plan) + R + 1, "first_call_s": first, "reps": reps}


def choose_cpu_n(n: int) -> int:
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 16 << 30
    m = n
    while m > 20 and 2 * (1 << m) * 8 > avail * 0.6:
        m -= 1
    return m


def config_of(args, plan, R, world=1):
    return {"workload": f"random circuit n={args.n} depth={args.depth} complex64 from |0>, reference LQR "
                        f"schedule nL={args.nl} ({len(plan)} tiles, {R} reorders), seed {args.seed}",
            "n": args.n, "depth": args.depth, "nL": args.nl, "tile_mode": args.mode,
            "l2": (f"state ({(8 << args.n) / 2**30:g} GiB) > L2 (126 MB): every sweep streams from HBM, "
                   "no flush needed" if (8 << args.n) > 126e6 else
                   f"state ({(8 << args.n) / 2**20:g} MiB) fits in L2: not an HBM measurement"),
            "parallelism": "replicas" if world > 1 else "single GPU"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="graphed", choices=["graphed", "cooperative", "sequential"])
    ap.add_argument("--n", type=int, default=30)
    ap.add_argument("--depth", type=int, default=100)
    ap.add_argument("--nl", type=int, default=20)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--jit", type=int, default=0, help="0 auto, 1 always, -1 never")
    ap.add_argument("--jit-lr", type=int, default=5)
    ap.add_argument("--jit-blocks", type=int, default=2)
    ap.add_argument("--jit-packed", type=int, default=0, help="FP32x2 arithmetic in the specialised kernels")
    ap.add_argument("--m", type=int, default=13)
    ap.add_argument("--k", type=int, default=3, help="lowest physical bits always staged")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-dense", action="store_true")
    ap.add_argument("--batch-count", type=int, default=512, help="instances of the batched variational workload")
    ap.add_argument("--no-fidelity", action="store_true")
    ap.add_argument("--n33", type=int, default=1, help="also time the n=33 circuit (64 GiB state)")
    ap.add_argument("--ref-units", type=int, default=16, help="reference arm: work units per step")
    ap.add_argument("--cold-async", type=int, default=1, help="time a new circuit structure's first call with "
                                                                "the generic kernel standing in while compiling")
    ap.add_argument("--dense-k", type=int, default=6, help="also time the circuit as fused k-qubit tensor-core "
                                                          "blocks (0: skip)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference_arm(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from frontierlabproject_b200 import build as B
    B.build()
    # cold starts are measured as cold: kernels compiled in this run go to an empty private cache
    # (an explicit QSIM_JIT_CACHE is respected)
    if "QSIM_JIT_CACHE" not in os.environ:
        import tempfile
        os.environ["QSIM_JIT_CACHE"] = tempfile.mkdtemp(prefix="qsim_jit_")
    from frontierlabproject_b200.backend import run_custom_backend
    from frontierlabproject_b200.qgpusim_cuda import StatevectorF32
    from frontierlabproject_b200.replicas import max_over_ranks, whole_job_rate

    hbm_peak, peak_kind = peaks()
    qc, plan, R = build_workload(args.n, args.depth, args.nl, args.seed)
    tiles = prepared_tiles(qc, plan, np.complex64)
    n = args.n
    sweep = 2 * (1 << n) * 8
    b_alg = (len(plan) + R + 1) * sweep

    sv = StatevectorF32(n)
    sv.set_config(m=args.m, k=args.k, jit=args.jit, jit_lr=args.jit_lr, jit_blocks=args.jit_blocks,
                  jit_packed=args.jit_packed)
    stream = torch.cuda.ExternalStream(sv.stream)
    apply = {"graphed": sv.apply_tile_graphed, "cooperative": sv.apply_tile_cooperative,
             "sequential": sv.apply_tile_dev}[args.mode]

    def step(ev):
        sv.reset()
        ev[0].record(stream)
        layout = list(range(n))
        for lay, batch in tiles:
            if lay != layout:
                sv.permute(layout, lay)
                layout = lay
            if batch is not None:
                apply(batch)
        sv.materialize()
        ev[1].record(stream)

    mk = lambda: [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    # cold start: the first step plans the schedule, compiles its kernels and captures the graph
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    step(mk())
    sv.synchronize()
    first_call_s = time.perf_counter() - t0
    first = sv.stats()
    for _ in range(max(0, args.warmup - 1)):
        step(mk())
    sv.synchronize()
    sv.reset_stats()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    evs = [mk() for _ in range(args.steps)]
    start.record(stream)
    for i in range(args.steps):
        step(evs[i])
    end.record(stream)
    sv.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = start.elapsed_time(end)
    pass_ms = sum(e[0].elapsed_time(e[1]) for e in evs)
    st = sv.stats()
    total_ms, pass_ms = max_over_ranks([total_ms, pass_ms], dist, "cuda")
    ms_step = total_ms / args.steps
    value = whole_job_rate(b_alg, ms_step / 1e3, world) / 1e9
    sweeps_step = (st["sweeps"] + st["gate_sweeps"]) / args.steps
    achieved = sweeps_step * sweep / (pass_ms / args.steps / 1e3) / 1e9
    launches_step = 1 + (st["sweeps"] - st["perm_sweeps"]) / args.steps + (1 if st["perm_sweeps"] else 0) \
        if args.mode == "graphed" else 1 + st["launches"] / args.steps

    # ---- fidelity of the timed circuit against double precision on the same GPU ----
    fid = None
    dfu = None
    if not args.no_fidelity:
        from frontierlabproject_b200.qgpusim_cuda import Statevector
        step(mk())
        sv.synchronize()
        sv64 = Statevector(n)
        t0 = time.perf_counter()
        layout = list(range(n))
        for lay, batch in prepared_tiles(qc, plan, np.complex128):
            if lay != layout:
                sv64.permute(layout, lay)
                layout = lay
            if batch is not None:
                sv64.apply_tile_graphed(batch)
        sv64.synchronize()
        t64 = time.perf_counter() - t0
        ov = sv64.inner(sv)
        n32, n64 = sv.norm_squared(), sv64.norm_squared()
        fid = {"fidelity_err_vs_fp64": max(0.0, 1.0 - abs(ov) ** 2 / (n32 * n64)),
               "norm_c64": n32, "norm_c128": n64,
               "reference": "the same schedule through the complex128 executor (generic pass kernel) on the same "
                            "GPU; 1 - |<psi64|psi32>|^2 / (|psi32|^2 |psi64|^2), FP64 on the device",
               "c128_run_s": t64}
        if args.dense_k:
            dfu = dense_fusion_bench(qc, plan, args.dense_k, sv64, hbm_peak)
        sv64.close()
        del sv64

    # ---- end to end through the public API (pinned host result) ----
    e2e = None
    if args.e2e_steps > 0:
        out = torch.empty(1 << n, dtype=torch.complex64, pin_memory=True).numpy()
        run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode=args.mode, sv=sv, out=out)
        ts = []
        for _ in range(args.e2e_steps):
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            _, met = run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode=args.mode, sv=sv,
                                        out=out)
            ts.append(time.perf_counter() - t0)
        te, = max_over_ranks([float(np.mean(ts))], dist, "cuda")
        h2d = sum(b.arr.nbytes + sum(k.nbytes for k in b._keep) for _, b in tiles if b is not None)
        e2e = {"value": whole_job_rate(b_alg, te, world) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int((1 << n) * 8), "circuit_time_s": te}
        del out
    sv.close()
    del sv

    adj = None
    if not args.no_adjoint:
        adj = adjoint_bench()
    bat = None
    if not args.no_batch:
        bat = batch_bench(args.batch_count)
    den = None
    if not args.no_dense:
        den = dense_bench(n)
    big = None
    if args.n33 and world == 1:
        big = n33_bench(args, hbm_peak)

    cold = None
    if args.cold_async and world == 1:
        cold = cold_start_async_bench(args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        ref = CpuReference(qc, plan, choose_cpu_n(n))
        b_alg_cpu = (len(plan) + R + 1) * 2 * (1 << ref.n_cpu) * 8
        ref.sample(4, 0)  # warm-up: first touch of the host state
        t_cpu, units, k = 0.0, 0, 0
        while t_cpu < args.cpu_budget:
            t, u = ref.sample(8, 1 + k)
            t_cpu += t
            units += u
            k += 1
        v = cpu_rate(ref, b_alg_cpu, t_cpu, units)
        cpu = {"value": v, "unit": "GB/s", "cores": ref.threads, "kind": "port", "sample": ref.describe(units, k),
               "seconds": t_cpu,
               "circuit_time_s_extrapolated": t_cpu / units * len(ref.units) * (1 << (n - ref.n_cpu))}
        del ref

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "c64", "data": "synthetic",
                "circuit_time_s": ms_step / 1e3,
                "config": config_of(args, plan, R, world),
                "sweeps_per_step": sweeps_step, "reference_sweeps_per_step": len(plan) + R + 1,
                "fidelity_err_vs_fp64": fid["fidelity_err_vs_fp64"] if fid else None, "fidelity": fid,
                "first_call_s": first_call_s, "first_call_compile_s": first["jit_compile_ms"] / 1e3,
                "first_call_async": cold,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                             "frac": achieved / hbm_peak, "traffic": None,
                             "traffic_note": "DRAM bytes per launch come from ncu captures of this kernel "
                                             "(profiles/), not from this run",
                             "kernel": ("qp_<key>_<pass> (pass kernel specialised at plan time)"
                                        if first["jit_compile_ms"] or (args.mode == "graphed" and args.jit >= 0
                                                                       and n >= 20)
                                        else "pass_kernel<float,5>"),
                             "peak_kind": peak_kind,
                             "algorithmic_bytes_per_sweep": sweep},
                "gpu_launches": int(round(launches_step * args.steps)),
                "clocks": clk, "e2e": e2e, "cpu_baseline": cpu, "n33": big, "adjoint": adj, "batch": bat,
                "dense_tc": den, "dense_fusion": dfu}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
