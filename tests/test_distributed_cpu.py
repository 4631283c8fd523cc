"""Sharded statevector over 2^g ranks (global qubits): the exchange plan of a reorder emulated
for all ranks in one process against the full-state scatter, and whole tile plans run on gloo
CPU ranks (world size 2 and 4) against the oracle, bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.distributed import plan_exchange
from oracle import statevector as O


def _scatter_bits(psi, perm):
    """out[sum_p bit_p(i) << perm[p]] = in[i] on a 1-D array."""
    n = psi.size.bit_length() - 1
    i = np.arange(psi.size, dtype=np.int64)
    j = np.zeros_like(i)
    for p in range(n):
        j |= ((i >> p) & 1) << perm[p]
    out = np.empty_like(psi)
    out[j] = psi
    return out


def _emulate_exchange(shards, plan):
    world = len(shards)
    shards = [_scatter_bits(s, plan.pre) for s in shards]
    out = []
    for r in range(world):
        parts = []
        for src in plan.sources(r):
            # the chunks src sends, in its buffer order; the one addressed to r
            off = 0
            for d, size in enumerate(plan.send_splits(src, world)):
                if d == r:
                    parts.append(shards[src][off:off + size])
                off += size
        out.append(np.concatenate(parts))
    return [_scatter_bits(s, plan.post) for s in out]


@pytest.mark.parametrize("n,g", [(6, 1), (7, 2), (8, 3), (9, 1), (9, 4)])
def test_exchange_plan_equals_full_scatter(n, g):
    rng = np.random.default_rng(n * 10 + g)
    L = n - g
    for trial in range(25):
        lo = list(rng.permutation(n))
        ln = list(rng.permutation(n))
        if trial == 0:
            ln = list(lo)
        psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
        want = O.permute_scatter(psi, lo, ln)
        plan = plan_exchange(lo, ln, n, g)
        shards = [psi[r << L:(r + 1) << L] for r in range(1 << g)]
        got = np.concatenate(_emulate_exchange(shards, plan))
        np.testing.assert_array_equal(got, want)
        for r in range(1 << g):  # every rank sends and receives a full shard
            assert sum(plan.send_splits(r, 1 << g)) == sum(plan.recv_splits(r, 1 << g)) == 1 << L
        if trial == 0:
            assert not plan.moves_data


class NumpyShard:
    """A rank's shard on the host; tiles through the oracle's per-gate arithmetic."""

    def __init__(self, n, g, rank):
        self.psi = np.zeros(1 << (n - g), dtype=np.complex128)
        if rank == 0:
            self.psi[0] = 1.0

    def apply_tile(self, tile, qmap, fuse):
        ops = O.tile_ops_from_tile(tile, qmap, np.complex128)
        for op in (O.fuse_ops(ops) if fuse else ops):
            if op[0] == "1q":
                O.apply_1q(self.psi, op[2], op[1])
            else:
                O.apply_2q(self.psi, op[3], op[1], op[2])

    def permute_local(self, perm):
        self.psi = _scatter_bits(self.psi, perm)

    def tensor(self):
        import torch
        return torch.from_numpy(self.psi)

    def recv_buffer(self):
        import torch
        return torch.empty(self.psi.size, dtype=torch.complex128)

    def load(self, t):
        self.psi = t.numpy().copy()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, case, q):
    import datetime
    import torch
    import torch.distributed as dist
    from frontierlabproject_b200.distributed import run_distributed
    from frontierlabproject_b200.transpiler import tile_circuit
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        n, depth, nl, seed = case
        g = world.bit_length() - 1
        qc = C.random_layered(n, depth, seed)
        _, plan = tile_circuit(qc, nl, native=False)
        shard = NumpyShard(n, g, rank)
        layout = run_distributed(qc, plan, shard, g)
        parts = [torch.empty(shard.psi.size, dtype=torch.complex128) for _ in range(world)]
        dist.all_gather(parts, torch.from_numpy(shard.psi))
        if rank == 0:
            q.put((layout, np.concatenate([p.numpy() for p in parts])))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("world,case", [(2, (10, 8, 6, 1)), (4, (11, 6, 7, 2))])
def test_sharded_tile_plan_matches_oracle_bitwise(world, case):
    from frontierlabproject_b200.transpiler import tile_circuit
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    layout, psi = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    n, depth, nl, seed = case
    qc = C.random_layered(n, depth, seed)
    _, plan = tile_circuit(qc, nl, native=False)
    ref, ref_layout = O.run_tile_plan(qc, plan, np.complex128)
    assert layout == ref_layout
    np.testing.assert_array_equal(psi, ref)
