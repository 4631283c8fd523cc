"""The sharded executor's GPU shard on one GPU (a one-rank NCCL group, g = 0: every reorder is a
local permutation through the in-place permutation passes, no exchange).  The exchange itself is
tested on gloo CPU ranks (tests/test_distributed_cpu.py); runs of two or more GPUs are not
measured (one GPU per call)."""
import datetime
import os
import socket

import numpy as np
import pytest

from frontierlabproject_b200 import circuits as C
from oracle import statevector as O

pytestmark = pytest.mark.gpu


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("f32", [True, False])
def test_gpu_shard_one_rank(f32):
    import torch.distributed as dist
    from frontierlabproject_b200.distributed import GpuShard, run_distributed
    from frontierlabproject_b200.transpiler import tile_circuit
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        qc = C.random_layered(14, 10, 4)
        _, plan = tile_circuit(qc, 9)
        shard = GpuShard(14, 0, 0, f32=f32)
        layout = run_distributed(qc, plan, shard, 0)
        ref, ref_layout = O.run_tile_plan(qc, plan, np.complex128)
        assert layout == ref_layout
        psi = shard.to_numpy()
        if f32:
            assert O.infidelity(ref, psi) <= 1e-5
        else:
            assert np.max(np.abs(psi - ref)) <= 1e-12
    finally:
        dist.destroy_process_group()
