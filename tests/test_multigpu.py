"""Host logic of the multi-GPU path on CPU: slab sharding and the final
gather, with two gloo ranks standing in for two GPUs (the FP64 oracle
stands in for each rank's GPU solve)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from mrtrix3_b200 import multigpu, synth


def test_slab_bounds_cover_and_balance():
    dims = (24, 20, 17)
    mask = synth.ellipsoid_mask(dims, 0.5)
    for world in (1, 2, 3, 4, 8):
        b = multigpu.slab_bounds(mask, dims, world)
        assert b[0][0] == 0 and b[-1][1] == mask.size
        assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
        counts = [int(mask[s:e].sum()) for s, e in b]
        assert sum(counts) == int(mask.sum())
        assert max(counts) - min(counts) <= 2 * dims[0] * dims[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import torch.distributed as dist

    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    v = synth.make_volume((6, 5, 8), 6, 60, 30.0, 8, 0.6, 123)
    sh = O.OracleShared(v.grad, synth.RESPONSE, synth.load_hr_dirs())

    def solve(dwi, mask):
        return sh.solve(dwi, mask=mask, nthreads=1)["F"].astype(np.float32)

    fod = multigpu.dwi2fod_distributed(v.dwi, v.mask, v.dims, 45, solve)
    if rank == 0:
        np.save(out_path, fod)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gather_equals_single_process(tmp_path):
    from oracle import oracle as O
    out = str(tmp_path / "fod.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    fod = np.load(out)
    v = synth.make_volume((6, 5, 8), 6, 60, 30.0, 8, 0.6, 123)
    ref = O.OracleShared(v.grad, synth.RESPONSE, synth.load_hr_dirs()).solve(v.dwi, mask=v.mask, nthreads=1)
    assert np.array_equal(fod, ref["F"].astype(np.float32))
