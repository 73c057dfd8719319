"""The slab-sharding driver (mrtrix3_b200/multigpu.py) with the GPU solve on
every rank: two gloo ranks, each deconvolving its mask-balanced z-slab with
csd_dwi2fod_host_phased, both on cuda:0 (one GPU is enough: the ranks'
kernels never wait on one another, and the one collective, the final
gather, runs on host tensors), gathered on rank 0.  Voxels are independent,
so the gathered volume equals one process's result bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mrtrix3_b200 import csd, multigpu, synth

pytestmark = pytest.mark.gpu

DIMS = (24, 20, 16)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _volume():
    return synth.make_volume(DIMS, 6, 60, (15.0, 40.0), 8, 0.6, 321)


def _worker(rank, world, port, out_path):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    v = _volume()
    sh = csd.make_shared(v.grad, synth.RESPONSE)

    def solve(dwi, mask):
        return csd.dwi2fod_csd_host_phased(sh, np.ascontiguousarray(dwi), None if mask is None else
                                           np.ascontiguousarray(mask))["fod"]

    fod = multigpu.dwi2fod_distributed(v.dwi, v.mask, v.dims, 45, solve)
    if rank == 0:
        np.save(out_path, fod)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gpu_solve_gather_equals_one_process(cuda, tmp_path):
    out = str(tmp_path / "fod.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    fod = np.load(out)
    v = _volume()
    sh = csd.make_shared(v.grad, synth.RESPONSE)
    ref = csd.dwi2fod_csd_host_phased(sh, v.dwi, v.mask)["fod"]
    assert np.array_equal(fod, ref)
    assert np.all(fod[v.mask == 0] == 0) and np.any(fod[v.mask != 0] != 0)
