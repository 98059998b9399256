"""Sharded search over 2 ranks (gloo, CPU): references are split by cost,
each rank aligns its share, results come back to rank 0 in the original
order and equal the unsharded result.  The per-rank compute here is the
oracle (the checker), standing in for the GPU library on a CPU-only box."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_fn(q, r):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    o = pyoracle.process_block(q, r, pyoracle.opts_from(refinement=0, convergence=2), nthreads=2)
    return o.out, o.tfm


def _worker(rank, world, port, q, r, outpath):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from gtalign_alpha_b200.shard import search_sharded
    res = search_sharded(q, r, _oracle_fn, rank, world)
    if rank == 0:
        np.savez(outpath, aln=res[0], tfm=res[1])
    dist.barrier()
    dist.destroy_process_group()


def test_lpt_shards_balance_and_cover():
    from gtalign_alpha_b200.shard import lpt_shards
    rng = np.random.default_rng(0)
    rl = rng.integers(30, 2000, size=1000)
    parts = lpt_shards(rl, [300, 200], 4)
    allidx = np.sort(np.concatenate(parts))
    assert np.array_equal(allidx, np.arange(1000))
    costs = [rl[p].sum() for p in parts]
    assert max(costs) / min(costs) < 1.01


def test_two_rank_search_equals_unsharded(tmp_path):
    import torch.multiprocessing as mp
    sys.path.insert(0, ROOT)
    from gtalign_alpha_b200 import synth
    wl = synth.config0(seed=21, n_refs=14, qlen=110, lmin=70, lmax=220)
    q, r = synth.pack(wl.queries), synth.pack(wl.refs)
    outpath = str(tmp_path / "res.npz")
    mp.start_processes(_worker, args=(2, _free_port(), q, r, outpath), nprocs=2,
                       join=True, start_method="spawn")
    got = np.load(outpath)
    aln, tfm = _oracle_fn(q, r)
    assert np.array_equal(got["aln"].view(np.uint32), aln.view(np.uint32))
    assert np.array_equal(got["tfm"].view(np.uint32), tfm.view(np.uint32))
