"""CPU: the replica path of multi-GPU runs (one process per rank, gloo here):
barrier and max-over-ranks of the step time, as bench.py uses them."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    import fem_pkg
    rep = fem_pkg.load_module("replicas")
    w, r, _, pg = rep.init_from_env("gloo", timeout_s=60)
    assert (w, r) == (world, rank)
    rep.barrier(pg)
    out[rank] = rep.max_over_ranks(1.5 + rank, pg)
    rep.barrier(pg)
    pg.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    assert dict(out) == {0: 2.5, 1: 2.5}


def test_single_rank_is_identity():
    import fem_pkg
    rep = fem_pkg.load_module("replicas")
    w, r, local, pg = rep.init_from_env()
    assert (w, r, local, pg) == (1, 0, 0, None)
    assert rep.max_over_ranks(3.25, pg) == 3.25
