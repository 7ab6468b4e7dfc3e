"""The multi-rank path on CPU: sample-range sharding + the film all-reduce, run
as two gloo ranks.  Each rank renders its shard of the frame with the oracle
(the checker, on the CPU) into a (2, H, W, 4) film; after the reduce, rank 0
compares with one oracle render of all the samples."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_package

W, H, SPP = 16, 16, 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        pt = load_package()
        import importlib

        scenes = importlib.import_module("pbrt_b200.scenes")
        D = importlib.import_module("pbrt_b200.distributed")
        from oracle.oracle import Oracle

        sc, cam = scenes.cornell(W, H)
        o = Oracle(pt)
        o.load(sc)
        film = D.new_film(H, W)
        for frame in range(2):
            off = D.sample_offset(frame, rank, world, SPP)
            s, _, _ = o.render(pt.render_params(W, H, SPP, cam, max_depth=8, sample_offset=off), threads=2)
            film[0] += torch.from_numpy(s)
        D.all_reduce_film(film)
        if rank == 0:
            full, _, _ = o.render(pt.render_params(W, H, 2 * world * SPP, cam, max_depth=8), threads=2)
            np.savez(out_path, film=film.numpy(), full=full, mean=D.resolve(film).numpy())
    finally:
        dist.destroy_process_group()


def test_sample_offsets_partition_the_frame():
    load_package()
    import importlib

    D = importlib.import_module("pbrt_b200.distributed")
    for world in (1, 2, 3, 8):
        seen = []
        for frame in range(3):
            for r in range(world):
                o = D.sample_offset(frame, r, world, 5)
                seen.extend(range(o, o + 5))
        assert sorted(seen) == list(range(3 * world * 5))
    with pytest.raises(ValueError):
        D.sample_offset(0, 2, 2, 4)


def test_two_rank_gloo_film_reduce(tmp_path):
    out = str(tmp_path / "r0.npz")
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    r = np.load(out)
    film, full = r["film"], r["full"]
    assert np.all(film[0][..., 3] == 8) and np.all(full[..., 3] == 8)
    # the same paths summed in a different order
    assert np.allclose(film[0] - film[1], full, rtol=2e-5, atol=1e-5)
    assert np.allclose(r["mean"], full[..., :3] / 8, rtol=2e-5, atol=1e-6)
