"""The multi-rank path on CPU: sample-range sharding and the per-frame film
reduce of bench.py's step loop (distributed.render_frame), run as two gloo
ranks.  Each rank renders its shard of each frame with the oracle (the
checker, on the CPU); after 3 frames, rank 0 compares the accumulated film
with one oracle render of all the samples, once with a device-style
accumulator and once with the end-to-end host film."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_package

W, H, SPP, FRAMES = 16, 16, 2, 3


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

        def render_into(P, film):  # the oracle stands in for libpt: adds its samples to the film
            s, _, st = o.render(P, threads=2)
            film[0] += torch.from_numpy(s)
            return s, 0.0, st

        def params(off):
            return pt.render_params(W, H, SPP, cam, max_depth=8, sample_offset=off)

        acc, shard = D.new_film(H, W), D.new_film(H, W)
        host = D.new_film(H, W)
        for frame in range(FRAMES):
            D.render_frame(render_into, params, acc, frame, rank, world, SPP, shard=shard)
        for frame in range(FRAMES):
            D.render_frame(render_into, params, None, frame, rank, world, SPP, shard=shard, host_acc=host)
        if rank == 0:
            full, _, _ = o.render(pt.render_params(W, H, FRAMES * world * SPP, cam, max_depth=8), threads=2)
            np.savez(out_path, film=acc.numpy(), host=host.numpy(), full=full, mean=D.resolve(acc).numpy())
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
    film, host, full = r["film"], r["host"], r["full"]
    n = FRAMES * 2 * SPP
    # every sample of the 3 frames counted exactly once
    assert np.all(film[0][..., 3] == n) and np.all(host[0][..., 3] == n) and np.all(full[..., 3] == n)
    # the same paths summed in a different order
    assert np.allclose(film[0] - film[1], full, rtol=2e-5, atol=1e-5)
    assert np.allclose(host[0] - host[1], full, rtol=2e-5, atol=1e-5)
    assert np.allclose(r["mean"], full[..., :3] / n, rtol=2e-5, atol=1e-6)


def test_render_frame_needs_a_shard_film():
    load_package()
    import importlib

    D = importlib.import_module("pbrt_b200.distributed")
    with pytest.raises(ValueError):
        D.render_frame(lambda P, f: None, lambda off: off, D.new_film(2, 2), 0, 0, 2, 1)


def test_bench_rejects_a_world_size_mismatch():
    """bench.py --gpus N must run on exactly N ranks."""
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--steps", "1"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode != 0 and "--gpus 2 but WORLD_SIZE=1" in (r.stderr + r.stdout)
