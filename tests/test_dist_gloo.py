"""The multi-GPU host logic of bench.py on CPU: two ranks over `gloo` (127.0.0.1).  Each rank
gets its own camera of the same scene (another azimuth: equal work, weak scaling), the barrier
passes, the time is the max over ranks and the throughput counts the rays of every rank."""
from __future__ import annotations

import math
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist

    import bench
    from kerrtrace_b200 import workloads
    try:
        r, w, local = bench.dist_setup("gloo")
        cfg, cam = bench.rank_camera(workloads, "c2", r, w)
        bench.barrier(w)
        t_max = bench.max_over_ranks(10.0 * (r + 1), w)      # rank 1 is the slower one
        out.put((r, list(cam.cam_pos), list(cam.fwd), cam.fov_scale, cfg.width * cfg.height, t_max,
                 bench.job_mrays_s(cfg.width * cfg.height, w, t_max)))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def test_two_gloo_ranks_render_their_own_view_and_share_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    if any(p.is_alive() for p in procs):
        for p in procs:
            p.kill()
        pytest.fail("a rank did not finish")
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(out.get(timeout=10) for _ in range(2))
    (r0, pos0, fwd0, fov0, n0, t0, v0), (r1, pos1, fwd1, fov1, n1, t1, v1) = res
    assert (r0, r1) == (0, 1)
    # same radius, inclination, FOV and frame size; a different azimuth
    rad = lambda p: math.sqrt(sum(c * c for c in p))  # noqa: E731
    assert abs(rad(pos0) - rad(pos1)) < 1e-4 * rad(pos0)
    assert abs(pos0[1] - pos1[1]) < 1e-4 * rad(pos0)
    assert abs(fov0 - fov1) < 1e-7 and n0 == n1
    assert math.dist(pos0, pos1) > 1.0
    # the camera still looks at the hole
    assert abs(sum(f * p for f, p in zip(fwd1, pos1)) / rad(pos1) + 1.0) < 1e-5
    # both ranks see the slowest rank's time; the job counts the rays of both
    assert t0 == t1 == 20.0
    assert abs(v0 - 2 * n0 / 0.020 / 1e6) < 1e-9 and v0 == v1
