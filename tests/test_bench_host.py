"""CPU: the multi-process (replica) plumbing of bench.py, on gloo with two ranks, and the reference arm's rule
that only rank 0 works under torchrun."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 3.0], world, "cpu")
        out[rank] = got
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_on_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == [2.0, 10.0, 3.0]


def test_max_over_ranks_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1, 2.5], 1) == [1.0, 2.5]


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_obj_scene_workload_round_trips_the_sphere(tmp_path):
    """The obj_scene workload's files hold the 1M displaced sphere exactly: loaded back by the library's scene
    loader, its triangles are the sphere workload's bit for bit (after the floor and lamp quads), the lamp is
    an area light and the camera comes from the .meta file."""
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    from diplodocus_b200 import scene_io as SI
    from diplodocus_b200 import scenes as S
    name, n, size = bench.write_obj_scene(str(tmp_path))
    sc = SI.load_obj_scene(str(tmp_path), name)
    tris, _ = S.displaced_sphere(n_rays=16)
    assert len(sc) == n == len(tris) + 4
    np.testing.assert_array_equal(sc.triangles()[4:].view(np.uint32), tris.view(np.uint32))
    assert [a.triangle_id for a in sc.area_lights] == [2, 3]
    assert sc.camera.fov == np.float32(0.9) and len(sc.point_lights) == 1


def test_trace_order_defaults_per_workload_and_the_flag_overrides_it():
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    ns = lambda w, o=None: argparse.Namespace(workload=w, trace_order=o)  # noqa: E731
    assert bench.trace_flags(ns("soup16m")) == 2          # DIPL_TRACE_COHERENT_ORDER
    assert bench.trace_flags(ns("displaced_sphere")) == 0
    assert bench.trace_flags(ns("soup16m", "given")) == 0
    assert bench.trace_flags(ns("displaced_sphere", "coherent")) == 2


def test_measured_traffic_is_reported_only_for_the_captured_configuration():
    sys.path.insert(0, ROOT)
    import bench
    n = 16777216
    per_ray = bench.measured_traffic("soup16m", "emc60", "trace", 1, 40, "coherent", n)
    assert per_ray is not None and per_ray > 0
    assert bench.measured_traffic("soup16m", "emc60", "trace", n, 40, "coherent", n) == round(
        bench.MEASURED_TRAFFIC[("soup16m", "emc60", "trace")]["per_unit"] * n)
    # another split budget, ray order, scene size or code has no measurement
    assert bench.measured_traffic("soup16m", "emc60", "trace", n, 0, "coherent", n) is None
    assert bench.measured_traffic("soup16m", "emc60", "trace", n, 40, "given", n) is None
    assert bench.measured_traffic("soup16m", "emc60", "trace", n, 40, "coherent", n // 4) is None
    assert bench.measured_traffic("soup16m", "morton30", "trace", n, 40, "coherent", n) is None
