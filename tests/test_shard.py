"""The multi-rank form of the render on CPU: ranks render disjoint sample ranges of one film
(rypath_b200.shard.sample_range) and merge their films over torch.distributed (gloo here, NCCL
between GPUs).  The oracle stands in for each rank's renderer; the merged film must equal the
film of one process that rendered every sample: counts exactly, FP64 sums to rounding.
"""

import datetime
import os
import socket

import numpy as np
import pytest

from oracle_lib import OracleScene, oracle, request
from rypath_b200 import abi, scenes, shard

W, H, SPP = 12, 10, 7


def oracle_film(scene, begin, count):
    lanes = OracleScene(scene).sample(request(W, H, count, sample_begin=begin), threads=1)
    film = np.zeros(W * H, abi.film_dtype())
    cie = np.ascontiguousarray(scenes.cie_xyz())
    assert oracle().or_film_add(lanes.ctypes.data, lanes.size, cie.ctypes.data, W * H, film.ctypes.data) == 0
    return film


def assert_same_film(got, want):
    np.testing.assert_array_equal(got["count"], want["count"])
    np.testing.assert_allclose(got["sum"] + got["correction"], want["sum"] + want["correction"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(got["weight_sum"] + got["weight_correction"],
                               want["weight_sum"] + want["weight_correction"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(got["square"], want["square"], rtol=1e-12, atol=0)


def test_sample_ranges_partition_the_film():
    for count in (0, 1, 7, 16, 1000):
        for world in (1, 2, 3, 8):
            ranges = [shard.sample_range(count, r, world, sample_begin=5) for r in range(world)]
            assert sum(c for _, c in ranges) == count
            assert ranges[0][0] == 5
            for (b0, c0), (b1, _) in zip(ranges, ranges[1:]):
                assert b0 + c0 == b1
            assert max(c for _, c in ranges) - min(c for _, c in ranges) <= 1
    with pytest.raises(ValueError):
        shard.sample_range(4, 2, 2)


def test_added_films_equal_one_render():
    scene = scenes.cornell_box(W, H, 1)
    whole = oracle_film(scene, 0, SPP)
    parts = [oracle_film(scene, *shard.sample_range(SPP, r, 3)) for r in range(3)]
    assert_same_film(shard.add_films(parts), whole)


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        scene = scenes.cornell_box(W, H, 1)
        begin, count = shard.sample_range(SPP, rank, world)
        merged = shard.merge_film(oracle_film(scene, begin, count))
        np.save(os.path.join(out_dir, f"merged{rank}.npy"), merged.view(np.uint8))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_merge_to_the_single_process_film(world, tmp_path):
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    whole = oracle_film(scenes.cornell_box(W, H, 1), 0, SPP)
    merged = [np.load(tmp_path / f"merged{r}.npy").view(abi.film_dtype()) for r in range(world)]
    for m in merged:
        assert m.tobytes() == merged[0].tobytes()  # the same film on every rank
    assert_same_film(merged[0], whole)


def _gpu_rank(rank, world, port, out_dir):
    import torch.distributed as dist

    from rypath_b200 import renderer

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        built = renderer.build_renderer(scenes.mixed_scene(W, H, 1, 6, subdivisions=3))
        assert built.status == abi.RP_SUCCESS, built.diagnostic
        begin, count = shard.sample_range(SPP, rank, world)
        st, diag, film = built.scene.render_film(renderer.RenderSettings(W, H, samples=count, batch_size=count, seed=1),
                                                 sample_begin=begin)
        assert st == abi.RP_SUCCESS, diag
        merged = shard.merge_film(film)
        np.save(os.path.join(out_dir, f"merged{rank}.npy"), merged.view(np.uint8))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_device_ranks_merge_to_the_single_render(tmp_path):
    """Two ranks rendering their sample ranges with the CUDA renderer (on one device, each its own
    independent launches), merged over gloo, equal one render of every sample."""
    import multiprocessing as mp

    from rypath_b200 import renderer

    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=_gpu_rank, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    built = renderer.build_renderer(scenes.mixed_scene(W, H, 1, 6, subdivisions=3))
    assert built.status == abi.RP_SUCCESS, built.diagnostic
    st, diag, whole = built.scene.render_film(renderer.RenderSettings(W, H, samples=SPP, batch_size=SPP, seed=1))
    assert st == abi.RP_SUCCESS, diag
    merged = np.load(tmp_path / "merged0.npy").view(abi.film_dtype())
    assert merged.tobytes() == np.load(tmp_path / "merged1.npy").view(abi.film_dtype()).tobytes()
    assert_same_film(merged, whole)
