"""Image-level sharding over ranks: the plan (partition, balance,
determinism) and the sharded driver on two gloo ranks on the CPU, with the
device computation replaced by a host stand-in."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from dmsc_b200.sharding import compute_dmsc_sharded, local_shard, shard_plan


def test_plan_is_a_balanced_partition():
    g = torch.Generator().manual_seed(3)
    shapes = [(int(h), int(w)) for h, w in torch.randint(1, 2048, (512, 2), generator=g)]
    for world in (1, 2, 3, 4, 8):
        plan = shard_plan(shapes, world)
        flat = sorted(i for p in plan for i in p)
        assert flat == list(range(len(shapes)))
        assert all(p == sorted(p) for p in plan)
        loads = [sum(shapes[i][0] * shapes[i][1] for i in p) for p in plan]
        biggest = max(h * w for h, w in shapes)
        assert max(loads) - min(loads) <= biggest  # LPT bound
        assert plan == shard_plan(list(shapes), world)
        assert [local_shard(shapes, world, r) for r in range(world)] == plan


def test_plan_edge_cases():
    assert shard_plan([], 4) == [[], [], [], []]
    assert shard_plan([(5, 5)], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        shard_plan([(1, 1)], 0)
    with pytest.raises(ValueError):
        local_shard([(1, 1)], 2, 2)


def _fake_compute(images, thresholds, duals, device, **kwargs):
    # stands in for the device batch: one tensor per image carrying what the
    # rank was given, so the test can check the routing
    return [torch.tensor([float(x.sum()), float(t), float(d), float(x.shape[0]), float(x.shape[1])])
            for x, t, d in zip(images, thresholds, duals)]


def _batch():
    g = torch.Generator().manual_seed(11)
    imgs = [torch.rand(int(h), int(w), generator=g) for h, w in torch.randint(1, 40, (9, 2), generator=g)]
    thr = [0.01 * i for i in range(9)]
    dual = [bool(i % 2) for i in range(9)]
    return imgs, thr, dual


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world)
        imgs, thr, dual = _batch()
        local = compute_dmsc_sharded(imgs, thr, dual, device="cpu", compute=_fake_compute)
        full = compute_dmsc_sharded(imgs, thr, dual, device="cpu", compute=_fake_compute, gather=True)
        q.put((rank, sorted(local), [v.tolist() for v in full]))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_driver_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, local, full = q.get(timeout=120)
        assert local != "error", full
        out[rank] = (local, full)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    imgs, thr, dual = _batch()
    plan = shard_plan([tuple(x.shape) for x in imgs], world)
    expect = [v.tolist() for v in _fake_compute(imgs, thr, dual, "cpu")]
    for r in range(world):
        assert out[r][0] == plan[r]
        assert out[r][1] == expect  # every rank gathers every image, in order
    assert sorted(out[0][0] + out[1][0]) == list(range(len(imgs)))


def test_single_rank_without_process_group():
    imgs, thr, dual = _batch()
    full = compute_dmsc_sharded(imgs, thr, dual, device="cpu", compute=_fake_compute, gather=True)
    assert [v.tolist() for v in full] == [v.tolist() for v in _fake_compute(imgs, thr, dual, "cpu")]
    with pytest.raises(ValueError):
        compute_dmsc_sharded(imgs, thr[:3], dual, device="cpu", compute=_fake_compute)
