"""The N>1 path on CPU: world_size-2 gloo ranks shard the shots, each images its shard (the
oracle stands in for the GPU engine), and the all-reduced images and misfit must equal the
single-process sums.  Plus the partition's invariants."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ds2d_b200 import synth
from ds2d_b200.shard import (reduce_images, reduce_images_device, reduce_scalar_f64, shard_loads,
                             shard_shots)
from oracle import pyoracle as po

ALLNX, ALLNZ, PML, NT, DX, DT = 48, 24, 8, 80, 10.0, 0.0008


def _case():
    vp, vs = synth.layered(ALLNX, ALLNZ, seed=5)
    shots = synth.uneven_shots(ALLNX, PML, 5, 20, 40, seed=9)
    w = synth.ricker(NT, 20.0, DT)
    rng = np.random.default_rng(2)
    adj = [(rng.standard_normal((s.ntr, NT)).astype(np.float32),
            rng.standard_normal((s.ntr, NT)).astype(np.float32)) for s in shots]
    return vp, vs, shots, w, adj


def _images_of(indices, vp, vs, shots, w, adj):
    tot = {k: np.zeros((ALLNX, ALLNZ)) for k in ("pp", "ps", "il")}
    misfit = 0.0
    for i in indices:
        s = shots[i]
        st = po.Setup(ALLNX, ALLNZ, s.nx, PML, DX, DX, DT)
        m = po.build_model(st, vp, vs, None, s.win_left, rbc=1, seed=3, shot_id=i)
        imgs = po.rtm(st, m, w, s, adj[i][0], adj[i][1], rbc=1)
        for k, im in zip(("pp", "ps", "il"), imgs):
            tot[k] += po.place(im, ALLNX, ALLNZ, s.win_left)
        misfit += float(np.sum(adj[i][0].astype(np.float64) ** 2))
    return tot, misfit


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        vp, vs, shots, w, adj = _case()
        mine = shard_shots(shots, world, rank, 0, PML, ALLNZ + 2 * PML, NT)
        imgs, misfit = _images_of(mine, vp, vs, shots, w, adj)
        red = reduce_images({k: v.astype(np.float32) for k, v in imgs.items()}, dist)
        mis = reduce_scalar_f64(misfit, dist)
        # the in-place path the GPU ranks take (device read-out, then one all-reduce of the
        # buffer), with a stand-in context whose read-out fills the buffer from this rank's sums
        import torch

        class _Ctx:
            def read_images_device(self, out, reset=True, which=None):
                for i, k in enumerate(which):
                    out[i].copy_(torch.from_numpy(imgs[k].astype(np.float32)))
                return out

        buf = torch.zeros((3, ALLNX, ALLNZ), dtype=torch.float32)
        reduce_images_device(_Ctx(), dist, buf, which=("pp", "ps", "il"))
        if rank == 0:
            np.savez(os.path.join(outdir, "red.npz"), misfit=mis,
                     dev=buf.numpy(), **red)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_partition_covers_every_shot_once_and_balances():
    shots = synth.uneven_shots(400, 20, 37, 100, 300, seed=4)
    for world in (1, 2, 3, 8):
        parts = [shard_shots(shots, world, r, 0, 20, 441, 4000) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(shots)))
        loads = shard_loads(shots, world, 0, 20, 441, 4000)
        assert max(loads) <= 4.0 / 3.0 * max(sum(loads) / world, max(
            (s.nx + 40) * 441 * 4000 for s in shots)) + 1
    with pytest.raises(ValueError):
        shard_shots(shots, 2, 2, 0, 20, 441, 4000)


def test_two_gloo_ranks_reduce_to_single_process_images(tmp_path):
    vp, vs, shots, w, adj = _case()
    want, want_mis = _images_of(range(len(shots)), vp, vs, shots, w, adj)
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = np.load(tmp_path / "red.npz")
    for i, k in enumerate(("pp", "ps", "il")):
        ref = want[k].astype(np.float32)
        assert np.linalg.norm(got[k] - ref) <= 1e-6 * np.linalg.norm(ref)
        assert np.linalg.norm(got["dev"][i] - ref) <= 1e-6 * np.linalg.norm(ref)
    assert abs(float(got["misfit"]) - want_mis) <= 1e-12 * abs(want_mis)
