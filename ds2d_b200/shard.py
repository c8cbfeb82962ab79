"""Multi-GPU host logic: one process per GPU, shots sharded across ranks, one image reduction.

Shots are independent within an LSRTM iteration; the reference farms them one at a time to MPI
workers and sums the per-shot gradient images on the master (main.cpp:896-1034, MPI_Reduce of
the images at :1038-1060).  Here every rank owns a static, cost-balanced shard of the shots,
runs all of them batched on its GPU, and the ranks exchange only the summed images (and the FP64
misfit) once per iteration with one all-reduce each.  The functions take a torch.distributed
module (NCCL on GPUs, gloo on CPU in the tests) so the same code runs in both."""
import numpy as np


def shot_cost(shot, nx_default, pml, nzpml, nt):
    """Cell-updates of one shot: its padded window (nx + 2 pml) x nzpml cells for nt steps."""
    nx = shot.nx if getattr(shot, "nx", 0) else nx_default
    return (nx + 2 * pml) * nzpml * nt


def shard_shots(shots, world, rank, nx_default, pml, nzpml, nt):
    """Indices of the shots rank `rank` of `world` owns, ascending.

    Greedy longest-processing-time assignment on shot_cost: shots sorted by decreasing cost (ties
    by index) go one by one to the least-loaded rank (ties by rank).  Deterministic, so every
    rank computes the same partition without communicating; every shot lands on exactly one
    rank; the heaviest rank carries at most 4/3 of the optimal makespan."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    costs = [shot_cost(s, nx_default, pml, nzpml, nt) for s in shots]
    order = sorted(range(len(shots)), key=lambda i: (-costs[i], i))
    load = [0] * world
    owner = [0] * len(shots)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(shots)) if owner[i] == rank]


def shard_loads(shots, world, nx_default, pml, nzpml, nt):
    """Total cost per rank of shard_shots' partition (for reporting the balance)."""
    return [sum(shot_cost(shots[i], nx_default, pml, nzpml, nt)
                for i in shard_shots(shots, world, r, nx_default, pml, nzpml, nt))
            for r in range(world)]


def reduce_images(images, dist, device="cpu"):
    """Sums the per-rank images over all ranks (one all-reduce of the stacked FP32 images).

    `images` maps names to equal-shape arrays; returns the same names with the global sums as
    numpy arrays.  Without a process group (dist None) the input is returned unchanged."""
    if dist is None:
        return {k: np.asarray(v) for k, v in images.items()}
    import torch
    names = list(images)
    t = torch.from_numpy(np.stack([np.ascontiguousarray(images[k], np.float32) for k in names]))
    t = t.to(device)
    dist.all_reduce(t)
    out = t.cpu().numpy()
    return {k: out[i] for i, k in enumerate(names)}


def reduce_images_device(ctx, dist, buf, which=("pp_grad", "ps_grad", "illumination")):
    """The GPU path of the reduction: the context's images are copied device to device into
    `buf` (a CUDA tensor [len(which)][allnx][allnz]) and summed over all ranks by one in-place
    NCCL all-reduce; nothing crosses PCIe.  The context stream must be torch's current stream
    (or synchronised with it) so the all-reduce sees the copies."""
    ctx.read_images_device(buf, reset=True, which=which)
    if dist is not None:
        dist.all_reduce(buf)
    return buf


def reduce_scalar_f64(value, dist, device="cpu"):
    """FP64 sum of one scalar over all ranks (misfit, CG dot products)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t)
    return float(t.item())
