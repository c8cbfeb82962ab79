"""Benchmark of the DS2D hot path on B200: elastic RTM with random boundaries.

Workload (one step): elastic RTM of a batch of 60 shots evenly spread along the surface of a
1201 x 401 model (dx = dz = 10 m, 40-cell random band -> 1281 x 481 padded cells, nt = 4000,
dt = 0.8 ms, 15 Hz Ricker), receivers on every column two cells below the surface: background
forward pass, interior reconstruction, adjoint pass and zero-lag imaging (3 propagations per
shot).  The true model is synthetic (8 dipping layers 2000-6000 m/s + 3 Gaussian lenses, seeded),
the migration model is it smoothed with sigma = 15 cells; observed data come from PML forward
modelling on the true model (untimed set-up).

Metric: Gcell-updates/s = shots * 1281 * 481 * 4000 * 3 / time, whole job (all ranks).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): every rank runs its own 60-shot batch (weak scaling) and the three images
are summed over ranks with one NCCL all-reduce per step, as the reference sums its gradients
over MPI ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CFG = dict(allnx=1201, allnz=401, pml=40, nt=4000, dx=10.0, dz=10.0, dt=0.0008, f0=15.0,
           shots=60, sz=0, gz=2, seed=2024)
# Reference-mode ELSRTM workload.  Counted propagations per shot: 6 (background, first- and
# second-order Born sets forward; background and first-order reconstruction and the adjoint
# backward); the reference also propagates a scattered adjoint that its runs leave at zero.
ELSRTM_SHOTS, ELSRTM_NT, ELSRTM_PROPS = 16, 2000, 6
TRAFFIC_CELLS_PER_SHOT = 1281 * 481  # padded cells of the grid the ncu traffic was captured on


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--shots", type=int, default=CFG["shots"])
    p.add_argument("--nt", type=int, default=CFG["nt"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-profile", action="store_true")
    p.add_argument("--ref-shots", type=int, default=2, help="shots per reference-arm step")
    p.add_argument("--no-autotune", action="store_true",
                   help="skip the launch-shape autotuner (library defaults)")
    p.add_argument("--set", default="",
                   help="library options applied after the autotuner, e.g. pair=1,pair_xr=96 "
                        "(profiling runs of one kernel variant)")
    p.add_argument("--workload", default="rtm",
                   choices=["rtm", "uneven", "lsrtm", "elsrtm", "acoustic", "unet"],
                   help="rtm: elastic RTM throughput, 60 shots 1201x401 (default); uneven: 256 "
                        "shots with their own aperture windows from a 4001x401 model; lsrtm: "
                        "learned vs plain CG-LSRTM; elsrtm: reference-mode ELSRTM iteration "
                        "(PML + boundary strips, Born modelling, NCC adjoint source), 16 shots "
                        "1201x401, nt 2000; acoustic: the CG-LSRTM normal operator L^T L on the "
                        "2001x601 grid (+20 band), 16 shots by default; unet: the preconditioner "
                        "network's forward pass and training step on one 2008x608 image")
    p.add_argument("--lsrtm-size", default="full", choices=["small", "full"],
                   help="full: 2001x601, 80 shots, nt 5000; small: 512x256, 40 shots, nt 2000")
    p.add_argument("--lsrtm-boundary", default="random", choices=["random", "pml"],
                   help="boundary of the LSRTM and acoustic workloads' operators: random band "
                        "(exact background "
                        "reversal) or the reference's PML with the background rebuilt from strips")
    p.add_argument("--lsrtm-strips", default="bf16", choices=["f32", "f16", "bf16"],
                   help="storage of the background's boundary strips with --lsrtm-boundary pml")
    p.add_argument("--pairs", type=int, default=192, help="training pairs of the preconditioner")
    p.add_argument("--train-steps", type=int, default=2000)
    p.add_argument("--trajectory", type=int, default=16,
                   help="training pairs along CG trajectories, this many iterates per model "
                        "(0: independent random models)")
    p.add_argument("--cg-iters", type=int, default=10)
    p.add_argument("--target", type=float, default=1e-2)
    return p.parse_args()


class Clocks:
    """Samples nvidia-smi SM clocks and throttle reasons while the timed region runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.stop = threading.Event()

    def _run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(timeout=6)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def workload(args, rank, world=1):
    """One model for all ranks; a survey of `shots` x world shots, of which this rank takes its
    cost-balanced shard (weak scaling: `shots` per GPU)."""
    from ds2d_b200 import synth
    from ds2d_b200.shard import shard_shots
    c = dict(CFG)
    c["nt"] = args.nt
    c["shots"] = args.shots
    uneven = getattr(args, "workload", "rtm") == "uneven"
    if uneven:  # 256 shots, windows U[400, 1500] cells, 4001x401 layered + lens model, 20-cell band
        c.update(allnx=4001, pml=20, wmin=400, wmax=1500)
        if args.shots == CFG["shots"]:
            c["shots"] = 256
    if getattr(args, "workload", "rtm") == "elsrtm":  # 40-cell PML, 16 shots, nt 2000 by default
        if args.shots == CFG["shots"]:
            c["shots"] = ELSRTM_SHOTS
        if args.nt == CFG["nt"]:
            c["nt"] = ELSRTM_NT
    vp, vs = synth.dipping_lenses(c["allnx"], c["allnz"], seed=c["seed"])
    vpm, vsm = synth.smooth(vp, 15.0), synth.smooth(vs, 15.0)
    w = synth.ricker(c["nt"], c["f0"], c["dt"])
    if uneven:
        survey = synth.uneven_shots(c["allnx"], c["pml"], c["shots"] * world, c["wmin"], c["wmax"],
                                    seed=c["seed"], sz=c["sz"], gz=c["gz"])
        c["nx"] = max(s.nx for s in survey)
    else:
        survey = synth.surface_shots(c["allnx"], c["allnx"], c["pml"], c["shots"] * world,
                                     sz=c["sz"], gz=c["gz"])
        c["nx"] = c["allnx"]
    mine = shard_shots(survey, world, rank, c["nx"], c["pml"], c["allnz"] + 2 * c["pml"], c["nt"])
    shots = [survey[i] for i in mine]
    return c, vp, vs, vpm, vsm, w, shots


def parse_set(text):
    """'k=v,k2=v2' -> {k: int(v)} (library options of --set)."""
    out = {}
    for item in filter(None, (x.strip() for x in text.split(","))):
        k, v = item.split("=")
        out[k.strip()] = int(v)
    return out


def job_updates(upd, dist, dev):
    """Cell-updates of one step summed over all ranks (shards of uneven windows differ)."""
    if dist is None:
        return upd
    import torch
    t = torch.tensor([float(upd)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def cells(c):
    return (c["allnx"] + 2 * c["pml"]) * (c["allnz"] + 2 * c["pml"])


def cpu_baseline(c, vpm, vsm, w, shot, obs_z, obs_x):
    """Oracle FP32 RTM of one shot on a bounded number of steps, all host cores."""
    from oracle import pyoracle as po
    nt = 120
    st = po.Setup(c["allnx"], c["allnz"], c["allnx"], c["pml"], c["dx"], c["dz"], c["dt"])
    m = po.build_model(st, vpm, vsm, None, shot.win_left, rbc=1, seed=c["seed"], shot_id=0)
    t0 = time.perf_counter()
    po.rtm(st, m, w[:nt], shot, obs_z[:, :nt], obs_x[:, :nt], 1, "f32")
    dt = time.perf_counter() - t0
    upd = 3.0 * cells(c) * nt
    return {"value": upd / dt / 1e9, "unit": "Gcell-updates/s", "cores": os.cpu_count(),
            "kind": "port",
            "sample": f"1 shot x {nt} steps of the 1281x481 RTM (3 propagations), oracle FP32, "
                      f"OpenMP on {os.cpu_count()} threads, {dt:.1f} s"}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measured_tensor_peak():
    """Dense BF16 tensor-core peak in TFLOP/s: the measured burst figure (a cuBLAS GEMM timed
    alone, the right denominator for a pass timed alone), else the earlier pool measurement."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def traffic_for(kernel, cells):
    """DRAM bytes (read + write) per launch of `kernel` over `cells` padded cells (all resident
    shots), from a committed ncu capture (profiles/traffic.json: bytes per shot of the captured
    1281x481 grid), else None.  A launch advances every resident cell by one step, so its traffic
    scales with the cells of the batch."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            per_shot = json.load(f)[kernel]["dram_bytes_per_shot"]
        return round(per_shot * cells / TRAFFIC_CELLS_PER_SHOT)
    except Exception:
        return None


def batch_cells(c, shots):
    """Padded cells of all shots of a batch (each shot's own window width)."""
    nz = c["allnz"] + 2 * c["pml"]
    return sum(((s.nx or c["nx"]) + 2 * c["pml"]) * nz for s in shots)  # nx 0: the grid's nx


def run_ours(args, rank, world, dist):
    import torch
    from ds2d_b200 import Elastic2D
    c, vp, vs, vpm, vsm, w, shots = workload(args, rank, world)
    dev = torch.cuda.current_device()
    ntr = max(s.ntr for s in shots)
    # Observed data: PML forward modelling on the true model (set-up, untimed).
    with Elastic2D(c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                   boundary="pml", max_shots=min(20, c["shots"]), max_ntr=ntr, device=dev) as fm:
        fm.set_models(vp, vs)
        fm.set_wavelet(w)
        obs_z, obs_x = fm.forward(shots)
    tuned = None
    if not args.no_autotune:
        # launch shape chosen by the project's autotuner on a short probe of the same batch
        from ds2d_b200.autotune import apply, tune_rtm
        tuned, tune_ms = tune_rtm(c["allnx"], c["allnz"], c["nx"], c["pml"], c["dx"], c["dz"],
                                  c["dt"], vpm, vsm, w, shots, max_ntr=ntr, seed=c["seed"],
                                  device=dev)
        print("autotune ms per probe step: " + json.dumps(tune_ms), file=sys.stderr, flush=True)
    e = Elastic2D(c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"],
                  boundary="random", max_shots=c["shots"], max_ntr=ntr, seed=c["seed"], device=dev)
    if tuned:
        apply(e, tuned)
    for k, v in parse_set(args.set).items():
        e.set_option(k, v)
        tuned = dict(tuned or {}, **{k: v})
    e.set_models(vpm, vsm)
    e.set_wavelet(w)
    # A non-default stream: the library captures each batch (time loops included) into a CUDA
    # graph, which the legacy default stream does not allow.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    e.set_stream(stream.cuda_stream)
    d_z = torch.from_numpy(obs_z).to(dev)
    d_x = torch.from_numpy(obs_x).to(dev)
    h_z = torch.from_numpy(obs_z).pin_memory()
    h_x = torch.from_numpy(obs_x).pin_memory()
    h2d = int(h_z.numel() + h_x.numel()) * 4
    img_bytes = 3 * c["allnx"] * c["allnz"] * 4

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    red_buf = torch.empty((3, c["allnx"], c["allnz"]), dtype=torch.float32, device=dev)

    def allreduce_images():
        # the one exchange step of the path: the images summed over every rank's shots, device
        # to device into red_buf and one in-place NCCL all-reduce (the library's stream is
        # torch's current stream)
        if dist is not None:
            from ds2d_b200.shard import reduce_images_device
            return reduce_images_device(e, dist, red_buf)
        return None

    # warm-up
    for _ in range(args.warmup):
        e.rtm_device(shots, d_z.data_ptr(), d_x.data_ptr())
    allreduce_images()
    e.read_images(reset=True)
    launches = e.last_launches
    upd = e.last_cell_updates
    # timed device-resident steps
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            e.rtm_device(shots, d_z.data_ptr(), d_x.data_ptr())
            allreduce_images()
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_upd = job_updates(upd, dist, dev) * args.steps
    value = total_upd / (ms / 1e3) / 1e9
    # end-to-end: host (pinned) data in, images out, through the public API
    e.read_images(reset=True)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e.rtm(shots, h_z.numpy(), h_x.numpy())
        if dist is not None:
            allreduce_images().cpu()  # the job's images, read back once per step
        else:
            e.read_images(reset=True, which=("pp_grad", "ps_grad", "illumination"))
    e1.record(stream)
    barrier()
    ms_e2e = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = total_upd / (ms_e2e / 1e3) / 1e9
    # per-kernel roofline from a profiled step (rank 0 only; profiling adds event overhead)
    roof = None
    if rank == 0 and not args.no_profile:
        e.profile(True)
        e.rtm_device(shots, d_z.data_ptr(), d_x.data_ptr())
        rep = e.profile_report()
        e.profile(False)
        tot = sum(v[1] for v in rep.values())
        name, (n, kms, by) = max(rep.items(), key=lambda kv: kv[1][1])
        peak, src = measured_peak()
        achieved = by / n / (kms / n / 1e3) / 1e9
        roof = {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": src,
                "traffic": traffic_for(name, batch_cells(c, shots)), "share": round(kms / tot, 4),
                "kernels": {k: {"launches": v[0], "ms": round(v[1], 3),
                                "GBps": round(v[2] / (v[1] / 1e3) / 1e9, 1) if v[1] > 0 else None}
                            for k, v in rep.items()}}
    out = None
    if rank == 0:
        out = {"metric": "Gcell-updates/s (elastic RTM, random boundary)", "value": round(value, 3),
               "unit": "Gcell-updates/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded dipping-layer + lens model, PML-modelled observed data)",
               "config": {"workload": (f"elastic RTM, random boundary, {c['shots']} shots per GPU"
                                       + (f" with windows U[{c['wmin']}, {c['wmax']}] cells"
                                          if "wmin" in c else "")),
                          "model": (f"{c['allnx']}x{c['allnz']} (+{c['pml']} band) "
                                    + (f"-> {cells(c)} padded cells" if "wmin" not in c else
                                       f"-> per-shot windows (nx + {2 * c['pml']}) x "
                                       f"{c['allnz'] + 2 * c['pml']} cells")),
                          "nt": c["nt"], "shots_per_gpu": c["shots"], "propagations_per_shot": 3,
                          "cell_updates_per_step": total_upd / args.steps, "parallelism": f"shots x{world}",
                          "l2": "inputs larger than L2 (wavefields of all resident shots, GBs)",
                          "launch_shape": tuned or "library defaults (autotuner skipped)"},
               "e2e": {"value": round(e2e, 3), "unit": "Gcell-updates/s",
                       "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": img_bytes},
               "gpu_launches": int(launches * args.steps),
               "clocks": clk.summary(), "roofline": roof}
        if not args.no_cpu_baseline and world == 1 and "wmin" not in c:
            n0 = shots[0].ntr
            out["cpu_baseline"] = cpu_baseline(c, vpm, vsm, w, shots[0], obs_z[:n0], obs_x[:n0])
    e.close()
    return out


def elsrtm_images(c):
    """Seeded reflectivity images (the current model update) of the ELSRTM workload."""
    from ds2d_b200 import synth
    pp = synth.reflectivity(c["allnx"], c["allnz"], seed=5, density=0.05, std=0.05)
    ps = 0.5 * synth.reflectivity(c["allnx"], c["allnz"], seed=6, density=0.05, std=0.05)
    return pp, ps


def run_elsrtm(args, rank, world, dist):
    """Reference-mode ELSRTM iteration (PML, boundary strips, Born modelling of two orders, NCC
    adjoint source, seven images) of this rank's shots, timed with CUDA events; the gradients
    are summed over ranks like the reference's MPI reduction."""
    import torch
    from ds2d_b200 import Elastic2D
    c, vp, vs, vpm, vsm, w, shots = workload(args, rank, world)
    dev = torch.cuda.current_device()
    ntr = max(s.ntr for s in shots)
    g = (c["allnx"], c["allnz"], c["nx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"])
    with Elastic2D(*g, boundary="pml", max_shots=len(shots), max_ntr=ntr, device=dev) as fm:
        fm.set_models(vp, vs)
        fm.set_wavelet(w)
        obs_z, obs_x = fm.forward(shots)
    img_pp, img_ps = elsrtm_images(c)
    e = Elastic2D(*g, boundary="pml", strips="f32", max_shots=len(shots), max_ntr=ntr, device=dev)
    e.set_models(vpm, vsm)
    e.set_wavelet(w)
    e.set_image(img_pp, img_ps)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    e.set_stream(stream.cuda_stream)
    d_z = torch.from_numpy(obs_z).to(dev)
    d_x = torch.from_numpy(obs_x).to(dev)
    h_z = torch.from_numpy(obs_z).pin_memory()
    h_x = torch.from_numpy(obs_x).pin_memory()
    h2d = int(h_z.numel() + h_x.numel()) * 4
    names = ("pp_grad", "ps_grad")
    img_bytes = len(names) * c["allnx"] * c["allnz"] * 4

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    red_buf = torch.empty((len(names), c["allnx"], c["allnz"]), dtype=torch.float32, device=dev)

    def reduce_grads():
        if dist is not None:
            from ds2d_b200.shard import reduce_images_device
            reduce_images_device(e, dist, red_buf, which=names)

    for _ in range(args.warmup):
        e.elsrtm_device(shots, d_z.data_ptr(), d_x.data_ptr(), 1)
    reduce_grads()
    e.read_images(reset=True)
    launches = e.last_launches
    upd = e.last_cell_updates
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            e.elsrtm_device(shots, d_z.data_ptr(), d_x.data_ptr(), 1)
            reduce_grads()
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_upd = job_updates(upd, dist, dev) * args.steps
    value = total_upd / (ms / 1e3) / 1e9
    # end to end: observed records from pinned host memory, gradients back to the host
    e.read_images(reset=True)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e.elsrtm(shots, h_z.numpy(), h_x.numpy(), 1)
        if dist is not None:
            reduce_grads()
            red_buf.cpu()
        else:
            e.read_images(reset=True, which=names)
    e1.record(stream)
    barrier()
    ms_e2e = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = total_upd / (ms_e2e / 1e3) / 1e9
    roof = None
    if rank == 0 and not args.no_profile:
        e.profile(True)
        e.elsrtm_device(shots, d_z.data_ptr(), d_x.data_ptr(), 1)
        rep = e.profile_report()
        e.profile(False)
        tot = sum(v[1] for v in rep.values())
        name, (n, kms, by) = max(rep.items(), key=lambda kv: kv[1][1])
        peak, src = measured_peak()
        achieved = by / n / (kms / n / 1e3) / 1e9
        roof = {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": src,
                "traffic": traffic_for(name, batch_cells(c, shots)), "share": round(kms / tot, 4),
                "kernels": {k: {"launches": v[0], "ms": round(v[1], 3),
                                "GBps": round(v[2] / (v[1] / 1e3) / 1e9, 1) if v[2] > 0 else None}
                            for k, v in rep.items()}}
    out = None
    if rank == 0:
        out = {"metric": "Gcell-updates/s (reference-mode ELSRTM)", "value": round(value, 3),
               "unit": "Gcell-updates/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded dipping-layer + lens model, PML-modelled observed "
                       "data, seeded reflectivity images)",
               "config": {"workload": f"reference-mode ELSRTM, PML + FP32 strips, {len(shots)} "
                                      "shots per GPU",
                          "model": f"{c['allnx']}x{c['allnz']} (+{c['pml']} PML) -> "
                                   f"{cells(c)} padded cells",
                          "nt": c["nt"], "shots_per_gpu": len(shots),
                          "propagations_per_shot": ELSRTM_PROPS,
                          "cell_updates_per_step": total_upd / args.steps, "parallelism": f"shots x{world}",
                          "l2": "inputs larger than L2 (wavefields of all resident shots, GBs)"},
               "e2e": {"value": round(e2e, 3), "unit": "Gcell-updates/s",
                       "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": img_bytes},
               "gpu_launches": int(launches * args.steps),
               "clocks": clk.summary(), "roofline": roof}
        if not args.no_cpu_baseline and world == 1:
            out["cpu_baseline"] = cpu_baseline_elsrtm(c, vpm, vsm, w, shots[0], obs_z, obs_x,
                                                      img_pp, img_ps)
    e.close()
    return out


def cpu_baseline_elsrtm(c, vpm, vsm, w, shot, obs_z, obs_x, img_pp, img_ps):
    """Oracle FP32 reference-mode ELSRTM of one shot on a bounded number of steps."""
    from oracle import pyoracle as po
    nt = 60
    st = po.Setup(c["allnx"], c["allnz"], c["allnx"], c["pml"], c["dx"], c["dz"], c["dt"])
    m = po.build_model(st, vpm, vsm, None, shot.win_left)
    dmp = po.window_image(st, img_pp, shot.win_left)
    dms = po.window_image(st, img_ps, shot.win_left)
    n0 = shot.ntr
    oz = np.ascontiguousarray(obs_z[:n0, :nt])
    ox = np.ascontiguousarray(obs_x[:n0, :nt])
    t0 = time.perf_counter()
    po.elsrtm(st, m, dmp, dms, w[:nt], shot, oz, ox, 1, precision="f32")
    dt = time.perf_counter() - t0
    upd = ELSRTM_PROPS * cells(c) * nt
    return {"value": upd / dt / 1e9, "unit": "Gcell-updates/s", "cores": os.cpu_count(),
            "kind": "port",
            "sample": f"1 shot x {nt} steps of the 1281x481 reference-mode ELSRTM, oracle FP32, "
                      f"OpenMP on {os.cpu_count()} threads, {dt:.1f} s"}


def run_reference_elsrtm(args, c, vp, vs, vpm, vsm, w, shots):
    """The reference's per-shot ELSRTM driver (ELSRTM_ROT_EXP_IMAGE_SINGLESHOT, its own CUDA
    kernels built for sm_100a) on a sample of the workload's shots; the driver call alone is
    timed with CUDA events (the harness's set-up of its FD2DGPU_ELASTIC object is not)."""
    from oracle import pyoracle as po
    sample = shots[:: max(1, len(shots) // args.ref_shots)][:args.ref_shots]
    img_pp, img_ps = elsrtm_images(c)
    g = (c["allnx"], c["allnz"], c["allnx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"])
    obs = [po.ref_forward(*g, vp, vs, w, s) for s in sample]
    for _ in range(args.warmup):
        po.ref_elsrtm(*g, vpm, vsm, w, img_pp, img_ps, sample[0], obs[0][0], obs[0][1], 1)
    tot = 0.0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for s, (oz, ox) in zip(sample, obs):
            tot += po.ref_elsrtm(*g, vpm, vsm, w, img_pp, img_ps, s, oz, ox, 1)["elapsed_ms"]
    wall = time.perf_counter() - t0
    upd = ELSRTM_PROPS * cells(c) * c["nt"] * len(sample) * args.steps
    v = upd / (tot / 1e3) / 1e9
    ve = upd / wall / 1e9
    return {"impl": "reference", "metric": "Gcell-updates/s (reference-mode ELSRTM)",
            "value": round(v, 3), "unit": "Gcell-updates/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(tot / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": "reference-mode ELSRTM, PML + strips",
                                            "shots_per_step": len(sample), "nt": c["nt"],
                                            "propagations_per_shot": ELSRTM_PROPS},
            "cpu_baseline": {"value": round(v, 3), "unit": "Gcell-updates/s", "cores": 1,
                             "kind": "reference",
                             "sample": f"{len(sample)} of the {len(shots)} shots per step, full "
                                       "nt, run by the reference's own per-shot driver and CUDA "
                                       "kernels (FD2DGPU.cu / born.cu built for sm_100a) on the "
                                       "same B200"},
            "e2e": {"value": round(ve, 3), "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_reference(args, rank, world):
    """The reference's own CUDA build (oracle/_ref) on a bounded sample of the same workload."""
    from oracle import pyoracle as po
    if rank != 0:
        return None
    if not po.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libds2dref.so was not built"}
    if args.workload not in ("rtm", "elsrtm"):
        return {"impl": "reference", "unavailable": "the reference runs one window width for all "
                "shots (main.cpp:1010-1017) and has no learned or CG-LSRTM path; its arm covers "
                "the RTM and ELSRTM workloads"}
    import torch  # noqa: F401
    c, vp, vs, vpm, vsm, w, shots = workload(args, 0)
    if args.workload == "elsrtm":
        return run_reference_elsrtm(args, c, vp, vs, vpm, vsm, w, shots)
    sample = shots[:: max(1, len(shots) // args.ref_shots)][:args.ref_shots]
    st = po.Setup(c["allnx"], c["allnz"], c["allnx"], c["pml"], c["dx"], c["dz"], c["dt"])
    # observed data with the reference's own PML forward modelling
    obs = [po.ref_forward(c["allnx"], c["allnz"], c["allnx"], c["pml"], c["nt"], c["dx"], c["dz"],
                          c["dt"], vp, vs, w, s) for s in sample]
    az = np.stack([o[0] for o in obs])
    ax = np.stack([o[1] for o in obs])
    pads = [po.build_model(st, vpm, vsm, None, s.win_left, rbc=1, seed=c["seed"], shot_id=i)
            for i, s in enumerate(sample)]
    vpp, vsp = np.stack([p[0] for p in pads]), np.stack([p[1] for p in pads])
    g = (c["allnx"], c["allnz"], c["allnx"], c["pml"], c["nt"], c["dx"], c["dz"], c["dt"])
    for _ in range(args.warmup):
        po.ref_rtm(*g, vpm, vsm, w, sample, az, ax, rbc=1, vp_pad=vpp, vs_pad=vsp)
    tot = 0.0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _, ms = po.ref_rtm(*g, vpm, vsm, w, sample, az, ax, rbc=1, vp_pad=vpp, vs_pad=vsp)
        tot += ms
    wall = time.perf_counter() - t0
    upd = 3.0 * cells(c) * c["nt"] * len(sample) * args.steps
    v = upd / (tot / 1e3) / 1e9
    ve = upd / wall / 1e9
    return {"impl": "reference", "metric": "Gcell-updates/s (elastic RTM, random boundary)",
            "value": round(v, 3), "unit": "Gcell-updates/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(tot / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": "elastic RTM, random boundary",
                                            "shots_per_step": len(sample), "nt": c["nt"]},
            "cpu_baseline": {"value": round(v, 3), "unit": "Gcell-updates/s", "cores": 1,
                             "kind": "reference",
                             "sample": f"{len(sample)} of the 60 shots per step, full nt, run by "
                                       "the reference's own CUDA kernels (FD2DGPU.cu / born.cu "
                                       "built for sm_100a) on the same B200, driven in the "
                                       "reference driver's order; random band injected"},
            "e2e": {"value": round(ve, 3), "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_acoustic(args):
    """The acoustic Born pair of CG-LSRTM (configs 3 / 5): L^T L (ds2d_ac_normal: background with
    the Born source, scattered set with records, background replay, fused reverse step) on the
    2001x601 grid with a 20-cell random band (or, with --lsrtm-boundary pml, the reference's PML
    and the background rebuilt from --lsrtm-strips boundary strips); shots evenly spread, nt from
    --nt (default 60 here, the profiling case).  Timed with CUDA events on the library's stream."""
    import torch
    from ds2d_b200 import Elastic2D, synth
    allnx, allnz, band = 2001, 601, 20
    nt = args.nt if args.nt != CFG["nt"] else 60
    nshots = args.shots if args.shots != CFG["shots"] else 16
    vp = np.broadcast_to(np.linspace(1800, 4500, allnz, dtype=np.float32), (allnx, allnz)).copy()
    w = synth.ricker(nt, 15.0, 0.0008)
    shots = synth.surface_shots(allnx, allnx, band, nshots)
    m = torch.from_numpy(synth.reflectivity(allnx, allnz, seed=4, density=0.05, std=0.05)).cuda()
    img = torch.zeros_like(m)
    with Elastic2D(allnx, allnz, allnx, band, nt, 10.0, 10.0, 0.0008,
                   boundary=args.lsrtm_boundary, strips=args.lsrtm_strips,
                   max_shots=nshots, max_ntr=allnx, seed=3) as e:
        opts = parse_set(args.set)
        for k, v in opts.items():
            e.set_option(k, v)
        e.set_models(vp, 0 * vp)
        e.set_wavelet(w)
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        e.set_stream(stream.cuda_stream)
        for _ in range(args.warmup):
            e.ac_normal_device(shots, m.data_ptr(), img.data_ptr())
        upd = e.last_cell_updates
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            e.ac_normal_device(shots, m.data_ptr(), img.data_ptr())
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
    out = {"metric": "Gcell-updates/s (acoustic L^T L)", "value": round(upd * args.steps / ms / 1e6, 3),
            "unit": "Gcell-updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (linear 1800-4500 m/s background, seeded sparse reflectivity)",
            "config": {"workload": "acoustic normal operator L^T L", "grid": "2001x601 (+20 band)",
                       "boundary": args.lsrtm_boundary,
                       "strips": args.lsrtm_strips if args.lsrtm_boundary == "pml" else None,
                       "shots": nshots, "nt": nt, "cell_updates_per_step": upd,
                       "options": opts}}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_acoustic(allnx, allnz, band, vp, w, shots[0])
    return out


def cpu_baseline_acoustic(allnx, allnz, pml, vp, w, shot):
    """The reference's own CPU acoustic stepper (main.cpp:602-727, OpenMP on all host threads) on
    the same padded grid with a 20-cell PML, a bounded number of steps (about 10 s of host work,
    from a 20-step probe); cell-updates per second of one propagation."""
    from oracle import pyoracle as po
    if not po.ref_available():
        return None
    st = po.Setup(allnx, allnz, allnx, pml, 10.0, 10.0, 0.0008)
    m = po.build_model(st, vp, 0 * vp, None, shot.win_left)
    damp = np.maximum(m[5], m[6])
    wave = np.tile(w, 200)  # long enough for any sample length
    _, probe = po.ref_cpu_acoustic(m[0], m[2], damp, wave[:20], shot.isx, shot.isz, 0.0008, 10.0, 10.0)
    steps = int(min(3000, max(50, 20 * 6.0 / max(probe, 1e-3))))
    _, sec = po.ref_cpu_acoustic(m[0], m[2], damp, wave[:steps], shot.isx, shot.isz, 0.0008, 10.0,
                                 10.0)
    cells = m[0].size
    return {"value": round(cells * steps / sec / 1e9, 4), "unit": "Gcell-updates/s",
            "cores": os.cpu_count(), "kind": "reference",
            "sample": f"the reference's staggered_grid_extrapolation_2d_pml (main.cpp:602), one "
                      f"acoustic propagation on the {m[0].shape[0]}x{m[0].shape[1]} padded grid, "
                      f"{steps} steps, OpenMP on {os.cpu_count()} threads, {sec:.1f} s"}


def run_unet(args):
    """The preconditioner network (4-level U-Net, 32 base channels, BF16 tensor cores) on one
    2008x608 image: forward pass and one training step (loss gradient + Adam), CUDA events."""
    import torch
    from ds2d_b200.unet import UNet, he_normal, layer_shapes
    h, w = 2008, 608
    x = torch.randn((1, h, w), device="cuda")
    t = torch.randn((1, h, w), device="cuda")
    y = torch.empty_like(x)
    flops = 0.0
    for lvl, (name, ws, _) in enumerate(layer_shapes(32)):
        k, _, co, ci = ws
        scale = 4 ** int(name[1]) // 4 if name[0] in "ed" else 1  # level l runs at 1/4^(l-1) pixels
        flops += 2.0 * h * w / scale * co * ci * k * k
    opts = parse_set(args.set)  # network options (e.g. tcgen05_wgrad=0)
    with UNet(base=32, max_n=1, max_h=h, max_w=w) as net:
        net.set_params(he_normal(5))
        for k, v in opts.items():
            net.set_option(k, v)
        for _ in range(args.warmup):
            net.forward(x.data_ptr(), y.data_ptr(), 1, h, w)
            net.loss_grad(x.data_ptr(), t.data_ptr(), 1, h, w)
        torch.cuda.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        for _ in range(args.steps):
            net.forward(x.data_ptr(), y.data_ptr(), 1, h, w)
        e1.record()
        for _ in range(args.steps):
            net.loss_grad(x.data_ptr(), t.data_ptr(), 1, h, w)
            net.adam_step()
        e2.record()
        torch.cuda.synchronize()
        fwd_ms = e0.elapsed_time(e1) / args.steps
        train_ms = e1.elapsed_time(e2) / args.steps
    tflops = flops / fwd_ms / 1e9
    peak, src = measured_tensor_peak()
    return {"metric": "U-Net forward TFLOP/s (BF16 tensor cores)", "value": round(tflops, 2),
            "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(fwd_ms, 3), "higher_is_better": True, "dtype": "bf16 (fp32 accumulate)",
            "roofline": {"bound": "tensor", "achieved": round(tflops, 2), "peak": peak, "unit": "TFLOP/s",
                         "frac": round(tflops / peak, 4), "peak_source": src, "traffic": None,
                         "scope": "whole forward pass (convolutions, layout kernels, output layer), "
                                  "CUDA events; the per-kernel split is in profiles/"},
            "data": "synthetic (random image)",
            "config": {"workload": "U-Net preconditioner", "image": f"{h}x{w}", "base_channels": 32,
                       "forward_gflop": round(flops / 1e9, 2), "train_step_ms": round(train_ms, 3),
                       "options": opts}}


def run_lsrtm(args):
    """Learned vs plain acoustic CG-LSRTM on one GPU: training pairs (random reflectivity -> Born
    data -> RTM image, 512x256, 40 shots) made by this code, U-Net training on the GPU, then
    ds2d_lsrtm_pcg with and without the network on the application grid."""
    import torch
    from ds2d_b200 import Elastic2D, precond, synth
    from ds2d_b200.unet import UNet, he_normal

    def log(msg):
        print(msg, file=sys.stderr, flush=True)

    dev = torch.cuda.current_device()
    f0, dt, dx, band = 15.0, 0.0008, 10.0, 20
    # ---- training pairs and training -------------------------------------------------------
    # Training survey: 512 columns at the application's depth, record length and shot spacing
    # (full: 600 deep, nt 5000, 20 shots ~ 25 cells apart like 80 shots over 2001 columns;
    # small: the application grid itself, 512x256, nt 2000, 40 shots).
    if args.lsrtm_size == "full":
        tnx, tnz, tnt, tshots = 512, 600, 5000, 20
    else:
        tnx, tnz, tnt, tshots = 512, 256, 2000, 40
    tr_shots = synth.surface_shots(tnx, tnx, band, tshots)
    bkw = dict(boundary=args.lsrtm_boundary, strips=args.lsrtm_strips)
    et = Elastic2D(tnx, tnz, tnx, band, tnt, dx, dx, dt, max_shots=tshots, max_ntr=tnx, seed=7,
                   device=dev, **bkw)
    opts = parse_set(args.set)  # library options of both contexts (e.g. ac_ckpt=500)
    for k, v in opts.items():
        et.set_option(k, v)
    vpt = precond.background(tnx, tnz, seed=1)
    et.set_models(vpt, np.zeros_like(vpt))
    et.set_wavelet(synth.ricker(tnt, f0, dt))
    t0 = time.perf_counter()
    if args.trajectory > 0:
        nmod = max(1, (args.pairs + 16) // args.trajectory)
        X, Y = precond.make_trajectory_pairs(et, tr_shots, nmod, args.trajectory, seed=11, log=log)
        args.pairs = X.shape[0] - 16
    else:
        X, Y = precond.make_pairs(et, tr_shots, args.pairs + 16, seed=11, log=log)
    t_pairs = time.perf_counter() - t0
    cells_pair = 5.0 * tshots * (tnx + 2 * band) * (tnz + 2 * band) * tnt
    et.close()
    anx, anz, ant, ashots = (2001, 601, 5000, 80) if args.lsrtm_size == "full" else (512, 256, 2000, 40)
    hp, wp = (anx + 7) // 8 * 8, (anz + 7) // 8 * 8
    net = UNet(base=32, max_n=8, max_h=max(128, hp), max_w=max(tnz, wp), device=dev)
    net.set_params(he_normal(5))
    t0 = time.perf_counter()
    hist = precond.train(net, X[:args.pairs], Y[:args.pairs], steps=args.train_steps, batch=8,
                         lr=1e-3, log=log)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    ev = precond.evaluate(net, X[args.pairs:], Y[args.pairs:])
    log(f"held-out fit error: network {ev['net']:.3f}, scaled RTM image {ev['rtm']:.3f}")
    del X, Y
    # ---- application: observed Born data of a sparse random reflectivity -------------------
    shots = synth.surface_shots(anx, anx, band, ashots)
    ea = Elastic2D(anx, anz, anx, band, ant, dx, dx, dt, max_shots=ashots, max_ntr=anx, seed=9,
                   device=dev, **bkw)
    for k, v in opts.items():
        ea.set_option(k, v)
    vpa = precond.background(anx, anz, seed=2)
    ea.set_models(vpa, np.zeros_like(vpa))
    ea.set_wavelet(synth.ricker(ant, f0, dt))
    rng = np.random.default_rng(17)
    m_true = torch.from_numpy(precond.random_reflectivity(anx, anz, rng, reflectors=0)).to(dev)
    ntr = sum(s.ntr for s in shots)
    dz = torch.zeros((ntr, ant), dtype=torch.float32, device=dev)
    dxr = torch.zeros_like(dz)
    ea.ac_born_device(shots, m_true.data_ptr(), dz.data_ptr(), dxr.data_ptr())
    res = {}
    for name, p in (("plain", None), ("learned", net)):
        m = torch.zeros_like(m_true)
        r, ms = ea.lsrtm_pcg(shots, dz.data_ptr(), dxr.data_ptr(), m.data_ptr(), args.cg_iters,
                             target=args.target, net=p)
        err = float(((m - m_true).norm() / m_true.norm()).item())
        hit = [t for t, v in zip(ms, r) if v <= args.target]

        def time_to(level):
            h = [t for t, v in zip(ms, r) if v <= level]
            return round(h[0] / 1e3, 2) if h else None
        res[name] = {"time_to_target_s": round(hit[0] / 1e3, 3) if hit else None,
                     "time_to_residual_s": {str(lv): time_to(lv)
                                            for lv in (0.5, 0.3, 0.2, 0.15, 0.1, 0.05, 0.02, 0.01)},
                     "iterations": len(r), "residual": [round(float(v), 5) for v in r],
                     "elapsed_s": [round(float(t) / 1e3, 2) for t in ms],
                     "image_rel_error_vs_true": round(err, 4)}
        log(f"{name}: residual {r[-1]:.4f} after {len(r)} iterations, {ms[-1] / 1e3:.1f} s")
    tp, tl = res["plain"]["time_to_target_s"], res["learned"]["time_to_target_s"]
    # equal-residual speed-up when both reach the target; otherwise the time the learned run needs
    # to reach the plain run's final residual, against the plain run's total time
    if tp is not None and tl is not None:
        speedup = tp / tl
        basis = "time to the target residual, plain / learned"
    else:
        rp = res["plain"]["residual"][-1]
        tl_eq = next((t for t, v in zip(res["learned"]["elapsed_s"], res["learned"]["residual"])
                      if v <= rp), None)
        speedup = res["plain"]["elapsed_s"][-1] / tl_eq if tl_eq else None
        basis = (f"target {args.target} not reached by both; time to the plain run's final "
                 f"residual {rp:.4g}, plain / learned")
    upd = 5.0 * ashots * (anx + 2 * band) * (anz + 2 * band) * ant
    return {"metric": "LSRTM time to 1e-2 relative data residual, learned vs plain (speed-up)",
            "value": round(speedup, 3) if speedup else None, "unit": "x", "basis": basis,
            "higher_is_better": True, "n_gpus": 1, "dtype": "f32 stencils, bf16 network, f64 CG",
            "data": "synthetic (seeded sparse reflectivity on a smooth 1800-4500 m/s background)",
            "config": {"workload": "acoustic CG-LSRTM", "grid": f"{anx}x{anz} (+{band} "
                       + ("random band)" if args.lsrtm_boundary == "random" else
                          f"PML, {args.lsrtm_strips} boundary strips with FP32 scales)"),
                       "shots": ashots, "nt": ant, "cg_iterations": args.cg_iters,
                       "target": args.target, "options": opts},
            "plain": res["plain"], "learned": res["learned"],
            "training": {"pairs": args.pairs, "grid": f"{tnx}x{tnz}", "shots": tshots, "nt": tnt,
                         "pair_generation_s": round(t_pairs, 1),
                         "pair_gcell_updates_per_s": round(cells_pair * (args.pairs + 16) / t_pairs / 1e9, 2),
                         "steps": args.train_steps, "batch": 8, "crop": "128 x full depth",
                         "training_s": round(t_train, 1),
                         "loss_first_last": [round(hist[0], 4), round(hist[-1], 4)],
                         "heldout_fit_error": {k: round(v, 4) for k, v in ev.items()}},
            "cg_iteration_cell_updates": upd}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out))
        return
    import torch
    torch.cuda.set_device(local)
    if args.workload in ("lsrtm", "acoustic", "unet"):
        if rank == 0:
            fn = {"lsrtm": run_lsrtm, "acoustic": run_acoustic, "unet": run_unet}[args.workload]
            print(json.dumps(fn(args)))
        return
    if world > 1:
        import datetime

        import torch.distributed as td
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = td
    out = (run_elsrtm if args.workload == "elsrtm" else run_ours)(args, rank, world, dist)
    if out is not None:
        print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
