"""Autotuner of the fused elastic kernels' launch shape (no counterpart in the reference, whose
launches are fixed 32x32 blocks).

The knobs are the rows marched per CTA (`xr`), the depth of the cp.async prefetch ring (`ring`),
the register / occupancy target (`occ`) and the threads per CTA (`cta`, 128 or 192) of the
one-column ring kernels, and, for the random boundary, the pair-blocked bulk-copy kernels
(`pair`) with their CTA widths (`pair_cta` backward, `pair_fcta` forward), rows per CTA
(`pair_xr`) and the backward step fused or split in two launches (`pair_split`); `pair` 2
takes the pair kernel for the forward step only, with the backward on the one-column kernel.
The forward step can also run time-blocked (`tb` = time steps per launch, 1-4, `tb_cta` = its
CTA width, `tb_bulk` = operand rows by bulk copy at depth 1-2): one launch advances the batch by
`tb` steps, reading and writing the state once.
The backward step can run warp-specialised (`bwd_ws` = threads per role, 96 / 128 / 192: the
source and adjoint wavefields on separate warps of one CTA), with one barrier per row step
(`bwd_1b`), and with its operand rows fed by bulk copies (`bwd_bulk`, CTA width `bwd_cta`).
Their best values depend on the grid, the number of resident shots and the boundary, so the
tuner times each candidate on a probe context with the caller's grid and batch but only
`probe_nt` time steps (an RTM of the same shots: one forward and one backward fused launch per
step), and returns the fastest setting; `apply` copies it onto the production context.  Everything runs through the public API on the GPU."""
import numpy as np

from .api import Elastic2D

_RING_BASE = {"pair": 0, "pair_split": 0, "pair_cta": 0, "pair_fcta": 0, "pair_xr": 0, "tb": 0,
              "tb_cta": 0, "tb_bulk": 1, "bwd_ws": 0, "bwd_1b": 0, "bwd_bulk": 0, "bwd_cta": 0}
_RING_SPACE = [
    {"ring": 4, "xr": 128, "occ": 0, "cta": 128}, {"ring": 4, "xr": 128, "occ": 0, "cta": 192},
    {"ring": 4, "xr": 64, "occ": 0, "cta": 128}, {"ring": 4, "xr": 256, "occ": 0, "cta": 192},
    {"ring": 2, "xr": 128, "occ": 0, "cta": 128}, {"ring": 4, "xr": 128, "occ": 1, "cta": 128},
]
# Pair-blocked kernels (random boundary only): backward CTA width x rows per CTA (0 = the
# library's wave-filling choice).
_PAIR_SPACE = ([{"pair": 2, "pair_split": 0, "pair_cta": 0, "pair_fcta": fcta, "pair_xr": xr,
                 "cta": cta}
                for fcta in (256, 64) for xr in (0, 143) for cta in (192, 128)] +
               [{"pair": 1, "pair_split": 0, "pair_cta": cta, "pair_fcta": 256, "pair_xr": xr}
                for cta in (256, 64) for xr in (0, 96)] +
               [{"pair": 1, "pair_split": 1, "pair_cta": 0, "pair_fcta": 256, "pair_xr": xr}
                for xr in (0, 96)])
# Time-blocked forward (random boundary only): depth 1-4 at the automatic CTA width, and the
# 512-thread single-strip CTAs at depth 1-2; the backward on the one-column ring kernel.
_TB_SPACE = ([{"tb": k, "tb_cta": 0, "cta": 192} for k in (1, 2, 3, 4)] +
             [{"tb": k, "tb_cta": 512, "cta": 192} for k in (1, 2)] +
             [{"tb": 2, "tb_cta": 0, "tb_bulk": 0, "cta": 192}])
# Backward variants (random boundary only) behind the two best forward kernels: warp-specialised
# (`bwd_ws` threads per role), the ring kernel with one barrier per row step (`bwd_1b`), and the
# ring fed by bulk copies (`bwd_bulk`, with either barrier count).
_WS_SPACE = ([{"tb": 2, "tb_cta": 0, "bwd_ws": kt} for kt in (96, 128, 192)] +
             [{"pair": 2, "pair_fcta": 256, "bwd_ws": kt} for kt in (96, 128, 192)] +
             [{"tb": 2, "tb_cta": 0, "bwd_1b": 1, "cta": cta} for cta in (128, 192)] +
             [{"pair": 2, "pair_fcta": 256, "bwd_1b": 1, "cta": cta} for cta in (128, 192)] +
             [{"tb": 2, "tb_cta": 0, "bwd_bulk": 1, "bwd_1b": one, "bwd_cta": bc}
              for one in (0, 1) for bc in (128, 192, 256)] +
             [{"tb": k, "tb_cta": tc, "bwd_bulk": 1, "bwd_cta": 0} for k in (1, 2) for tc in (256, 512)] +
             [{"pair": 2, "pair_fcta": 256, "bwd_bulk": 1, "bwd_1b": one, "bwd_cta": bc}
              for one in (0, 1) for bc in (128, 192, 256)] +
             [{"tb": 2, "tb_cta": 0, "bwd_bulk": 1, "bwd_1b": 1, "bwd_cta": 256, "pair_xr": pxr}
              for pxr in (96, 128, 192)])
_RING_DEFAULTS = {"ring": 4, "xr": 128, "occ": 0, "cta": 0, "tb": 0, "tb_cta": 0, "tb_bulk": 1,
                  "bwd_ws": 0, "bwd_1b": 0, "bwd_bulk": 0, "bwd_cta": 0}


def default_space(boundary="random"):
    """Full option sets (every knob named, so no setting carries over between candidates)."""
    space = [dict(_RING_BASE, **c) for c in _RING_SPACE]
    if boundary == "random":
        space = ([dict(_RING_DEFAULTS, **c) for c in _PAIR_SPACE] +
                 [{**_RING_DEFAULTS, **_RING_BASE, **c} for c in _TB_SPACE + _WS_SPACE] + space)
    return space


DEFAULT_SPACE = default_space("random")


def tune_rtm(allnx, allnz, nx, pml, dx, dz, dt, vp, vs, wavelet, shots, boundary="random",
             max_ntr=None, seed=0, device=0, probe_nt=48, space=None, repeats=2):
    """Times every setting of `space` on an RTM of `shots` with probe_nt steps; returns
    (best setting, {setting key: ms per step})."""
    import torch
    space = space or default_space(boundary)
    max_ntr = max_ntr or max(s.ntr for s in shots)
    w = np.asarray(wavelet, np.float32)[:probe_nt]
    timings = {}
    with Elastic2D(allnx, allnz, nx, pml, probe_nt, dx, dz, dt, boundary=boundary,
                   max_shots=len(shots), max_ntr=max_ntr, seed=seed, device=device) as e:
        e.set_models(vp, vs)
        e.set_wavelet(w)
        stream = torch.cuda.Stream(device=device)
        e.set_stream(stream.cuda_stream)
        ntr = sum(s.ntr for s in shots)
        az = torch.zeros((ntr, probe_nt), dtype=torch.float32, device=f"cuda:{device}")
        for cfg in space:
            for k, v in cfg.items():
                e.set_option(k, v)
            e.rtm_device(shots, az.data_ptr(), az.data_ptr())  # warm-up (and graph capture)
            torch.cuda.synchronize(device)
            best = float("inf")
            for _ in range(repeats):
                ev0 = torch.cuda.Event(enable_timing=True)
                ev1 = torch.cuda.Event(enable_timing=True)
                ev0.record(stream)
                e.rtm_device(shots, az.data_ptr(), az.data_ptr())
                ev1.record(stream)
                torch.cuda.synchronize(device)
                best = min(best, ev0.elapsed_time(ev1) / probe_nt)
            timings[key(cfg)] = best
            e.read_images(reset=True)
    best_cfg = min(space, key=lambda c: timings[key(c)])
    return dict(best_cfg), timings


def key(cfg):
    return ",".join(f"{k}={cfg[k]}" for k in sorted(cfg))


def apply(ctx, cfg):
    for k, v in cfg.items():
        ctx.set_option(k, v)
