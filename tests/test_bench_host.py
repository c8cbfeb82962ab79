"""Host-side logic of bench.py (no GPU): the workloads it measures, their per-rank shards, the
roofline inputs it reads from committed files."""
import json
import os

import numpy as np

import bench
from ds2d_b200.shard import shard_shots


class _Args:
    def __init__(self, workload="rtm", shots=bench.CFG["shots"], nt=bench.CFG["nt"]):
        self.workload, self.shots, self.nt = workload, shots, nt


def test_rtm_workload_is_the_configured_survey_sharded_without_overlap():
    world = 2
    seen = []
    for rank in range(world):
        c, vp, vs, vpm, vsm, w, shots = bench.workload(_Args(nt=50), rank, world)
        assert (c["allnx"], c["allnz"], c["pml"]) == (1201, 401, 40)
        assert vp.shape == (1201, 401) and vpm.shape == vp.shape and len(w) == 50
        assert len(shots) == c["shots"] == 60
        seen += [(s.win_left, s.isx) for s in shots]
    assert len(set(seen)) == 120  # 60 shots per rank, a 120-shot survey, no shot twice


def test_uneven_workload_matches_its_config():
    c, vp, vs, vpm, vsm, w, shots = bench.workload(_Args(workload="uneven", nt=10), 0, 1)
    assert (c["allnx"], c["allnz"], c["pml"], len(shots)) == (4001, 401, 20, 256)
    widths = [s.nx for s in shots]
    assert min(widths) >= 400 and max(widths) <= 1500 and c["nx"] == max(widths)
    assert all(0 <= s.win_left and s.win_left + s.nx <= 4001 for s in shots)
    parts = [shard_shots(shots, 4, r, c["nx"], 20, 441, 10) for r in range(4)]
    assert sorted(i for p in parts for i in p) == list(range(256))


def test_elsrtm_workload_matches_its_config():
    c, vp, vs, vpm, vsm, w, shots = bench.workload(_Args(workload="elsrtm"), 0, 1)
    assert (c["allnx"], c["allnz"], c["pml"], c["nt"]) == (1201, 401, 40, bench.ELSRTM_NT)
    assert len(shots) == c["shots"] == bench.ELSRTM_SHOTS and len(w) == bench.ELSRTM_NT
    pp, ps = bench.elsrtm_images(c)
    assert pp.shape == ps.shape == (1201, 401) and np.abs(pp).max() > 0


def test_roofline_inputs():
    peak, src = bench.measured_peak()
    path = os.path.join(bench.ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        assert src == "measured" and peak == float(json.load(open(path))["hbm_gbs"])
    else:
        assert src == "fallback"
    # committed per-shot DRAM traffic scales with the resident shots of a launch
    cell = bench.TRAFFIC_CELLS_PER_SHOT
    t16, t60 = bench.traffic_for("bwd_fused", 16 * cell), bench.traffic_for("bwd_fused", 60 * cell)
    assert t16 and t60 and abs(t60 / t16 - 60 / 16) < 1e-6
    assert bench.traffic_for("no_such_kernel", 60 * cell) is None
    # uneven windows: traffic follows the batch's padded cells, not its shot count
    c, _, _, _, _, _, shots = bench.workload(_Args(workload="uneven", nt=10), 0, 1)
    assert bench.batch_cells(c, shots) == sum((s.nx + 40) * 441 for s in shots)


def test_autotuner_candidates_name_every_knob():
    """Every candidate of the launch-shape autotuner sets every knob the space uses, so no
    setting carries over from the candidate timed before it; the space holds the time-blocking
    depths 1-4 and the backward variants."""
    from ds2d_b200 import autotune
    for boundary in ("random", "pml"):
        space = autotune.default_space(boundary)
        keys = {tuple(sorted(c)) for c in space}
        assert len(keys) == 1, keys
        assert len({autotune.key(c) for c in space}) == len(space)  # no candidate twice
    space = autotune.default_space("random")
    assert {c["tb"] for c in space} == {0, 1, 2, 3, 4}
    assert {c["bwd_bulk"] for c in space} == {0, 1} and {c["bwd_1b"] for c in space} == {0, 1}
    assert {c["bwd_cta"] for c in space} >= {128, 192, 256}


def test_tensor_peak_reads_the_measured_burst_figure():
    """The U-Net line's roofline denominator: the measured BF16 burst figure when the peaks file
    is there, the earlier pool measurement otherwise; a plausible B200 dense figure either way."""
    import bench
    peak, src = bench.measured_tensor_peak()
    assert src in ("measured", "fallback")
    assert 1000.0 < peak < 2500.0
