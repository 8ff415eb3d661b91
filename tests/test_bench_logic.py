"""The bench's measurement arithmetic, on the CPU: padded sizes, the
algorithmic work each kernel family is credited with, and which DRAM-traffic
capture a bench line cites."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from gbm3d_b200 import autotune, options  # noqa: E402


def _opts(**kw):
    o = options.resolve_opts({"profile": "default"})
    o.update(autotune.BASELINE)
    o.update(kw)
    return o


TUNED7 = dict(refStride=8, refStrideWie=7, matchSpins=[0], matchSpinsWie=[0], cycleSpin=1, staleWeights=False)


@pytest.mark.parametrize("kw,side", [({}, 4097), (dict(refStride=8, refStrideWie=7), 4096),
                                      (dict(refStride=8, refStrideWie=6), 4112),
                                      (dict(refStride=8, refStrideWie=8), 4096)])
def test_padded_side(kw, side):
    """Smallest size >= 4096 at which both reference grids end at the border."""
    o = _opts(**kw)
    p = bench.padded_side(o)
    assert p == side
    s1, s2 = options.strides(o)
    assert (p - 8) % s1 == 0 and (p - 8) % s2 == 0


def test_match_flops_and_tensor_bytes():
    """Matching is credited N_ref * W^2 * d^2 * 3 flop per step and spin."""
    o = _opts(**TUNED7)
    kt = {"match": (2, 1.0)}
    _, work = bench.roofline(o, kt, {}, 1965.0)
    refs1 = ((4096 - 8) // 8 + 1) ** 2
    refs2 = ((4096 - 8) // 7 + 1) ** 2
    assert work["match"]["algorithmic_per_step"] == (refs1 + refs2) * 32 * 32 * 64 * 3
    assert work["match"]["achieved"] == pytest.approx(work["match"]["algorithmic_per_step"] / 1e-3 / 1e12)
    assert work["match"]["peak"] == pytest.approx(148 * 128 * 2 * 1965e6 / 1e12)


def test_traffic_capture_matches_the_option_set():
    """The tuned option sets cite their own 2048^2 capture scaled by the padded
    area; any other set cites the dense 1024^2 capture scaled by references."""
    kt = {"match": (2, 5.0), "aggregate": (2, 1.0)}
    roof, _ = bench.roofline(_opts(**TUNED7), kt, {}, 1965.0)
    side, table = bench.TRAFFIC_TUNED_2048[(8, 7, (0,), (0,), 1, 32)]
    assert roof["kernel"] == "match"
    assert roof["traffic"] == pytest.approx(table["match"] * (4096 / side) ** 2)
    assert "2048x2048" in roof["traffic_source"]
    roof, _ = bench.roofline(_opts(), kt, {}, 1965.0)
    refs = ((4097 - 8) // 3 + 1) ** 2
    assert roof["traffic"] == pytest.approx(bench.TRAFFIC_1024["match"] * refs / bench.REFS_1024)
    assert "1024x1024" in roof["traffic_source"]


def test_measured_hbm_peak_is_used_when_present():
    o = _opts(**TUNED7)
    _, work = bench.roofline(o, {"wiener": (1, 1.0)}, {"hbm_gbs": 7000.0}, 1965.0)
    assert work["wiener"]["peak"] == 7000.0 and work["wiener"]["unit"] == "GB/s"
    _, work = bench.roofline(o, {"wiener": (1, 1.0)}, {}, 1965.0)
    assert work["wiener"]["peak"] == 6650.0


def _replica_rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")      # rank 1 is the slower one
    form = bench.bcast_from_rank0("tuned" if rank == 0 else "plain", dist)
    value = bench.replica_value(world, 16.777216, ms)
    with open(os.path.join(out, f"r{rank}.txt"), "w") as f:
        f.write(f"{ms} {form} {value}")
    dist.barrier()
    dist.destroy_process_group()


def test_replica_mode_two_ranks(tmp_path):
    """bench.py --gpus 2 as two gloo ranks on the CPU: every rank reports the
    slowest rank's time, takes rank 0's choice of form, and the whole-job
    value counts both ranks' images."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_replica_rank, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        ms, form, value = open(tmp_path / f"r{r}.txt").read().split()
        assert float(ms) == 15.0 and form == "tuned"
        assert abs(float(value) - 2 * 16.777216 / 0.015) < 1e-9
