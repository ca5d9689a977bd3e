"""Host-side checks of bench.py's bookkeeping: the clock summary and the roofline inputs read from
profiles/ (no GPU)."""
import json
import pathlib

import pytest

import bench

ROOT = pathlib.Path(__file__).resolve().parent.parent


def test_clock_summary_reports_median_and_every_reason_seen():
    clk = bench.Clocks(0)
    bits = bench.Clocks.REASON_BITS
    clk.max_mhz = 1965.0
    clk.samples = [(1965.0, 0), (1950.0, bits["sw_power_cap"]), (1800.0, bits["hw_slowdown"] | bits["sw_power_cap"])]
    s = clk.summary()
    assert s["sm_mhz"] == 1950.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]


def test_clock_summary_without_samples_says_so():
    s = bench.Clocks(0).summary()
    assert s["samples"] == 0 and s["reasons"] == ["unsampled"]


@pytest.mark.parametrize("kernel", ["list_scan", "density_lambda", "correction_project"])
def test_dram_traffic_of_the_gather_passes_is_recorded(kernel):
    traffic = bench.traffic_from_profiles(kernel)
    assert traffic is not None and traffic > 16 * 1048576   # at least the iterate read once at 1M particles


def test_issue_roofline_uses_the_recorded_instruction_count():
    instructions = bench.profile_figure("warp_instructions_per_launch", "list_scan")
    assert instructions is not None and instructions > 0
    r = bench.issue_roofline("list_scan", 0.25)
    mhz = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["sm_max_mhz"] if (ROOT / "MEASURED_PEAKS.json").exists() else 1965.0
    peak = 148 * 4 * mhz * 1e-3
    assert r["peak"] == pytest.approx(peak, rel=1e-3)
    assert r["achieved"] == pytest.approx(instructions / 0.25e-3 / 1e9, rel=1e-3)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"], rel=1e-3)
    assert bench.issue_roofline("no_such_kernel", 0.25) is None


def test_profile_figures_name_the_command_that_made_them():
    text = (ROOT / "profiles" / "substep_dam_break_1m.md").read_text()
    assert "ncu --set full --clock-control none" in text and "ncu --metrics gpu__time_duration.sum --clock-control none" in text


def _max_rank(rank, world, port, out):
    import os
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # every rank reports its own time; the job's time is the slowest rank's
        out[rank] = bench.max_over_ranks(1.5 + rank, world)
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_takes_the_slowest_rank():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_max_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert dict(out) == {0: 2.5, 1: 2.5}

