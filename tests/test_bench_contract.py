"""bench.py's host-side pieces that shape its JSON line: the autotuner choice
it reports, the dominant kernel and DRAM traffic it reads from the committed
ncu summaries, and the clock summary's throttle reasons."""

import subprocess
import sys
from pathlib import Path

import bench

ROOT = Path(__file__).resolve().parent.parent


def test_tuned_batch_reads_the_autotuner_report():
    line = ("device 0 shape 1x256x256 starts 32 storage 0: batch 8 (resident (15 clusters of 8 "
            "CTAs at once): 0.48 ms, 32: 0.286 ms, 16: 0.248 ms, 8: 0.233 ms)")
    assert bench.tuned_batch(line) == 8
    assert bench.tuned_batch(line.replace("batch 8 (", "resident (")) == "resident"
    assert bench.tuned_batch("device 0 shape 1x64x64 starts 8 storage 0: batch 8 (...)") is None
    assert bench.tuned_batch("") is None


def test_dominant_kernel_and_traffic_come_from_the_committed_summaries():
    dominant = bench.profile_value("dominant_kernel")
    assert dominant in ("modulus", "update")
    traffic = bench.ncu_traffic(dominant)
    assert traffic is not None and traffic > 0
    # the launch list names the kernel with the larger share
    text = (ROOT / "profiles" / "launch_list_gaussians_256x256_32starts.md").read_text()
    shares = {}
    for row in text.splitlines():
        # (the last template argument, when present, is the CTAs per SM)
        if row.startswith("| `column_pass_kernel<256, 3, float, float2, 8"):
            shares["modulus"] = float(row.split("|")[4].strip().rstrip("%"))
        if row.startswith("| `fast_pass_kernel<256, 1, 4, float, float2, float2>`"):
            shares["update"] = float(row.split("|")[4].strip().rstrip("%"))
    assert set(shares) == {"modulus", "update"}
    assert max(shares, key=shares.get) == dominant


def test_clock_summary_flags_throttle_reasons(tmp_path):
    sampler = bench.ClockSampler(0)
    sampler.path = tmp_path / "clocks.csv"
    sampler.path.write_text(
        "0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active\n"
        "0, 1800, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active\n")
    sampler.proc = object()  # the samples are already on disk
    summary = sampler.summary()
    assert summary["sm_max_mhz"] == 1965.0
    assert summary["reasons"] == ["sw_power_cap"]


def test_reference_arm_on_a_non_zero_rank_prints_nothing():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"],
                         env={"RANK": "1", "PATH": "/usr/bin:/bin"}, capture_output=True,
                         text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0
    assert out.stdout.strip() == ""
