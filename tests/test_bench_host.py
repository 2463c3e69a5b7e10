"""Host-side logic of the bench: the algorithmic byte counts behind the roofline figures and the
parsing of the nvidia-smi clock record that decides whether a timed run is kept."""
import bench


def test_algorithmic_bytes_of_the_precision_snapshot():
    # 26 B per sample, 24 B per row, 8 B per channel, 32 B per plane cell, 4 B per pixel
    n_s, rows, chans, G, N = 8_372_224, 130_816, 64, 3072, 2048
    b = bench.algorithmic_bytes(n_s, rows, chans, 1, G, N)
    assert b == 217_677_824 + 3_139_584 + 512 + 301_989_888 + 16_777_216 == 539_585_024
    assert bench.algorithmic_bytes(n_s, rows, chans, 8, G, N) - b == 7 * 32 * G * G
    # gridding stage: a 16 B record per gridded sample, one 8 B write per plane cell
    assert bench.grid_kernel_bytes(7_017_770, 1, G) == 16 * 7_017_770 + 8 * G * G == 187_781_792


def test_clock_record_summary(tmp_path):
    rows = [
        "0, 1965, 1965, 812.4, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 990.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 995.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, [N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",  # unreadable sample
        "garbage",
    ]
    p = tmp_path / "clocks.csv"
    p.write_text("\n".join(rows) + "\n")
    s = bench.ClockSampler(0)
    s.path = str(p)
    out = s.summary()
    assert out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0 and out["samples"] == 3
    assert out["reasons"] == ["sw_power_cap"]
    assert not p.exists()  # the temporary record is removed once summarised


def test_clock_record_flags_thermal_slowdown(tmp_path):
    p = tmp_path / "clocks.csv"
    p.write_text("0, 1410, 1965, 1000.0, 0x0000000000000060, Active, Not Active, Active, Active\n")
    s = bench.ClockSampler(0)
    s.path = str(p)
    out = s.summary()
    assert out["reasons"] == ["hw_slowdown", "sw_power_cap", "sw_thermal_slowdown"]
    assert out["sm_mhz"] == 1410.0


def test_missing_clock_record_reads_unsampled(tmp_path):
    s = bench.ClockSampler(0)
    s.path = str(tmp_path / "absent.csv")
    assert s.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
