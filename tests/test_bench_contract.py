"""CPU tests of bench.py's host side: the reference arm's JSON line (it runs
the reference algorithm on the host cores, so it needs no GPU) and the
parsing of the nvidia-smi clock record that every GPU line carries."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "3", "--edge", "48"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [x for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "site_updates_per_s" and d["unit"] == "site-updates/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] >= 3 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference")
    assert cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_clock_record_summary(tmp_path):
    """The nvidia-smi fallback's CSV and the summary every GPU line carries:
    median SM clock, the reasons seen in any sample, the sample count."""
    import bench

    path = tmp_path / "clocks.csv"
    rows = [  # index, sm, max sm, power, active, hw, hw thermal, sw thermal, sw power cap
        "0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1890, 1965, 998.0, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1845, 1965, 1001.2, 0x4, Not Active, Not Active, Not Active, Active",
        "garbage line",
    ]
    path.write_text("\n".join(rows) + "\n")
    samples, smax = bench.ClockSampler.parse_smi_csv(str(path))
    assert smax == 1965.0 and len(samples) == 3
    cs = bench.ClockSampler(0)
    cs.samples, cs.sm_max, cs.source = samples, smax, "nvidia-smi"
    s = cs.summary()
    assert s == {"sm_mhz": 1890.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"],
                 "samples": 3, "source": "nvidia-smi"}
    assert cs.summary() == s  # computed once, kept
    # NVML reason bits: hardware slowdown and thermal reasons are named
    cs = bench.ClockSampler(0)
    cs.samples = [(1500.0, 0x8 | 0x4), (1600.0, 0x40), (1700.0, 0x0)]
    cs.sm_max, cs.source = 1965.0, "nvml"
    assert cs.summary()["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_power_cap"]
    assert cs.summary()["sm_mhz"] == 1600.0
