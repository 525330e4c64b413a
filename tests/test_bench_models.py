"""The algorithmic byte counts behind bench.py's roofline fractions, on the
CPU: the per-cell figures that the kernel documentation states, and the
fraction arithmetic (achieved = bytes / event time, frac = achieved / peak)."""
import pytest

import bench


def test_pcg_bytes_per_cell():
    # FP64, 2 red-black sweeps on level 0 and 3 on the coarser levels
    assert bench.pcg_bytes(1, 0) == 58  # set-up
    # per CG iteration: CG 113, four sweeps of 49, transfers 43, coarser levels (6 x 49 + 43) / 7
    per = bench.pcg_bytes(1, 1) - bench.pcg_bytes(1, 0)
    assert per == pytest.approx(113 + 4 * 49 + 43 + (6 * 49 + 43) / 7.0)
    assert per == pytest.approx(400.142857, abs=1e-6)
    # FP32 storage: CG 57, sweeps 25, transfers 21.5
    per32 = bench.pcg_bytes(1, 1, wbytes=4) - bench.pcg_bytes(1, 0, wbytes=4)
    assert per32 == pytest.approx(57 + 4 * 25 + 21.5 + (6 * 25 + 21.5) / 7.0)


def test_energy_bytes_per_cell():
    # one FP64 energy step with one BiCGStab iteration (two V-cycles)
    assert bench.energy_bytes(1, 1) == pytest.approx(1415.057, abs=1e-3)


def test_kernel_classes_fractions():
    dims = (256, 128, 128)
    ncell = dims[0] * dims[1] * dims[2]
    nface = (dims[0] + 1) * dims[1] * dims[2] + dims[0] * (dims[1] + 1) * dims[2] + dims[0] * dims[1] * (dims[2] + 1)
    phases = {"momentum": 0.8, "p_assembly": 0.1, "p_solve": 5.0, "correction": 0.1, "energy": 1.5}
    kc = bench.kernel_classes(phases, 7, dims, 2, 6650.0)
    expect = {"momentum": 49.0 * nface * 2 * 2, "p_assembly": 89.0 * ncell, "p_solve": bench.pcg_bytes(ncell, 7),
              "correction": 97.0 * ncell, "energy": bench.energy_bytes(ncell, 1)}
    for k, b in expect.items():
        assert kc[k]["algorithmic_bytes"] == b, k
        gbs = b / (phases[k] * 1e-3) / 1e9
        assert kc[k]["achieved_gbs"] == pytest.approx(gbs), k
        assert kc[k]["frac"] == pytest.approx(gbs / 6650.0), k


def _fake_smi(tmp_path, lines):
    """An nvidia-smi stand-in that prints the given CSV lines in a loop every
    50 ms, as `nvidia-smi --query-gpu=... -lms` does."""
    script = tmp_path / "nvidia-smi"
    body = "".join("echo '%s'\n" % ln for ln in lines)
    script.write_text("#!/bin/bash\nwhile true; do\n%s sleep 0.05\ndone\n" % body)
    script.chmod(0o755)
    return str(tmp_path)


def test_clock_sampler_reads_the_loop(tmp_path, monkeypatch):
    """bench.ClockSampler keeps the samples taken inside the timed region
    (median SM clock, the maximum, the throttle reasons that were active)."""
    import os
    import time
    d = _fake_smi(tmp_path, ["1965, 1965, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
                             "1800, 1965, 0x0000000000000004, Not Active, Not Active, Not Active, Active"])
    monkeypatch.setenv("PATH", d + os.pathsep + os.environ["PATH"])
    c = bench.ClockSampler(0)
    c.start()
    time.sleep(0.4)
    out = c.stop()
    assert out["samples"] >= 2
    assert out["sm_max_mhz"] == 1965.0
    assert out["sm_mhz"] in (1800.0, 1965.0)
    assert out["reasons"] == ["sw_power_cap"]


def test_clock_sampler_without_nvidia_smi(tmp_path, monkeypatch):
    """No nvidia-smi on the PATH: the line says the clocks went unsampled."""
    monkeypatch.setenv("PATH", str(tmp_path))
    c = bench.ClockSampler(0)
    c.start()
    assert c.stop() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}


def test_clock_sampler_nvml(monkeypatch):
    """The NVML path: SM clock and the clock-event bit mask read every 10 ms,
    the reasons named from the mask."""
    import time

    class FakeNvml:
        NVML_CLOCK_SM = 1

        def __init__(self):
            self.n = 0

        def nvmlDeviceGetMaxClockInfo(self, h, which):
            return 1965

        def nvmlDeviceGetClockInfo(self, h, which):
            self.n += 1
            return 1965 if self.n % 2 else 1800

        def nvmlDeviceGetCurrentClocksEventReasons(self, h):
            return 0x4 | 0x1  # sw_power_cap, idle

    fake = FakeNvml()
    monkeypatch.setattr(bench, "_nvml_open", lambda index: (fake, object()))
    c = bench.ClockSampler(0)
    c.start()
    time.sleep(0.2)
    out = c.stop()
    assert out["samples"] >= 5
    assert out["sm_max_mhz"] == 1965.0
    assert out["sm_mhz"] in (1800.0, 1965.0)
    assert out["reasons"] == ["sw_power_cap"]
