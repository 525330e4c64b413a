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
