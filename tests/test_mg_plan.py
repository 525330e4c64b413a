"""The placement of the V-cycle's coarse levels in block 0's shared memory
(mg::plan_stage), checked on the host: a small program compiled from
tests/mg_plan/plan.cu prints the plan for a grid, which must follow the rule
(every level from the first of at most 2048 cells on, less the finest of
them while their x and rhs exceed 64 KB), with 16-byte aligned,
non-overlapping arrays inside the staging area; after them the couplings of
the coarsest of those levels, as many as fit in 160 KB in all."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def plan_exe(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    exe = str(tmp_path_factory.mktemp("mg_plan") / "plan")
    r = subprocess.run([nvcc, "-std=c++17", "-O1", os.path.join(HERE, "mg_plan", "plan.cu"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _levels(n):
    out = [tuple(n)]
    while out[-1][0] * out[-1][1] * out[-1][2] > 64:
        out.append(tuple((v + 1) // 2 for v in out[-1]))
    return out


def _expected(n, size):
    lv = _levels(n)

    def b(d):
        return ((d[0] + 2) * (d[1] + 2) * (d[2] + 2) * size + 15) // 16 * 16

    ls = 0
    while ls < len(lv) - 1 and lv[ls][0] * lv[ls][1] * lv[ls][2] > 2048:
        ls += 1
    tot = sum(2 * b(d) for d in lv[ls:])
    while tot > 65536 and ls < len(lv) - 1:
        tot -= 2 * b(lv[ls])
        ls += 1
    sro = len(lv)
    while sro > ls and tot + 3 * b(lv[sro - 1]) <= 160 * 1024:
        sro -= 1
        tot += 3 * b(lv[sro])
    return len(lv), ls, tot, [b(d) for d in lv], sro


@pytest.mark.parametrize("n", [(256, 128, 128), (512, 256, 256), (48, 24, 24), (16, 8, 8), (512, 4, 4),
                               (4, 4, 4), (2048, 1, 1), (100, 37, 3)])
def test_stage_plan(plan_exe, n):
    r = subprocess.run([plan_exe, *map(str, n)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    for line in r.stdout.strip().splitlines():
        head, ro = line.split("|")
        f, g = head.split(), ro.split()
        size, L, ls, stage = map(int, f[:4])
        eL, els, etot, sizes, esro = _expected(n, size)
        assert (L, ls, stage, int(g[0])) == (eL, els, etot, esro), (n, size)
        assert 0 < stage <= 160 * 1024
        spans = []
        for l, off in zip(range(ls, L), f[4:]):
            sx, sr = map(int, off.split(":"))
            assert sx % 16 == 0 and sr % 16 == 0
            spans += [(sx, sx + sizes[l]), (sr, sr + sizes[l])]
        assert len(g) - 1 == L - esro
        for l, off in zip(range(esro, L), g[1:]):
            for o in map(int, off.split(":")):
                assert o % 16 == 0
                spans.append((o, o + sizes[l]))
        spans.sort()
        assert spans[0][0] == 0 and spans[-1][1] == stage
        assert all(a[1] <= b[0] for a, b in zip(spans, spans[1:]))
