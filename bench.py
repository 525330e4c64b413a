"""Benchmark: SIMPLE-CHT outer iterations per second on one B200 (or N
independent replicas, one per GPU).

Workload: 256x128x128 cells (4.19M) channel 2x1x1 with 8 seeded solid blocks
(edges 8-24 cells, seed 0), the reference's FP64 outer step (lid-driven
SIMPLE with first-order upwind momentum, HYPRE-rule CG pressure correction on
the frozen matrix, fluid and solid energy, interface swap).  Synthetic input
generated in-repo; the state (>500 MB of FP64 arrays) is larger than L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line.  `--impl reference` times the CPU restatement of the
reference algorithm (oracle/, single-threaded: Gauss-Seidel in lexicographic
order is sequential) on a bounded sample of the same workload.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "SIMPLE outer iterations/s (FP64, reference-faithful CHT step)"
UNIT = "iter/s"
PEAKS_FILE = os.path.join(HERE, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def workload_deck():
    from hsolver_b200 import cases
    return cases.config2(seed=0)


CONFIG = {"workload": "channel 256x128x128 (4.19M cells), 8 seeded blocks (edges 8-24), reference SIMPLE-CHT step",
          "grid": [256, 128, 128], "blocks": 8, "seed": 0, "precision": "fp64",
          "pressure_solver": "CG (HYPRE PCG rule, rtol 1e-5, maxiter 1000, frozen matrix)",
          "l2_policy": "state arrays > 500 MB, larger than L2 (126 MB)", "parallelism": "replicas"}


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._th = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

        def run():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.samples.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)

        self._th = threading.Thread(target=run, daemon=True)
        self._th.start()

    def stop(self):
        self._stop.set()
        if self._th:
            self._th.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit())
        mx = max(float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].strip() == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.samples)}


def cg_bytes_per_launch(nfluid, iters):
    """Compulsory HBM bytes of one pressure-correction launch (k_pcorr):
    setup reads u*,v*,w* and writes r, p, x (49 B/cell incl. the mask);
    each iteration streams r, p, x, 3 coefficients + mask and writes p, s, x
    (73 B), then r, s + mask and writes r (25 B); the final x update 24 B."""
    return nfluid * (49 + 98 * iters + 24)


def run_gpu(args):
    import torch
    import hsolver_b200

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    deck = workload_deck()
    g = hsolver_b200.Solver(deck, device=local)
    g.init()
    nfluid = int((g.fluid_empty() == 0).sum())
    stream = torch.cuda.ExternalStream(g.stream(), device=local)

    for _ in range(args.warmup):
        g.step(1)
    g.sync()
    c0 = g.counters()
    g.profile(True)
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    phases, nsteps = g.profile_read()
    g.profile(False)
    c1 = g.counters()
    st = g.step(0, stats=True)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # end to end through the C ABI with pinned host buffers: a fresh solver
    # replays the same outer steps; every step uploads the solver state from
    # pinned memory, runs one outer step and reads the state back
    state = ["u_star", "v_star", "w_star", "p_temp", "t_temp", "p"]
    ge = hsolver_b200.Solver(deck, device=local)
    ge.init()
    for _ in range(args.warmup):
        ge.step(1)
    host = {f: torch.empty(ge.field_size(f), dtype=torch.float64, pin_memory=True) for f in state}
    for f in state:
        ge.field(f, out=host[f].numpy())
    L = hsolver_b200.load()
    ids = hsolver_b200.FIELDS
    h2d = sum(host[f].numel() * 8 for f in state)
    e2e_steps = args.steps

    def e2e_step():
        for f in state:
            p = ctypes.cast(host[f].data_ptr(), ctypes.POINTER(ctypes.c_double))
            if L.hs_set_field(ge.h, ids[f], p, host[f].numel()) != 0:
                raise RuntimeError(L.hs_last_error(ge.h).decode())
        ge.step(1)
        for f in state:
            p = ctypes.cast(host[f].data_ptr(), ctypes.POINTER(ctypes.c_double))
            if L.hs_get_field(ge.h, ids[f], p, host[f].numel()) != 0:
                raise RuntimeError(L.hs_last_error(ge.h).decode())

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    ge.close()
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())

    # the mixed-precision pressure solve (FP32 multigrid V-cycle inside FP64
    # CG) on the same case and steps, device-timed the same way
    mixed = None
    if not args.no_variants:
        gm = hsolver_b200.Solver(deck, hsolver_b200.default_params(pressure_solver=hsolver_b200.PSOLVE_MGCG),
                                 device=local)
        gm.init()
        for _ in range(args.warmup):
            gm.step(1)
        gm.sync()
        sm = torch.cuda.ExternalStream(gm.stream(), device=local)
        gm.profile(True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m0.record(sm)
        gm.step(args.steps)
        m1.record(sm)
        m1.synchronize()
        mms = m0.elapsed_time(m1)
        mph, mn = gm.profile_read()
        mst = gm.step(0, stats=True)
        if dist:
            t = torch.tensor([mms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            mms = float(t.item())
        mixed = {"pressure_solver": "CG + FP32 multigrid V-cycle, FP64 recurrences", "value": world * args.steps / (mms * 1e-3),
                 "unit": UNIT, "ms_per_step": mms / args.steps,
                 "phase_ms_per_step": {k: v / max(1, mn) for k, v in mph.items()}, "pcg_iters_last": mst["pcg_iters"]}
        gm.close()

    if rank == 0:
        peak, peak_kind = hbm_peak()
        iters = c1["pcg_iters"] - c0["pcg_iters"]
        solves = max(1, c1["pcg_solves"] - c0["pcg_solves"])
        cg_ms = phases["pressure"] / max(1, nsteps)
        bytes_launch = cg_bytes_per_launch(nfluid, iters / solves)
        achieved = bytes_launch / (cg_ms * 1e-3) / 1e9 if cg_ms > 0 else None
        out = {
            "metric": METRIC, "value": world * args.steps / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded in-repo case generator)",
            "config": CONFIG,
            "e2e": {"value": world * e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
            "roofline": {"bound": "hbm", "kernel": "k_pcorr (pressure-correction CG, one launch per outer step)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": None,
                         "peak_source": peak_kind, "algorithmic_bytes_per_launch": bytes_launch,
                         "cg_iters_per_launch": iters / solves, "launch_ms": cg_ms},
            "phase_ms_per_step": {k: v / max(1, nsteps) for k, v in phases.items()},
            "sweeps_per_step": {k: (c1[k] - c0[k]) / max(1, args.steps) for k in ["sweeps_u", "sweeps_v", "sweeps_w", "sweeps_t"]},
            "last_step": {k: st[k] for k in ["pcg_iters", "pcg_relres", "sweeps_t", "sweeps_solid_max"]},
            "gpu_launches": 17 * args.steps,
            "variants": {"mixed_mgcg": mixed},
            "clocks": clk,
        }
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(deck, 1)
        print(json.dumps(out), flush=True)
    g.close()
    if dist:
        dist.destroy_process_group()


def cpu_baseline(deck, steps):
    """The oracle (CPU FP64 restatement of the reference, one thread) on one
    outer step of the same case."""
    from oracle import oracle
    o = oracle.OracleCase(deck)
    o.init()
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    return {"value": steps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "%d outer step(s) of the bench case after init (first steps), %.1f s" % (steps, dt)}


def run_reference(args):
    """CPU arm: the reference algorithm restated in C (oracle/), since the
    reference's own single-rank build cannot run a case with 8 solid blocks
    (its nParts = 1 decomposition keeps one solid region, mesh/mesh.cpp:2365)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    deck = workload_deck()
    o = oracle.OracleCase(deck)
    o.init()
    warm = min(args.warmup, 1)
    steps = max(1, min(args.steps, 2))
    o.step(warm)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    v = steps / dt
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": steps, "warmup": warm,
        "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded in-repo case generator)", "config": CONFIG, "impl": "reference",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": "%d outer step(s) after %d warm-up step(s); the sequential Gauss-Seidel "
                                   "of the reference uses one thread" % (steps, warm)},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
