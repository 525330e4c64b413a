"""Benchmark: SIMPLE conjugate-heat-transfer outer iterations per second on
one B200 (or N independent replicas, one per GPU).

Workload (the at-scale drop-in configuration): 256x128x128 cells (4.19M)
channel 2x1x1, inlet plug flow u = 1, zero-gradient outlet, no-slip walls,
Re = 400, Pr = 0.71, 8 seeded solid blocks (edges 8-24 cells, seed 0) with a
heat source q ~ U[0.5, 2] and k_solid/k_fluid ~ U[10, 1000] per block;
relaxation 0.7 / 0.3 / 0.9; FP64 throughout (the plain form); pressure
correction by multigrid-preconditioned CG to the reference's rtol 1e-5
(fluid_solver.h:1874); energy over fluid and solid by multigrid-preconditioned
BiCGStab to 0.5 of its initial residual per outer step (the temperature is
one-way coupled; its residual stays an order below the momentum residuals).
(The number of outer steps to a 1e-6 global residual is the same, 1393, for
p' rtol 1e-8 .. 1e-3 and energy 1e-2 .. 0.5: SIMPLE's rate is set by the
relaxation; the stop test includes the FP64 energy residual.)  Synthetic input generated
in-repo; the state (~790 MB on the device) is larger than L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--no-cpu-baseline] [--no-variants]
  python bench.py --probe NAME [--steps K] [--mixed] [--p-tol X] [--t-tol X]
                  [--t-maxiter N] [--p-level0 L] [--conv C] [--ri X]

Prints one JSON line.  Variants on the same GPU: the mixed-precision form,
the adjoint/forward cost of the energy gradient, wall time to a global
residual of 1e-6 (the 256x128x128 case, config 1 and config 3; the first is
also `time_to_1e-6` and `speedup_mixed` at the top level), the
reference-faithful lid-cavity step on the same grid, the reference's own
compiled code against the GPU on the reference's deck (`like_for_like`),
the 512x256x256 case, the momentum convection schemes with buoyancy
(`convection`) and the z-slab pressure-correction solve on 1, 2 and 4 slabs
of this GPU (`sharded_p_solve`).  `--gpus N` > 1 without a launcher reruns itself
under torch.distributed.run with N ranks (independent replicas, one per
GPU).  `--impl reference` times the CPU restatement (oracle/, FP64, OpenMP on
every host thread, the count in cpu_baseline.cores) on 1-2 outer steps of the
same workload with the reference's inner-solver settings; it loads no part
of the CUDA library.
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

METRIC = "SIMPLE outer iterations/s (channel conjugate heat transfer, FP64)"
UNIT = "iter/s"
PEAKS_FILE = os.path.join(HERE, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
NAME = "config2"
# inner solves of the at-scale case (config 1 keeps the library defaults,
# p' rtol 1e-8 as its specification states): p' to rtol 1e-5, and one
# BiCGStab iteration (two V-cycles) of the energy per outer step.  Neither
# changes the number of outer steps to a global residual of 1e-6 on this case
# (1393 for p' rtol 1e-8 to 1e-3 and for an energy solve to 1e-2 per step):
# SIMPLE's rate is set by the relaxation, and the energy residual stays an
# order below the momentum residuals.
SOLVER = {"p_tol": 1e-5, "t_tol": 0.5, "t_maxiter": 1}
CONFIG = {"workload": "channel 256x128x128 (4.19M cells), 8 seeded heated blocks (edges 8-24, q U[0.5,2], "
                      "k_s/k_f U[10,1000]), Re 400, SIMPLE-CHT outer step",
          "grid": [256, 128, 128], "blocks": 8, "seed": 0, "precision": "fp64", "re": 400, "pr": 0.71,
          "relaxation": {"u": 0.7, "p": 0.3, "T": 0.9}, "momentum": "FOU, 2 red-black GS sweeps",
          "pressure_solver": "CG + multigrid V-cycle (FP64; 2 red-black sweeps each way on the finest level, 3 on the coarser), rtol 1e-5 (the reference's HYPRE setting)",
          "energy_solver": "BiCGStab + multigrid V-cycle (FP64), one iteration per outer step",
          "l2_policy": "state ~790 MB on the device, larger than L2 (126 MB)", "parallelism": "replicas"}
# red-black sweeps before and after the coarse correction on the finest level
# of the p' V-cycle, one more on the coarser levels (the library default,
# hs_channel_params.p_mg_sweeps = 0)
MG_SWEEPS = 2
# launches per outer step: 4 momentum passes, p' assembly, residual finalize,
# p' solve, correction, energy assembly, energy BiCGStab, energy relaxation
LAUNCHES_PER_STEP = 11
# DRAM bytes per CG iteration of k_ch_pcg on this case, from one ncu capture
# (profiles/k_ch_pcg_config2.md: 18.30 GB per 8-iteration launch)
PCG_TRAFFIC_PER_ITER = 18.30e9 / 8


def workload(name=NAME, seed=0, host_side=False):
    """The seeded deck of a configuration, its Reynolds number, the k ratio
    per block and q per cell.  The cell types come from the product's case
    model (hs_case_*), or from the oracle's when host_side is set: the CPU
    arms load no part of the CUDA library."""
    from hsolver_b200 import cases
    deck = cases.CONFIGS[name](seed) if name in ("config2", "config4", "config5") else cases.CONFIGS[name]()
    if host_side:
        from oracle import oracle
        ctype, region = oracle.OracleCase(deck).cell_types()
    else:
        import hsolver_b200
        ctype, region = hsolver_b200.Case(deck).cell_types()
    re_, k, q = cases.block_physics(name, ctype, region, seed)
    return deck, re_, k, q, ctype


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def _nvml_open(index):
    """NVML and the handle of CUDA device `index` (found by its PCI address,
    since NVML numbers the GPUs without regard to CUDA_VISIBLE_DEVICES)."""
    import pynvml
    import torch
    pynvml.nvmlInit()
    pr = torch.cuda.get_device_properties(index)
    try:
        h = pynvml.nvmlDeviceGetHandleByPciBusId("%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id))
    except Exception:
        u = str(pr.uuid)
        h = pynvml.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
    return pynvml, h


class ClockSampler:
    """SM clocks and throttle reasons during the timed region: read through
    NVML every 10 ms by a thread (reading only), or, where NVML cannot be
    opened, from one nvidia-smi process in its loop mode (every 100 ms;
    start() then returns once its first sample is in, at most 3 s, and only
    later samples are kept)."""

    QUERY = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, index):
        self.index = index
        self.samples = []  # (time, sm MHz, max MHz, [reason names])
        self._proc = None
        self._th = None
        self._stop = threading.Event()
        self._t0 = 0.0

    def _start_nvml(self):
        nv, h = _nvml_open(self.index)
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons

        def sample():
            sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
            bits = int(get_reasons(h))
            self.samples.append((time.perf_counter(), sm, mx, [n for n, b in self.REASONS if bits & b]))

        sample()  # fails here, before the thread, if NVML cannot read the device

        def run():
            while not self._stop.wait(0.01):
                try:
                    sample()
                except Exception:
                    return

        self._th = threading.Thread(target=run, daemon=True)
        self._th.start()

    def _start_smi(self):
        self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        num = lambda v: float(v) if v.replace(".", "").isdigit() else None  # noqa: E731

        def run():
            for line in self._proc.stdout:
                f = [x.strip() for x in line.strip().split(",")]
                if len(f) >= 7:
                    self.samples.append((time.perf_counter(), num(f[0]), num(f[1]),
                                         [n for (n, _), v in zip(self.REASONS, f[3:7]) if v == "Active"]))

        self._th = threading.Thread(target=run, daemon=True)
        self._th.start()
        t_end = time.perf_counter() + 3.0
        while not self.samples and time.perf_counter() < t_end and self._proc.poll() is None:
            time.sleep(0.01)

    def start(self):
        try:
            self._start_nvml()
        except Exception:
            self.samples = []
            try:
                self._start_smi()
            except Exception:
                self._proc = None
        self._t0 = time.perf_counter()

    def stop(self):
        self._stop.set()
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        if self._th:
            self._th.join(timeout=5)
        # the samples taken in the region (or, for a region shorter than the
        # sampling interval, the last one before it)
        region = [x for x in self.samples if x[0] >= self._t0] or \
            [x for x in self.samples if x[0] < self._t0][-1:]
        if not region:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(x[1] for x in region if x[1] is not None)
        mxs = [x[2] for x in region if x[2] is not None]
        reasons = sorted({n for x in region for n in x[3]})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": max(mxs) if mxs else None,
                "reasons": reasons, "samples": len(region)}


def pcg_bytes(ncell, iters, wbytes=8, sweeps=MG_SWEEPS):
    """Algorithmic HBM bytes of one pressure-correction solve, per cell, with
    w bytes per stored value (8 in the FP64 form, 4 in the mixed form's FP32
    storage): the compulsory-traffic model in which every input array of a
    kernel is read once and every output written once, neighbours hitting in
    cache, masks at 1 byte:
      set-up: couplings 3w and the solid mask read, level-0 mask written,
        r read, diagonal and the V-cycle's seed written -> 7w + 2;
      per CG iteration:
        the fused CG (A p with <s, p>; x, r update with <r, r>; p update):
          14w + 1 (113 B in FP64);
        a red-black smoother sweep (both colours) on level 0: x, rhs, three
          couplings and the mask read, x written -> 6w + 1 (49 B in FP64),
          `sweeps` of them before and after the coarse correction;
        restriction and prolongation: 5.375w (43 B in FP64);
        the coarser levels (one sweep more each way) add 1/7 of their own
          per-cell bytes."""
    w = wbytes
    setup = 7 * w + 2
    cg = 14 * w + 1
    pair = 6 * w + 1
    transfer = 5.375 * w

    def level(sw):
        return 2 * sw * pair + transfer

    return ncell * (setup + iters * (cg + level(sweeps) + level(sweeps + 1) / 7.0))


def energy_bytes(ncell, iters, w=8, mw=8):
    """Compulsory HBM bytes of one energy step per cell (FP64 form: Krylov
    vectors w = 8 and V-cycle values mw = 8 bytes; the operator rows, the
    assembly's inputs and T are FP64), each array once per pass:
      assembly: k, q, three face velocities, solid mask read (41), nine
        operator arrays written (72), level 0 of the hierarchy (conductance
        and flux per axis) written (6 mw);
      hierarchy build: level 0 read, coarser levels written (~6.9 mw);
      first residual: rhs, seven operator arrays, x read; r, r^, p, v
        written (64 + 5w);
      per BiCGStab iteration: p update with the V-cycle seed (4w + 8mw), two
        V-cycles (level 0: three half-sweeps of 9 mw, restriction 8.25 mw,
        prolongation mw/8, coarser levels 1/7: ~40.4 mw each), two operator
        products (56 + mw + 3w each), s update with its seed (3w + 8mw), x
        and r update (8w);
      relaxation: T and x read, T written (16 + w)."""
    assemble = 41 + 72 + 6 * mw
    build = 6.9 * mw
    r0 = 64 + 5 * w
    vc = (3 * 9 + 8.25 + 0.125) * mw * 8.0 / 7.0
    it = (4 * w + 8 * mw) + 2 * vc + 2 * (56 + mw + 3 * w) + (3 * w + 8 * mw) + 8 * w
    return ncell * (assemble + build + r0 + iters * it + 16 + w)


def kernel_classes(phases, iters_mean, dims, mom_sweeps, peak, energy_iters=1):
    """Achieved HBM bandwidth of each phase of the outer step on its
    algorithmic bytes (FP64 form; each array counted once per pass):
      momentum: 49 B per face per red-black pass (u^n of the three
        components, p, u*, mask; u* written), 2 passes per sweep;
      p' assembly: 89 B per cell (u*, v*, w*, d of the three components,
        mask; three couplings and b written);
      p' solve: pcg_bytes();
      correction: 97 B per cell (u*, d per face of the three components,
        p', p and the solid mask read; u, v, w and p written);
      energy: energy_bytes() with the step's BiCGStab iterations."""
    nx, ny, nz = dims
    ncell = nx * ny * nz
    nface = (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)
    model = {"momentum": 49.0 * nface * 2 * mom_sweeps, "p_assembly": 89.0 * ncell,
             "p_solve": pcg_bytes(ncell, iters_mean), "correction": 97.0 * ncell,
             "energy": energy_bytes(ncell, energy_iters)}
    out = {}
    for k, b in model.items():
        ms = phases.get(k, 0.0)
        gbs = b / (ms * 1e-3) / 1e9 if ms > 0 else None
        out[k] = {"algorithmic_bytes": b, "ms": ms, "achieved_gbs": gbs, "frac": (gbs / peak) if gbs else None}
    return out


def time_steps(torch, g, steps, local):
    stream = torch.cuda.ExternalStream(g.stream(), device=local)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    st = g.step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1), st


def profiled_steps(g, steps):
    """per-phase ms per step and the p' iterations of each step"""
    g.profile(True)
    iters = []
    for _ in range(steps):
        iters.append(g.step(1)["pcg_iters"])
    ph, n = g.profile_read()
    g.profile(False)
    return {k: v / max(1, n) for k, v in ph.items()}, iters


def max_over_ranks(torch, dist, v):
    """The largest value over the ranks (NCCL on the GPU, gloo on the host)."""
    if not dist:
        return v
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_gpu(args):
    import numpy as np
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
    deck, re_, k, q, ctype = workload()
    ncell = int(ctype.size)

    def make(precision=0, **kw):
        g = hsolver_b200.Channel(deck, device=local, re=re_, precision=precision, **SOLVER, **kw)
        g.set_solid(k, q)
        g.init()
        return g

    g = make(0)
    g.step(args.warmup)
    g.sync()
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    ms, st = time_steps(torch, g, args.steps, local)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = max_over_ranks(torch, dist, ms)
    phases, iters = profiled_steps(g, 3)
    dev_bytes = g.device_bytes()

    # adjoint / forward of the energy gradient on the current (frozen) flow
    adj = None
    if not args.no_variants:
        J, dq, dk, info = g.adjoint(tol=1e-8)
        adj = {"J": J, "fwd_iters": info["fwd_iters"], "adj_iters": info["adj_iters"], "fwd_ms": info["fwd_ms"],
               "adj_ms": info["adj_ms"], "adjoint_over_forward": info["adj_ms"] / info["fwd_ms"],
               "note": "forward energy solve from T = t_in to rtol 1e-8, then the transposed solve to the "
                       "gradients on the device (their copies to the host excluded); CUDA events"}
    g.close()

    # end to end through the public API with pinned host buffers: a fresh
    # solver replays the same outer steps; each step uploads u, v, w, p, T,
    # runs one outer step and reads them back
    state = ["u", "v", "w", "p", "T"]
    ge = make(0)
    ge.step(args.warmup)
    host = {f: torch.empty(ge.field_size(f), dtype=torch.float64, pin_memory=True) for f in state}
    for f in state:
        ge.field(f, out=host[f].numpy())
    L = hsolver_b200.load()
    ids = hsolver_b200.CH_FIELDS
    h2d = sum(host[f].numel() * 8 for f in state)

    def e2e_step():
        for f in state:
            p = ctypes.cast(host[f].data_ptr(), ctypes.POINTER(ctypes.c_double))
            if L.hs_channel_set_field(ge.h, ids[f], p, host[f].numel()) != 0:
                raise RuntimeError(L.hs_last_error(None).decode())
        ge.step(1)
        for f in state:
            p = ctypes.cast(host[f].data_ptr(), ctypes.POINTER(ctypes.c_double))
            if L.hs_channel_get_field(ge.h, ids[f], p, host[f].numel()) != 0:
                raise RuntimeError(L.hs_last_error(None).decode())

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(torch, dist, time.perf_counter() - t0)
    ge.close()

    variants = {}
    if not args.no_variants:
        gm = make(1)
        gm.step(args.warmup)
        gm.sync()
        if dist:
            dist.barrier()
        mms, mst = time_steps(torch, gm, args.steps, local)
        mms = max_over_ranks(torch, dist, mms)
        mph, miters = profiled_steps(gm, 3)
        variants["mixed"] = {"precision": "FP32 fields/sweeps/V-cycles, FP64 residual refinement, dots, coarsest solve",
                             "value": world * args.steps / (mms * 1e-3), "unit": UNIT, "ms_per_step": mms / args.steps,
                             "speedup_vs_fp64": ms / mms, "phase_ms_per_step": mph, "pcg_iters": miters,
                             "device_bytes": gm.device_bytes()}
        gm.close()
        variants["adjoint"] = adj
        variants["time_to_residual"] = time_to_residual(args, hsolver_b200, local)
        variants["reference_physics"] = reference_physics(args, torch, hsolver_b200, local, dist)
        variants["like_for_like"] = like_for_like(torch, hsolver_b200, local)
        variants["config5"] = config5(torch, hsolver_b200, local)
        variants["convection"] = convection(torch, hsolver_b200, local)
        variants["sharded_p_solve"] = sharded_p_solve(local)

    if rank == 0:
        peak, peak_kind = hbm_peak()
        it_mean = sum(iters) / max(1, len(iters))
        pms = phases["p_solve"]
        b = pcg_bytes(ncell, it_mean)
        achieved = b / (pms * 1e-3) / 1e9 if pms > 0 else None
        out = {
            "metric": METRIC, "value": world * args.steps / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded in-repo case generator)",
            "config": CONFIG,
            "e2e": {"value": world * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
            "roofline": {"bound": "hbm", "kernel": "k_ch_pcg (pressure correction, multigrid-preconditioned CG, "
                                                 "one cooperative launch per outer step)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                         "traffic": PCG_TRAFFIC_PER_ITER * it_mean,
                         "traffic_source": "ncu dram bytes of 3 launches (8 iterations each), per iteration x "
                                           "this launch's iterations", "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": b,
                         "pcg_iters_per_launch": it_mean, "launch_ms": pms},
            "phase_ms_per_step": phases,
            "kernel_classes": kernel_classes(phases, it_mean, CONFIG["grid"], 2, peak),
            "last_step": {"pcg_iters": st["pcg_iters"], "t_iters": st["t_iters"], "global_residual": st["global"]},
            "device_bytes": dev_bytes,
            "gpu_launches": LAUNCHES_PER_STEP * args.steps,
            "variants": variants,
            "clocks": clk,
        }
        ttr = variants.get("time_to_residual", {}).get(NAME)
        if ttr:
            # the specification's headline: wall time to a global residual of
            # 1e-6 on this case, FP64 and mixed, and their ratio
            out["time_to_1e-6"] = {"fp64_s": ttr["fp64"]["seconds"], "mixed_s": ttr["mixed"]["seconds"],
                                   "steps": [ttr["fp64"]["steps"], ttr["mixed"]["steps"]],
                                   "converged": [ttr["fp64"]["converged"], ttr["mixed"]["converged"]],
                                   "mixed_vs_fp64_rel_l2": ttr["mixed_vs_fp64_rel_l2"]}
            out["speedup_mixed"] = ttr.get("speedup_mixed")
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline()
        print(json.dumps(out), flush=True)
    if dist:
        dist.destroy_process_group()


def time_to_residual(args, hsolver_b200, local):
    """Wall time of hs_channel_solve_to(1e-6) for the FP64 and mixed forms, and
    the per-field relative L2 difference of the two converged states: the
    bench case (256x128x128, the specification's target), config 1
    (48x24x24) and config 3 (the same on a tanh-stretched grid, maximum cell
    aspect ratio 20: the mixed-precision configuration)."""
    import numpy as np
    out = {}
    cases_ = [(NAME, args.residual_max), ("config1", 2000), ("config3", 3000)]
    for name, cap in cases_:
        deck, re_, k, q, _ = workload(name)
        res, fields = {}, {}
        for prec, key in ((0, "fp64"), (1, "mixed")):
            g = hsolver_b200.Channel(deck, device=local, re=re_, precision=prec, **(SOLVER if name == NAME else {}))
            g.set_solid(k, q)
            g.init()
            g.sync()
            t0 = time.perf_counter()
            ok, steps, st = g.solve_to(1e-6, cap)
            g.sync()
            res[key] = {"converged": ok, "steps": steps, "seconds": time.perf_counter() - t0, "global": st["global"]}
            fields[key] = {f: g.field(f) for f in ("u", "v", "w", "p", "T")}
            g.close()
        if res["fp64"]["converged"] and res["mixed"]["converged"]:
            res["speedup_mixed"] = res["fp64"]["seconds"] / res["mixed"]["seconds"]
        res["mixed_vs_fp64_rel_l2"] = {
            f: float(np.linalg.norm(fields["mixed"][f] - fields["fp64"][f]) / max(np.linalg.norm(fields["fp64"][f]), 1e-300))
            for f in ("u", "v", "w", "p", "T")}
        out[name] = res
    return out


def convection(torch, hsolver_b200, local):
    """The momentum convection schemes and buoyancy on the bench case: the
    outer step with hybrid, and with QUICK (deferred correction) plus a
    Boussinesq term along +z at Richardson number 1, beside first-order
    upwind (the reference's scheme, the bench's headline); 3 warm-up and 10
    timed steps each, per-phase times of 3 more."""
    deck, re_, k, q, _ = workload()
    out = {}
    for name, kw in (("upwind", {}), ("hybrid", {"conv": 1}), ("quick_buoyancy", {"conv": 2, "ri": 1.0}),
                     ("quick_buoyancy_mixed", {"conv": 2, "ri": 1.0, "precision": 1})):
        g = hsolver_b200.Channel(deck, device=local, re=re_, **SOLVER, **kw)
        g.set_solid(k, q)
        g.init()
        g.step(3)
        ms, st = time_steps(torch, g, 10, local)
        phases, iters = profiled_steps(g, 3)
        out[name] = {"value": 10 / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / 10,
                     "momentum_ms_per_step": phases["momentum"], "pcg_iters": iters}
        g.close()
    return out


def sharded_p_solve(local, dims=(256, 128, 128)):
    """The z-slab pressure-correction solve (hs_slab_*, slabs.slab_pcg_solve)
    on this GPU: a seeded channel-like system of the bench case's size (face
    couplings U[0.5, 2], walls, inlet and outlet faces) to rtol 1e-5 cut into
    1, 2 and 4 slabs whose halo planes are copied between them (the
    multi-GPU form moves the same planes over NCCL), with block Jacobi alone
    (the iteration count grows with the slab count) and with the global
    coarse correction on 4^3-cell aggregates; the per-iteration time
    includes the host's sums of every dot product (one synchronisation per
    pass)."""
    import numpy as np
    from hsolver_b200 import slabs
    nx, ny, nz = dims
    rng = np.random.default_rng(0)
    gx = rng.uniform(0.5, 2.0, (nz, ny, nx + 1))
    gy = rng.uniform(0.5, 2.0, (nz, ny + 1, nx))
    gz = rng.uniform(0.5, 2.0, (nz + 1, ny, nx))
    gx[:, :, 0] = 0.0
    gy[:, 0, :] = gy[:, -1, :] = 0.0
    gz[0] = gz[-1] = 0.0
    b = rng.standard_normal((nz, ny, nx))
    out = {"workload": "p' system %dx%dx%d, rtol 1e-5, slabs on one GPU" % dims}
    for n in (1, 2, 4):
        for two_level in (False, True):
            parts = []
            for r in range(n):
                k0, k1 = slabs.slab_bounds(nz, n, r)
                sl = slabs.SlabPCG(nx, ny, k1 - k0, device=local, coarse=(4, k0, nz) if two_level else None)
                sl.set_system(gx[k0:k1], gy[k0:k1], gz[k0:k1 + 1], b[k0:k1])
                parts.append(sl)
            slabs.slab_pcg_solve(parts, tol=1e-5, maxiter=2000)  # warm-up (builds the hierarchies)
            t0 = time.perf_counter()
            it, rel = slabs.slab_pcg_solve(parts, tol=1e-5, maxiter=2000)
            dt = time.perf_counter() - t0
            for sl in parts:
                sl.close()
            out["slabs_%d%s" % (n, "_two_level" if two_level else "")] = {
                "iters": it, "relres": rel, "ms": dt * 1e3, "ms_per_iter": dt * 1e3 / max(it, 1)}
    return out


def config5(torch, hsolver_b200, local):
    """The large single-GPU case: 512x256x256 (33.5M cells), 32 seeded blocks
    (edges 8-48, q U[0.1,5], k_s/k_f U[10,1000]), Re 1000.  Both forms:
    device footprint and step time (3 timed steps after 2 warm-up steps),
    per-phase times of 2 more steps with the p' solve's fraction of the HBM
    bandwidth on its algorithmic bytes (FP64 form: every kernel class), and
    the energy adjoint / forward on the flow frozen after those steps (the
    specification's converged flow takes thousands of outer steps here; the
    cost ratio is a property of the operator, not of convergence)."""
    deck, re_, k, q, _ = workload("config5")
    dims = (512, 256, 256)
    ncell = dims[0] * dims[1] * dims[2]
    peak, _ = hbm_peak()
    out = {"workload": "channel 512x256x256 (33.5M cells), 32 seeded blocks, Re 1000"}
    for prec, key in ((0, "fp64"), (1, "mixed")):
        g = hsolver_b200.Channel(deck, device=local, re=re_, precision=prec, **SOLVER)
        g.set_solid(k, q)
        g.init()
        g.step(2)
        ms, st = time_steps(torch, g, 3, local)
        phases, iters = profiled_steps(g, 2)
        it_mean = sum(iters) / len(iters)
        pb = pcg_bytes(ncell, it_mean, 8 if prec == 0 else 4)
        r = {"device_bytes": g.device_bytes(), "ms_per_step": ms / 3, "pcg_iters": st["pcg_iters"],
             "t_iters": st["t_iters"], "phase_ms_per_step": phases,
             "p_solve_frac": pb / (phases["p_solve"] * 1e-3) / 1e9 / peak if phases.get("p_solve") else None}
        if prec == 0:
            r["kernel_classes"] = kernel_classes(phases, it_mean, dims, 2, peak)
        J, dq, dk, info = g.adjoint(tol=1e-8)
        r["adjoint"] = {"fwd_iters": info["fwd_iters"], "adj_iters": info["adj_iters"], "fwd_ms": info["fwd_ms"],
                        "adj_ms": info["adj_ms"], "adjoint_over_forward": info["adj_ms"] / info["fwd_ms"]}
        out[key] = r
        g.close()
    return out


def reference_physics(args, torch, hsolver_b200, local, dist):
    """The reference-faithful lid-cavity SIMPLE step on the same grid (the
    reference's own physics and solvers), device-timed."""
    from hsolver_b200 import cases
    g = hsolver_b200.Solver(cases.config2(seed=0), device=local)
    g.init()
    g.step(args.warmup)
    g.sync()
    ms, _ = time_steps(torch, g, args.steps, local)
    ms = max_over_ranks(torch, dist, ms)
    g.close()
    return {"workload": "lid-driven SIMPLE-CHT step of the reference (FP64, HYPRE-rule CG rtol 1e-5, frozen matrix, "
                        "lexicographic Gauss-Seidel), same 256x128x128 grid",
            "value": args.steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / args.steps}


REF_DRIVER = os.path.join(HERE, "oracle", "_ref", "ref_driver")
DECKS = os.path.join(HERE, "tests", "golden", "decks")


def like_for_like(torch, hsolver_b200, local, deck_name="example13", steps=3):
    """The reference's own code against the GPU on one computation: the
    reference's lid-cavity SIMPLE step (its FluidSolver / MobSolver / Solver
    sources compiled single-rank against the in-repo MPI / HYPRE shims,
    oracle/_ref/ref_driver, one host core) and the reference-faithful GPU
    step (hs_step), which reproduces it bit for bit without the pressure
    solve and to 1e-9 with it, on the reference's own deck, the same outer
    steps from the initial state.  The CPU time per step is the reference's
    clock() measurement (solver.h:51-58) around the loop body of
    Solver::solve (solver.h:55-154); the GPU's by CUDA events."""
    import tempfile
    deck_path = os.path.join(DECKS, deck_name + ".in")
    if not os.path.exists(REF_DRIVER):
        return {"unavailable": "oracle/_ref/ref_driver not built (needs the reference tree at build time)"}
    with tempfile.TemporaryDirectory() as work:
        r = subprocess.run([REF_DRIVER, deck_path, os.path.join(work, "wd"), "-", "time:%d" % steps],
                           capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        return {"unavailable": "ref_driver exited %d" % r.returncode}
    ref = json.loads(r.stdout.strip().splitlines()[-1])
    with open(deck_path) as f:
        g = hsolver_b200.Solver(f.read(), device=local)
    g.init()
    stream = torch.cuda.ExternalStream(g.stream(), device=local)
    gpu_ms, its = [], []
    for _ in range(steps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = g.step(1, stats=True)
        e1.record(stream)
        e1.synchronize()
        gpu_ms.append(e0.elapsed_time(e1))
        its.append(st["pcg_iters"])
    g.close()
    cpu_s = [s["clock_s"] for s in ref["steps"]]
    return {"deck": deck_name + ".in (the reference's own deck)", "steps": steps,
            "reference_cpu_s_per_step": cpu_s, "reference_wall_s_per_step": [s["wall_s"] for s in ref["steps"]],
            "reference_pcg_iters": [s["pcg_iters"] for s in ref["steps"]], "reference_cores": 1,
            "reference_setup_s": ref["setup_s"], "gpu_ms_per_step": gpu_ms, "gpu_pcg_iters": its,
            "speedup": (sum(cpu_s) * 1e3) / sum(gpu_ms),
            "parity": "GPU state bit-identical to the reference's without the pressure solve, rel. L2 <= 1e-9 with it "
                      "(tests/test_gpu_parity.py, tests/test_oracle_golden.py)"}


# The CPU step's inner solves as the reference configures its own: the p'
# system by CG without a preconditioner to rtol 1e-5 with at most 1000
# iterations (HYPRE PCG, fluid_solver.h:1871-1875), the energy to the GPU
# step's 0.5 reduction with at most 100 iterations (the reference's sweep cap
# for its energy Gauss-Seidel, fluid_solver.h:794-881).  The tolerances are
# the GPU step's; the CPU's solvers are the reference's, so the iteration
# counts differ and the ratio measures solver and hardware together.
CPU_SOLVER = {"p_tol": 1e-5, "p_maxiter": 1000, "t_tol": 0.5, "t_maxiter": 100}


def cpu_threads():
    from oracle import oracle
    L = oracle.lib()
    L.or_threads.restype = ctypes.c_int
    return int(L.or_threads())


def cpu_case():
    """The bench case on the FP64 C oracle (OpenMP on every host thread),
    initialised; classification by the oracle (no CUDA library is loaded)."""
    from oracle import oracle
    deck, re_, k, q, _ = workload(host_side=True)
    o = oracle.ChannelCase(deck, re=re_, **CPU_SOLVER)
    o.set_solid(k, q)
    o.init()
    return o


def cpu_steps(o, n):
    """Seconds of each of n outer steps and the solver iterations they took."""
    dts, its = [], []
    for _ in range(n):
        t0 = time.perf_counter()
        o.step(1)
        dts.append(time.perf_counter() - t0)
        st = o.stats()
        its.append([st["pcg_iters"], st["t_iters"]])
    return dts, its


CPU_SAMPLE_NOTE = ("outer steps of the bench case from the initial state by the FP64 C oracle (OpenMP, %d threads): "
                   "the same discretisation and outer step as the GPU, with the reference's inner solvers (p' by CG "
                   "without preconditioner, rtol 1e-5, at most 1000 iterations, fluid_solver.h:1871-1875; energy by "
                   "Jacobi BiCGStab to 0.5, at most 100 iterations); (p', energy) iterations per step %s")


def cpu_baseline():
    o = cpu_case()
    dts, its = cpu_steps(o, 1)
    return {"value": 1.0 / dts[0], "unit": UNIT, "cores": cpu_threads(), "kind": "port",
            "sample": "1 of the " + CPU_SAMPLE_NOTE % (cpu_threads(), its), "seconds": dts}


def run_reference(args):
    """CPU arm: the channel step restated in C (oracle/), the only CPU
    implementation of this physics (the reference solves a lid cavity with
    no inlet, heat source or conductivity ratio), with the reference's own
    inner-solver settings; a bounded sample of 1-2 outer steps (about 20-40 s
    each on the host) from the initial state.  Under torchrun only rank 0
    runs it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps = max(1, min(args.steps, 2))
    o = cpu_case()
    dts, its = cpu_steps(o, steps)
    dt = sum(dts)
    v = steps / dt
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": steps, "warmup": 0,
        "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded in-repo case generator)", "config": CONFIG, "impl": "reference",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cpu_threads(), "kind": "port",
                         "sample": "%d " % steps + CPU_SAMPLE_NOTE % (cpu_threads(), its), "seconds": dts},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def probe(args):
    """A few outer steps of one case on one GPU, printing the p' and energy
    iterations of every step: the command the profiles name (ncu runs it on a
    small case).  NAME: config1 .. config5 (the seeded configurations with
    their block physics; config2 is the bench case), `reference` (the
    reference-faithful lid-cavity step on the 256x128x128 grid), or
    NXxNYxNZ:K (a 2x1x1 channel with K seeded blocks of edges 8-20, seed 1,
    the bench case's block physics)."""
    import hsolver_b200
    from hsolver_b200 import cases
    t0 = time.perf_counter()
    if args.probe == "reference":
        g = hsolver_b200.Solver(cases.config2(seed=0))
        g.init()
        st = g.step(args.steps, stats=True)
        g.sync()
        print("ok reference steps %d pcg_iters %d (%.2f s)" % (args.steps, st["pcg_iters"], time.perf_counter() - t0))
        return
    if args.probe in cases.CONFIGS:
        deck, re_, k, q, _ = workload(args.probe)
    else:
        dims, nb = args.probe.split(":")
        nx, ny, nz = (int(v) for v in dims.split("x"))
        deck = cases.channel(nx, ny, nz, cases.place_blocks((nx, ny, nz), int(nb), 8, 20, seed=1))
        ctype, region = hsolver_b200.Case(deck).cell_types()
        re_, k, q = cases.block_physics("config2", ctype, region)
    kw = {}
    if args.p_tol is not None:
        kw["p_tol"] = args.p_tol
    if args.t_tol is not None:
        kw["t_tol"] = args.t_tol
    if args.t_maxiter is not None:
        kw["t_maxiter"] = args.t_maxiter
    if args.p_level0 is not None:
        kw["p_level0"] = args.p_level0
    if args.conv is not None:
        kw["conv"] = args.conv
    if args.ri is not None:
        kw["ri"] = args.ri
    g = hsolver_b200.Channel(deck, re=re_, precision=hsolver_b200.PREC_MIXED if args.mixed else hsolver_b200.PREC_FP64,
                             **kw)
    g.set_solid(k, q)
    g.init()
    its = []
    g.profile(True)
    for _ in range(args.steps):
        st = g.step(1)
        its.append((st["pcg_iters"], st["t_iters"]))
    g.sync()
    ph, n = g.profile_read()
    print("ok channel %s steps %d (pcg, energy) iterations per step %s (%.2f s); ms per step %s"
          % (args.probe, args.steps, its, time.perf_counter() - t0,
             {k: round(v / max(n, 1), 3) for k, v in ph.items()}))


def replica_check(args):
    """The replica plumbing on the host: every rank joins a gloo group and
    rank 0 prints the max over ranks of 10 + rank (what the N-GPU bench does
    with its event times), with the world size."""
    import datetime
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    rank, world = dist.get_rank(), dist.get_world_size()
    v = max_over_ranks(torch, dist, 10.0 + rank)
    if rank == 0:
        print(json.dumps({"replica_check": True, "n_gpus": world, "max_ms": v}), flush=True)
    dist.destroy_process_group()


def spawn_replicas(args, argv):
    """--gpus N > 1 without a launcher: rerun this command under
    torch.distributed.run with N ranks on this node (127.0.0.1, a free port),
    one per GPU; rank 0 prints the JSON line.  Returns the launcher's exit
    status."""
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + list(argv)
    return subprocess.run(cmd).returncode


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--residual-max", type=int, default=4000,
                    help="outer-step cap of the 256x128x128 time-to-residual runs")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--probe", default=None, metavar="NAME", help="run a few steps of one case (see probe())")
    ap.add_argument("--mixed", action="store_true", help="--probe: the mixed-precision form")
    ap.add_argument("--p-tol", type=float, default=None, help="--probe: p' relative tolerance")
    ap.add_argument("--t-tol", type=float, default=None, help="--probe: energy relative tolerance")
    ap.add_argument("--t-maxiter", type=int, default=None, help="--probe: energy iteration cap")
    ap.add_argument("--p-level0", type=int, default=None, help="--probe: finest p' level form (0 the default, 1 grid-wide, 2 z-marching)")
    ap.add_argument("--conv", type=int, default=None, help="--probe: momentum convection (0 upwind, 1 hybrid, 2 QUICK)")
    ap.add_argument("--ri", type=float, default=None, help="--probe: Richardson number of the buoyancy term (along +z)")
    ap.add_argument("--replica-check", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args(argv)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and args.probe is None:
        sys.exit(spawn_replicas(args, argv))
    if args.replica_check:
        replica_check(args)
    elif args.probe is not None:
        probe(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
