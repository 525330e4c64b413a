"""Run a few outer steps of a seeded case on one GPU (profiling and timing
probe; the profiles in profiles/ name this command).

  python -m hsolver_b200.probe --grid 192 96 96 --blocks 4 --steps 3 [--mixed]
  python -m hsolver_b200.probe --reference --steps 2      # lid-cavity path, 256x128x128
  python -m hsolver_b200.probe --config config2 --p-tol 1e-5 --t-tol 1e-1 --steps 3   # bench case

Channel case: a 2x1x1 channel with `--blocks` seeded solid blocks (edges
8-20 cells), Re 400, q U[0.5,2], k_s/k_f U[10,1000], the library's default
solver settings.  `--config NAME`: one of the seeded configurations of
hsolver_b200.cases with its block physics (config2 is bench.py's case).
`--reference`: the reference-faithful step on the 256x128x128 grid with 8
seeded blocks.  Prints the p' and energy iterations of every step.
"""
import argparse
import time


def main(argv=None):
    import hsolver_b200
    from hsolver_b200 import cases
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=[192, 96, 96])
    ap.add_argument("--blocks", type=int, default=4)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--reference", action="store_true")
    ap.add_argument("--config", default=None)
    ap.add_argument("--p-tol", type=float, default=None)
    ap.add_argument("--t-tol", type=float, default=None)
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    if a.reference:
        g = hsolver_b200.Solver(cases.config2(seed=0))
        g.init()
        st = g.step(a.steps, stats=True)
        g.sync()
        print("ok reference steps %d pcg_iters %d (%.2f s)" % (a.steps, st["pcg_iters"], time.perf_counter() - t0))
        return
    if a.config:
        deck = cases.CONFIGS[a.config](0) if a.config in ("config2", "config4", "config5") else cases.CONFIGS[a.config]()
        ctype, region = hsolver_b200.Case(deck).cell_types()
        re_, k, q = cases.block_physics(a.config, ctype, region, 0)
        label = a.config
    else:
        nx, ny, nz = a.grid
        deck = cases.channel(nx, ny, nz, cases.place_blocks((nx, ny, nz), a.blocks, 8, 20, seed=a.seed))
        ctype, region = hsolver_b200.Case(deck).cell_types()
        re_, k, q = cases.block_physics("config2", ctype, region)
        label = "%dx%dx%d" % (nx, ny, nz)
    kw = {}
    if a.p_tol is not None:
        kw["p_tol"] = a.p_tol
    if a.t_tol is not None:
        kw["t_tol"] = a.t_tol
    g = hsolver_b200.Channel(deck, re=re_, precision=hsolver_b200.PREC_MIXED if a.mixed else hsolver_b200.PREC_FP64,
                             **kw)
    g.set_solid(k, q)
    g.init()
    its = []
    for _ in range(a.steps):
        st = g.step(1)
        its.append((st["pcg_iters"], st["t_iters"]))
    g.sync()
    print("ok channel %s steps %d (pcg, energy) iterations per step %s (%.2f s)"
          % (label, a.steps, its, time.perf_counter() - t0))


if __name__ == "__main__":
    main()
