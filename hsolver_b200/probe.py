"""Run a few outer steps of a seeded case on one GPU (profiling and timing
probe; the profiles in profiles/ name this command).

  python -m hsolver_b200.probe --grid 192 96 96 --blocks 4 --steps 3 [--mixed]
  python -m hsolver_b200.probe --reference --steps 2      # lid-cavity path, 256x128x128

Channel case: a 2x1x1 channel with `--blocks` seeded solid blocks (edges
8-20 cells), Re 400, q U[0.5,2], k_s/k_f U[10,1000], the library's default
solver settings.  `--reference`: the reference-faithful step on the
256x128x128 grid with 8 seeded blocks.
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
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    if a.reference:
        g = hsolver_b200.Solver(cases.config2(seed=0))
        g.init()
        st = g.step(a.steps, stats=True)
        g.sync()
        print("ok reference steps %d pcg_iters %d (%.2f s)" % (a.steps, st["pcg_iters"], time.perf_counter() - t0))
        return
    nx, ny, nz = a.grid
    deck = cases.channel(nx, ny, nz, cases.place_blocks((nx, ny, nz), a.blocks, 8, 20, seed=a.seed))
    ctype, region = hsolver_b200.Case(deck).cell_types()
    re_, k, q = cases.block_physics("config2", ctype, region)
    g = hsolver_b200.Channel(deck, re=re_, precision=hsolver_b200.PREC_MIXED if a.mixed else hsolver_b200.PREC_FP64)
    g.set_solid(k, q)
    g.init()
    st = g.step(a.steps)
    g.sync()
    print("ok channel %dx%dx%d steps %d pcg_iters %d t_iters %d (%.2f s)"
          % (nx, ny, nz, a.steps, st["pcg_iters"], st["t_iters"], time.perf_counter() - t0))


if __name__ == "__main__":
    main()
