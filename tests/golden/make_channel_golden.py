"""Converged state of configuration 3 (the tanh-stretched channel, cell
aspect ratio up to 20) from the C oracle, for the GPU's converged-state
parity test: the oracle steps until its global residual is at most 1e-6 and
its fields u, v, w, p, T are stored with the step count in
channel_config3_converged.npz.  Runs on the CPU (the oracle's OpenMP
threads); about a minute.  Usage: python tests/golden/make_channel_golden.py"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)


def main():
    import bench
    from oracle import oracle
    deck, re_, k, q, _ = bench.workload("config3")
    o = oracle.ChannelCase(deck, re=re_)
    o.set_solid(k, q)
    o.init()
    steps = 0
    while True:
        o.step(1)
        steps += 1
        if steps > 5 and o.stats()["global"] <= 1e-6:
            break
        if steps >= 3000:
            raise SystemExit("oracle did not converge")
    fields = {f: o.field(f) for f in ("u", "v", "w", "p", "T")}
    np.savez_compressed(os.path.join(HERE, "channel_config3_converged.npz"), steps=steps,
                        global_residual=o.stats()["global"], **fields)
    print("steps", steps, "global", o.stats()["global"])


if __name__ == "__main__":
    main()
