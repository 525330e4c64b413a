"""Regenerate the golden fixtures from the reference's own sources.

Runs oracle/_ref/ref_driver (the reference's FluidSolver / MobSolver /
Solver compiled single-rank against the shims in oracle/ref/shim; build it
with `make -C oracle/ref`) on every deck in tests/golden/decks and stores:

* golden_<deck>.npz: full state arrays after the listed outer steps (small
  decks), keys "<step>/<array>";
* golden_digests.json: per-array SHA-256 of the raw FP64 bytes, the L2 norm
  and the PCG iteration count for larger decks, where full arrays would not
  be small fixtures.

Needs the reference tree, named by the REF environment variable when the
driver is not built yet; run it where that tree is, never on the GPU box.
Usage: REF=<reference tree> python tests/golden/make_golden.py [--only DECK]
(one deck's digests, merged into the existing file) [--proc] (the processor
files of decks/small.in, tests/golden/proc_small).
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
from oracle.oracle import read_dump  # noqa: E402

DRIVER = os.path.join(REPO, "oracle", "_ref", "ref_driver")
FULL = {"small": [1, 2, 5], "inner": [1, 5, 20], "quirk": [1, 3]}
DIGEST = {"config1": [1, 2, 5], "config3": [1, 3], "example13": [1, 2, 10], "example21": [1]}
KEEP = ["u_star", "v_star", "w_star", "up", "vp", "wp", "p_temp", "t_temp", "ux", "uy", "uz", "p", "t",
        "id", "fluid.empty", "fluid.t_boundary", "fluid.t_halo", "solid.t_temp", "solid.t", "solid.empty",
        "solid.t_boundary", "solid.t_halo", "fluid.meta", "solid.meta", "pcg_iters"]


def run(deck, steps, work):
    prefix = os.path.join(work, "d")
    subprocess.run([DRIVER, os.path.join(HERE, "decks", deck + ".in"), os.path.join(work, "wd"), prefix,
                    ",".join(str(s) for s in steps)], check=True, stdout=subprocess.DEVNULL)
    return {s: read_dump("%s.step%d.bin" % (prefix, s)) for s in steps}


def digest_entries(res):
    out = {}
    for s, d in res.items():
        ent = {}
        for k in KEEP:
            if k in d and d[k].dtype == np.float64:
                ent[k] = {"sha256": hashlib.sha256(d[k].tobytes()).hexdigest(),
                          "l2": float(np.linalg.norm(d[k])), "n": int(d[k].size)}
        ent["pcg_iters"] = int(d["pcg_iters"][0])
        out[str(s)] = ent
    return out


def write_processor_fixture():
    """proc_small/processor0/{cells,faces,boundary}.txt: the processor files
    the reference's decompose step writes for decks/small.in (nParts = 1),
    read back by the drop-in CYCASMesh in tests/test_drop_in.py."""
    import shutil
    with tempfile.TemporaryDirectory() as work:
        wd = os.path.join(work, "wd")
        subprocess.run([DRIVER, os.path.join(HERE, "decks", "small.in"), wd, "-", "time:1"], check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        out = os.path.join(HERE, "proc_small", "processor0")
        os.makedirs(out, exist_ok=True)
        for name in ("cells.txt", "faces.txt", "boundary.txt"):
            shutil.copyfile(os.path.join(wd, "processor0", name), os.path.join(out, name))


def main():
    if not os.path.exists(DRIVER):
        ref = os.environ.get("REF")
        if not ref:
            sys.exit("set REF to the reference source tree (the driver oracle/_ref/ref_driver is built from it)")
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle", "ref"), "REF=" + ref], check=True)
    if len(sys.argv) > 1 and sys.argv[1] == "--proc":
        write_processor_fixture()
        return
    if len(sys.argv) > 2 and sys.argv[1] == "--only":
        # regenerate one deck's digests and merge them into the existing file
        deck = sys.argv[2]
        path = os.path.join(HERE, "golden_digests.json")
        with open(path) as f:
            digests = json.load(f)
        with tempfile.TemporaryDirectory() as work:
            digests[deck] = digest_entries(run(deck, DIGEST[deck], work))
        with open(path, "w") as f:
            json.dump(digests, f, indent=1, sort_keys=True)
        return
    digests = {}
    for deck, steps in FULL.items():
        with tempfile.TemporaryDirectory() as work:
            res = run(deck, steps, work)
        arrays = {}
        for s, d in res.items():
            for k in KEEP:
                if k in d:
                    arrays["%d/%s" % (s, k)] = d[k]
        np.savez_compressed(os.path.join(HERE, "golden_%s.npz" % deck), **arrays)
    for deck, steps in DIGEST.items():
        with tempfile.TemporaryDirectory() as work:
            digests[deck] = digest_entries(run(deck, steps, work))
    with open(os.path.join(HERE, "golden_digests.json"), "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
