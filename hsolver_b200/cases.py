"""Seeded synthetic cases written as hsolver `.in` decks.

The deck format is the reference's (mesh/mesh.cpp:1616-1796): `xgrid`,
`ygrid`, `zgrid` point lists, `mobs` boxes of 1-based inclusive cell ranges
`i0,i1,j0,j1,k0,k1`, `walls` (8 ints) and `holes` (13 ints); every value
carries a trailing comma, because the reference's reader drops a final value
without one (mesh/mesh.cpp:1677).
"""
import numpy as np


def _fmt(vals):
    return ",".join(repr(float(v)) for v in vals) + ","


def deck_text(xs, ys, zs, blocks=(), walls=(), holes=()):
    """Render a deck; `blocks` are 1-based inclusive (i0,i1,j0,j1,k0,k1)."""
    s = "xgrid = " + _fmt(xs) + "\n\n"
    s += "ygrid = " + _fmt(ys) + "\n\n"
    s += "zgrid = " + _fmt(zs) + "\n\n"
    s += "mobs =\n" + "".join("    " + ",".join(str(int(v)) for v in b) + ",\n" for b in blocks) + "\n"
    s += "walls =\n" + "".join("    " + ",".join(str(int(v)) for v in w) + ",\n" for w in walls) + "\n"
    s += "holes= " + "".join(",".join(str(int(v)) for v in h) + ",\n" for h in holes) + "\n\nends\n"
    return s


def uniform(n, length):
    return np.linspace(0.0, length, n + 1)


def tanh_clustered(n, length, max_aspect, other_spacing):
    """Wall-clustered points y_j = L/2 (1 + tanh(b(2j/n - 1)) / tanh(b)), with b
    chosen so that the largest cell aspect ratio (other_spacing / smallest
    cell) equals `max_aspect`."""
    def pts(b):
        t = np.arange(n + 1) / n
        return 0.5 * length * (1.0 + np.tanh(b * (2 * t - 1)) / np.tanh(b))

    lo, hi = 1e-6, 20.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        ar = other_spacing / np.min(np.diff(pts(mid)))
        if ar > max_aspect:
            hi = mid
        else:
            lo = mid
    p = pts(0.5 * (lo + hi))
    p[0], p[-1] = 0.0, length
    return p


def place_blocks(shape, k, edge_lo, edge_hi, seed, margin_x=1):
    """Rejection-sample k non-overlapping boxes (>= 1-cell gap between boxes,
    >= margin_x cells clear of the x = 0 and x = Nx planes); returns 1-based
    inclusive boxes."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    boxes = []
    tries = 0
    while len(boxes) < k:
        tries += 1
        if tries > 100000:
            raise RuntimeError("could not place %d blocks" % k)
        e = rng.integers(edge_lo, edge_hi + 1, size=3)
        e = np.minimum(e, [nx - 2 * margin_x, ny, nz])
        o = [rng.integers(margin_x, nx - margin_x - e[0] + 1), rng.integers(0, ny - e[1] + 1),
             rng.integers(0, nz - e[2] + 1)]
        lo = np.array(o)
        hi = lo + e                                    # half-open 0-based
        ok = True
        for b in boxes:
            blo = np.array([b[0] - 1, b[2] - 1, b[4] - 1])
            bhi = np.array([b[1], b[3], b[5]])
            if np.all(lo < bhi + 1) and np.all(blo < hi + 1):
                ok = False
                break
        if ok:
            boxes.append((int(lo[0] + 1), int(hi[0]), int(lo[1] + 1), int(hi[1]), int(lo[2] + 1), int(hi[2])))
    return boxes


def channel(nx, ny, nz, blocks, lx=2.0, ly=1.0, lz=1.0, ys=None, zs=None):
    return deck_text(uniform(nx, lx), ys if ys is not None else uniform(ny, ly),
                     zs if zs is not None else uniform(nz, lz), blocks)


def config1():
    """48x24x24 channel 2x1x1, one block over cells x 16-24, y 0-8, z 8-16
    (0-based half-open), i.e. the deck line 17,24,1,8,9,16."""
    return channel(48, 24, 24, [(17, 24, 1, 8, 9, 16)])


def config2(seed=0):
    """256x128x128 channel, 8 seeded blocks with edges in [8, 24] cells."""
    return channel(256, 128, 128, place_blocks((256, 128, 128), 8, 8, 24, seed))


def config3():
    """Config-1 geometry on a tanh wall-clustered grid in y and z (max cell
    aspect ratio 20)."""
    dx = 2.0 / 48
    return channel(48, 24, 24, [(17, 24, 1, 8, 9, 16)], ys=tanh_clustered(24, 1.0, 20.0, dx),
                   zs=tanh_clustered(24, 1.0, 20.0, dx))


def config4(seed=0):
    """128x64x64 channel, 4 seeded blocks with edges in [8, 24] cells."""
    return channel(128, 64, 64, place_blocks((128, 64, 64), 4, 8, 24, seed))


def config5(seed=0):
    """512x256x256 channel, 32 seeded blocks with edges in [8, 48] cells."""
    return channel(512, 256, 256, place_blocks((512, 256, 256), 32, 8, 48, seed))


CONFIGS = {"config1": config1, "config2": config2, "config3": config3, "config4": config4, "config5": config5}


# Physics of the seeded configurations: Reynolds number and per-block
# conductivity ratio / heat-source ranges.
PHYSICS = {
    "config1": {"re": 100.0, "k": (100.0, 100.0), "q": (1.0, 1.0)},
    "config2": {"re": 400.0, "k": (10.0, 1000.0), "q": (0.5, 2.0)},
    "config3": {"re": 100.0, "k": (100.0, 100.0), "q": (1.0, 1.0)},
    "config4": {"re": 400.0, "k": (10.0, 1000.0), "q": (0.5, 2.0)},
    "config5": {"re": 1000.0, "k": (10.0, 1000.0), "q": (0.1, 5.0)},
}


def block_physics(name, ctype, region, seed=0):
    """(re, k_ratio per solid region, q per cell) for a configuration: one
    uniform draw per block (regions in the order of their lowest cell index),
    q constant inside each block and zero in the fluid."""
    ph = PHYSICS[name]
    ctype = np.asarray(ctype)
    region = np.asarray(region)
    nreg = int(region[ctype == 1].max()) + 1 if np.any(ctype == 1) else 0
    rng = np.random.default_rng(1000 + seed)
    k = rng.uniform(ph["k"][0], ph["k"][1], nreg)
    qb = rng.uniform(ph["q"][0], ph["q"][1], nreg)
    q = np.where(ctype == 1, qb[np.maximum(region, 0)], 0.0)
    return ph["re"], k, q
