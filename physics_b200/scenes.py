"""Synthetic scenes of the benchmark configurations.

The reference ships no datasets for this path; every scene is generated here
from a seed.  Random draws use SplitMix64, the same generator as the
reference's replay RNG (crates/phy-core/src/replay.rs:29-52), vectorised: the
n-th draw of a stream seeded with `s` is mix(s + (n+1) * 0x9E3779B97F4A7C15).

Scenes (positions as an (N, 3) float64 array, insertion order):

* ``quickstart_dam`` — the README quick-start block: SphParams::defaults(),
  fill_box((-1,1,-1), (1,3,1), 0.3, 0.1): 7x7x7 = 343 particles (spacing 0.3
  is larger than h = 0.2, so only the self term contributes to the density).
* ``dam_break(nx, ny, nz, box)`` — a jittered cubic lattice of spacing
  s = h/2 = 0.1 at ((i+0.5)s, (j+0.5)s, (k+0.5)s), each coordinate jittered by
  (2u-1) * 0.05 s with u drawn in the order i -> j -> k, then x, y, z (seed
  0xC0FFEE); zero velocity; mass = lattice_mass(s); bounds [0, box]^3;
  SphParams::defaults() otherwise.  The standard sizes:
    - 80x160x80  = 1,024,000 particles, box 32,   dt 0.005  (plain f64 at scale)
    - 128x256x128 = 4,194,304 particles, box 51.2, dt 0.0025 (precision form)
    - 32x64x32   = 65,536 particles,    box 12.8, dt 0.005  (differentiation form)
* ``batch_scenes(n_scenes, nmin, nmax)`` — independent dam breaks of uneven
  size for the batched form: per scene five draws of the stream seeded with
  BATCH_SEED (scene-major): target count log-uniform in [nmin, nmax], box
  aspect per axis uniform in [0.5, 2], fill fraction (block volume / box
  volume) uniform in [0.2, 0.5].  The block keeps the box's aspect, sits in
  the low corner and is the dam-break lattice above (jitter seed SEED + 1 +
  scene index); bounds [0, box extent] per axis.  The standard batch is 256
  scenes in [2000, 200000] stepped 200 times at dt 0.005.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
SEED = 0xC0FFEE
BATCH_SEED = 0xBA7C4ED
SPACING = 0.1


def splitmix64(seed: int, start: int, count: int) -> np.ndarray:
    """Draws start .. start+count-1 of SplitMix64 seeded with `seed` (replay.rs:40-46)."""
    with np.errstate(over="ignore"):
        n = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + n * GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, start: int, count: int) -> np.ndarray:
    """Rng::next_f64 (replay.rs:48-52): top 53 bits / 2^53."""
    return (splitmix64(seed, start, count) >> np.uint64(11)).astype(np.float64) / float(1 << 53)


@dataclass
class Scene:
    name: str
    pos: np.ndarray
    vel: np.ndarray
    mass: float
    bounds_min: tuple
    bounds_max: tuple
    dt: float
    steps: int

    @property
    def n(self) -> int:
        return self.pos.shape[0]


def quickstart_positions() -> np.ndarray:
    """fill_box((-1,1,-1), (1,3,1), 0.3, 0.1) (world.rs:124-144), float-accumulated."""
    lo = (-1.0 + 0.1, 1.0 + 0.1, -1.0 + 0.1)
    hi = (1.0 - 0.1, 3.0 - 0.1, 1.0 - 0.1)
    d = 0.3
    out = []
    x = lo[0]
    while x <= hi[0]:
        y = lo[1]
        while y <= hi[1]:
            z = lo[2]
            while z <= hi[2]:
                out.append((x, y, z))
                z = z + d
            y = y + d
        x = x + d
    return np.asarray(out, np.float64)


def lattice_mass(s: float, h: float = 0.2, rest: float = 1000.0) -> float:
    """FluidWorld::lattice_mass (world.rs:148-169) with kernels of the same h."""
    import math
    h2 = h * h
    h3 = h2 * h
    h6 = h3 * h3
    h9 = h6 * h3
    c = 315.0 / (64.0 * math.pi * h9)
    n_shell = int(math.ceil(h / s)) + 1
    total = 0.0
    for i in range(-n_shell, n_shell + 1):
        for j in range(-n_shell, n_shell + 1):
            for l in range(-n_shell, n_shell + 1):
                r = s * math.sqrt(float(i * i + j * j + l * l))
                if r < h:
                    diff = h2 - r * r
                    total = total + c * diff * diff * diff
    return rest / total if total > 0.0 else 0.02


def dam_break_positions(nx: int, ny: int, nz: int, spacing: float = SPACING, seed: int = SEED,
                        jitter: float = 0.05) -> np.ndarray:
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    base = np.stack([(i + 0.5) * spacing, (j + 0.5) * spacing, (k + 0.5) * spacing], axis=-1).reshape(-1, 3)
    n = base.shape[0]
    u = uniform01(seed, 0, 3 * n).reshape(n, 3)
    return base + (2.0 * u - 1.0) * (jitter * spacing)


def dam_break(nx: int, ny: int, nz: int, box: float, dt: float, steps: int, seed: int = SEED) -> Scene:
    pos = dam_break_positions(nx, ny, nz, SPACING, seed)
    return Scene(name=f"dam_break_{nx}x{ny}x{nz}", pos=pos, vel=np.zeros_like(pos), mass=lattice_mass(SPACING),
                 bounds_min=(0.0, 0.0, 0.0), bounds_max=(box, box, box), dt=dt, steps=steps)


def config(name: str) -> Scene:
    """The benchmark scenes by name."""
    if name == "quickstart":
        pos = quickstart_positions()
        return Scene("quickstart_dam", pos, np.zeros_like(pos), lattice_mass(0.3), (-5.0, -5.0, -5.0),
                     (5.0, 5.0, 5.0), 0.01, 200)
    if name == "plain_1m":
        return dam_break(80, 160, 80, 32.0, 0.005, 500)
    if name == "comp_4m":
        return dam_break(128, 256, 128, 51.2, 0.0025, 1000)
    if name == "grad_64k":
        return dam_break(32, 64, 32, 12.8, 0.005, 100)
    if name.startswith("dam_"):  # dam_NX_NY_NZ: a small case of the same recipe
        nx, ny, nz = (int(v) for v in name.split("_")[1:4])
        return dam_break(nx, ny, nz, max(nx, ny, nz) * SPACING * 2.0, 0.005, 100)
    raise KeyError(name)


@dataclass
class BatchScene:
    pos: np.ndarray
    bounds_min: tuple
    bounds_max: tuple

    @property
    def n(self) -> int:
        return self.pos.shape[0]


def partition_scenes(counts, nparts: int) -> list:
    """Scenes split over `nparts` GPUs by particle count (greedy bin packing: the
    largest scene first, each to the part holding the fewest particles, ties to the
    lowest part).  Returns one ascending list of scene indices per part; every part's
    load is within the largest scene of the mean."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    order = sorted(range(len(counts)), key=lambda i: (-int(counts[i]), i))
    load = [0] * nparts
    parts = [[] for _ in range(nparts)]
    for i in order:
        k = min(range(nparts), key=lambda p: (load[p], p))
        parts[k].append(i)
        load[k] += int(counts[i])
    return [sorted(p) for p in parts]


def batch_scenes(n_scenes: int = 256, nmin: int = 2000, nmax: int = 200000, seed: int = BATCH_SEED,
                 spacing: float = SPACING) -> list:
    """The batched form's scenes (see the module docstring)."""
    u = uniform01(seed, 0, 5 * n_scenes).reshape(n_scenes, 5)
    out = []
    for sc in range(n_scenes):
        target = np.exp(np.log(nmin) + u[sc, 0] * (np.log(nmax) - np.log(nmin)))
        aspect = 0.5 + 1.5 * u[sc, 1:4]
        fill = 0.2 + 0.3 * u[sc, 4]
        volume = target * spacing ** 3 / fill
        edge = (volume / float(np.prod(aspect))) ** (1.0 / 3.0)
        box = edge * aspect
        counts = np.maximum(1, np.round(box * fill ** (1.0 / 3.0) / spacing)).astype(int)
        pos = dam_break_positions(int(counts[0]), int(counts[1]), int(counts[2]), spacing, SEED + 1 + sc)
        out.append(BatchScene(pos, (0.0, 0.0, 0.0), tuple(float(b) for b in box)))
    return out
