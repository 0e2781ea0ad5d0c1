"""Seeded synthetic inputs for the standalone pressure-Poisson cases.

The cases are the unit-cube Poisson problems with immersed spheres and the
sphere/ellipsoid flow boxes.  Everything is generated from a counter-based
SplitMix64 stream, so the same seed gives the same bodies and right-hand side
in numpy, in C and on any machine:

* ``splitmix64(x)``: the published SplitMix64 finaliser (Steele, Lea, Flood,
  "Fast splittable pseudorandom number generators", OOPSLA 2014).
* uniform doubles: top 53 bits of the stream word times 2**-53.
* normal variates: Box-Muller on two uniforms of the same counter pair.

Level-set sign convention: phi > 0 inside a body (the reference's
calcLevelSetSphere, flow_sphere_task_description.h:57-74); several bodies are
merged by max, i.e. min of (|x - c| - r).
"""
from __future__ import annotations

import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 output for counter words ``x`` (uint64 array)."""
    with np.errstate(over="ignore"):
        z = (np.asarray(x, dtype=np.uint64) + _GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniforms(seed: int, stream: int, count: int) -> np.ndarray:
    """``count`` uniforms in [0, 1) from stream ``stream`` of ``seed``."""
    base = np.uint64((seed * 0x100000001B3 + stream * 0x1000193) & 0xFFFFFFFFFFFFFFFF)
    with np.errstate(over="ignore"):
        ctr = base + np.arange(count, dtype=np.uint64) * _GOLDEN
    return (splitmix64(ctr) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def normals(seed: int, stream: int, count: int) -> np.ndarray:
    """``count`` i.i.d. N(0, 1) variates (Box-Muller)."""
    u = uniforms(seed, stream, 2 * count).reshape(count, 2)
    u1 = 1.0 - u[:, 0]                      # (0, 1]
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u[:, 1])


def four_spheres(seed: int, count: int = 4, rmin: float = 0.05, rmax: float = 0.15,
                 cmin: float = 0.2, cmax: float = 0.8):
    """Sphere list [(cx, cy, cz, r)] with radii U[rmin, rmax] and centres
    U[cmin, cmax]^3 (the standalone Poisson geometry generator)."""
    u = uniforms(seed, 1, 4 * count).reshape(count, 4)
    out = []
    for k in range(count):
        r = rmin + (rmax - rmin) * u[k, 0]
        c = cmin + (cmax - cmin) * u[k, 1:4]
        out.append((float(c[0]), float(c[1]), float(c[2]), float(r)))
    return out


def random_rotation(u3: np.ndarray) -> np.ndarray:
    """Uniform random rotation from three uniforms (Shoemake's quaternion
    method, Graphics Gems III)."""
    a, b, c = (float(v) for v in u3)
    q = (math.sqrt(1 - a) * math.sin(2 * math.pi * b), math.sqrt(1 - a) * math.cos(2 * math.pi * b),
         math.sqrt(a) * math.sin(2 * math.pi * c), math.sqrt(a) * math.cos(2 * math.pi * c))
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def ellipsoids(seed: int, count: int, box, amin: float = 0.3, amax: float = 0.8):
    """Ellipsoids with semi-axes U[amin, amax], random rotations and centres in
    the first third (in x) of ``box`` = (Lx, Ly, Lz)."""
    u = uniforms(seed, 2, 9 * count).reshape(count, 9)
    Lx, Ly, Lz = box
    out = []
    for k in range(count):
        ax = amin + (amax - amin) * u[k, 0:3]
        c = np.array([u[k, 3] * Lx / 3.0, 0.25 * Ly + 0.5 * Ly * u[k, 4], 0.25 * Lz + 0.5 * Lz * u[k, 5]])
        c[0] = max(c[0], ax.max() + 0.5)
        out.append((c, ax, random_rotation(u[k, 6:9])))
    return out


def connected_fluid(rowptr: np.ndarray, col: np.ndarray, val: np.ndarray, pins) -> np.ndarray:
    """Mask of the cells that the operator couples (through nonzero
    off-diagonal coefficients) to the first pinned cell's neighbourhood.

    A cut-cell Laplacian can hold fluid pockets sealed off by bodies and cut
    cells whose every face fraction is zero (zero rows).  Those blocks are
    singular, so a compatible right-hand side must vanish on them."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components
    n = rowptr.size - 1
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    keep = (val != 0.0) & (rows != col)
    pinset = {int(p) for p in pins}
    keep &= ~np.isin(rows, list(pinset))      # pinned rows are identity rows
    g = csr_matrix((np.ones(int(keep.sum())), (rows[keep], col[keep])), shape=(n, n))
    _, lab = connected_components(g, directed=True, connection="weak")
    sizes = np.bincount(lab)
    main = int(np.argmax(sizes))
    mask = lab == main
    mask[list(pinset)] = False
    return mask


def poisson_rhs(seed: int, celltype: np.ndarray, pins, fluid_mask: np.ndarray | None = None) -> np.ndarray:
    """Right-hand side of the standalone Poisson case: i.i.d. N(0, 1) on the
    fluid cells of the main connected fluid region, mean removed over those
    cells, zero on solid cells, sealed pockets and the pinned rows.
    ``celltype`` uses the reference's CellTypes codes (SolidCell == 0);
    ``fluid_mask`` (from :func:`connected_fluid`) selects the main region."""
    n = celltype.size
    b = normals(seed, 3, n)
    fluid = celltype.reshape(-1) != 0
    if fluid_mask is not None:
        fluid &= fluid_mask
    b[~fluid] = 0.0
    for p in pins:
        fluid[int(p)] = False
        b[int(p)] = 0.0
    b[fluid] -= b[fluid].mean()
    return b
