"""Seeded synthetic specimens for the benchmark configurations.

No structure files ship with the reference, so every workload is generated
here from its crystallographic description (or, for amorphous carbon, by
seeded random sequential addition).  Each builder returns ``(Z, x, y, z)``
as int32 / float32 arrays in Angstrom.
"""
from __future__ import annotations

import numpy as np

BASE_SEED = 0x5EED2026


def _tile(frac: np.ndarray, Zc: np.ndarray, cell: tuple[float, float, float], reps: tuple[int, int, int]):
    ix, iy, iz = np.meshgrid(np.arange(reps[0]), np.arange(reps[1]), np.arange(reps[2]), indexing="ij")
    shifts = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(np.float64)
    pos = (shifts[:, None, :] + frac[None, :, :]).reshape(-1, 3) * np.asarray(cell)
    Z = np.tile(Zc, shifts.shape[0]).astype(np.int32)
    return Z, pos[:, 0].astype(np.float32), pos[:, 1].astype(np.float32), pos[:, 2].astype(np.float32)


def srtio3(nx: int = 4, ny: int = 4, nz: int = 20, a: float = 3.905):
    """SrTiO3 perovskite: Sr (0,0,0), Ti (1/2,1/2,1/2), O at the face centres."""
    frac = np.array([[0, 0, 0], [0.5, 0.5, 0.5], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    Zc = np.array([38, 22, 8, 8, 8])
    return _tile(frac, Zc, (a, a, a), (nx, ny, nz))


def silicon_110(nx: int = 8, ny: int = 6, nz: int = 50, a: float = 5.431):
    """Si viewed along [110]: orthogonal 4-atom cell a/sqrt2 x a x a/sqrt2
    (x = [1-10]/2, y = [001], z = [110]/2) repeated nx x ny x nz."""
    conv = np.array([[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0],
                     [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75], [0.75, 0.75, 0.25]])
    ex = np.array([1, -1, 0]) / 2.0
    ey = np.array([0, 0, 1.0])
    ez = np.array([1, 1, 0]) / 2.0
    basis = np.stack([ex, ey, ez], axis=1)  # columns: cell vectors in units of a
    inv = np.linalg.inv(basis)
    pts = []
    for i in range(-2, 3):
        for j in range(-2, 3):
            for k in range(-2, 3):
                for p in conv:
                    f = inv @ (p + np.array([i, j, k]))
                    f = np.round(f, 9) % 1.0
                    pts.append(tuple(np.round(f, 6)))
    frac = np.array(sorted(set(pts)))
    assert frac.shape[0] == 4, frac
    cell = (a / np.sqrt(2), a, a / np.sqrt(2))
    return _tile(frac, np.full(4, 14), cell, (nx, ny, nz))


def gan_wurtzite_11_20(nx: int = 10, ny: int = 6, nz: int = 40, a: float = 3.189, c: float = 5.185,
                       u: float = 0.377):
    """GaN wurtzite viewed along [11-20]: orthohexagonal 8-atom cell
    a*sqrt3 x c x a (x = [1-100], y = [0001], z = [11-20])."""
    # hexagonal positions: Ga (1/3,2/3,0), (2/3,1/3,1/2); N shifted by u along c
    hexf = [(1 / 3, 2 / 3, 0.0, 31), (2 / 3, 1 / 3, 0.5, 31), (1 / 3, 2 / 3, u, 7), (2 / 3, 1 / 3, 0.5 + u, 7)]
    A1 = np.array([a, 0, 0])
    A2 = np.array([-a / 2, a * np.sqrt(3) / 2, 0])
    A3 = np.array([0, 0, c])
    # orthohexagonal cell: X = A1 + 2 A2 (length a*sqrt3), Y = A3 (c), Z = A1 (a)
    X, Y, Zv = A1 + 2 * A2, A3, A1
    M = np.stack([X, Y, Zv], axis=1)
    inv = np.linalg.inv(M)
    pts = {}
    for i in range(-3, 4):
        for j in range(-3, 4):
            for k in range(-2, 3):
                for fx, fy, fz, Zn in hexf:
                    r = (fx + i) * A1 + (fy + j) * A2 + (fz + k) * A3
                    f = np.round(inv @ r, 9) % 1.0
                    pts[tuple(np.round(f, 6))] = Zn
    frac = np.array(list(pts.keys()))
    Zc = np.array(list(pts.values()))
    assert frac.shape[0] == 8, frac.shape
    return _tile(frac, Zc, (np.linalg.norm(X), c, a), (nx, ny, nz))


def amorphous_carbon(size=(50.0, 50.0, 200.0), density: float = 0.1, min_sep: float = 1.2,
                     seed: int = BASE_SEED + 2):
    """Carbon atoms placed uniformly at random at `density` atoms/A^3 with a
    minimum separation (random sequential addition on a cell list, seeded)."""
    rng = np.random.default_rng(seed)
    L = np.asarray(size, np.float64)
    n_target = int(round(density * L.prod()))
    cs = min_sep
    ncell = np.maximum((L / cs).astype(int), 1)
    grid: dict[tuple[int, int, int], list[int]] = {}
    pos = np.empty((n_target, 3))
    n = 0
    r2 = min_sep * min_sep
    while n < n_target:
        cand = rng.random((4096, 3)) * L
        for p in cand:
            c = tuple(np.minimum((p / cs).astype(int), ncell - 1))
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        lst = grid.get((c[0] + dx, c[1] + dy, c[2] + dz))
                        if lst:
                            q = pos[lst]
                            if np.any(((q - p) ** 2).sum(axis=1) < r2):
                                ok = False
                                break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                pos[n] = p
                grid.setdefault(c, []).append(n)
                n += 1
                if n == n_target:
                    break
    Z = np.full(n_target, 6, np.int32)
    return Z, pos[:, 0].astype(np.float32), pos[:, 1].astype(np.float32), pos[:, 2].astype(np.float32)


def random_atoms(n: int, size=(10.0, 10.0, 10.0), Zs=(6, 8, 14, 38), seed: int = BASE_SEED):
    """Small random structures for tests (no minimum separation)."""
    rng = np.random.default_rng(seed)
    xyz = rng.random((n, 3)) * np.asarray(size)
    Z = rng.choice(np.asarray(Zs), n).astype(np.int32)
    return Z, xyz[:, 0].astype(np.float32), xyz[:, 1].astype(np.float32), xyz[:, 2].astype(np.float32)


def write_xyz(path: str, Z, x, y, z, symbols: dict[int, str] | None = None, comment_line: bool = True):
    """Write an .xyz file.  comment_line=False writes the layout the reference
    reader expects (count and comment on the first line)."""
    sym = symbols or {1: "H", 6: "C", 7: "N", 8: "O", 14: "Si", 22: "Ti", 31: "Ga", 38: "Sr"}
    with open(path, "w") as f:
        f.write(f"{len(Z)}\ncomment\n" if comment_line else f"{len(Z)} comment\n")
        for zz, a, b, c in zip(Z, x, y, z):
            f.write(f"{sym[int(zz)]} {float(a):.6f} {float(b):.6f} {float(c):.6f}\n")
