"""BCC lattice set-up on the host (the part of MISA-MD's job the plugin relies on).

Index convention (MISA-MD's, which the reference kernels assume): x is doubled,
so unit cell (cx, cy, cz) holds sites gx = 2 cx (corner) and gx = 2 cx + 1
(body centre); the ideal position of site (gx, gy, gz) is
(gx a0/2, (gy + (gx&1)/2) a0, (gz + (gx&1)/2) a0).  "Box order" is
((gz * ny) + gy) * (2 nx) + gx.
"""
from __future__ import annotations

import numpy as np

from ._abi import ATOM_DTYPE, MbDeviceDomain, check, i64ptr, lib

KB_EV = 8.617333262e-5           # eV / K
FTM2V = 9.64853321233e-3         # (eV/A)/amu -> A/fs^2
MVV2E = 1.0 / FTM2V              # amu A^2/fs^2 -> eV


def ideal_positions(cells: tuple[int, int, int], a0: float) -> np.ndarray:
    nx, ny, nz = cells
    gz, gy, gx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(2 * nx), indexing="ij")
    h = 0.5 * (gx & 1)
    pos = np.stack([0.5 * a0 * gx, a0 * (gy + h), a0 * (gz + h)], axis=-1)
    return pos.reshape(-1, 3)


def bcc_box(cells: tuple[int, int, int], a0: float, atom_type: int = 0) -> np.ndarray:
    """Perfect lattice in box order (mb_atom_element records)."""
    pos = ideal_positions(cells, a0)
    a = np.zeros(pos.shape[0], dtype=ATOM_DTYPE)
    a["id"] = np.arange(1, pos.shape[0] + 1)
    a["type"] = atom_type
    a["x"] = pos
    return a


def add_vacancies(box: np.ndarray, fraction: float, seed: int) -> np.ndarray:
    """Vacate round(fraction * n) sites chosen uniformly without replacement."""
    rng = np.random.default_rng(seed)
    n = int(round(fraction * box.shape[0]))
    idx = rng.choice(box.shape[0], size=n, replace=False) if n else np.zeros(0, dtype=np.int64)
    box["type"][idx] = -1
    box["v"][idx] = 0.0
    return np.sort(idx)


# the six octahedral sites of a BCC unit cell, in units of a0
OCTAHEDRAL = np.array([[0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5],
                       [0.5, 0.0, 0.0], [0.0, 0.5, 0.0], [0.0, 0.0, 0.5]])


def octahedral_interstitials(n: int, cells: tuple[int, int, int], a0: float, seed: int,
                             atom_type: int = 0, first_id: int = 1 << 40) -> np.ndarray:
    """n interstitial atoms at distinct random octahedral sites."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = cells
    total = nx * ny * nz * 6
    pick = rng.choice(total, size=n, replace=False) if n else np.zeros(0, dtype=np.int64)
    kind = pick % 6
    cell = pick // 6
    cx, cy, cz = cell % nx, (cell // nx) % ny, cell // (nx * ny)
    pos = (np.stack([cx, cy, cz], axis=-1) + OCTAHEDRAL[kind]) * a0
    itl = np.zeros(n, dtype=ATOM_DTYPE)
    itl["id"] = first_id + np.arange(n)
    itl["type"] = atom_type
    itl["x"] = pos
    return itl


def maxwell_boltzmann(box: np.ndarray, itl: np.ndarray | None, temperature: float, mass: float, seed: int) -> None:
    """Gaussian velocities at `temperature`, zero net momentum, rescaled to exactly
    (3N - 3)/2 kB T of kinetic energy (A/fs)."""
    rng = np.random.default_rng(seed)
    live = box["type"] >= 0
    n_live = int(live.sum())
    n_itl = 0 if itl is None else itl.shape[0]
    sigma = np.sqrt(KB_EV * temperature * FTM2V / mass)
    v = rng.normal(0.0, sigma, size=(n_live + n_itl, 3))
    v -= v.mean(axis=0)
    n = n_live + n_itl
    ke = 0.5 * mass * np.sum(v * v) * MVV2E
    target = 0.5 * (3 * n - 3) * KB_EV * temperature
    if ke > 0 and temperature > 0:
        v *= np.sqrt(target / ke)
    box["v"][live] = v[:n_live]
    box["v"][~live] = 0.0
    if n_itl:
        itl["v"] = v[n_live:]


def kinetic_energy(box: np.ndarray, itl: np.ndarray | None, mass: float) -> float:
    live = box["type"] >= 0
    ke = np.sum(box["v"][live] ** 2)
    if itl is not None and itl.shape[0]:
        ke += np.sum(itl["v"] ** 2)
    return 0.5 * mass * ke * MVV2E


# ------------------------------------------------------------ drop-in layout
def domain(cells: tuple[int, int, int], ghost: tuple[int, int, int], start=(0, 0, 0)) -> MbDeviceDomain:
    """The converted _hipDeviceDomain of a single periodic box (ghost in doubled x)."""
    bx, by, bz = 2 * cells[0], cells[1], cells[2]
    gx, gy, gz = ghost
    return MbDeviceDomain(gx, gy, gz, bx, by, bz, bx + 2 * gx, by + 2 * gy, bz + 2 * gz, 0,
                          start[0], start[1], start[2])


def box_to_ext(box: np.ndarray, cells: tuple[int, int, int], ghost: tuple[int, int, int], a0: float,
               out: np.ndarray | None = None) -> np.ndarray:
    """Ghost-extended AoS array (the host's lattice with its periodic ghost fill)."""
    bx, by, bz = 2 * cells[0], cells[1], cells[2]
    gx, gy, gz = ghost
    ex, ey, ez = bx + 2 * gx, by + 2 * gy, bz + 2 * gz
    L = np.array([cells[0] * a0, cells[1] * a0, cells[2] * a0])
    zz, yy, xx = np.meshgrid(np.arange(ez) - gz, np.arange(ey) - gy, np.arange(ex) - gx, indexing="ij")
    sx, sy, sz = np.mod(xx, bx), np.mod(yy, by), np.mod(zz, bz)
    src = ((sz * by + sy) * bx + sx).reshape(-1)
    ext = out if out is not None else np.empty(ex * ey * ez, dtype=ATOM_DTYPE)
    ext[:] = box[src]
    shift = np.stack([(xx - sx) // bx * L[0], (yy - sy) // by * L[1], (zz - sz) // bz * L[2]], axis=-1).reshape(-1, 3)
    ext["x"] += shift
    return ext


def ext_to_box(ext: np.ndarray, cells: tuple[int, int, int], ghost: tuple[int, int, int]) -> np.ndarray:
    bx, by, bz = 2 * cells[0], cells[1], cells[2]
    gx, gy, gz = ghost
    ex, ey = bx + 2 * gx, by + 2 * gy
    e = ext.reshape(bz + 2 * gz, ey, ex)
    return np.ascontiguousarray(e[gz:gz + bz, gy:gy + by, gx:gx + bx]).reshape(-1)


def stencil_linear(a0: float, reach: float, ext_x: int, ext_y: int, cap: int = 320):
    """Reference-style (even, odd) linear neighbour offsets for an ext array."""
    even = np.zeros(cap, dtype=np.int64)
    odd = np.zeros(cap, dtype=np.int64)
    import ctypes
    n = ctypes.c_int(0)
    check(lib().mb_stencil_linear(a0, reach, ext_x, ext_y, i64ptr(even), i64ptr(odd), cap, ctypes.byref(n)))
    return even[:n.value].copy(), odd[:n.value].copy()


def ghost_for_reach(a0: float, reach: float) -> tuple[int, int, int]:
    """Smallest (doubled-x, y, z) ghost widths covering a stencil of this reach."""
    e, o = stencil_linear(a0, reach, 1 << 20, 1 << 10)
    offs = np.concatenate([e, o])
    dz = np.rint(offs / float(1 << 30)).astype(np.int64)
    rem = offs - dz * (1 << 30)
    dy = np.rint(rem / float(1 << 20)).astype(np.int64)
    dx = rem - dy * (1 << 20)
    gx = int(np.abs(dx).max())
    gx += gx & 1
    return gx, int(np.abs(dy).max()), int(np.abs(dz).max())
