"""Tabulated EAM potentials for the misa_b200 library (host side).

``fe_analytic`` builds the synthetic Fe potential the benchmarks use:
phi(r) = A (rc - r)^2 (1 + B r), f(r) = (rc - r)^2, F(rho) = -sqrt(rho),
tabulated on uniform knots r in [0, rc] and rho in [0, rho_max].
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import _abi


@dataclasses.dataclass
class EamTables:
    n_types: int
    dr: float
    drho: float
    cutoff: float
    f: np.ndarray    # [n_types, nr]
    F: np.ndarray    # [n_types, nrho]
    phi: np.ndarray  # [n_types*(n_types+1)//2, nr]

    @property
    def nr(self) -> int:
        return self.f.shape[1]

    @property
    def nrho(self) -> int:
        return self.F.shape[1]

    def as_c(self) -> _abi.MbEamTables:
        """ctypes view; keeps references to the arrays on the returned struct."""
        f = np.ascontiguousarray(self.f, dtype=np.float64)
        F = np.ascontiguousarray(self.F, dtype=np.float64)
        phi = np.ascontiguousarray(self.phi, dtype=np.float64)
        t = _abi.MbEamTables(self.n_types, f.shape[1], F.shape[1], 0, self.dr, self.drho, self.cutoff,
                             _abi.dptr(f), _abi.dptr(F), _abi.dptr(phi))
        t._keep = (f, F, phi)
        return t


def fe_analytic(nr: int = 5000, nrho: int = 5000, cutoff: float = 5.6, rho_max: float = 50.0,
                A: float = 0.8, B: float = -0.2) -> EamTables:
    r = np.linspace(0.0, cutoff, nr)
    rho = np.linspace(0.0, rho_max, nrho)
    f = (cutoff - r) ** 2
    phi = A * (cutoff - r) ** 2 * (1.0 + B * r)
    F = -np.sqrt(rho)
    return EamTables(1, cutoff / (nr - 1), rho_max / (nrho - 1), cutoff, f[None, :], F[None, :], phi[None, :])


def alloy_analytic(n_types: int = 3, nr: int = 2000, nrho: int = 2000, cutoff: float = 5.6,
                   rho_max: float = 200.0) -> EamTables:
    """A multi-type variant of the same analytic family (types differ by scale)."""
    r = np.linspace(0.0, cutoff, nr)
    rho = np.linspace(0.0, rho_max, nrho)
    f = np.stack([(1.0 + 0.15 * a) * (cutoff - r) ** 2 for a in range(n_types)])
    F = np.stack([-(1.0 + 0.1 * a) * np.sqrt(rho) for a in range(n_types)])
    rows = []
    for a in range(n_types):
        for b in range(a, n_types):
            rows.append((0.8 + 0.05 * (a + b)) * (cutoff - r) ** 2 * (1.0 - 0.2 * r))
    return EamTables(n_types, cutoff / (nr - 1), rho_max / (nrho - 1), cutoff, f, F, np.stack(rows))


# ------------------------------------------------------------------ potential files
# The tabulated-EAM file formats MISA-MD and other MD codes read for Fe-Cu-Ni style
# alloys.  Tables are on knots r_k = k dr (k = 0 .. Nr-1) and rho_k = k drho; the pair
# term is stored as r * phi(r) (setfl) or through an effective charge Z(r) with
# r * phi = 27.2 * 0.529 * Z_i Z_j (funcfl, Hartree * Bohr in eV * A).
HARTREE_BOHR = 27.2 * 0.529


def _numbers(lines):
    for ln in lines:
        for tok in ln.split():
            yield float(tok)


def _phi_from_rphi(rphi: np.ndarray, dr: float) -> np.ndarray:
    """phi(r) from knot values of r * phi(r); the r = 0 knot copies the first interior one
    (pairs never get that close)."""
    r = np.arange(rphi.shape[-1]) * dr
    phi = np.empty_like(rphi)
    phi[..., 1:] = rphi[..., 1:] / r[1:]
    phi[..., 0] = phi[..., 1]
    return phi


def _pair_row(a: int, b: int, n: int) -> int:
    """Row of pair (a, b) in the packed upper triangle (0,0),(0,1),..,(0,n-1),(1,1),..."""
    if a > b:
        a, b = b, a
    return a * n - a * (a - 1) // 2 + (b - a)


def read_setfl(path) -> tuple[EamTables, dict]:
    """Read a multi-element setfl file (LAMMPS ``eam/alloy`` layout): 3 comment lines;
    ``N el_1 .. el_N``; ``Nrho drho Nr dr cutoff``; per element a line ``Z mass a0
    lattice`` followed by Nrho values of F and Nr values of f; then the pair terms r*phi
    for i = 0..N-1, j = 0..i.  Returns the tables and {elements, masses, numbers,
    lattice_constants, lattices}."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    head = lines[3].split()
    n = int(head[0])
    if n < 1 or n > 3:
        raise ValueError(f"{path}: {n} elements (the device tables take 1 to 3)")
    elements = head[1:1 + n]
    if len(elements) != n:
        raise ValueError(f"{path}: line 4 names {len(elements)} elements, expected {n}")
    g = lines[4].split()
    nrho, drho, nr, dr, cutoff = int(g[0]), float(g[1]), int(g[2]), float(g[3]), float(g[4])
    F = np.zeros((n, nrho))
    f = np.zeros((n, nr))
    meta = {"elements": elements, "numbers": [], "masses": [], "lattice_constants": [], "lattices": []}
    pos = 5
    rest = []
    for a in range(n):
        h = lines[pos].split()
        meta["numbers"].append(int(float(h[0])))
        meta["masses"].append(float(h[1]))
        meta["lattice_constants"].append(float(h[2]) if len(h) > 2 else 0.0)
        meta["lattices"].append(h[3] if len(h) > 3 else "")
        pos += 1
        need = nrho + nr
        vals = []
        while len(vals) < need:
            if pos >= len(lines):
                raise ValueError(f"{path}: element {elements[a]} table is truncated")
            vals.extend(float(t) for t in lines[pos].split())
            pos += 1
        if len(vals) != need:
            raise ValueError(f"{path}: element {elements[a]} table has {len(vals)} values, expected {need}")
        F[a] = vals[:nrho]
        f[a] = vals[nrho:]
    rest = list(_numbers(lines[pos:]))
    npair = n * (n + 1) // 2
    if len(rest) != npair * nr:
        raise ValueError(f"{path}: {len(rest)} pair values, expected {npair * nr}")
    rphi = np.asarray(rest).reshape(npair, nr)
    phi = np.zeros((npair, nr))
    q = 0
    for i in range(n):  # file order: (0,0), (1,0), (1,1), (2,0), ...
        for j in range(i + 1):
            phi[_pair_row(i, j, n)] = _phi_from_rphi(rphi[q], dr)
            q += 1
    return EamTables(n, dr, drho, cutoff, f, F, phi), meta


def write_setfl(path, t: EamTables, elements=None, numbers=None, masses=None, lattice_constants=None,
                lattices=None, comment: str = "misa_b200 tables") -> None:
    """Write tables as a setfl file (values at full double precision, 5 per line)."""
    n = t.n_types
    elements = elements or [f"E{a}" for a in range(n)]
    numbers = numbers or [26] * n
    masses = masses or [55.845] * n
    lattice_constants = lattice_constants or [2.855] * n
    lattices = lattices or ["bcc"] * n
    r = np.arange(t.nr) * t.dr

    def block(vals):
        vals = np.asarray(vals, dtype=np.float64)
        return "\n".join(" ".join(f"{v:.17g}" for v in vals[k:k + 5]) for k in range(0, vals.size, 5))

    out = [comment, "", "", f"{n} " + " ".join(elements),
           f"{t.nrho} {t.drho:.17g} {t.nr} {t.dr:.17g} {t.cutoff:.17g}"]
    for a in range(n):
        out.append(f"{numbers[a]} {masses[a]:.17g} {lattice_constants[a]:.17g} {lattices[a]}")
        out.append(block(t.F[a]))
        out.append(block(t.f[a]))
    for i in range(n):
        for j in range(i + 1):
            out.append(block(r * t.phi[_pair_row(i, j, n)]))
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def read_funcfl(path) -> tuple[EamTables, dict]:
    """Read a single-element funcfl file (LAMMPS ``eam`` layout): 1 comment line;
    ``Z mass a0 lattice``; ``Nrho drho Nr dr cutoff``; Nrho values of F, Nr values of the
    effective charge Z(r), Nr values of f.  phi(r) = 27.2 * 0.529 * Z(r)^2 / r."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    h = lines[1].split()
    g = lines[2].split()
    nrho, drho, nr, dr, cutoff = int(g[0]), float(g[1]), int(g[2]), float(g[3]), float(g[4])
    vals = list(_numbers(lines[3:]))
    if len(vals) != nrho + 2 * nr:
        raise ValueError(f"{path}: {len(vals)} table values, expected {nrho + 2 * nr}")
    F = np.asarray(vals[:nrho])
    Z = np.asarray(vals[nrho:nrho + nr])
    f = np.asarray(vals[nrho + nr:])
    phi = _phi_from_rphi(HARTREE_BOHR * Z * Z, dr)
    meta = {"numbers": [int(float(h[0]))], "masses": [float(h[1])],
            "lattice_constants": [float(h[2]) if len(h) > 2 else 0.0], "lattices": [h[3] if len(h) > 3 else ""]}
    return EamTables(1, dr, drho, cutoff, f[None, :], F[None, :], phi[None, :]), meta
