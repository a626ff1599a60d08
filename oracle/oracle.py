"""ctypes binding of the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE ONLY.

Used by tests/, the smoke check and the bench's CPU-baseline leg as the checker.
It declares its own record and domain types (same bytes as the reference's
_cuAtomElement and _hipDeviceDomain, src/kernel_types.h:40-64) and imports nothing
from the product package.

PARITY UNPINNED against the reference itself (it cannot be built here); pinned by
analytic known answers, finite differences and NVE conservation in
tests/test_oracle.py.
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

ATOM = np.dtype([
    ("id", "<i8"), ("type", "<i4"), ("pad_", "<i4"),
    ("x", "<f8", (3,)), ("v", "<f8", (3,)), ("f", "<f8", (3,)),
    ("rho", "<f8"), ("df", "<f8"),
])


class Domain(C.Structure):
    _fields_ = [("ghost_size_x", C.c_int32), ("ghost_size_y", C.c_int32), ("ghost_size_z", C.c_int32),
                ("box_size_x", C.c_int32), ("box_size_y", C.c_int32), ("box_size_z", C.c_int32),
                ("ext_size_x", C.c_int32), ("ext_size_y", C.c_int32), ("ext_size_z", C.c_int32),
                ("pad_", C.c_int32),
                ("box_index_start_x", C.c_int64), ("box_index_start_y", C.c_int64),
                ("box_index_start_z", C.c_int64)]


class MdParams(C.Structure):
    _fields_ = [("a0", C.c_double), ("mass", C.c_double), ("dt", C.c_double), ("cutoff", C.c_double),
                ("itl_margin", C.c_double)]


class Energy(C.Structure):
    _fields_ = [("pe", C.c_double), ("ke", C.c_double)]


_PD = C.POINTER(C.c_double)
_PI64 = C.POINTER(C.c_int64)
_P = C.c_void_p


def build() -> pathlib.Path:
    src = [HERE / "eam_oracle.c", HERE / "eam_oracle.h"]
    if not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in src):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        sig = {
            "orc_spline_coeffs": (None, [_PD, C.c_int, C.c_double, _PD]),
            "orc_pot_create": (_P, [C.c_int, C.c_int, C.c_double, C.c_int, C.c_double, C.c_double, _PD, _PD, _PD]),
            "orc_pot_destroy": (None, [_P]),
            "orc_rho_of_r": (C.c_double, [_P, C.c_int, C.c_double]),
            "orc_drho_of_r": (C.c_double, [_P, C.c_int, C.c_double]),
            "orc_phi_of_r": (C.c_double, [_P, C.c_int, C.c_int, C.c_double]),
            "orc_dphi_of_r": (C.c_double, [_P, C.c_int, C.c_int, C.c_double]),
            "orc_F_of_rho": (C.c_double, [_P, C.c_int, C.c_double]),
            "orc_dF_of_rho": (C.c_double, [_P, C.c_int, C.c_double]),
            "orc_stencil_build": (C.c_int, [C.POINTER(Domain), C.c_double, C.c_double, _PI64, _PI64, C.c_int]),
            "orc_rho_pass": (None, [_P, C.POINTER(Domain), _P, _PI64, C.c_size_t, _PI64, C.c_size_t, C.c_double]),
            "orc_df_pass": (None, [_P, C.POINTER(Domain), _P]),
            "orc_force_pass": (None, [_P, C.POINTER(Domain), _P, _PI64, C.c_size_t, _PI64, C.c_size_t, C.c_double]),
            "orc_md_run_convert": (C.c_int, [_P, C.POINTER(Domain), _P, _P, C.c_int, C.c_int, _PI64, C.c_size_t,
                                             _PI64, C.c_size_t, C.POINTER(MdParams), C.c_int, C.c_double,
                                             C.c_double, _PI64]),
            "orc_convert": (C.c_int, [C.POINTER(Domain), C.c_double, _P, _P, C.c_int, C.c_int, C.c_double,
                                      C.c_double, _PI64]),
            "orc_rho_pass_half": (None, [_P, C.POINTER(Domain), _P, _PI64, C.c_size_t, _PI64, C.c_size_t,
                                         C.c_double]),
            "orc_force_pass_half": (None, [_P, C.POINTER(Domain), _P, _PI64, C.c_size_t, _PI64, C.c_size_t,
                                           C.c_double]),
            "orc_ghost_fill": (None, [C.POINTER(Domain), _P, _PD, C.c_int]),
            "orc_compute_forces": (None, [_P, C.POINTER(Domain), _P, _P, C.c_int, _PI64, C.c_size_t, _PI64,
                                          C.c_size_t, C.POINTER(MdParams), C.POINTER(Energy)]),
            "orc_md_run": (None, [_P, C.POINTER(Domain), _P, _P, C.c_int, _PI64, C.c_size_t, _PI64, C.c_size_t,
                                  C.POINTER(MdParams), C.c_int, C.POINTER(Energy)]),
            "orc_num_threads": (C.c_int, []),
            "orc_set_threads": (None, [C.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_PD)


def _i(a: np.ndarray):
    assert a.dtype == np.int64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_PI64)


def _a(a: np.ndarray):
    assert a.dtype == ATOM and a.flags["C_CONTIGUOUS"], a.dtype
    return C.c_void_p(a.ctypes.data)


def spline_coeffs(y: np.ndarray, dx: float) -> np.ndarray:
    y = np.ascontiguousarray(y, dtype=np.float64)
    out = np.zeros((y.size, 7))
    lib().orc_spline_coeffs(_d(y), y.size, dx, _d(out))
    return out


def make_domain(cells, ghost, start=(0, 0, 0)) -> Domain:
    bx, by, bz = 2 * cells[0], cells[1], cells[2]
    gx, gy, gz = ghost
    return Domain(gx, gy, gz, bx, by, bz, bx + 2 * gx, by + 2 * gy, bz + 2 * gz, 0, *start)


class Pot:
    def __init__(self, n_types, dr, drho, cutoff, f, F, phi):
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (f, F, phi)]
        f, F, phi = self._keep
        self.h = lib().orc_pot_create(n_types, f.shape[-1], dr, F.shape[-1], drho, cutoff, _d(f), _d(F), _d(phi))
        if not self.h:
            raise ValueError("oracle rejected the tables")
        self.cutoff = cutoff

    @classmethod
    def from_tables(cls, t) -> "Pot":
        return cls(t.n_types, t.dr, t.drho, t.cutoff, t.f, t.F, t.phi)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_pot_destroy(self.h)
            self.h = None

    def rho(self, t, r):
        return lib().orc_rho_of_r(self.h, t, r)

    def drho(self, t, r):
        return lib().orc_drho_of_r(self.h, t, r)

    def phi(self, a, b, r):
        return lib().orc_phi_of_r(self.h, a, b, r)

    def dphi(self, a, b, r):
        return lib().orc_dphi_of_r(self.h, a, b, r)

    def F(self, t, rho):
        return lib().orc_F_of_rho(self.h, t, rho)

    def dF(self, t, rho):
        return lib().orc_dF_of_rho(self.h, t, rho)


def stencil(dom: Domain, a0: float, reach: float):
    cap = 512
    e = np.zeros(cap, dtype=np.int64)
    o = np.zeros(cap, dtype=np.int64)
    n = lib().orc_stencil_build(C.byref(dom), a0, reach, _i(e), _i(o), cap)
    if n < 0:
        raise ValueError("stencil build failed")
    return e[:n].copy(), o[:n].copy()


def rho_pass(pot: Pot, dom: Domain, ext: np.ndarray, even, odd, cutoff: float) -> None:
    lib().orc_rho_pass(pot.h, C.byref(dom), _a(ext), _i(even), even.size, _i(odd), odd.size, cutoff)


def df_pass(pot: Pot, dom: Domain, ext: np.ndarray) -> None:
    lib().orc_df_pass(pot.h, C.byref(dom), _a(ext))


def force_pass(pot: Pot, dom: Domain, ext: np.ndarray, even, odd, cutoff: float) -> None:
    lib().orc_force_pass(pot.h, C.byref(dom), _a(ext), _i(even), even.size, _i(odd), odd.size, cutoff)


def convert(dom: Domain, a0: float, ext: np.ndarray, itl: np.ndarray, n_itl: int, d_conv: float, d_rec: float,
            counters: np.ndarray | None = None) -> int:
    """Lattice <-> interstitial bookkeeping after a step (orc_convert): itl is a buffer
    whose length is the capacity, its first n_itl records the list; returns the new
    count.  counters (int64[3]) accumulates conversions, recombinations, refusals."""
    c = np.zeros(3, dtype=np.int64) if counters is None else counters
    assert c.dtype == np.int64 and c.size == 3
    return int(lib().orc_convert(C.byref(dom), a0, _a(ext), _a(itl), n_itl, itl.shape[0], d_conv, d_rec, _i(c)))


def md_run_convert(pot: Pot, dom: Domain, ext: np.ndarray, itl: np.ndarray, n_itl: int, even, odd, mp: MdParams,
                   nsteps: int, d_conv: float, d_rec: float, counters: np.ndarray | None = None) -> int:
    """nsteps steps with the lattice <-> interstitial bookkeeping after every drift
    (orc_md_run_convert); itl is a buffer of capacity len(itl).  Returns the new count."""
    c = np.zeros(3, dtype=np.int64) if counters is None else counters
    return int(lib().orc_md_run_convert(pot.h, C.byref(dom), _a(ext), _a(itl), n_itl, itl.shape[0], _i(even),
                                        even.size, _i(odd), odd.size, C.byref(mp), nsteps, d_conv, d_rec, _i(c)))


def half_stencil(st: np.ndarray) -> np.ndarray:
    """One offset of each opposite pair: the offsets that are positive as linear
    indices (lexicographically positive (dz, dy, dx)), in their original order."""
    return np.ascontiguousarray(st[st > 0])


def rho_pass_half(pot: Pot, dom: Domain, ext: np.ndarray, even, odd, cutoff: float) -> None:
    """Newton's-third-law rho pass (orc_rho_pass_half): shares to box and ghost records."""
    lib().orc_rho_pass_half(pot.h, C.byref(dom), _a(ext), _i(even), even.size, _i(odd), odd.size, cutoff)


def force_pass_half(pot: Pot, dom: Domain, ext: np.ndarray, even, odd, cutoff: float) -> None:
    """Newton's-third-law force pass (orc_force_pass_half)."""
    lib().orc_force_pass_half(pot.h, C.byref(dom), _a(ext), _i(even), even.size, _i(odd), odd.size, cutoff)


def fold_ghosts(dom: Domain, ext: np.ndarray, field: str) -> np.ndarray:
    """Box-order copy of `field` with every ghost record's value added to the box site
    it images under the periodic wrap: what the host's reverse ghost communication
    does on a single periodic rank."""
    ex, ey, ez = dom.ext_size_x, dom.ext_size_y, dom.ext_size_z
    gx, gy, gz = dom.ghost_size_x, dom.ghost_size_y, dom.ghost_size_z
    bx, by, bz = dom.box_size_x, dom.box_size_y, dom.box_size_z
    a = ext[field].reshape((ez, ey, ex) + ext[field].shape[1:])
    out = np.zeros((bz, by, bx) + ext[field].shape[1:])
    zi = (np.arange(ez) - gz) % bz
    yi = (np.arange(ey) - gy) % by
    xi = (np.arange(ex) - gx) % bx
    np.add.at(out, (zi[:, None, None], yi[None, :, None], xi[None, None, :]), a)
    return out.reshape((bz * by * bx,) + ext[field].shape[1:])


def ghost_fill(dom: Domain, ext: np.ndarray, box_len, mask: int) -> None:
    L = np.ascontiguousarray(box_len, dtype=np.float64)
    lib().orc_ghost_fill(C.byref(dom), _a(ext), _d(L), mask)


def md_params(a0, mass, dt, cutoff, itl_margin=1.0) -> MdParams:
    return MdParams(a0, mass, dt, cutoff, itl_margin)


def compute_forces(pot: Pot, dom: Domain, ext: np.ndarray, itl: np.ndarray, even, odd, mp: MdParams):
    e = Energy()
    n = 0 if itl is None else itl.shape[0]
    itl_p = _a(itl) if n else None
    lib().orc_compute_forces(pot.h, C.byref(dom), _a(ext), itl_p, n, _i(even), even.size, _i(odd), odd.size,
                             C.byref(mp), C.byref(e))
    return e.pe, e.ke


def md_run(pot: Pot, dom: Domain, ext: np.ndarray, itl: np.ndarray, even, odd, mp: MdParams, nsteps: int,
           record: bool = True):
    """nsteps velocity-Verlet steps, state updated in place.  With record=True the
    forces are first re-evaluated at the starting positions and an (nsteps+1, 2)
    array of (pe, ke) is returned; with record=False the forces in the records must
    be current and nothing else is computed (one force evaluation per step)."""
    es = (Energy * (nsteps + 1))() if record else None
    n = 0 if itl is None else itl.shape[0]
    itl_p = _a(itl) if n else None
    lib().orc_md_run(pot.h, C.byref(dom), _a(ext), itl_p, n, _i(even), even.size, _i(odd), odd.size, C.byref(mp),
                     nsteps, es)
    return np.array([[e.pe, e.ke] for e in es]) if record else None


def set_threads(n: int) -> None:
    lib().orc_set_threads(n)


def num_threads() -> int:
    return lib().orc_num_threads()
