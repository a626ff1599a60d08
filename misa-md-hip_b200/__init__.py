"""misa_b200: B200-native EAM hot path of MISA-MD (host-side Python mirror).

The compute path is the CUDA library ``libmisa_b200.so`` (csrc/, built for
sm_100a); this package only binds its C ABI (include/misa_b200.h) with ctypes and
sets up lattices.  Importing it does not need a GPU; every compute call does, and
raises if the library or the device is missing (there is no CPU fallback).

Two ways in:
  * ``Hooks`` — the misa-md-hip plugin interface (rho / df / force passes on the
    host's ghost-extended AoS lattice), for a MISA-MD-style host loop;
  * ``Sim``   — device-resident molecular dynamics of one lattice.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi, lattice, potential
from ._abi import ATOM_DTYPE, MB_PREC_FP64, MB_PREC_MIXED, MbError, check, lib, ptr

__all__ = ["ATOM_DTYPE", "MB_PREC_FP64", "MB_PREC_MIXED", "MbError", "Hooks", "Sim", "Ensemble", "lattice", "potential",
           "lib", "build"]


def build(force: bool = False, verbose: bool = False):
    from . import builder
    return builder.build(force=force, verbose=verbose)


class Hooks:
    """The drop-in plugin interface (misa-md-hip src/hip_arch_acc_imp.cpp:28-225)."""

    def __init__(self, device: int = 0):
        check(lib().mb_env_init(device))

    def domain_init(self, dom: _abi.MbDeviceDomain) -> None:
        check(lib().mb_domain_init(C.byref(dom)))

    def nei_offset_init(self, even: np.ndarray, odd: np.ndarray) -> None:
        even = np.ascontiguousarray(even, dtype=np.int64)
        odd = np.ascontiguousarray(odd, dtype=np.int64)
        check(lib().mb_nei_offset_init(_abi.i64ptr(even), even.size, _abi.i64ptr(odd), odd.size))

    def pot_init(self, tables: potential.EamTables) -> None:
        t = tables.as_c()
        check(lib().mb_pot_init(C.byref(t)))

    def rho_calc(self, atoms: np.ndarray, cutoff: float) -> None:
        assert atoms.dtype == ATOM_DTYPE
        check(lib().mb_eam_rho_calc(ptr(atoms), cutoff))

    def df_calc(self, atoms: np.ndarray, cutoff: float) -> None:
        check(lib().mb_eam_df_calc(ptr(atoms), cutoff))

    def df_from_rho(self, atoms: np.ndarray) -> None:
        check(lib().mb_eam_df_from_rho(ptr(atoms)))

    def set_half_neighbour(self, enable: bool) -> None:
        """The reference's USE_NEWTONS_THIRD_LOW build at run time (half stencils; rho
        and f shares written to box and ghost records); nei_offset_init must follow."""
        check(lib().mb_set_half_neighbour(int(enable)))

    def force_calc(self, atoms: np.ndarray, cutoff: float) -> None:
        assert atoms.dtype == ATOM_DTYPE
        check(lib().mb_eam_force_calc(ptr(atoms), cutoff))

    def set_batches(self, batches: int) -> None:
        """-b/--batches: z-slabs the rho and force hooks stream the array in (1: the
        library chooses)."""
        check(lib().mb_cli_set_batches(int(batches)))

    def last_timing(self) -> tuple[float, float]:
        k, c = C.c_float(), C.c_float()
        check(lib().mb_hook_last_timing(C.byref(k), C.byref(c)))
        return k.value, c.value

    @staticmethod
    def clean() -> None:
        check(lib().mb_env_clean())


class Sim:
    """Device-resident MD of one periodic BCC lattice (+ interstitials)."""

    def __init__(self, cells, tables: potential.EamTables, lattice_const: float = 2.855, mass: float = 55.845,
                 dt: float = 1.0, cutoff: float | None = None, stencil_skin: float = 0.7,
                 precision: int = MB_PREC_FP64, max_interstitials: int = 0, slab: tuple[int, int] | None = None):
        """slab = (z_first, z_count): this sim holds only those unit cells along z of the
        periodic lattice `cells` (one rank of a z-slab decomposition, mb_sim_create_slab)."""
        self.cells = tuple(int(c) for c in cells)
        self.lattice_const = lattice_const
        self.mass = mass
        self.dt = dt
        cfg = _abi.MbSimConfig(self.cells[0], self.cells[1], self.cells[2], precision, lattice_const, mass, dt,
                               tables.cutoff if cutoff is None else cutoff, stencil_skin, max_interstitials, 0)
        t = tables.as_c()
        h = C.c_void_p()
        if slab is None:
            check(lib().mb_sim_create(C.byref(cfg), C.byref(t), C.byref(h)))
            nz = self.cells[2]
        else:
            check(lib().mb_sim_create_slab(C.byref(cfg), C.byref(t), int(slab[0]), int(slab[1]), C.byref(h)))
            nz = int(slab[1])
        self.slab = slab
        self._h = h
        self.n_box = 2 * self.cells[0] * self.cells[1] * nz
        self.n_itl = 0
        self.max_interstitials = max_interstitials

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().mb_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, box: np.ndarray, itl: np.ndarray | None = None) -> None:
        assert box.dtype == ATOM_DTYPE and box.shape[0] == self.n_box
        n = 0 if itl is None else int(itl.shape[0])
        itl_p = ptr(np.ascontiguousarray(itl)) if n else None
        check(lib().mb_sim_upload(self._h, ptr(np.ascontiguousarray(box)), itl_p, n))
        self.n_itl = n

    def download(self) -> tuple[np.ndarray, np.ndarray]:
        box = np.zeros(self.n_box, dtype=ATOM_DTYPE)
        itl = np.zeros(max(1, self.max_interstitials), dtype=ATOM_DTYPE)
        n = C.c_int32(0)
        check(lib().mb_sim_download(self._h, ptr(box), ptr(itl), C.byref(n)))
        return box, itl[:n.value].copy()

    def run(self, nsteps: int, energy_every: int = 0) -> None:
        check(lib().mb_sim_run(self._h, nsteps, energy_every))
        check(lib().mb_sim_sync(self._h))

    def energies(self) -> np.ndarray:
        n = C.c_int32(0)
        check(lib().mb_sim_energies(self._h, None, 0, C.byref(n)))
        out = np.zeros((max(1, n.value), 3))
        check(lib().mb_sim_energies(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), n.value, C.byref(n)))
        return out[:n.value]

    def time_steps(self, nsteps: int) -> float:
        ms = C.c_float()
        check(lib().mb_sim_time_steps(self._h, nsteps, C.byref(ms)))
        return ms.value

    def kernel_times(self) -> tuple[float, float]:
        a, b = C.c_float(), C.c_float()
        check(lib().mb_sim_kernel_times(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def step_host(self, box: np.ndarray, itl: np.ndarray | None = None) -> None:
        """One full step through host buffers (box / itl updated in place)."""
        n = 0 if itl is None else int(itl.shape[0])
        check(lib().mb_sim_step_host(self._h, ptr(box), ptr(itl) if n else None, n))

    def set_host_slabs(self, n_slabs: int) -> None:
        """z-slabs step_host streams the box in (0 automatic, 1 one piece, else at most
        that many)."""
        check(lib().mb_sim_set_host_slabs(self._h, int(n_slabs)))

    def host_slabs(self) -> int:
        """Slabs the next step_host takes."""
        n = C.c_int32(0)
        check(lib().mb_sim_host_slabs(self._h, C.byref(n)))
        return n.value

    def info(self) -> dict:
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().mb_sim_info(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return {"n_sites": a.value, "n_stencil": b.value, "device_bytes": c.value}

    def set_graphs(self, enable: bool) -> None:
        check(lib().mb_sim_set_graphs(self._h, int(enable)))

    # -- z-slab decomposition (decomp.py drives these)
    def halo_bytes(self, what: int) -> int:
        """Bytes of one halo message: what 1 positions, 2 df, 3 site codes."""
        b = C.c_int64()
        check(lib().mb_sim_halo_bytes(self._h, what, C.byref(b)))
        return b.value

    def halo_pack(self, what: int, side: int, device_ptr: int) -> None:
        check(lib().mb_sim_halo_pack(self._h, what, side, C.c_void_p(device_ptr)))

    def halo_unpack(self, what: int, side: int, device_ptr: int, z_shift: float = 0.0) -> None:
        check(lib().mb_sim_halo_unpack(self._h, what, side, C.c_void_p(device_ptr), z_shift))

    def phase(self, phase: int, energy: bool = False) -> None:
        """0: rho / df; 1: forces + velocity-Verlet + drift (mb_sim_slab_phase)."""
        check(lib().mb_sim_slab_phase(self._h, phase, int(energy)))

    def clear_energies(self) -> None:
        check(lib().mb_sim_clear_energies(self._h))

    def sync(self) -> None:
        """Wait for the sim's queued device work (mb_sim_sync)."""
        check(lib().mb_sim_sync(self._h))


    def set_conversion(self, convert_distance: float, recombine_distance: float) -> None:
        """Atoms farther than convert_distance from their site join the interstitial
        list after each step; interstitials within recombine_distance of a vacant site
        take it (mb_sim_set_conversion).  convert_distance 0 switches it off."""
        check(lib().mb_sim_set_conversion(self._h, convert_distance, recombine_distance))

    def conversion_stats(self) -> dict:
        c = np.zeros(4, dtype=np.int64)
        n = C.c_int32(0)
        check(lib().mb_sim_conversion_stats(self._h, _abi.i64ptr(c), C.byref(n)))
        return {"converted": int(c[0]), "recombined": int(c[1]), "refused": int(c[2]), "dropped": int(c[3]),
                "n_itl": n.value}


class Ensemble:
    """Many independent periodic lattices advanced together in mixed precision: one
    CUDA graph per timestep advances every lattice (C ABI: mb_ensemble_*)."""

    def __init__(self, tables: potential.EamTables, lattice_const: float = 2.855, mass: float = 55.845,
                 dt: float = 1.0, cutoff: float | None = None, stencil_skin: float = 0.7,
                 hbm_budget_bytes: int = 0, max_lattices: int = 0):
        self.lattice_const = lattice_const
        cfg = _abi.MbEnsembleConfig(lattice_const, mass, dt, tables.cutoff if cutoff is None else cutoff,
                                    stencil_skin, int(hbm_budget_bytes), int(max_lattices), 0)
        t = tables.as_c()
        h = C.c_void_p()
        check(lib().mb_ensemble_create(C.byref(cfg), C.byref(t), C.byref(h)))
        self._h = h
        self._cells: dict[int, tuple] = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().mb_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @staticmethod
    def lattice_bytes(cells, max_interstitials: int = 0) -> int:
        spec = _abi.MbLatticeSpec(*[int(c) for c in cells], int(max_interstitials))
        b = C.c_int64()
        check(lib().mb_ensemble_lattice_bytes(C.byref(spec), C.byref(b)))
        return b.value

    def add(self, cells, box: np.ndarray, itl: np.ndarray | None = None, steps: int = 0,
            max_interstitials: int | None = None) -> int:
        cells = tuple(int(c) for c in cells)
        n = 0 if itl is None else int(itl.shape[0])
        cap = n if max_interstitials is None else max_interstitials
        spec = _abi.MbLatticeSpec(cells[0], cells[1], cells[2], cap)
        slot = C.c_int32()
        box = np.ascontiguousarray(box)
        itl_c = np.ascontiguousarray(itl) if n else None
        check(lib().mb_ensemble_add(self._h, C.byref(spec), ptr(box), ptr(itl_c) if n else None, n, int(steps),
                                    C.byref(slot)))
        self._cells[slot.value] = (cells, cap)
        return slot.value

    def remove(self, slot: int) -> None:
        check(lib().mb_ensemble_remove(self._h, slot))
        self._cells.pop(slot, None)

    def set_steps(self, slot: int, steps_target: int) -> None:
        check(lib().mb_ensemble_set_steps(self._h, slot, int(steps_target)))

    def advance(self, max_launches: int, energy_every: int = 0) -> int:
        n = C.c_int32()
        check(lib().mb_ensemble_advance(self._h, max_launches, energy_every, C.byref(n)))
        return n.value

    def run(self, nsteps: int, energy_every: int = 0) -> None:
        check(lib().mb_ensemble_run(self._h, nsteps, energy_every))
        check(lib().mb_ensemble_sync(self._h))

    def sync(self) -> None:
        check(lib().mb_ensemble_sync(self._h))

    def set_conversion(self, convert_distance: float, recombine_distance: float) -> None:
        """mb_sim_set_conversion for every lattice (mb_ensemble_set_conversion)."""
        check(lib().mb_ensemble_set_conversion(self._h, convert_distance, recombine_distance))

    def conversion_stats(self, slot: int) -> dict:
        c = np.zeros(4, dtype=np.int64)
        n = C.c_int32(0)
        check(lib().mb_ensemble_conversion_stats(self._h, slot, _abi.i64ptr(c), C.byref(n)))
        return {"converted": int(c[0]), "recombined": int(c[1]), "refused": int(c[2]), "dropped": int(c[3]),
                "n_itl": n.value}

    def download(self, slot: int) -> tuple[np.ndarray, np.ndarray]:
        cells, cap = self._cells[slot]
        box = np.zeros(2 * cells[0] * cells[1] * cells[2], dtype=ATOM_DTYPE)
        itl = np.zeros(max(1, cap), dtype=ATOM_DTYPE)
        n = C.c_int32()
        check(lib().mb_ensemble_download(self._h, slot, ptr(box), ptr(itl), C.byref(n)))
        return box, itl[:n.value].copy()

    def status(self, slot: int) -> tuple[int, int, int]:
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().mb_ensemble_status(self._h, slot, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def energies(self, slot: int) -> np.ndarray:
        n = C.c_int32()
        check(lib().mb_ensemble_energies(self._h, slot, None, 0, C.byref(n)))
        out = np.zeros((max(1, n.value), 3))
        check(lib().mb_ensemble_energies(self._h, slot, out.ctypes.data_as(C.POINTER(C.c_double)), n.value,
                                         C.byref(n)))
        return out[:n.value]

    def time(self, nsteps: int) -> float:
        ms = C.c_float()
        check(lib().mb_ensemble_time(self._h, nsteps, C.byref(ms)))
        return ms.value

    def set_policy(self, policy: int) -> None:
        check(lib().mb_ensemble_set_policy(self._h, policy))

    def autotune(self, steps: int = 5) -> tuple[int, float]:
        p, ms = C.c_int32(), C.c_float()
        check(lib().mb_ensemble_autotune(self._h, steps, C.byref(p), C.byref(ms)))
        return p.value, ms.value

    def info(self) -> dict:
        a, b, c, d = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32()
        check(lib().mb_ensemble_info(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        return {"n_sites": a.value, "n_tiles": b.value, "device_bytes": c.value, "n_slots": d.value}

    def set_graphs(self, enable: bool) -> None:
        check(lib().mb_ensemble_set_graphs(self._h, int(enable)))

    def set_mode(self, mode: int) -> None:
        """0: split kernels where their stencil applies (default), 1: persistent, 2: split."""
        check(lib().mb_ensemble_set_mode(self._h, mode))

    def set_wait_limit(self, barrier_polls: int) -> None:
        """Polls a grid barrier of the persistent kernel makes before giving up with
        MB_ERR_TIMEOUT (mb_ensemble_set_wait_limit); negative restores the default."""
        check(lib().mb_ensemble_set_wait_limit(self._h, int(barrier_polls)))

    def kernel_times(self) -> tuple[float, float, int]:
        """(density ms, force ms, kernels per step) of one step; see mb_ensemble_kernel_times."""
        a, b, n = C.c_float(), C.c_float(), C.c_int32()
        check(lib().mb_ensemble_kernel_times(self._h, C.byref(a), C.byref(b), C.byref(n)))
        return a.value, b.value, n.value
