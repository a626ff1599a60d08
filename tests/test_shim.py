"""The MISA-MD hook shim (misa-md-hip_b200/shim/hip_hooks_misa_b200.cpp), compiled with
g++ against stand-in declarations of the host's types (tests/shim/arch/arch_imp.h) and
linked with the library, the way a MISA-MD build links it.

CPU: the shim compiles, exports every hook under the reference's (C++) names, and the
-b/--batches option reaches the library.  GPU: rho -> df -> force through the hip_*
names, with the host's r * phi pair tables converted by hip_pot_init, match the oracle."""
from __future__ import annotations

import ctypes as C
import pathlib
import shutil
import subprocess

import numpy as np
import pytest

import misa_b200 as mb
from oracle import oracle as orc
from scenarios import A0, make, rel_err

ROOT = pathlib.Path(__file__).resolve().parents[1]
SHIM = ROOT / "misa-md-hip_b200" / "shim" / "hip_hooks_misa_b200.cpp"
DRIVER = ROOT / "tests" / "shim" / "shim_driver.cpp"
MIRROR = ROOT / "tests" / "shim" / "arch" / "arch_imp.h"
OUT = ROOT / "tests" / "shim" / "_build" / "libshim_test.so"
HOOKS = [
    "hip_env_init()", "hip_env_clean()", "hip_domain_init(comm::BccDomain const*)",
    "hip_nei_offset_init(NeighbourIndex<long> const*)", "hip_pot_init(eam*)",
    "hip_eam_rho_calc(eam*, _type_atom_list_collection, double)",
    "hip_eam_df_calc(eam*, _type_atom_list_collection, double)",
    "hip_eam_force_calc(eam*, _type_atom_list_collection, double)",
    "hip_create_atoms_mem(void**, unsigned long, long, long, long)", "hip_release_atoms_mem(void*)",
    "hip_cli_options(args::ArgumentParser&)", "hip_cli_options_parse(args::ArgumentParser&)",
    "__kernel_calRho_wrapper(dim3, dim3, _cuAtomElement*, _hipDeviceNeiOffsets, double)",
    "__kernel_calDf_wrapper(dim3, dim3, _cuAtomElement*)",
    "__kernel_calForce_wrapper(dim3, dim3, _cuAtomElement*, _hipDeviceNeiOffsets, double)",
]


def _cuda_include() -> str:
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return str(pathlib.Path(nvcc).resolve().parents[1] / "include")


def build_shim() -> pathlib.Path:
    deps = [SHIM, DRIVER, MIRROR, ROOT / "include" / "misa_b200.h", mb._abi.LIB_PATH]
    if OUT.exists() and all(d.stat().st_mtime <= OUT.stat().st_mtime for d in deps):
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-Werror",
           f"-I{ROOT / 'tests' / 'shim'}", f"-I{ROOT / 'include'}", f"-I{_cuda_include()}",
           str(SHIM), str(DRIVER), f"-L{mb._abi.LIB_PATH.parent}", "-lmisa_b200",
           "-Wl,-rpath,$ORIGIN/../../../misa-md-hip_b200", "-o", str(OUT)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"shim build failed:\n{' '.join(cmd)}\n{r.stderr}")
    return OUT


@pytest.fixture(scope="module")
def shim():
    mb.lib()  # the library the shim links, loaded first
    L = C.CDLL(str(build_shim()))
    _P, _I64P, _DP = C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_double)
    L.drive_env_init.argtypes = [C.c_char_p, C.c_int]
    L.drive_env_clean.argtypes = [C.c_char_p, C.c_int]
    L.drive_cli.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
    L.drive_setup.argtypes = [_I64P, _I64P, _I64P, _I64P, C.c_int, _I64P, C.c_int, C.c_int, C.c_int, C.c_double,
                              C.c_int, C.c_double, _DP, _DP, _DP, C.c_char_p, C.c_int]
    L.drive_pass.argtypes = [C.c_int, _P, C.c_double, C.c_char_p, C.c_int]
    L.drive_atoms_mem.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.c_char_p, C.c_int]
    return L


def _call(fn, *args):
    err = C.create_string_buffer(1024)
    rc = fn(*args, err, 1024)
    if rc:
        raise RuntimeError(err.value.decode())


def test_shim_compiles_and_exports_every_hook_under_the_reference_names():
    lib = build_shim()
    out = subprocess.run(["nm", "-D", "-C", "--defined-only", str(lib)], capture_output=True, text=True,
                         check=True).stdout
    defined = {line.split(" ", 2)[2] for line in out.splitlines() if line.count(" ") >= 2}
    missing = [h for h in HOOKS if h not in defined]
    assert not missing, missing


def test_shim_batches_option_reaches_the_library(shim):
    try:
        _call(shim.drive_cli, b"4")
        assert mb.lib().mb_cli_batches() == 4
        _call(shim.drive_cli, None)  # no -b: the value stays
        assert mb.lib().mb_cli_batches() == 4
    finally:
        mb.check(mb.lib().mb_cli_set_batches(1))


def test_shim_turns_errors_into_exceptions(shim):
    # a pass before any set-up is refused by the library and thrown by the hook
    _call(shim.drive_env_clean)  # whatever an earlier test set up is gone
    ext = np.zeros(8, dtype=mb.ATOM_DTYPE)
    with pytest.raises(RuntimeError, match="hip_eam_rho_calc"):
        _call(shim.drive_pass, 0, ext.ctypes.data, 5.6)


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _setup(shim, sc, start):
    dom = mb.lattice.domain(sc.cells, sc.ghost, start)
    even, odd = mb.lattice.stencil_linear(A0, sc.reach, dom.ext_size_x, dom.ext_size_y)
    t = sc.tables
    r = np.arange(t.nr) * t.dr
    rphi = np.ascontiguousarray(t.phi * r)  # what the host's setfl tables hold
    phi = np.empty_like(rphi)  # what hip_pot_init hands the library
    phi[:, 1:] = rphi[:, 1:] / r[1:]
    phi[:, 0] = phi[:, 1]
    box = np.array([dom.box_size_x, dom.box_size_y, dom.box_size_z], dtype=np.int64)
    ghost = np.array([dom.ghost_size_x, dom.ghost_size_y, dom.ghost_size_z], dtype=np.int64)
    st = np.array(start, dtype=np.int64)
    f = np.ascontiguousarray(t.f, dtype=np.float64)
    F = np.ascontiguousarray(t.F, dtype=np.float64)
    _call(shim.drive_setup, _ptr(box, C.c_int64), _ptr(ghost, C.c_int64), _ptr(st, C.c_int64),
          _ptr(even, C.c_int64), even.size, _ptr(odd, C.c_int64), odd.size, t.n_types, t.nr, t.dr, t.nrho, t.drho,
          _ptr(f, C.c_double), _ptr(F, C.c_double), _ptr(rphi, C.c_double))
    pot = orc.Pot(t.n_types, t.dr, t.drho, t.cutoff, t.f, t.F, phi)
    return orc.make_domain(sc.cells, sc.ghost, start), even, odd, pot


@pytest.mark.gpu
@pytest.mark.parametrize("n_types,start", [(1, (0, 0, 0)), (3, (1, 0, 0))])
def test_shim_hooks_match_oracle(shim, n_types, start):
    sc = make(cells=(7, 6, 5), temperature=900.0, vacancy=0.02, n_types=n_types, seed=27, jitter=0.1)
    _call(shim.drive_env_init)
    try:
        odom, even, odd, pot = _setup(shim, sc, start)
        ext = sc.ext()
        eo = ext.copy().view(orc.ATOM)
        _call(shim.drive_pass, 0, ext.ctypes.data, sc.cutoff)
        _call(shim.drive_pass, 1, ext.ctypes.data, sc.cutoff)  # full-neighbour build: no-op
        L = [sc.cells[0] * A0, sc.cells[1] * A0, sc.cells[2] * A0]
        orc.ghost_fill(odom, ext.view(orc.ATOM), L, 2)  # the host's df ghost exchange
        _call(shim.drive_pass, 2, ext.ctypes.data, sc.cutoff)
        orc.rho_pass(pot, odom, eo, even, odd, sc.cutoff)
        orc.ghost_fill(odom, eo, L, 2)
        orc.force_pass(pot, odom, eo, even, odd, sc.cutoff)
        bg = mb.lattice.ext_to_box(ext, sc.cells, sc.ghost)
        bo = mb.lattice.ext_to_box(eo.view(mb.ATOM_DTYPE), sc.cells, sc.ghost)
        live = bo["type"] >= 0
        assert rel_err(bg["rho"][live], bo["rho"][live]) < 1e-12
        assert rel_err(bg["df"][live], bo["df"][live]) < 1e-12
        assert rel_err(bg["f"][live], bo["f"][live]) < 1e-10
        created, released = C.c_int(), C.c_int()
        _call(shim.drive_atoms_mem, 10, 8, 6, C.byref(created), C.byref(released))
        assert created.value == 1 and released.value == 1
    finally:
        _call(shim.drive_env_clean)
