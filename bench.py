#!/usr/bin/env python
"""Benchmark of the MISA-MD EAM hot path on B200: atom-steps/s.

A "step" is one velocity-Verlet timestep of the whole lattice (rho/df pass, force
pass with the integration fused, interstitial passes), state resident in HBM.

Default workload (the scale configuration): BCC Fe 128^3 unit cells
(4,194,304 sites), 0.5% of sites vacated (seed 7), 200 interstitial atoms at random
octahedral sites (seed 7), 300 K, dt = 1 fs, plain FP64, synthetic analytic
potential tabulated at 5000 knots.  `--config mixed` runs the 200^3-cell mixed
precision configuration instead.

Multi-GPU: every rank advances its own independent replica (the path does not
shard; no collective on the data path): value = all ranks' atom-steps / max time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib.util
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
A0, MASS, RC, SKIN, DT = 2.855, 55.845, 5.6, 0.7, 1.0

# algorithmic figures per atom-step (device-resident SoA, stored force):
#   rho pass   reads x (24) + type (4), writes df (8)                        = 36 B
#   force pass reads x, type, df, v, f_old (84), writes x, v, f (72)         = 156 B
#   flops: 58 pairs x (20 rho + 50 force) + 30 per atom                      = 4090
BYTES_RHO, BYTES_FORCE = 36, 156
BYTES_MIXED_RHO, BYTES_MIXED_FORCE = 32, 128  # mixed: df and f stored as FP32
BYTES_MIXED = BYTES_MIXED_RHO + BYTES_MIXED_FORCE
FLOP_RHO, FLOP_FORCE = 58 * 20, 58 * 50 + 30

# velocity_seed: seed of the Maxwell-Boltzmann draw; seed: vacancies and interstitial
# sites.  oracle: the same workload's name in oracle/workload.py (the CPU reference arm
# builds it there, from the same seeds, without loading this package).
WORKLOADS = {
    "scale": dict(name="fe_bcc_128c_vac0.5pct_itl200_300K_fp64", cells=(128, 128, 128), temperature=300.0,
                  vacancy=0.005, n_itl=200, seed=7, velocity_seed=1007, precision="fp64", oracle="fe128"),
    "mixed": dict(name="fe_bcc_200c_vac0.5pct_itl763_900K_mixed", cells=(200, 200, 200), temperature=900.0,
                  vacancy=0.005, n_itl=763, seed=7, velocity_seed=1007, precision="mixed", oracle="fe200"),
    "scale_mixed": dict(name="fe_bcc_128c_vac0.5pct_itl200_300K_mixed", cells=(128, 128, 128), temperature=300.0,
                        vacancy=0.005, n_itl=200, seed=7, velocity_seed=1007, precision="mixed", oracle="fe128"),
    "small": dict(name="fe_bcc_20c_600K_fp64", cells=(20, 20, 20), temperature=600.0, vacancy=0.0, n_itl=0,
                  seed=42, velocity_seed=42, precision="fp64", oracle="fe20"),
}


def _package():
    if "misa_b200" in sys.modules:
        return sys.modules["misa_b200"]
    pkg_dir = ROOT / "misa-md-hip_b200"
    spec = importlib.util.spec_from_file_location("misa_b200", pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["misa_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def build_state(mb, wl: dict, cells=None):
    cells = cells or wl["cells"]
    box = mb.lattice.bcc_box(cells, A0)
    mb.lattice.add_vacancies(box, wl["vacancy"], wl["seed"])
    scale = (cells[0] * cells[1] * cells[2]) / float(np.prod(wl["cells"]))
    n_itl = int(round(wl["n_itl"] * scale))
    itl = mb.lattice.octahedral_interstitials(n_itl, cells, A0, wl["seed"])
    mb.lattice.maxwell_boltzmann(box, itl, wl["temperature"], MASS, wl["velocity_seed"])
    return box, itl


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
        except Exception:
            pass
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def ncu_l1tex(kernel: str) -> dict | None:
    """L1TEX data-stage throughput (% of peak) of `kernel` from the committed ncu summary:
    the on-chip resource the lattice passes are bound by (their DRAM traffic is at or below
    the algorithmic bytes)."""
    p = ROOT / "profiles" / "traffic.json"
    try:
        d = json.loads(p.read_text())[kernel]
        return {"frac": d["l1tex_throughput_pct"] / 100.0, "source": d["source"]}
    except Exception:
        return None


def ncu_traffic(kernel: str, n_atoms: int) -> float | None:
    """DRAM bytes per launch of `kernel` from the committed ncu summary, scaled from the
    profiled atom count to n_atoms (traffic grows in proportion to the lattice)."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())[kernel]
        return float(d["dram_bytes_per_launch"]) * n_atoms / float(d["atoms"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows: list[list[str]] = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return self

        def pump():
            for line in self.proc.stdout:
                self.rows.append([c.strip() for c in line.split(",")])

        self.thread = threading.Thread(target=pump, daemon=True)
        self.thread.start()
        return self

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 4 + k and r[4 + k].lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, value: float) -> float:
    if pg is None:
        return value
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def cpu_oracle_rate(wl: dict, warmup: int, steps: int, threads: int | None = None) -> dict:
    """Atom-steps/s of the CPU oracle (the reference's lattice EAM step restated in C,
    OpenMP over sites) on the whole workload: the lattice and its defects are built by
    oracle/workload.py from the workload's seeds, the forces at the start are computed
    (untimed), then `warmup` untimed and `steps` timed velocity-Verlet steps, each one
    rho / df / force evaluation of every atom.  Loads the oracle only, never this
    package."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as orc
    from oracle import workload as W
    if threads:
        orc.set_threads(threads)
    box, itl = W.config_state(wl["oracle"])
    run = W.OracleRun(box, itl, wl["cells"], reach=RC + SKIN)
    del box
    if warmup:
        run.steps(warmup)
    t0 = time.perf_counter()
    run.steps(steps)
    dt = time.perf_counter() - t0
    n_cells = "x".join(str(c) for c in wl["cells"])
    return {"value": run.n_atoms * steps / dt, "unit": "atom-steps/s", "cores": orc.num_threads(), "kind": "port",
            "sample": f"the whole workload ({n_cells} cells, {run.n_atoms} atoms): {warmup} untimed + {steps} "
                      f"timed steps of the C oracle, OpenMP over sites", "ms_per_step": dt / steps * 1e3}


def run_reference(args, wl) -> None:
    """The reference's CPU implementation of the path (the C oracle port: the
    reference's own CPU EAM path lives in the MISA-MD host, which is not available) on
    the same workload as the GPU arm, with every host thread: W untimed and K timed
    steps of the whole lattice.  Under torchrun only rank 0 runs it."""
    if "oracle" not in wl:
        print(json.dumps({"impl": "reference", "unavailable": "the CPU reference arm times the single-lattice "
                          "configurations (scale, small, mixed, scale_mixed)"}), flush=True)
        return
    cpu = cpu_oracle_rate(wl, args.warmup, args.steps, os.cpu_count())
    value = cpu["value"]
    line = {
        "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": cpu["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lattice, analytic tabulated potential)",
        "impl": "reference",
        "config": {"workload": wl["name"], "cells": list(wl["cells"])},
        "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def hooks_e2e(mb, wl, box, device: int, pairs: int = 5) -> dict:
    """rho + force through the drop-in hooks (mb_eam_rho_calc, mb_eam_force_calc) on the
    host's ghost-extended AoS array in page-locked memory, the calls a MISA-MD timestep
    makes; one rho + force pair counts as one step of the box's atoms."""
    cells = wl["cells"]
    ghost = mb.lattice.ghost_for_reach(A0, RC + SKIN)
    h = mb.Hooks(device)
    dom = mb.lattice.domain(cells, ghost)
    h.domain_init(dom)
    even, odd = mb.lattice.stencil_linear(A0, RC + SKIN, dom.ext_size_x, dom.ext_size_y)
    h.nei_offset_init(even, odd)
    h.pot_init(mb.potential.fe_analytic())
    ext0 = mb.lattice.box_to_ext(box, cells, ghost, A0)
    n = ext0.shape[0]
    p = C.c_void_p()
    alloc = C.c_int()
    mb.check(mb.lib().mb_create_atoms_mem(C.byref(p), 104, n, 1, 1, C.byref(alloc)))
    try:
        ext = np.ctypeslib.as_array((C.c_uint8 * (104 * n)).from_address(p.value)).view(mb.ATOM_DTYPE)
        ext[:] = ext0
        h.rho_calc(ext, RC)  # warm-up pair
        h.force_calc(ext, RC)
        t0 = time.perf_counter()
        for _ in range(pairs):
            h.rho_calc(ext, RC)
            h.force_calc(ext, RC)
        dt = time.perf_counter() - t0
        k_ms, c_ms = h.last_timing()
    finally:
        rel = C.c_int()
        mb.check(mb.lib().mb_release_atoms_mem(p, C.byref(rel)))
        mb.Hooks.clean()
    rows = ((dom.box_size_z - 1) * dom.ext_size_y + dom.box_size_y - 1) * dom.ext_size_x + dom.box_size_x
    atoms = int((box["type"] >= 0).sum())
    return {"value": atoms * pairs / dt, "unit": "atom-steps/s", "ms_per_pair": dt / pairs * 1e3, "pairs": pairs,
            "h2d_bytes_per_step": 2 * 104 * n, "d2h_bytes_per_step": 2 * 104 * rows,
            "slabs": int(mb.lib().mb_cli_batches()) if mb.lib().mb_cli_batches() > 1 else "automatic",
            "last_force_pass_ms": {"device_work_span": k_ms, "rest": c_ms},
            "api": "mb_eam_rho_calc + mb_eam_force_calc (host ghost-extended AoS array, page-locked)"}


def run_ours(args, mb, wl, world, rank, local, pg) -> None:
    mb.check(mb.lib().mb_env_init(local))
    precision = mb.MB_PREC_FP64 if wl["precision"] == "fp64" else mb.MB_PREC_MIXED
    box, itl = build_state(mb, wl)
    n_atoms = int((box["type"] >= 0).sum()) + itl.shape[0]
    sim = mb.Sim(wl["cells"], mb.potential.fe_analytic(), lattice_const=A0, mass=MASS, dt=DT, cutoff=RC,
                 stencil_skin=SKIN, precision=precision, max_interstitials=max(1, itl.shape[0]))
    sim.upload(box, itl)
    info = sim.info()
    if args.settle:
        # untimed steps from the fresh lattice to the thermally disordered state a run
        # spends its time in: at the fresh lattice all lanes of a warp read the same
        # spline knots, later they read random knots (shared-memory bank conflicts), and
        # the lattice passes take ~6% longer
        sim.run(args.settle)
    sim.run(max(args.warmup, 3))  # W >= 3 untimed warm-up steps (graph capture happens here)

    clocks = ClockSampler(local).start()
    barrier(pg)
    ms = sim.time_steps(args.steps)
    barrier(pg)
    clk = clocks.stop()
    ms = reduce_max(pg, ms)
    total_atom_steps = n_atoms * args.steps * world
    value = total_atom_steps / (ms * 1e-3)

    # per-kernel device time (CUDA events on the sim's stream, outside the timed region)
    rho_ms, force_ms = sim.kernel_times()
    peaks = measured_peaks()
    f64 = C.c_double()
    f32 = C.c_double()
    probe = C.CDLL(str(ROOT / "misa-md-hip_b200" / "libmb_probe.so"))
    if probe.mb_probe_fma_peaks(C.byref(f64), C.byref(f32)) != 0:
        raise RuntimeError("the FMA peak probe failed")
    if precision == mb.MB_PREC_FP64:
        kname, kbytes, kflops, kms = "k_force64 (force + velocity-Verlet)", BYTES_FORCE * n_atoms, FLOP_FORCE, force_ms
        fpeak, fname = f64.value, "fp64"
    elif rho_ms > 0:
        # split kernels (one large lattice): density pass, then force + integration
        kname, kbytes, kflops, kms = ("k_mx_force (mixed force + velocity-Verlet)", BYTES_MIXED_FORCE * n_atoms,
                                      FLOP_FORCE, force_ms)
        fpeak, fname = f32.value, "fp32"
    else:
        # one persistent launch holds the rho, force and integration phases
        kname, kbytes, kflops, kms = ("k_ens_step (rho + force + velocity-Verlet, one persistent launch)",
                                      BYTES_MIXED * n_atoms, FLOP_RHO + FLOP_FORCE, force_ms)
        fpeak, fname = f32.value, "fp32"
    achieved = kbytes / (kms * 1e-3) / 1e9
    traffic = ncu_traffic(kname.split()[0], n_atoms)
    roofline = {
        "kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
        "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
        "traffic": traffic, "algorithmic_bytes_per_launch": kbytes, "launch_ms": kms,
        fname: {"achieved_tflops": kflops * n_atoms / (kms * 1e-3) / 1e12, "peak_tflops": fpeak,
                "frac": kflops * n_atoms / (kms * 1e-3) / 1e12 / fpeak,
                "peak_source": "measured FMA-chain probe (libmb_probe.so)"},
        "fp64_peak_tflops": f64.value, "fp32_peak_tflops": f32.value,
        "l1tex": ncu_l1tex(kname.split()[0]),
    }
    if rho_ms > 0:
        rb = BYTES_RHO if precision == mb.MB_PREC_FP64 else BYTES_MIXED_RHO
        roofline["rho_kernel"] = {"kernel": "k_rho64" if precision == mb.MB_PREC_FP64 else "k_mx_rho",
                                  "launch_ms": rho_ms, "achieved_gbs": rb * n_atoms / (rho_ms * 1e-3) / 1e9,
                                  "achieved_tflops": FLOP_RHO * n_atoms / (rho_ms * 1e-3) / 1e12}

    # end to end through the public host-buffer entry point: every step uploads the
    # lattice records from pinned host memory and reads the updated records back
    e2e = hooks = None
    if precision == mb.MB_PREC_FP64:
        n_box = box.shape[0]
        p = C.c_void_p()
        alloc = C.c_int()
        mb.check(mb.lib().mb_create_atoms_mem(C.byref(p), 104, n_box, 1, 1, C.byref(alloc)))
        host = np.ctypeslib.as_array((C.c_uint8 * (104 * n_box)).from_address(p.value)).view(mb.ATOM_DTYPE)
        b2, i2 = sim.download()
        host[:] = b2
        k_e2e = max(3, min(args.steps, 20))
        sim.step_host(host, i2)  # warm-up
        barrier(pg)
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            sim.step_host(host, i2)
        e2e_s = time.perf_counter() - t0
        barrier(pg)
        e2e_s = reduce_max(pg, e2e_s)
        rel = C.c_int()
        mb.check(mb.lib().mb_release_atoms_mem(p, C.byref(rel)))
        e2e = {"value": n_atoms * k_e2e * world / e2e_s, "unit": "atom-steps/s",
               "h2d_bytes_per_step": 104 * (n_box + i2.shape[0]), "d2h_bytes_per_step": 104 * (n_box + i2.shape[0]),
               "steps": k_e2e, "api": "mb_sim_step_host (pinned host AoS records in, updated records out)"}
        if world == 1:
            try:
                hooks = hooks_e2e(mb, wl, b2, local)
            except Exception as e:  # an extra figure: reported, never fatal to the bench line
                hooks = {"error": str(e)[:300]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference arm's measurement (same lattice, same threads), with fewer steps
        c = cpu_oracle_rate(wl, 1, 4, os.cpu_count())
        cpu = {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")}
    mixed = None
    if precision == mb.MB_PREC_FP64 and not args.no_mixed:
        mixed = mixed_comparison(args, mb, wl, box, itl, n_atoms, value / world, pg)
    sim.close()
    n_itl = int(itl.shape[0])
    del box, itl
    # the batched-ensemble and serving configurations, measured in the same run
    ensemble = serving = None
    if world == 1 and not args.no_extras:
        try:
            ensemble = ensemble_measure(mb, args.steps, args.warmup)
        except Exception as e:  # an extra figure: reported, never fatal to the bench line
            ensemble = {"error": str(e)[:300]}
        try:
            serving = serve_measure(mb, args.serve_requests, max_seconds=args.serve_seconds)
        except Exception as e:
            serving = {"error": str(e)[:300]}
    if precision == mb.MB_PREC_FP64:
        launches_per_step = 6 if n_itl else 2  # itl clear, itl mark, rho, itl rho, force, itl force
    elif rho_ms > 0:  # split: itl clear, bin, mark, rho, itl rho, force, itl force, bookkeeping
        launches_per_step = 8 if n_itl else 3
    else:
        launches_per_step = 1
    if rank == 0:
        line = {
            "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if precision == mb.MB_PREC_FP64 else "f32+f64",
            "data": "synthetic (seeded lattice, analytic tabulated potential)",
            "config": {"workload": wl["name"], "cells": list(wl["cells"]), "atoms_per_gpu": n_atoms,
                       "stencil": info["n_stencil"], "replicas": world,
                       "l2": f"state {info['device_bytes'] / 1e6:.0f} MB per GPU > 126 MB L2 (no flush needed)",
                       "timed_state": f"after {args.settle} untimed settling steps from the fresh lattice"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches_per_step * args.steps,
            "clocks": clk,
        }
        if mixed is not None:
            line["mixed"] = mixed
        if hooks is not None:
            line["hooks"] = hooks
        if ensemble is not None:
            line["ensemble"] = ensemble
        if serving is not None:
            line["serve"] = serving
        print(json.dumps(line), flush=True)


def mixed_comparison(args, mb, wl, box, itl, n_atoms, fp64_rate, pg) -> dict:
    """Mixed precision on the same lattice: atom-steps/s, speed-up over the plain FP64
    path and the relative force RMS error against the FP64 forces at the same state
    (the workload after 100 FP64 steps, so that the lattice is thermally disordered)."""
    t = mb.potential.fe_analytic()
    with mb.Sim(wl["cells"], t, lattice_const=A0, mass=MASS, dt=DT, cutoff=RC, stencil_skin=SKIN,
                precision=mb.MB_PREC_FP64, max_interstitials=max(1, itl.shape[0])) as s:
        s.upload(box, itl)
        s.run(100)
        tbox, titl = s.download()
    forces = {}
    for prec in (mb.MB_PREC_FP64, mb.MB_PREC_MIXED):
        with mb.Sim(wl["cells"], t, lattice_const=A0, mass=MASS, dt=DT, cutoff=RC, stencil_skin=SKIN, precision=prec,
                    max_interstitials=max(1, itl.shape[0])) as s:
            s.upload(tbox, titl)
            s.run(0)
            b, i = s.download()
            forces[prec] = np.concatenate([b["f"][b["type"] >= 0], i["f"]])
    f64, f32 = forces[mb.MB_PREC_FP64], forces[mb.MB_PREC_MIXED]
    err = float(np.sqrt(np.sum((f32 - f64) ** 2) / np.sum(f64 ** 2)))
    with mb.Sim(wl["cells"], t, lattice_const=A0, mass=MASS, dt=DT, cutoff=RC, stencil_skin=SKIN,
                precision=mb.MB_PREC_MIXED, max_interstitials=max(1, itl.shape[0])) as s:
        if args.settle:
            s.upload(tbox, titl)  # timed in the same thermally disordered state as the FP64 path
        else:
            s.upload(box, itl)
        s.run(max(args.warmup, 3))
        barrier(pg)
        ms = s.time_steps(args.steps)
        barrier(pg)
        ms = reduce_max(pg, ms)
        rho_ms, force_ms = s.kernel_times()
    rate = n_atoms * args.steps / (ms * 1e-3)
    if rho_ms > 0:
        kern = {"kernels": "k_mx_rho, k_mx_force (+ interstitial and bookkeeping kernels), one CUDA graph per step",
                "rho_ms": rho_ms, "force_ms": force_ms}
    else:
        kern = {"kernels": "k_ens_step (one persistent launch per step)", "step_ms": force_ms}
    return {"value": rate * (int(os.environ.get("WORLD_SIZE", "1"))), "unit": "atom-steps/s",
            "ms_per_step": ms / args.steps, "speedup_vs_fp64": rate / fp64_rate,
            "force_rms_rel_err_vs_fp64": err, "force_err_state": "workload after 100 FP64 steps",
            "timed_state": "workload after 100 FP64 steps" if args.settle else "fresh workload",
            "dtype": "f32 pairs + two-sum, f64 state", **kern}


def run_nve(args, mb, world, rank, local, pg) -> None:
    """The mixed-precision NVE run of the 200^3-cell workload (16 M atoms, 900 K, 0.5%
    vacancies, 763 interstitials): --nve-equil + --nve-steps steps with the total energy
    recorded and the relative force RMS error against the FP64 path checked every
    --check-every steps.  At each check the mixed state (positions, velocities, mixed
    forces at those positions) is read back and the FP64 path evaluates the forces at the
    same positions; the FP64 path matches the CPU oracle to ~1e-15
    (tests/test_gpu_parity.py).  Atoms that leave their lattice site move to the
    interstitial list and back (mb_sim_set_conversion, on unless --no-conversion; 1.0 A
    and 0.5 A by default: thermal excursions at 900 K reach ~0.7 A with this potential,
    while an atom hopping to a neighbouring vacancy passes 1.24 A from its site).
    Energy drift is reported over the --nve-steps production steps after the
    equilibration (E(t) - E(t_eq)) / N in eV/atom, plus the offset from step 0: a run
    started from a perfect lattice moves about 1e-5 eV/atom within its first few hundred
    steps while kinetic and potential energy equilibrate (the O(dt^2) velocity-Verlet
    energy error, the same in the FP64 path)."""
    mb.check(mb.lib().mb_env_init(local))
    wl = dict(WORKLOADS["mixed"])
    if args.nve_itl is not None:  # interstitial count override (0: vacancies only)
        wl["n_itl"] = args.nve_itl
        wl["name"] = wl["name"].replace("itl763", f"itl{args.nve_itl}")
    if args.nve_precision == "fp64":
        wl["name"] = wl["name"].replace("mixed", "fp64")
    box, itl = build_state(mb, wl)
    n_atoms = int((box["type"] >= 0).sum()) + itl.shape[0]
    tables = mb.potential.fe_analytic()
    conversion = not args.no_conversion
    cap = itl.shape[0] + (4096 if conversion else 0)
    kw = dict(lattice_const=A0, mass=MASS, dt=DT, cutoff=RC, stencil_skin=args.nve_skin,
              max_interstitials=max(1, cap))
    every = max(1, args.check_every)
    total = args.nve_equil + args.nve_steps
    prec = mb.MB_PREC_FP64 if args.nve_precision == "fp64" else mb.MB_PREC_MIXED
    mixed = mb.Sim(wl["cells"], tables, precision=prec, **kw)
    # the checks evaluate both paths on the read-back state (same positions, same
    # lattice / interstitial membership): a fresh probe of the run's precision and the
    # FP64 reference, neither doing bookkeeping
    probe = mb.Sim(wl["cells"], tables, precision=prec, **kw)
    ref = mb.Sim(wl["cells"], tables, precision=mb.MB_PREC_FP64, **kw)
    mixed.upload(box, itl)
    if conversion:
        mixed.set_conversion(args.conv_distance, args.rec_distance)
    del box, itl
    steps_done, rms, rms_steps, e_rec = 0, [], [], []
    t_md = 0.0
    mixed.run(0, energy_every=every)  # priming pass: forces and the step-0 energies
    e_rec.append(mixed.energies())  # each run() keeps only its own energy samples
    clocks = ClockSampler(local).start()
    while True:
        b, i = mixed.download()
        live = b["type"] >= 0
        probe.upload(b, i)
        probe.run(0)
        pb, pi = probe.download()
        f32 = np.concatenate([pb["f"][live], pi["f"]])
        ref.upload(b, i)
        ref.run(0)
        rb, ri = ref.download()
        f64 = np.concatenate([rb["f"][live], ri["f"]])
        rms.append(float(np.sqrt(np.sum((f32 - f64) ** 2) / np.sum(f64 ** 2))))
        rms_steps.append(steps_done)
        del b, i, pb, pi, rb, ri, f32, f64, live
        if steps_done >= total:
            break
        n = min(every, total - steps_done)
        t0 = time.perf_counter()
        mixed.run(n, energy_every=every)
        t_md += time.perf_counter() - t0
        steps_done += n
        e_rec.append(mixed.energies())
    clk = clocks.stop()
    e = np.concatenate([x for x in e_rec if x.size], axis=0)
    conv = mixed.conversion_stats() if conversion else None
    mixed.close()
    probe.close()
    ref.close()
    etot = e[:, 1] + e[:, 2]
    e0 = float(etot[0])
    drift = (etot - e0) / n_atoms
    prod = e[:, 0] >= args.nve_equil
    eq = float(etot[prod][0]) if prod.any() else e0
    drift_prod = (etot[prod] - eq) / n_atoms if prod.any() else np.zeros(1)
    slope = float(np.polyfit(e[prod, 0], etot[prod] / n_atoms, 1)[0]) if prod.sum() > 2 else 0.0
    if rank == 0:
        print(json.dumps({
            "metric": "atom-steps/s", "value": n_atoms * steps_done * world / t_md, "unit": "atom-steps/s",
            "n_gpus": world, "steps": steps_done, "warmup": 0, "ms_per_step": t_md * 1e3 / max(1, steps_done),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == mb.MB_PREC_FP64 else "f32+f64",
            "data": "synthetic (seeded lattice, analytic tabulated potential)",
            "config": {"workload": wl["name"] + "_nve", "cells": list(wl["cells"]), "atoms_per_gpu": n_atoms,
                       "stencil_skin": args.nve_skin, "convert_distance": args.conv_distance if conversion else None,
                       "recombine_distance": args.rec_distance if conversion else None,
                       "check_every": every, "timing": "wall clock of the MD segments (energy steps included)"},
            "force_rms_rel_err_vs_fp64": {"max": max(rms), "mean": float(np.mean(rms)), "final": rms[-1],
                                          "steps": rms_steps, "values": rms},
            "energy_drift_ev_per_atom": {
                "production_steps": args.nve_steps, "equilibration_steps": args.nve_equil,
                "production_max_abs": float(np.max(np.abs(drift_prod))), "production_final": float(drift_prod[-1]),
                "production_fit_slope_x_steps": slope * args.nve_steps,
                "offset_from_step0_max_abs": float(np.max(np.abs(drift))), "final_from_step0": float(drift[-1]),
                "steps": e[:, 0].astype(int).tolist(), "values_from_step0": drift.tolist()},
            "conversion": conv,
            "bars": {"force_rms": 1e-6, "drift": 1e-5}, "clocks": clk, "cpu_baseline": None, "e2e": None,
            "gpu_launches": None}), flush=True)


ENSEMBLE_DESC = ("512 independent periodic BCC Fe lattices, edges uniform in [8, 40] cells (seed 11), "
                 "300-1200 K, 0-1% vacancies, mixed precision, every lattice advanced by the same launches "
                 "of each step (one CUDA graph per step)")


def ensemble_measure(mb, steps: int, warmup: int, pg=None, autotune: bool = True, clocks_device=None) -> dict:
    """The batched ensemble: 512 lattices with edges uniform in [8, 40] cells (seed 11),
    temperature uniform in [300, 1200] K, 0-1% vacancies, mixed precision.  The
    autotuner picks between the split kernels and the tile policies of the persistent
    kernel; `steps` launches are timed with CUDA events (max over ranks)."""
    rng = np.random.default_rng(11)
    n_lat = 512
    edges = rng.integers(8, 41, size=(n_lat, 3))
    temps = rng.uniform(300.0, 1200.0, size=n_lat)
    vacs = rng.uniform(0.0, 0.01, size=n_lat)
    ens = mb.Ensemble(mb.potential.fe_analytic(), lattice_const=A0, mass=MASS, dt=DT, cutoff=RC, stencil_skin=SKIN)
    n_atoms = 0
    for k in range(n_lat):
        cells = tuple(int(e) for e in edges[k])
        box = mb.lattice.bcc_box(cells, A0)
        mb.lattice.add_vacancies(box, float(vacs[k]), 1000 + k)
        mb.lattice.maxwell_boltzmann(box, None, float(temps[k]), MASS, 5000 + k)
        ens.add(cells, box, steps=0)
        n_atoms += int((box["type"] >= 0).sum())
    policy, tune_ms = ens.autotune(5) if autotune else (None, None)
    ens.run(max(warmup, 3))
    clocks = ClockSampler(clocks_device).start() if clocks_device is not None else None
    barrier(pg)
    ms = ens.time(steps)
    barrier(pg)
    clk = clocks.stop() if clocks else None
    ms = reduce_max(pg, ms)
    rho_ms, force_ms, kernels = ens.kernel_times()
    info = ens.info()
    ens.close()
    peaks = measured_peaks()
    split = rho_ms > 0
    if split:
        kname, kbytes, kms = "k_mx_force (mixed force + velocity-Verlet, every lattice)", BYTES_MIXED_FORCE, force_ms
    else:
        kname, kbytes, kms = "k_ens_step (one persistent launch)", BYTES_MIXED, force_ms
    achieved = kbytes * n_atoms / (kms * 1e-3) / 1e9
    roofline = {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                "traffic": ncu_traffic(kname.split()[0] + "_ensemble", n_atoms), "launch_ms": kms,
                "algorithmic_bytes_per_launch": kbytes * n_atoms}
    if split:
        roofline["rho_kernel"] = {"kernel": "k_mx_rho", "launch_ms": rho_ms,
                                  "achieved_gbs": BYTES_MIXED_RHO * n_atoms / (rho_ms * 1e-3) / 1e9}
    return {"value": n_atoms * steps / (ms * 1e-3), "unit": "atom-steps/s", "ms_per_step": ms / steps,
            "steps": steps, "lattices": n_lat, "atoms": n_atoms, "roofline": roofline, "gpu_launches": kernels * steps,
            "kernels": "split (k_mx_rho, k_mx_force, linear item walk)" if split else
            f"persistent k_ens_step, tile policy {policy}",
            "autotune_best_ms_5_steps": tune_ms, "clocks": clk,
            "l2": f"state {info['device_bytes'] / 1e6:.0f} MB > 126 MB L2 (no flush needed)",
            "dtype": "f32 pairs + two-sum, f64 state", "workload": ENSEMBLE_DESC}


def run_ensemble(args, mb, world, rank, local, pg) -> None:
    mb.check(mb.lib().mb_env_init(local))
    e = ensemble_measure(mb, args.steps, args.warmup, pg, clocks_device=local)
    if rank == 0:
        print(json.dumps({
            "metric": "atom-steps/s", "value": e["value"] * world, "unit": "atom-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": e["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded lattices)",
            "config": {"workload": "ensemble_512_lattices_8to40c_mixed", "lattices": e["lattices"],
                       "atoms_per_gpu": e["atoms"], "kernels": e["kernels"],
                       "autotune_best_ms_5_steps": e["autotune_best_ms_5_steps"], "l2": e["l2"]},
            "roofline": e["roofline"], "gpu_launches": e["gpu_launches"], "clocks": e["clocks"],
            "cpu_baseline": None, "e2e": None}), flush=True)


def serve_measure(mb, n_requests: int, max_seconds: float = 600.0, clocks_device=None) -> dict:
    """Continuous-batching serving of a Poisson request stream (50 req/s, seed 13; atoms
    log-uniform in [1e3, 2e6], steps uniform in [100, 5000], 300-1200 K, 0-1% vacancies)
    under a 160 GB HBM admission budget: the first n_requests requests, arriving on the
    wall clock, each lattice built on a worker thread and uploaded when memory allows."""
    from misa_b200 import serve
    reqs = serve.poisson_stream(n_requests, rate=50.0, seed=13)
    srv = serve.Server(hbm_budget_bytes=160 << 30, chunk=50)
    clocks = ClockSampler(clocks_device).start() if clocks_device is not None else None
    stats = srv.serve(reqs, realtime=True, max_seconds=max_seconds)
    clk = clocks.stop() if clocks else None
    srv.close()
    return {"value": stats["atom_steps_per_s"], "unit": "atom-steps/s", "requests": n_requests,
            "completed": stats["completed"], "rejected": stats["rejected"], "unfinished": stats["unfinished"],
            "latency_p50_s": stats["latency_p50_s"], "latency_p99_s": stats["latency_p99_s"],
            "makespan_s": stats["makespan_s"], "admit_stall_s": stats["admit_stall_s"],
            "gpu_launches": stats["launches"], "clocks": clk, "dtype": "f32 pairs + two-sum, f64 state",
            "admission": {"order": srv.order, "batch_atoms": srv.batch_atoms},
            "workload": "Poisson 50 req/s (seed 13), atoms log-uniform [1e3, 2e6], steps uniform [100, 5000], "
                        "300-1200 K, 0-1% vacancies, 160 GB HBM budget, continuous batching, shortest remaining "
                        "work admitted first under a batch target of sites in flight"}


def run_serve(args, mb, world, rank, local, pg) -> None:
    mb.check(mb.lib().mb_env_init(local))
    sv = serve_measure(mb, args.requests, clocks_device=local)
    if rank == 0:
        print(json.dumps({
            "metric": "atom-steps/s", "value": sv["value"] * world, "unit": "atom-steps/s",
            "n_gpus": world, "steps": sv["gpu_launches"], "warmup": 0, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic request stream",
            "config": {"workload": "serve_poisson50_seed13", "requests": args.requests,
                       "completed": sv["completed"], "rejected": sv["rejected"]},
            "latency_p50_s": sv["latency_p50_s"], "latency_p99_s": sv["latency_p99_s"],
            "makespan_s": sv["makespan_s"], "admit_stall_s": sv["admit_stall_s"], "admission": sv["admission"],
            "gpu_launches": sv["gpu_launches"], "clocks": sv["clocks"], "cpu_baseline": None, "e2e": None}),
              flush=True)


def run_decomp(args, mb, world, rank, local, pg) -> None:
    """One 128^3-cell lattice (0.5% vacancies, seed 7, 300 K; no interstitials: slabs hold
    none) split into z-slabs over the N ranks (strong scaling): every step exchanges the
    ghost layers of positions and of df with the neighbouring ranks (NCCL point-to-point
    on device buffers, misa_b200.decomp) around the rho and force phases.  Timed on the
    wall clock between synchronised points (exchanges and their host synchronisations
    included), max over ranks."""
    import torch

    from misa_b200 import decomp
    mb.check(mb.lib().mb_env_init(local))
    wl = dict(WORKLOADS["scale"], n_itl=0)
    box, _ = build_state(mb, wl)
    n_atoms = int((box["type"] >= 0).sum())
    dev = torch.device("cuda", local) if torch.cuda.is_available() else None
    bufs = lambda n: torch.empty(n, dtype=torch.uint8, device=dev)  # noqa: E731
    r = decomp.SlabRank(wl["cells"], mb.potential.fe_analytic(), rank, world, bufs, lattice_const=A0, mass=MASS,
                        dt=DT, cutoff=RC, stencil_skin=SKIN)
    ex = decomp.TorchExchange(pg, rank, world) if world > 1 else None
    sync = torch.cuda.synchronize if dev is not None else None
    try:
        r.upload(box)
        decomp.exchange_codes([r], ex, sync)
        for _ in range(max(args.warmup, 3)):
            decomp.step_all([r], ex, sync=sync)
        r.sim.sync()
        clocks = ClockSampler(local).start()
        barrier(pg)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            decomp.step_all([r], ex, sync=sync)
        r.sim.sync()
        dt = time.perf_counter() - t0
        barrier(pg)
        clk = clocks.stop()
    finally:
        r.close()
    dt = reduce_max(pg, dt)
    if rank == 0:
        print(json.dumps({
            "metric": "atom-steps/s", "value": n_atoms * args.steps / dt, "unit": "atom-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded lattice, analytic tabulated potential)",
            "config": {"workload": "fe_bcc_128c_vac0.5pct_300K_fp64_zslabs", "cells": list(wl["cells"]),
                       "atoms": n_atoms, "slabs": r.parts,
                       "timing": "wall clock between synchronised points, ghost-layer exchanges included"},
            # rho and force per step, plus 4 halo packs and 4 unpacks when the slabs exchange
            "gpu_launches": (2 + (8 if world > 1 else 0)) * args.steps, "clocks": clk, "cpu_baseline": None,
            "e2e": None}), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(WORKLOADS) + ["ensemble", "serve", "nve", "decomp"], default="scale")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--settle", type=int, default=100,
                    help="untimed steps before the warm-up, so that the lattice is timed thermally disordered "
                         "(0: time from the fresh lattice)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision comparison")
    ap.add_argument("--requests", type=int, default=64, help="requests served by --config serve")
    ap.add_argument("--no-extras", action="store_true",
                    help="default line without the ensemble and serve objects")
    ap.add_argument("--serve-requests", type=int, default=64, help="requests of the default line's serve object")
    ap.add_argument("--serve-seconds", type=float, default=90.0,
                    help="wall-time cap of the default line's serve object")
    ap.add_argument("--nve-steps", type=int, default=10000, help="steps of --config nve")
    ap.add_argument("--check-every", type=int, default=100, help="force / energy check interval of --config nve")
    ap.add_argument("--nve-precision", choices=["mixed", "fp64"], default="mixed", help="path run by --config nve")
    ap.add_argument("--nve-itl", type=int, default=None, help="interstitials of --config nve (default 763)")
    ap.add_argument("--nve-equil", type=int, default=1000, help="equilibration steps before the drift window")
    ap.add_argument("--no-conversion", action="store_true", help="--config nve without lattice <-> interstitial moves")
    ap.add_argument("--conv-distance", type=float, default=1.0,
                    help="--config nve: an atom this far (A) from its site joins the interstitial list")
    ap.add_argument("--nve-skin", type=float, default=1.3,
                    help="--config nve: stencil skin (A); at 900 K thermal excursions reach ~0.7 A with this "
                         "potential, so the stencil must cover twice that (1.3 A: every site closer than 6.9 A, "
                         "complete up to 1.39 A of combined displacement)")
    ap.add_argument("--rec-distance", type=float, default=0.5,
                    help="--config nve: an interstitial this close (A) to a vacant site takes it")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    wl = WORKLOADS.get(args.config, {"name": args.config})
    if args.impl == "reference":
        # CPU only: no process group, no GPU, no product library; rank 0 alone measures
        if int(os.environ.get("RANK", "0")) == 0:
            run_reference(args, wl)
        return
    world, rank, local, pg = dist_setup()
    mb = _package()
    try:
        if args.config == "ensemble":
            run_ensemble(args, mb, world, rank, local, pg)
        elif args.config == "serve":
            run_serve(args, mb, world, rank, local, pg)
        elif args.config == "nve":
            run_nve(args, mb, world, rank, local, pg)
        elif args.config == "decomp":
            run_decomp(args, mb, world, rank, local, pg)
        else:
            run_ours(args, mb, wl, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
