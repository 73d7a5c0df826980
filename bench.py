"""Benchmark of the multislice hot path: slice-steps/s at 1024^2.

Workload (the 1-GPU configuration of the metric): amorphous carbon slab
50 x 50 x 200 A, Z = 6 atoms placed uniformly at random at 0.1 atoms/A^3
(~50,000 atoms, minimum separation 1.2 A, seeded), 1024 x 1024 FP32-complex
grid, 100 slices of 2 A, 300 kV, conventional (3D-integrated) potential.
Synthetic seeded input stands in for a structure file.

One bench step = one pass of the slice stack: 100 slice steps
psi <- IFFT(P * FFT(exp(i sigma V) * psi)) over the device-resident potential
stack (400 MB, larger than L2, so every step streams its V from HBM).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  `value` is device time (CUDA events on the
engine's stream) of K steps, max over ranks; `e2e` times the same metric
through the C ABI with host buffers: atoms in, binning, potential build,
the 100 slices, exit wave out.  Multi-GPU runs are independent replicas
(weak scaling): a single specimen does not shard, frozen-phonon passes and
probe positions do.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GRID = 1024
SLICE_DZ = 2.0
KV = 300.0
CS = 1.2e7
SIZE = (50.0, 50.0, 200.0)
METRIC = "slice-steps/s @1024^2 (conventional multislice, fused path)"
UNIT = "slice-steps/s"
BYTES_PER_PX_STEP = 20  # read+write psi (complex64) + read V (float)


def workload(size=SIZE):
    from cudamultislice_b200 import structures as S

    Z, x, y, z = S.amorphous_carbon(size, density=0.1, min_sep=1.2)
    return Z, x, y, z


FORCED_PLAN = -1  # profiling: FFT plan variant forced on every leg's engine (-1: autotuned)


def new_sim(device: int):
    from cudamultislice_b200 import ManagedMultisliceSimulation

    sim = ManagedMultisliceSimulation(device=device)
    if FORCED_PLAN >= 0:
        sim.SetFFTPlan(FORCED_PLAN)
    return sim


def configure(sim, atoms, fparams, grid=GRID):
    Z, x, y, z = atoms
    sim.SetAtoms(Z, x, y, z)
    sim.UploadBinnedAtoms()
    sim.GetParameterisation(fparams)
    sim.ApplyMicroscopeParameters(KV, 0.0, 0.0, 0.0, CS, 0.1, 30.0, 20.0)
    # pixel 0 at the structure's corner: offset = the 2 A box padding
    ps = SIZE[0] / grid
    sim.SetCalculationVariables(ps, 0.0, grid, grid, sim.GetSizeX(), sim.GetSizeY(), sim.GetSizeZ(), 2.0, 2.0)
    sim.PreCalculateFrequencies()
    sim.InitialiseWavefunctions(SLICE_DZ)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [q.strip() for q in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def allreduce_max(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def stem_leg(fparams, device: int, nprobes: int = 256, batch: int = 0) -> dict:
    """STEM probes/s on the GaN [11-20] HAADF configuration: 10 x 6 x 40
    orthohexagonal cells (19,200 atoms), 1024^2 grid, 1.5945 A slices, 300 kV,
    25 mrad, Cs = 0, df = 0, annular detector 70-200 mrad; a subset of the
    128 x 128 raster, probes batched through the fused passes.  A probe is one
    position through all slices, including probe generation and detection."""
    import numpy as np

    from cudamultislice_b200 import structures as S

    Z, x, y, z = S.gan_wurtzite_11_20(10, 6, 40)
    sim = new_sim(device)
    sim.SetAtoms(Z, x, y, z)
    sim.UploadBinnedAtoms()
    sim.GetParameterisation(fparams)
    sim.ApplyMicroscopeParameters(300.0, 0.0, 0.0, 0.0, 0.0, 0.1, 30.0, 25.0)
    ps = float(sim.GetSizeX()) / GRID
    sim.STEMSetCalculationVariables(ps, 0.0, GRID, GRID, sim.GetSizeX(), sim.GetSizeY(), sim.GetSizeZ())
    sim.PreCalculateFrequencies()
    sim.InitialiseWavefunctions(1.5945)
    nsl = sim.BuildPotentialStack()
    # probe positions: a 128 x 128 raster over the cell area, first `nprobes`
    gx = np.linspace(0, GRID - 1, 128).astype(np.int32)
    px, py = np.meshgrid(gx, gx)
    px, py = px.ravel()[:nprobes], py.ravel()[:nprobes]
    out = {}
    for name, path, n in (("fused", 0, nprobes), ("plain", 1, max(nprobes // 16, 8))):
        sim.SetSlicePath(path)
        sim.StemRaster(px[:64], py[:64], 70.0, 200.0, batch=batch)  # warm-up / tuning
        t0 = time.perf_counter()
        sig = sim.StemRaster(px[:n], py[:n], 70.0, 200.0, batch=batch)
        dt = time.perf_counter() - t0
        out[name] = {"probes_per_s": n / dt, "probes": int(n), "slices": int(nsl)}
        if name == "fused":
            out["signal_mean"] = float(np.mean(sig))
            tb, tl = sim.RasterTuning()
            out["tuned"] = {"probes_per_launch": tb, "slices_in": "batched persistent loop" if tl else "per-pass kernels"}
    sim.close()
    step_s = 1.0 / (out["fused"]["probes_per_s"] * nsl)
    algo = 32 * GRID * GRID  # per probe-slice step: psi r/w in both passes (t shared, L2)
    peak, peak_kind = measured_peaks()
    return {"value": out["fused"]["probes_per_s"], "unit": "probes/s",
            "slice_steps_per_s": out["fused"]["probes_per_s"] * nsl,
            "roofline": {"bound": "hbm", "achieved": algo / step_s / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": algo / step_s / 1e9 / peak, "peak_source": peak_kind,
                         "algorithmic_bytes": "32 B per pixel per probe-slice step (wave read and written by "
                                              "the row and the column pass; the shared transmission is an L2 hit)"},
            "plain_value": out["plain"]["probes_per_s"],
            "speedup_fused_vs_plain": out["fused"]["probes_per_s"] / out["plain"]["probes_per_s"],
            "tuned": out["fused"].get("tuned"),
            "config": f"GaN [11-20] 10x6x40 cells ({len(Z)} atoms), {GRID}^2, {nsl} slices of 1.5945 A, 300 kV, "
                      f"25 mrad, HAADF 70-200 mrad, {nprobes} probes of the 128x128 raster, "
                      f"batch {'tuned on the device' if batch <= 0 else batch}",
            "timing": "host clock around ms_stem_raster (synchronous), potential stack resident"}


def mixed_leg(fparams, device: int, n1024: int = 256, n512: int = 256, batch: int = 64) -> dict:
    """The mixed-grid STEM configuration: GaN [11-20] 10 x 6 x 40 cells on
    1024^2 together with the same crystal cropped to 5 x 3 x 40 cells on 512^2
    (1.5945 A slices, 300 kV, 25 mrad, HAADF 70-200 mrad), `n1024` probes of
    the 128 x 128 raster and `n512` of the 64 x 64 raster, run as two concurrent
    branches of one CUDA graph (ms_stem_raster_concurrent) against the same two
    rasters one after the other.  Device time."""
    import numpy as np

    from cudamultislice_b200 import stem_raster_concurrent
    from cudamultislice_b200 import structures as S

    sims, pos = [], []
    for cells, grid, nr, npr in (((10, 6, 40), 1024, 128, n1024), ((5, 3, 40), 512, 64, n512)):
        Z, x, y, z = S.gan_wurtzite_11_20(*cells)
        sim = new_sim(device)
        sim.SetAtoms(Z, x, y, z)
        sim.UploadBinnedAtoms()
        sim.GetParameterisation(fparams)
        sim.ApplyMicroscopeParameters(300.0, 0.0, 0.0, 0.0, 0.0, 0.1, 30.0, 25.0)
        ps = float(sim.GetSizeX()) / grid
        sim.STEMSetCalculationVariables(ps, 0.0, grid, grid, sim.GetSizeX(), sim.GetSizeY(), sim.GetSizeZ())
        sim.PreCalculateFrequencies()
        sim.InitialiseWavefunctions(1.5945)
        sim.BuildPotentialStack()
        g = np.linspace(0, grid - 1, nr).astype(np.int32)
        px, py = np.meshgrid(g, g)
        pos.append((px.ravel()[:npr], py.ravel()[:npr]))
        sims.append(sim)
    nprobes = n1024 + n512
    res = {}
    for b in (0, 16, batch):  # 0: each handle's tuned batch (and loop or per-pass choice)
        stem_raster_concurrent(sims, [(p[0][:max(b, 16)], p[1][:max(b, 16)]) for p in pos], 70.0, 200.0, b)  # warm-up
        _, ms_conc = stem_raster_concurrent(sims, pos, 70.0, 200.0, b)
        ms_seq = 0.0
        for sim, p in zip(sims, pos):
            _, ms1 = stem_raster_concurrent([sim], [p], 70.0, 200.0, b)
            ms_seq += ms1
        res[b] = (nprobes / (ms_conc / 1000.0), nprobes / (ms_seq / 1000.0))
    for sim in sims:
        sim.close()
    best = max(max(v) for v in res.values())
    return {"value": best, "unit": "probes/s",
            "by_batch": {("tuned" if b == 0 else str(b)): {"together": c, "sequential": q,
                                                            "together_over_sequential": c / q}
                         for b, (c, q) in res.items()},
            "together": "two handles on supported grids with equal slice counts and the batched loop: one persistent "
                        "cooperative launch per round over both rasters; otherwise concurrent CUDA-graph branches",
            "config": f"GaN [11-20]: 10x6x40 cells on 1024^2 ({n1024} probes) + 5x3x40 cells on 512^2 "
                      f"({n512} probes), 1.5945 A slices, 300 kV, 25 mrad, HAADF 70-200 mrad",
            "timing": "device time of one CUDA-graph launch: both rasters as concurrent branches, or one after "
                      "the other; value = the faster arrangement"}


def c1_leg(fparams, device: int, reps: int = 20) -> dict:
    """The reference's own small case: SrTiO3 4 x 4 x 20 cells (1,600 atoms),
    256^2 over 15.62 A, 40 slices of 1.9525 A, 200 kV, exit wave.  The fused
    slice loop is one CUDA-graph launch (ms_run_conventional); the plain path
    runs the reference's launch sequence.  Device time of the slice loop,
    potential stack resident."""
    from cudamultislice_b200 import structures as S

    n = 256
    Z, x, y, z = S.srtio3(4, 4, 20)
    sim = new_sim(device)
    sim.SetAtoms(Z, x, y, z)
    sim.UploadBinnedAtoms()
    sim.GetParameterisation(fparams)
    sim.ApplyMicroscopeParameters(200.0, -500.0, 0.0, 0.0, 1.0e7, 0.1, 30.0, 20.0)
    sim.SetCalculationVariables(3.905 * 4 / n, -500.0, n, n, sim.GetSizeX(), sim.GetSizeY(), sim.GetSizeZ(),
                                2.0, 2.0)
    sim.PreCalculateFrequencies()
    sim.InitialiseWavefunctions(1.9525)
    out = {}
    for name, path in (("fused", 0), ("plain", 1)):
        sim.SetSlicePath(path)
        nsl = sim.RunConventional()
        best = None
        for _ in range(reps):
            sim.RunConventional()
            t = sim.LastDeviceMs()
            best = t if best is None else min(best, t)
        out[name] = nsl / (best / 1000.0)
    sim.close()
    return {"value": out["fused"], "unit": "slice-steps/s", "plain_value": out["plain"],
            "speedup_fused_vs_plain": out["fused"] / out["plain"],
            "config": f"SrTiO3 4x4x20 cells (1600 atoms), {n}^2, {nsl} slices of 1.9525 A, 200 kV",
            "timing": "device time of the slice loop (best of 20; fused: one CUDA-graph launch)"}


def grid4096_leg(fparams, device: int, steps_per: int = 20, reps: int = 3) -> dict:
    """The bench workload's specimen (a-C 50 x 50 x 200 A, 300 kV) sampled on
    4096^2 (0.0122 A pixels): the conventional slice loop over the resident
    potential stack (100 slices, 6.7 GB), fused passes against the plain path
    (cuFFT + one kernel per operation).  Device time, inputs far above L2."""

    n = 4096
    sim = new_sim(device)
    configure(sim, workload(), fparams, grid=n)
    nsl = sim.BuildPotentialStack()
    out = {}
    for name, path in (("fused", 0), ("plain", 1)):
        sim.SetSlicePath(path)
        sim.TimeSlices(steps_per, 1, breakdown=False)
        ms, _, _ = sim.TimeSlices(steps_per, reps, breakdown=False)
        out[name] = steps_per * reps / (ms / 1000.0)
    sim.SetSlicePath(0)
    _, row_ms, col_ms = sim.TimeSlices(steps_per, 1, breakdown=True)
    fft_plan = sim.FFTPlan(1)
    sim.close()
    peak, peak_kind = measured_peaks()
    step_gbs = BYTES_PER_PX_STEP * n * n * out["fused"] / 1e9
    return {"value": out["fused"], "unit": "slice-steps/s", "plain_value": out["plain"],
            "speedup_fused_vs_plain": out["fused"] / out["plain"],
            "row_pass_ms": row_ms, "col_pass_ms": col_ms,
            "row_pass_gbs": 20 * n * n / (row_ms / 1000.0) / 1e9, "col_pass_gbs": 16 * n * n / (col_ms / 1000.0) / 1e9,
            "step_achieved_gbs": step_gbs, "step_frac": step_gbs / peak, "peak_source": peak_kind,
            "fft_plan": {"row_variant": fft_plan[0], "col_variant": fft_plan[1]},
            "config": f"a-C 50x50x200 A, {n}^2, {nsl} slices of {SLICE_DZ} A, {KV:g} kV, potential stack resident",
            "timing": f"device time, {reps} x {steps_per} slices after one untimed pass per path"}


def grid4096_profile_leg(fparams, device: int, reps: int = 4) -> dict:
    """A small case of the 4096^2 slice loop for kernel captures: a-C slab
    50 x 50 x 16 A (8 slices of 2 A, 512 MB potential stack), 300 kV, fused
    conventional slice loop, `reps` passes over the stack."""
    n = 4096
    sim = new_sim(device)
    configure(sim, workload((50.0, 50.0, 16.0)), fparams, grid=n)
    nsl = sim.BuildPotentialStack()
    ms, _, _ = sim.TimeSlices(nsl, reps, breakdown=False)
    sim.close()
    return {"slices": nsl, "slice_steps_per_s": nsl * reps / (ms / 1000.0)}


def fd_leg(fparams, device: int, steps: int = 400, reps: int = 3) -> dict:
    """Finite-difference multislice on the bench workload's specimen (a-C
    50 x 50 x 200 A, 1024^2, 300 kV) at dz = 0.5 A (the slice thickness / 4,
    400 steps through the slab): whole runs of MultisliceStep (ms_run_fd) over
    the resident band-limited potential planes, the fused passes (one CUDA
    graph, two passes per step) against the reference's launch sequence
    (cuFFT + one kernel per operation).  Device time of each run; the
    potential planes are built once per path before timing (reported apart).
    The reference's own step is the stable bound of its quadratic
    (U.cu:1815-1846), also reported."""
    atoms = workload()
    sim = new_sim(device)
    configure(sim, atoms, fparams)
    sim.InitialiseWavefunctions()
    try:
        auto_steps = sim.GetSlices(False)  # the reference's stable FD step count (U.cu:1815-1846)
    except Exception:  # no stable step for these conditions
        auto_steps = 0
    auto_dz = (float(sim.GetSizeZ())) / max(auto_steps, 1) if auto_steps else None
    out = {}
    for name, path in (("fused", 0), ("plain", 1)):
        sim.SetSlicePath(path)
        sim.InitialiseWavefunctions()
        sim.SetFDdz(SLICE_DZ / 4)
        t0 = time.perf_counter()
        sim.RunFD(steps)  # builds the band-limited planes, then runs
        build_s = time.perf_counter() - t0
        best = None
        for _ in range(reps):
            sim.InitialiseWavefunctions()
            sim.RunFD(steps)
            t = sim.LastDeviceMs()
            best = t if best is None else min(best, t)
        out[name] = {"steps_per_s": steps / (best / 1000.0), "run_ms": best, "first_run_with_planes_s": build_s}
    sim.SetSlicePath(0)
    sim.close()
    return {"value": out["fused"]["steps_per_s"], "unit": "FD steps/s", "plain_value": out["plain"]["steps_per_s"],
            "speedup_fused_vs_plain": out["fused"]["steps_per_s"] / out["plain"]["steps_per_s"],
            "dz_A": SLICE_DZ / 4, "steps": steps,
            "reference_stable_dz": {"steps": int(auto_steps), "dz_A_approx": auto_dz,
                                    "note": "the reference's automatic step from its stability quadratic; the "
                                            "workload's dz/4 = 0.5 A is the step asked for"},
            "config": "a-C 50x50x200 A (50k atoms), 1024^2, 300 kV, FD dz 0.5 A, band-limited potential planes "
                      "resident (built once per path)",
            "timing": "device time (CUDA events) of ms_run_fd, best of 3 runs after the run that builds the planes",
            "detail": out}


def focal_profile_leg(fparams, device: int) -> dict:
    """A reduced inverse-problem case for kernel captures: SrTiO3 4 x 4 x 10
    cells on 512^2, 200 kV, one focal-series gradient (8 defoci, 20 slices,
    dL/dxy) -- one potential build per slice and one potential adjoint per slice."""
    import numpy as np

    from cudamultislice_b200 import structures as S

    n = 512
    Z, x, y, z = S.srtio3(4, 4, 10)
    sim = new_sim(device)
    sim.SetAtoms(Z, x, y, z)
    sim.UploadBinnedAtoms()
    sim.GetParameterisation(fparams)
    sim.ApplyMicroscopeParameters(200.0, 0.0, 0.0, 0.0, 1.0e7, 0.1, 30.0, 20.0)
    sim.SetCalculationVariables(3.905 * 4 / n, 0.0, n, n, sim.GetSizeX(), sim.GetSizeY(), sim.GetSizeZ(), 2.0, 2.0)
    sim.PreCalculateFrequencies()
    sim.InitialiseWavefunctions(1.9525)
    df = np.linspace(-800.0, 600.0, 8).astype(np.float32)
    L, _, gxy = sim.FocalSeriesGrad(df, np.ones((8, n, n), np.float32), 20, want_v=False)
    ms = sim.LastDeviceMs()
    sim.close()
    return {"loss": L, "grad_abs_sum": float(np.abs(gxy).sum()), "device_ms": ms}


def adjoint_leg(fparams, device: int, reps: int = 3) -> dict:
    """Differentiable focal series on the inverse-problem workload: SrTiO3
    4 x 4 x 50 cells (4,000 atoms), 512^2 over the 15.62 A cell, 100 slices of
    1.9525 A, 200 kV, Cs 1 mm, 20 mrad, 8 CTF images at defocus -80..+60 nm;
    targets are the images of the same crystal with seeded position errors
    (sigma 0.1 A in x, y, z); L2 loss.  Device time (CUDA events) of the
    forward (potential build + 100 slices + 8 images + loss) against forward +
    adjoint (dL/dV of every slice, dL/dxy of every atom, sqrt(S)-slice
    checkpointing), potentials rebuilt on every call as in one optimisation
    step; and the same pair with the potential stack resident (dL/dV only)."""
    import numpy as np

    from cudamultislice_b200 import structures as S

    n, nslices = 512, 100
    df = np.linspace(-800.0, 600.0, 8).astype(np.float32)
    Z, x, y, z = S.srtio3(4, 4, 50)
    rng = np.random.default_rng(2026)
    pert = [(a + rng.normal(0.0, 0.1, a.size)).astype(np.float32) for a in (x, y, z)]
    sim = new_sim(device)

    def setup(xx, yy, zz):
        sim.SetAtoms(Z, xx, yy, zz)
        sim.UploadBinnedAtoms()
        sim.GetParameterisation(fparams)
        sim.ApplyMicroscopeParameters(200.0, 0.0, 0.0, 0.0, 1.0e7, 0.1, 30.0, 20.0)
        sim.SetCalculationVariables(3.905 * 4 / n, 0.0, n, n, sim.GetSizeX(), sim.GetSizeY(), sim.GetSizeZ(),
                                    2.0, 2.0)
        sim.PreCalculateFrequencies()
        sim.InitialiseWavefunctions(1.9525)

    setup(*pert)
    _, T = sim.FocalSeries(df, np.zeros((8, n, n), np.float32), nslices, images=True)
    setup(x, y, z)

    def timed(fn, rebuild):
        best = None
        for k in range(reps + 1):
            if rebuild:
                sim.UploadBinnedAtoms()
            fn()
            if k > 0:
                t = sim.LastDeviceMs()
                best = t if best is None else min(best, t)
        return best

    import torch

    ksq = int(np.ceil(np.sqrt(nslices)))
    fwd = timed(lambda: sim.FocalSeries(df, T, nslices), True)
    fwd_res = timed(lambda: sim.FocalSeries(df, T, nslices), False)
    out = {}
    # sqrt(S) checkpoints (each segment recomputed once), then the automatic
    # default, which stores every wave when they fit in 1/8 of free memory
    for name, k in (("sqrt_checkpoints", ksq), ("default", 0)):
        sim.SetCheckpoint(k)
        grad = timed(lambda: sim.FocalSeriesGrad(df, T, nslices, want_v=True, want_xy=True), True)
        grad_res = timed(lambda: sim.FocalSeriesGrad(df, T, nslices, want_v=True, want_xy=False), False)
        out[name] = {"grad_ms": grad, "grad_over_forward": grad / fwd, "resident_grad_dV_ms": grad_res,
                     "resident_grad_over_forward": grad_res / fwd_res}
    free_b, _ = torch.cuda.mem_get_info(device)
    auto_k = 1 if nslices * n * n * 8 <= free_b // 8 else ksq
    loss = sim.FocalSeries(df, T, nslices)
    sim.close()
    sq = out["sqrt_checkpoints"]
    return {
        "config": f"SrTiO3 4x4x50 cells ({len(Z)} atoms), {n}^2, {nslices} slices of 1.9525 A, 200 kV, "
                  "8 defoci -80..+60 nm, targets from seeded 0.1 A position errors",
        "forward_ms": fwd, "grad_ms": sq["grad_ms"], "grad_over_forward": sq["grad_over_forward"],
        "checkpoint_stride": ksq,
        "potentials_resident": {"forward_ms": fwd_res, "grad_dV_ms": sq["resident_grad_dV_ms"],
                                "grad_over_forward": sq["resident_grad_over_forward"]},
        "default_stride": {"stride": auto_k, **out["default"]},
        "loss": loss,
        "timing": "device time (CUDA events on the engine stream), best of 3 after a warm-up call",
    }


def tds_leg(fparams, device: int, nconf: int = 16, batch: int = 16) -> dict:
    """Frozen-phonon series on the batched-TDS workload: Si [110], 8 x 6 x 50
    orthogonal 4-atom cells (9,600 atoms), 512^2 square pixels over 32.6 A, 1.92 A slices,
    200 kV, u_rms 0.076 A (seeded Philox), sum of centred |FFT(psi)| and the
    mean CTF image; `nconf` of the 64 configurations timed (device time),
    `batch` configurations per launch on the fused path, one at a time on the
    plain path.  Reports configurations/s and slice-steps/s (potential build
    included: every configuration has its own potentials)."""
    from cudamultislice_b200 import structures as S

    n = 512
    Z, x, y, z = S.silicon_110(8, 6, 50)
    sim = new_sim(device)
    sim.SetAtoms(Z, x, y, z)
    sim.UploadBinnedAtoms()
    sim.GetParameterisation(fparams)
    sim.ApplyMicroscopeParameters(200.0, 0.0, 0.0, 0.0, 1.0e7, 0.1, 30.0, 20.0)
    ps = 6 * 5.431 / n
    sim.SetCalculationVariables(ps, 0.0, n, n, sim.GetSizeX(), sim.GetSizeY(), sim.GetSizeZ(), 2.0, 2.0)
    sim.PreCalculateFrequencies()
    sim.InitialiseWavefunctions(1.92)
    nsl = sim.GetSlices(True)
    out = {}
    for name, path, nc, b in (("fused", 0, nconf, batch), ("plain", 1, max(nconf // 4, 2), 1)):
        sim.SetSlicePath(path)
        sim.FrozenPhonon(0x5EED2026, 0, min(b, nc), 0.076, batch=b)  # warm-up / tuning
        sim.FrozenPhonon(0x5EED2026, 0, nc, 0.076, batch=b)
        ms = sim.LastDeviceMs()
        out[name] = {"configs_per_s": nc / (ms / 1000.0), "slice_steps_per_s": nc * nsl / (ms / 1000.0),
                     "configs": nc, "batch": b, "ms": ms}
    sim.SetSlicePath(0)
    sim.close()
    return {"value": out["fused"]["configs_per_s"], "unit": "configs/s",
            "slice_steps_per_s": out["fused"]["slice_steps_per_s"],
            "plain_value": out["plain"]["configs_per_s"],
            "speedup_fused_vs_plain": out["fused"]["configs_per_s"] / out["plain"]["configs_per_s"],
            "config": f"Si [110] 8x6x50 cells ({len(Z)} atoms), {n}^2, {nsl} slices of 1.92 A, 200 kV, "
                      f"u_rms 0.076 A, {nconf} of 64 configurations, batch {batch}",
            "timing": "device time (CUDA events) of ms_frozen_phonon, potential build of every configuration "
                      "included", "detail": out}


MID_SLICES = 10  # CPU-baseline sample: this many slices from the middle of the slab


def potential_leg(fparams, device: int, reps: int = 3) -> dict:
    """The workload's potential stack (102 slices, 1024^2, 50k atoms) built by
    the separable kernel (the default) and by the per-sub-plane kernel: device
    time of ms_build_potential_stack, best of `reps` rebuilds after a first
    build that tunes each kernel's tile shape."""
    atoms = workload()
    out = {}
    for mode, name in ((2, "separable"), (1, "per_subplane")):
        sim = new_sim(device)
        sim.SetPotentialSum(mode)
        configure(sim, atoms, fparams)
        nsl = sim.BuildPotentialStack()
        best = float("inf")
        for _ in range(reps):
            sim.UploadBinnedAtoms()
            sim.BuildPotentialStack()
            best = min(best, sim.LastDeviceMs())
        out[name] = {"stack_ms": best, "us_per_slice": 1000.0 * best / nsl, "slices": nsl,
                     "kernel_ran": {1: "per sub-plane", 2: "separable"}[sim.PotentialSum()[0]]}
        sim.close()
    return {"value": out["separable"]["us_per_slice"], "unit": "us per slice",
            "speedup_separable_vs_per_subplane": out["per_subplane"]["stack_ms"] / out["separable"]["stack_ms"],
            "config": "a-C 50x50x200 A (50k atoms), 1024^2, 102 slices of 2 A (binnedAtomPKernel3 semantics)",
            "timing": "device time (CUDA events) of ms_build_potential_stack, best of 3 rebuilds",
            "detail": out}


def mid_range(S: int, k: int = MID_SLICES) -> range:
    """Iterations of the k slices centred in an S-slice stack."""
    a = max(1, S // 2 - k // 2 + 1)
    return range(a, min(S, a + k - 1) + 1)


def cpu_full_run(atoms, fparams, threads: int) -> dict:
    """The FP64 OpenMP oracle on the host cores over every slice of the
    workload (potential build + transmission + propagation per slice), each
    slice timed; returns the exit wave for the error check, the mid-slab
    sample's rate, and the rate of the slice step alone (transmission and
    propagation on a stored potential, as `value` times the GPU)."""
    import numpy as np

    from oracle import oracle

    oracle.build()
    oracle.set_threads(threads)
    orc = oracle.OracleSimulation()
    configure(orc, atoms, fparams)
    S = orc.GetSlices(True)
    times = []
    for i in range(1, S + 1):
        t0 = time.perf_counter()
        orc.MultisliceStepConventional(i)
        times.append(time.perf_counter() - t0)
    wave = orc.Wave()
    mid = mid_range(S)
    V = orc.PotentialConventional(mid[0])
    t0 = time.perf_counter()
    for i in mid:
        orc.StepGivenPotential(i, V)
    step_only = len(mid) / (time.perf_counter() - t0)
    orc.close()
    return {"wave": wave, "slices": S, "mid": (mid[0], mid[-1]),
            "mid_rate": len(mid) / sum(times[i - 1] for i in mid), "step_only_rate": step_only,
            "total_s": sum(times)}


def run_reference(args, world, rank):
    """--impl reference: the reference path's CPU implementation (the FP64
    OpenMP port in oracle/; the reference itself has no CPU path) on all host
    threads, each step a bounded sample of the same workload."""
    if rank != 0:
        return
    from cudamultislice_b200 import FPARAMS

    from oracle import oracle

    atoms = workload()
    threads = os.cpu_count() or 1
    oracle.build()
    oracle.set_threads(threads)
    orc = oracle.OracleSimulation()
    configure(orc, atoms, FPARAMS)
    mid = list(mid_range(orc.GetSlices(True)))
    per_step = 2  # slices per step, cycling through the mid-slab sample

    def step(k):
        for j in range(per_step):
            orc.MultisliceStepConventional(mid[(k * per_step + j) % len(mid)])

    for k in range(args.warmup):
        step(k)
    total = 0.0
    for k in range(args.steps):
        t0 = time.perf_counter()
        step(args.warmup + k)
        total += time.perf_counter() - t0
    orc.close()
    value = per_step * args.steps / total
    sample = (f"{per_step} slices per step cycling through slices {mid[0]}-{mid[-1]} of the slab "
              "(potential build + transmission + propagation per slice)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128 (FP64)",
        "data": "synthetic (seeded)", "config": config_dict(len(atoms[0])),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_dict(natoms: int) -> dict:
    return {
        "workload": f"amorphous carbon 50x50x200 A, 0.1 atoms/A^3 ({natoms} C, seeded), 1024x1024 grid, "
                    "100 slices x 2 A, 300 kV, conventional potential (binnedAtomPKernel3 semantics)",
        "grid": GRID, "slices_per_step": 100, "slice_dz_A": SLICE_DZ, "kV": KV, "atoms": natoms,
        "parallelism": "replicas", "l2": "inputs larger than L2: 400 MB potential stack streamed per pass",
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="profiling mode: set-up plus the timed slice loop only (no e2e, plain or CPU legs)")
    ap.add_argument("--fft-plan", type=int, default=-1,
                    help="profiling mode and --leg runs: force this FFT plan variant (default: the autotuner's choice)")
    ap.add_argument("--leg", choices=["stem", "adjoint", "tds", "mixed", "focal_profile", "c1", "fd", "grid4096",
                                       "grid4096_profile", "potential"],
                    help="run one secondary leg alone and print its JSON (exploration)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.leg:
        from cudamultislice_b200 import FPARAMS

        global FORCED_PLAN
        FORCED_PLAN = args.fft_plan

        leg = {"stem": stem_leg, "adjoint": adjoint_leg, "tds": tds_leg, "mixed": mixed_leg,
               "focal_profile": focal_profile_leg, "c1": c1_leg, "fd": fd_leg,
               "grid4096": grid4096_leg, "grid4096_profile": grid4096_profile_leg,
               "potential": potential_leg}[args.leg](FPARAMS, local)
        if rank == 0:
            print(json.dumps({"leg": args.leg, **leg}), flush=True)
        return

    from cudamultislice_b200 import FPARAMS, ManagedMultisliceSimulation

    atoms = workload()
    sim = ManagedMultisliceSimulation(device=local)
    configure(sim, atoms, FPARAMS)
    nsl = sim.BuildPotentialStack()
    assert nsl >= 100
    if args.profile and args.fft_plan >= 0:
        sim.SetFFTPlan(args.fft_plan)
    fft_plan = sim.FFTPlan(1)
    steps_per = 100  # slices per bench step (the workload's 100 slices of 2 A)
    for _ in range(max(args.warmup, 3)):
        sim.TimeSlices(steps_per, 1, breakdown=False)

    import torch

    torch.cuda.set_device(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.25)
    l0 = sim.LaunchCount()
    total_ms, _, _ = sim.TimeSlices(steps_per, args.steps, breakdown=False)
    launches = sim.LaunchCount() - l0
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    total_ms = allreduce_max(total_ms, world)
    slice_steps = steps_per * args.steps * world
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_mode": True, "value": slice_steps / (total_ms / 1000.0), "unit": UNIT,
                              "gpu_launches": launches}), flush=True)
        sim.close()
        return
    value = slice_steps / (total_ms / 1000.0)

    # roofline of the dominant kernel.  With the persistent slice loop (one
    # cooperative launch per bench step = 100 slices) that is the loop kernel
    # itself: its launch duration is the step time; algorithmic bytes per
    # launch = 100 slices x 20 B per pixel (psi read + written, V read).
    N = GRID * GRID
    peak, peak_kind = measured_peaks()
    step_ms = total_ms / (steps_per * args.steps)
    loop_on = launches == args.steps
    traffic = None
    traffic_file = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(traffic_file):
        with open(traffic_file) as f:
            traffic = json.load(f)
    if loop_on:
        launch_ms = total_ms / args.steps
        algo = steps_per * BYTES_PER_PX_STEP * N
        achieved = algo / (launch_ms / 1000.0) / 1e9
        roofline = {"bound": "hbm", "kernel": "k_slice_loop (persistent cooperative slice loop: per slice a row "
                    "phase IFFT_row, x exp(i sigma V), FFT_row and a column phase FFT_col, x P(k), IFFT_col, "
                    "grid barriers between them)", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_kind,
                    "traffic": (traffic or {}).get("slice_loop_per_launch"),
                    "launch_ms": launch_ms, "slices_per_launch": steps_per,
                    "algorithmic_bytes_per_launch": algo,
                    "timing": "CUDA events on the engine stream around the timed launches, one launch per step"}
    else:
        _, row_ms, col_ms = sim.TimeSlices(steps_per, 1, breakdown=True)
        row_bytes, col_bytes = 20 * N, 16 * N
        dom = ("row pass", row_ms, row_bytes) if row_ms >= col_ms else ("column pass", col_ms, col_bytes)
        achieved = dom[2] / (dom[1] / 1000.0) / 1e9
        roofline = {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_kind, "traffic": None, "launch_ms": dom[1]}
    roofline["step_achieved_gbs"] = BYTES_PER_PX_STEP * N / (step_ms / 1000.0) / 1e9
    roofline["step_frac"] = roofline["step_achieved_gbs"] / peak

    # the same loop on one launch per pass (the fused passes without the
    # persistent kernel), and those passes timed back to back on their own
    sim.SetSliceLoop(False)
    sim.TimeSlices(steps_per, 1, breakdown=False)
    pp_ms, _, _ = sim.TimeSlices(steps_per, args.steps, breakdown=False)
    rv, cv = sim.FFTPlan(1)
    row_us = sim.TimePass(0, 7, rv, 1, 200)  # A_INV | A_MULT_T | A_FWD
    col_us = sim.TimePass(1, 2, cv, 1, 200)  # B_PROPAGATE
    sim.SetSliceLoop(True)
    per_pass = {"value": steps_per * args.steps / (pp_ms / 1000.0), "unit": UNIT,
                "row_pass_us_back_to_back": row_us, "col_pass_us_back_to_back": col_us,
                "row_pass_frac": 20 * N / (row_us * 1e-6) / 1e9 / peak,
                "col_pass_frac": 16 * N / (col_us * 1e-6) / 1e9 / peak,
                "plan": {"row_variant": rv, "col_variant": cv},
                "note": "k_pass_a / k_pass_b launched per pass (programmatic dependent launch); per-pass times "
                        "from ms_time_pass, each pass launched back to back on its own"}

    # plain path (cuFFT + one kernel per operation) on the same GPU and stack
    sim.SetSlicePath(1)
    sim.TimeSlices(steps_per, 1, breakdown=False)
    plain_ms, _, _ = sim.TimeSlices(steps_per, args.steps, breakdown=False)
    plain_value = steps_per * args.steps / (plain_ms / 1000.0)
    sim.SetSlicePath(0)

    # end to end through the C ABI with host buffers (pinned, as a serving
    # process keeps its staging buffers)
    import numpy as np

    def pinned(a):
        t = torch.empty(a.shape, dtype=getattr(torch, a.dtype.name), pin_memory=True)
        v = t.numpy()
        v[...] = a
        return v, t

    hosts = [pinned(a) for a in atoms]
    Z, x, y, z = (v for v, _ in hosts)
    out_host, out_t = pinned(np.zeros((GRID, GRID), np.complex64))
    h2d = Z.nbytes + x.nbytes + y.nbytes + z.nbytes
    e2e_times = []
    for k in range(min(args.steps, 20) + 1):
        t0 = time.perf_counter()
        sim.SetAtoms(Z, x, y, z)
        sim.UploadBinnedAtoms()
        sim.InitialiseWavefunctions(SLICE_DZ)
        ns = sim.RunConventional()
        psi = sim.ExitWave(out=out_host)
        dt = time.perf_counter() - t0
        if k > 0:
            e2e_times.append(dt)
    e2e_s = allreduce_max(sum(e2e_times), world)
    e2e_value = ns * len(e2e_times) * world / e2e_s

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 (FP32 complex)", "data": "synthetic (seeded)",
        "config": config_dict(len(Z)), "clocks": clk, "gpu_launches": launches,
        "fft_plan": ({"slice_loop": "packed 32-point plan (variant 3), one warp per line, both phases"} if loop_on
                     else {"row_variant": fft_plan[0], "col_variant": fft_plan[1],
                           "selected_by": "on-device autotuner"}),
        "roofline": roofline,
        "plain_path": {"value": plain_value, "unit": UNIT, "speedup_fused_vs_plain": value / world / plain_value},
        "per_pass_path": per_pass,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(psi.nbytes),
                "note": "host clock around the synchronous C-ABI calls: atoms in from pinned host memory, "
                        "binning, potential stack (100 slices) built while each built slice is stepped on a second stream, "
                        "exit wave out to pinned host memory"},
    }

    if rank == 0:  # secondary legs: one GPU, after the collective timing
        out["stem"] = stem_leg(FPARAMS, local)
        out["adjoint"] = adjoint_leg(FPARAMS, local)
        out["tds"] = tds_leg(FPARAMS, local)
        out["stem_mixed"] = mixed_leg(FPARAMS, local)
        out["c1"] = c1_leg(FPARAMS, local)
        out["fd"] = fd_leg(FPARAMS, local)
        out["grid4096"] = grid4096_leg(FPARAMS, local)
        out["potential"] = potential_leg(FPARAMS, local)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cb = cpu_full_run(atoms, FPARAMS, threads)
        sim.InitialiseWavefunctions(SLICE_DZ)
        assert sim.RunConventional() == cb["slices"]
        psi_gpu = sim.ExitWave().astype(np.complex128)
        err = float(np.linalg.norm(psi_gpu - cb["wave"]) / np.linalg.norm(cb["wave"]))
        a, b = cb["mid"]
        out["cpu_baseline"] = {
            "value": cb["mid_rate"], "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"FP64 OpenMP oracle on {threads} threads, slices {a}-{b} of the {cb['slices']}-slice "
                      "workload (potential build + transmission + propagation), timed inside the full run "
                      "that the error check uses",
            "slice_step_only": {"value": cb["step_only_rate"], "unit": UNIT,
                                "what": "transmission + propagation on a stored potential (as `value` is timed "
                                        "on the GPU), the same mid-slab slices"},
            "full_run_s": cb["total_s"]}
        out["err_vs_fp64"] = {"value": err, "after_slices": cb["slices"],
                              "path": "fused slice loop (ms_run_conventional) from atoms to exit wave",
                              "definition": "||psi - psi64||_2 / ||psi64||_2 on the exit wave"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    sim.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
