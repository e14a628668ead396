#!/usr/bin/env python
"""Time steps/s of the body-fitted IGA Navier-Stokes solve on one B200.

Workload (default --workload c3, the config the metric's mixed-vs-FP64
comparison is quoted on): the Y-bifurcation -- parent R 2.0 mm, L 20 mm;
daughters R 1.59 mm (Murray), L 16 mm, half-angle 35 deg; swept half-disc
O-grids, 199,800 tricubic elements, 217,271 control points; rho = 1060 kg/m^3,
mu = 3.5e-3 Pa s, backward Euler dt = 2e-3 s; parabolic inflow scaled by a
seeded Fourier waveform (mean 0.15 m/s + 4 harmonics, amplitudes U(0, 0.05),
seed 0, 1 Hz); each daughter outlet a 0D RCR model (R1 1e8, C 1e-10, R2 1e9
SI, zero initial pressure); no-slip walls.  Other workloads: c2 (the
51,200-element pulsatile tube), c1 (the 1,280-element cylinder), c2-100 (a
12,800-element section, profiling), c5 (16 independent tubes as one mesh).
Inputs are synthetic (seeded generator), stated in `data`.

A "step" is one physical time step: Newton to ||r|| <= 1e-8 ||r_0|| (FP64
residual) with the exact tangent, each linear solve AMG-preconditioned
FGMRES(64) -- by default (--forcing ew) to an Eisenstat-Walker forcing
tolerance, with the step's Dirichlet values lifted into the state first so
that r_0 is the PDE residual, and in the tensor-core modes the previous
iteration's tangent kept while Newton contracts within 100x the linear
tolerance (--tangent-reuse 0 turns that off); --forcing fixed solves every system to a
true-residual rtol of 1e-8 as the reference (the AMG's dense coarse inverse
rebuilt every third linear solve, its fine-level data on every solve; both
precisions).  Outlet pressures follow the RCR models by the relaxed fixed
point (relaxation 1, tolerance 1e-8 + 1e-6 |P|), updated inside the Newton
loop (--outlet-coupling newton; "outer" runs the reference's loop of Newton
solves), with the models' dP/dQ terms in the Newton Jacobian.  --precision
bf16x3 (default): tangent contracted on the tcgen05 tensor cores with
split-BF16 operands (hi + lo, three products, FP32 accumulation), FP32
Jacobian for SpMV and the preconditioner, FP32 Krylov basis, FP64 residual,
vectors and refinement; --precision mixed: plain BF16 operands (a tangent
accurate to about 1e-2, so Newton contracts more slowly on the coupled
system); --precision tf32: TF32 operands; --precision fp64: every array FP64.

Legs of one run (rank 0 prints one JSON line):
  value     device-timed (CUDA events on the solver stream) with every input
            resident in HBM; the matrix (3.1 GB FP32 at C3) exceeds L2, so no
            flush.
  e2e       the same steps again, from the same starting state, through the
            C ABI with pinned host inputs (inlet Dirichlet values) and the
            state read back every step.
  roofline  per-kernel CUDA-event timing of the timed region: the tensor-core
            (or FP64) assembly, SpMV, the AMG V-cycle and the Krylov
            orthogonalisation (HBM-bound); the dominant one by share.
  fp64_gpu  (mixed only) the plain FP64 GPU solver on the warm-up steps from
            the same initial state (same outlet coupling), run with the fixed
            1e-8 tolerance and in the mixed arm's forcing mode; the faster of
            the two is reported (both values under "variants") with its Newton
            and FGMRES counts and the relative L2 error of the mixed solution
            against it after every step.
  cpu_baseline  the reference's own element code (oracle/_ref) and the CPU
            restatement of block-Jacobi GMRES on a bounded sample, all host
            cores, scaled to time steps/s.
  --impl reference  only the CPU reference arm, as its own line.

--workload transport: the two-species transport of the reference's `transport`
command on the C3 Y-bifurcation, its own JSON line.  The velocity is that of
one mixed Navier-Stokes step of C3 from rest (the flow the reference's
`solve` chain hands to transport); a step is rhs = P c, the inlet values set,
and L c' = rhs by block-Jacobi GMRES(50) to rtol 1e-8, warm-started.  value:
device-timed steps with L and P resident in HBM (L alone 1.6 GB, beyond L2);
e2e: the whole job through the C ABI from host buffers (velocity, mask and
inlet values uploaded, assembly, the steps, the final state read back),
steps / wall time; fp64_gpu: the same steps with the FP64 solver (the
default arm keeps an FP32 copy of L for the Arnoldi SpMV, FP64 everywhere
else); cpu_baseline: the CPU restatement of the step (2x2 SpMV +
block-Jacobi GMRES) on all host cores for a bounded number of iterations,
scaled by the GPU's iterations per step.

Multi-GPU: the single-mesh path does not shard ("replicas only"): under
torchrun every rank runs an independent replica; value = total steps / max
time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "NS time steps/s at rel.res 1e-8: learned+mixed vs plain FP64 GPU; SpMV GB/s"
RHO, MU, DT = 1060.0, 3.5e-3, 2e-3
# DRAM bytes (read + write) per 4x4 block of one FP32-Jacobian SpMV launch, measured with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum = 202,687,488 B on the 12,800-element section,
# 2,919,695 blocks); the launch streams the matrix once, so traffic scales with the block count.
SPMV_FP32_DRAM_BYTES_PER_BLOCK = 202687488 / 2919695
# The same for the transport's 2x2 block-Jacobi SpMV with the FP32 copy of L (59,472,384 B on the same
# section's 2,919,695 blocks).
TRANSPORT_SPMV_FP32_DRAM_BYTES_PER_BLOCK = 59472384 / 2919695


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


def sustained_bf16():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("bf16_tflops_sustained", d["bf16_tflops"]))
    return 1400.0


# The batched-tube workload: 64 seeded tubes, straight or helical, 1k-30k elements (log-uniform).
C5_TUBES = 64
C5_BATCH = dict(seed=0, min_elements=1000, max_elements=30000, helical=0.5, log_sizes=True)


def c5_specs():
    from tubularflowiga_b200 import meshgen
    return meshgen.tube_batch_specs(C5_TUBES, **C5_BATCH)


def tube_part(specs, world, rank):
    """The tubes rank `rank` of `world` solves: greedy longest-first packing on the tube cost model, so
    the GPUs get about equal work; no tube is split, so the ranks exchange nothing while solving."""
    from tubularflowiga_b200 import meshgen
    return meshgen.pack_tubes([meshgen.tube_cost(s) for s in specs], world)[rank]


def gather_tube_metrics(dist, tube_ids, metrics):
    """Per-tube metrics of every rank, in tube order, on every rank (one all_gather of Python objects;
    identity without a process group)."""
    local = list(zip([int(k) for k in tube_ids], metrics))
    if dist is None:
        return [m for _, m in sorted(local)]
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, local)
    return [m for _, m in sorted(item for part in parts for item in part)]


def workload(name, world=1, rank=0):
    from tubularflowiga_b200 import meshgen
    if name == "c2-100":
        tube = meshgen.straight_tube(1.5e-3, 7.5e-3, core=8, ring=2, layers=100)
        desc = ("pulsatile tube cross-section of the 51,200-element case, 100 layers (12,800 elements), "
                "R 1.5 mm, L 7.5 mm, same inflow (profiling case)")
        return tube, desc, meshgen.fourier_waveform(0)
    if name == "c5":
        specs = c5_specs()
        part = tube_part(specs, world, rank)
        batch = meshgen.tube_batch(C5_TUBES, indices=part, **C5_BATCH)
        batch.tube_ids = part
        desc = ("batch of %d independent tubes (seed 0), half of them helical (centreline curvature radius "
                "U(10, 40) mm): R U(0.5, 3) mm, L U(10, 40) R, 4x4-core O-grid, 1k-30k tricubic elements each "
                "(log-uniform; %d in all, %d on this rank's GPU), Re U(50, 800), a seeded Fourier inflow per "
                "tube; each GPU's tubes (greedy cost packing) as one disjoint-union mesh with per-tube Newton "
                "tests" % (C5_TUBES, sum(s.elements for s in specs), batch.mesh.elements))
        return batch, desc, [meshgen.fourier_waveform(k) for k in part]
    if name == "c4":
        tree = meshgen.binary_tree()
        desc = ("binary tree (seed 0) of depth 4 (15 segments, 8 outlets): root R 2.5 mm along +z, daughter "
                "radii by Murray's law x U(0.9, 1.1), lengths U(8, 12) R, branch angles U(30, 80) deg in "
                "alternating planes; swept O-grid regions (8x8 core + 3-cell ring, 2^m per segment above 2^m "
                "outlets), %d tricubic elements; traction-free outlets; C2's Fourier inflow"
                % tree.mesh.elements)
        return tree, desc, meshgen.fourier_waveform(0)
    if name == "c3":
        y = meshgen.y_bifurcation()
        desc = ("Y-bifurcation %d tricubic elements: parent R 2.0 mm L 20 mm, daughters R 1.59 mm L 16 mm at "
                "half-angle 35 deg, swept half-disc O-grids (6x12 core + 3-cell ring per half) x 308 + 247 "
                "layers; RCR outlets R1 1e8, C 1e-10, R2 1e9 (SI); C2's Fourier inflow" % y.mesh.elements)
        return y, desc, meshgen.fourier_waveform(0)
    if name == "c1":
        tube = meshgen.straight_cylinder_1280()
        desc = ("straight cylinder 1,280 tricubic elements (4x4 core + 16-cell ring) x 40 layers, "
                "R 1.5 mm, L 30 mm, steady inflow peak 0.2 m/s")
        wave = None
    else:
        tube = meshgen.pulsatile_tube_51200()
        desc = ("pulsatile tube 51,200 tricubic elements (8x8 core + 2x32-cell ring) x 400 layers, "
                "R 1.5 mm, L 30 mm, Fourier inflow mean 0.15 m/s + 4 harmonics U(0,0.05) seed 0")
        wave = meshgen.fourier_waveform(0)
    return tube, desc, wave


def max_over_ranks(dist, values, device):
    """Each rank's device-timed milliseconds -> their maximum over all ranks (one all-reduce that every
    rank takes; identity without a process group)."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def replica_throughput(world, steps, ms):
    """Whole-job time steps/s of `world` independent replicas that each took `steps` steps, timed by the
    slowest rank (`ms`, milliseconds)."""
    return world * steps / (ms / 1e3)


def step_dt(name):
    """Time step of a workload: the 1,280-element cylinder 1e-3 s; the tube batch 1e-4 s, because its
    smallest fast tubes (R 0.5 mm at Re 800, about 1.5 m/s) reach an axial CFL of 70 at 2e-3 s;
    otherwise 2e-3 s."""
    return {"c1": 1e-3, "c5": 1e-4}.get(name, DT)


# Per-workload solver settings of both arms.  The binary tree's Newton test is one decade tighter: at
# rel.res 1e-10 its mixed and FP64 arms accepted states up to 2.3e-8 apart in pressure (traction-free
# outlets, 600k elements).  Its coarse level has 1,762 point blocks (7,048 unknowns), whose dense inverse
# took 19% of the step when rebuilt every third refresh (0.3% every ninth); the tube batch is as large.
# The tube batch tests every tube against its own first residual (per-tube Newton tests and per-tube
# FGMRES) one decade tighter too: at rel.res 1e-10 the largest tubes' pressure was resolved only to
# 1.7e-7 by either precision (the two FP64 forcing modes differed by 2.9e-7), at 1e-11 to 2.0e-8 (their
# FP64 modes 2.8e-8 apart) with velocity within 8e-11; 1e-12 lies below what the largest tubes' FP64
# residual can reach.
NEWTON_RTOL = {"c4": 1e-11, "c5": 1e-11}
COARSE_PERIOD = {"c4": 9, "c5": 9}


def outlet_models(name):
    """RCR outlets of the Y-bifurcation (labels 2 and 3, zero initial pressure), else None."""
    if name != "c3":
        return None
    from tubularflowiga_b200 import api
    return [api.Outlet.rcr(label, 1e8, 1e-10, 1e9) for label in (2, 3)]


# Outlet coupling of the bench: the relaxed fixed point with relaxation 1 (rigid walls and a Dirichlet
# inflow fix the total outlet flow, so it reaches the reference's tolerance in two Newton loops; the
# reference's 0.5 would need about 20 here, more than its cap of 12).
OUTLET_RELAXATION = 1.0


def outlet_step(ns, outlets, coupling):
    """One step with outlet models: the reference's outer loop (a Newton loop per outlet iteration) or the
    pressures updated inside one Newton loop; both accept at the same tolerances."""
    if coupling == "outer":
        return ns.step_outlets(outlets, OUTLET_RELAXATION)
    return ns.step_outlets_coupled(outlets, OUTLET_RELAXATION)


def boundary(obj, wave):
    """(vmask, pmask, velocity_at(t)) of a workload: one tube with one waveform, or a tube batch whose
    tubes each scale their own peak velocity by their own seeded waveform (normalised to mean 1)."""
    from tubularflowiga_b200 import api
    if isinstance(wave, list):
        def velocity_at(t):
            factors = [inlet_factor(w, t) / w["mean"] for w in wave]
            return api.batch_boundary_conditions(obj, factors)[2]
        vmask, pmask, _ = api.batch_boundary_conditions(obj)
        return vmask, pmask, velocity_at
    vmask, pmask, profile = api.tube_boundary_conditions(obj, 1.0)
    return vmask, pmask, lambda t: inlet_factor(wave, t) * profile


def inlet_factor(wave, t):
    if wave is None:
        return 0.2
    th = 2 * np.pi * (t % wave["period"]) / wave["period"] + wave["phase"]
    return wave["mean"] + sum(c * np.cos((k + 1) * th) + s * np.sin((k + 1) * th)
                              for k, (c, s) in enumerate(zip(wave["cosine"], wave["sine"])))


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1])); mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_counts(tube, blocks):
    """Per-launch algorithmic bytes / flops (SpMV: 8 B values + 4 B column index per block entry set)."""
    n = tube.mesh.nodes
    N = 4 * n
    b_spmv = blocks * (16 * 8 + 4) + 4 * (n + 1) + N * 8 + N * 8
    b_bjac = n * 16 * 8                      # fused block-Jacobi apply: the 4x4 inverse per node
    nen = np.diff(tube.mesh.element_offsets).astype(np.float64)
    f_asm = float((8192.0 * nen * nen).sum())
    return b_spmv, b_bjac, f_asm


# Newton iterations per step and GMRES iterations per Newton iteration of the reference's own solver
# algorithm on each workload -- exact-tangent Newton to rel.res 1e-8 with a fresh tangent every iteration,
# every linear system to rtol 1e-8 by left block-Jacobi GMRES(200) with the 5000-iteration cap
# (iga_cuda.cu:956-1054, Gmres.hpp:69-213) -- recorded on the GPU by this library in that mode:
#   python bench.py --record-reference-counts --workload W --steps 3
# The CPU arm prices those counts at its own measured element and GMRES-iteration costs.
REFERENCE_COUNTS = {
    "c3": {"newton_per_step": 6.0, "gmres_per_newton": 3068.3,
           "recorded": "B200, outlets held at their initial 0 Pa: step 1 converged in 6 Newton iterations with "
                       "3526, 3696, 2703, 2657, 2657 and 3171 GMRES iterations; the first linear system of step 2 "
                       "stopped at the 5000-iteration cap (preconditioned residual 2.7e-2 of its start), where the "
                       "reference command exits with 'Navier-Stokes GMRES failed'.  The arm prices step 1."},
    "c2-100": {"newton_per_step": 2.0, "gmres_per_newton": 381.0,
               "recorded": "B200: steps 1-3 converged in 5, 3 and 2 Newton iterations (GMRES 211-287, 294-389, "
                           "362-400); the arm prices step 3"},
}


class CpuReference:
    """The reference's CPU path for one workload, set up once: its own element code (oracle/_ref, OpenMP
    over all host cores; the CPU restatement where the reference build is absent) and the CPU restatement
    of block-Jacobi GMRES(200) (Gmres.hpp:69-213) on the workload's full block pattern.

    A sample times a bounded part of one time step -- the assembly of the first `elements` elements and
    `iterations` GMRES iterations -- and extrapolates it to a whole step of `newton` Newton iterations with
    `gmres` GMRES iterations each: step = newton x (E x t_element + gmres x t_iteration)."""

    def __init__(self, tube, state, prev):
        from oracle import oracle as O
        self.O = O
        self.mesh = tube.mesh
        self.state, self.prev = state, prev
        m = tube.mesh
        self.P = O.Pattern(m.nodes, m.element_offsets, m.connectivity)
        self.kind = "reference" if O.ref_available() else "port"
        self.threads = O.ref().ref_max_threads() if self.kind == "reference" else O.max_threads()
        # GMRES operand: 4 I diagonal blocks plus small off-diagonal entries (the cost of an iteration
        # does not depend on the values); tiled from a 1 Mi-value random block so that filling the
        # multi-GB array is a memory copy
        rng = np.random.default_rng(0)
        vals = np.resize(rng.standard_normal(1 << 20) * 1e-3, self.P.blocks * 16)
        vals.reshape(-1, 4, 4)[self.P.diagonal] += np.eye(4) * 4.0
        self.vals = vals
        self.rhs = rng.standard_normal(4 * m.nodes)
        self.elements, self.iterations = max(self.threads, 64), 10

    def _time_assembly(self, count):
        m = self.mesh
        t0 = time.perf_counter()
        if self.kind == "reference":
            self.O.ref_assemble(m, self.P, self.state, self.prev, RHO, MU, DT, 0, count)
        else:
            self.O.assemble(m, self.P, self.state, self.prev, RHO, MU, DT)
        return time.perf_counter() - t0

    def _time_gmres(self, iterations):
        t0 = time.perf_counter()
        self.O.gmres_bjacobi(self.P, self.vals, self.rhs, restart=200, maxit=iterations, rtol=1e-300)
        return time.perf_counter() - t0

    def calibrate(self, budget_s):
        """Sample sizes for which one sample takes about budget_s (doubling from small sizes)."""
        m = self.mesh
        count = max(self.threads, 64)
        while True:
            count = min(count, m.elements) if self.kind == "reference" else m.elements
            if self._time_assembly(count) > 0.45 * budget_s or count >= m.elements:
                break
            count *= 2
        iters = 5
        while True:
            if self._time_gmres(iters) > 0.45 * budget_s or iters >= 400:
                break
            iters *= 2
        self.elements, self.iterations = count, iters

    def sample(self, newton, gmres):
        t_el = self._time_assembly(self.elements) / self.elements
        t_it = self._time_gmres(self.iterations) / self.iterations
        t_step = newton * (t_el * self.mesh.elements + gmres * t_it)
        return {
            "value": 1.0 / t_step, "unit": "time steps/s", "cores": int(self.threads), "kind": self.kind,
            "sample": (f"reference element assembly of {self.elements} of {self.mesh.elements} elements "
                       f"({t_el * 1e3:.2f} ms/element wall on {self.threads} threads) and {self.iterations} "
                       f"block-Jacobi GMRES(200) iterations of the CPU restatement on the full "
                       f"{4 * self.mesh.nodes}-DOF pattern ({t_it * 1e3:.1f} ms/iteration: the first Arnoldi "
                       f"steps of a cycle, cheaper than the cycle's average, so the step time is a lower bound); "
                       f"extrapolated to a step of {newton:.2f} Newton x (assembly + {gmres:.0f} GMRES "
                       f"iterations), the counts of the reference's algorithm recorded on the GPU"),
            "sample_s": t_el * self.elements + t_it * self.iterations, "step_s": t_step,
        }


def reference_counts(name):
    c = REFERENCE_COUNTS.get(name)
    if c is None:
        raise SystemExit("no recorded reference-algorithm counts for workload " + name)
    return c["newton_per_step"], c["gmres_per_newton"]


def record_reference_counts(args):
    """Newton and GMRES counts of the reference's solver algorithm on a workload (FP64, block-Jacobi
    GMRES(200) to rtol 1e-8 with its 5000-iteration cap, Newton to rel.res 1e-8 with the tangent of every
    iterate, Dirichlet values lifted by the first update), one JSON line per step; stops at the first
    failure, as the reference command does."""
    import torch
    torch.cuda.set_device(0)
    from tubularflowiga_b200 import api
    tube, desc, wave = workload(args.workload)
    mesh = api.Mesh(tube.mesh)
    vmask, pmask, velocity_at = boundary(tube, wave)
    dt = step_dt(args.workload)
    ns = api.NavierStokes(mesh, precision=api.FP64, preconditioner=api.BLOCK_JACOBI, density=RHO, viscosity=MU,
                          dt=dt, nonlinear_rtol=1e-8, nonlinear_atol=1e-300, mass_rtol=1e-3, gmres_restart=200,
                          gmres_max_iterations=5000, gmres_rtol=1e-8, newton_forcing=0, tangent_reuse_factor=0.0)
    ns.set_dirichlet(vmask, pmask, velocity_at(0.0))
    ns.set_tractions({label: 0.0 for label in getattr(tube, "outlet_labels", (2, 3) if args.workload == "c3"
                                                       else (2,))})
    s0 = api.initial_state(vmask, velocity_at(0.0))
    ns.set_state(s0, s0)
    for k in range(args.steps):
        ns.set_dirichlet_values(velocity_at((k + 1) * dt).ravel())
        ns.commit_step()
        initial, gmres, status = -1.0, [], "converged"
        for _ in range(30):
            try:
                r = ns.newton_iteration(initial)
            except api.TfigaError as e:
                gmres.append(5000)
                status = "failed: " + str(e)
                break
            if initial < 0:
                initial = r["residual_l2"]
            if r["converged"]:
                break
            gmres.append(r["linear_iterations"])
        else:
            status = "no convergence in 30 Newton iterations"
        print(json.dumps({"workload": args.workload, "step": k + 1, "newton": len(gmres), "gmres": gmres,
                          "status": status}), flush=True)
        if status != "converged":
            break
    ns.close()
    return 0


def run_reference_arm(args, world, rank):
    if rank != 0:
        return 0
    tube, desc, wave = workload(args.workload)
    from tubularflowiga_b200 import api
    n = tube.mesh.nodes
    vmask, pmask, velocity_at = boundary(tube, wave)
    s0 = api.initial_state(vmask, velocity_at(0.0))
    newton, lin = reference_counts(args.workload)
    cpu = CpuReference(tube, s0, s0)
    # each timed step is one bounded sample of the step, sized so that the whole run stays within a few
    # minutes; the warm-up steps calibrate the sample size
    budget = max(2.0, min(args.ref_budget, 150.0 / max(1, args.steps)))
    for _ in range(max(1, args.warmup)):
        cpu.calibrate(budget)
    t0 = time.perf_counter()
    samples = [cpu.sample(newton, lin) for _ in range(args.steps)]
    wall = time.perf_counter() - t0
    res = dict(samples[-1])
    res["value"] = float(np.mean([r["value"] for r in samples]))
    line = {"metric": METRIC, "value": res["value"], "unit": "time steps/s", "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 / res["value"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": {"workload": desc, "elements": tube.mesh.elements, "nodes": n,
                       "solver": "reference CPU element code + CPU block-Jacobi GMRES(200); Newton and GMRES "
                                 "counts of the reference's algorithm recorded on the GPU",
                       "parallelism": "replicas only"},
            "extrapolated": {"note": "each timed step runs a bounded sample of the full step and is "
                                     "extrapolated to it, so ms_per_step x steps exceeds the run's wall time",
                             "sample_s_per_step": float(np.mean([r["sample_s"] for r in samples])),
                             "sampled_wall_s": wall, "newton_per_step": newton, "gmres_per_newton": lin,
                             "counts_recorded": REFERENCE_COUNTS[args.workload]["recorded"]},
            "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": res["value"], "unit": "time steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


TRANSPORT_METRIC = "two-species transport time steps/s (backward Euler, block-Jacobi GMRES(50) rtol 1e-8)"
# Transport coefficients of the transport workload (SI): a small solute (D 1e-9 m^2/s) exchanging with an
# advected species (k+ 1/s, k- 0.1/s, k'+ 0.5/s), inlet values N0 1, N+ 0.5, artificial diffusion 1e-6 m^2/s,
# dt 2e-3 s as the flow.
TRANSPORT = dict(diffusion=1e-9, vplus=1.0, kplus=1.0, kminus=0.1, detach_plus=0.5, dt=2e-3, n0_bc=1.0,
                 nplus_bc=0.5, artificial_diffusion=1e-6)


def flow_velocity(api, mesh, tube, wave):
    """Nodal velocity [n, 3] after one mixed Navier-Stokes step of C3 from rest."""
    ns = api.NavierStokes(mesh, precision=api.MIXED_BF16X3, density=RHO, viscosity=MU, dt=DT,
                          nonlinear_rtol=1e-8, nonlinear_atol=1e-300, gmres_restart=64, gmres_max_iterations=5000,
                          gmres_rtol=1e-8, preconditioner=api.AMG, amg_coarse_period=3, newton_forcing=1,
                          tangent_reuse_factor=100.0)
    vmask, pmask, velocity_at = boundary(tube, wave)
    ns.set_dirichlet(vmask, pmask, velocity_at(0.0))
    s0 = api.initial_state(vmask, velocity_at(0.0))
    ns.set_state(s0, s0)
    outlets = [api.Outlet(**m.as_dict()) for m in outlet_models("c3")]
    inlet = np.ascontiguousarray(velocity_at(DT).ravel(), np.float64)
    api.check(api.lib().tfiga_ns_set_dirichlet_values(ns._h, api.C.c_void_p(inlet.ctypes.data), None))
    ns.commit_step()
    outlet_step(ns, outlets, "newton")
    v = ns.get_state().reshape(-1, 4)[:, :3].copy()
    ns.close()
    return v


def transport_cpu_reference(mesh, left, previous, state, iterations_per_step, budget_iterations=30):
    """CPU restatement of one transport step on all host cores: 2x2 SpMV P c and block-Jacobi GMRES(50) run
    for a bounded number of iterations, scaled to the GPU's iterations per step."""
    from oracle import oracle as O
    ro, cols, diag = mesh.pattern()
    t0 = time.perf_counter()
    rhs = O.transport_spmv(ro, cols, previous, state)
    t_spmv = time.perf_counter() - t0
    t0 = time.perf_counter()
    _, its, _ = O.transport_gmres(ro, cols, diag, left, rhs, state, restart=50, maxit=budget_iterations,
                                  rtol=1e-300)
    t_gmres = time.perf_counter() - t0
    its = max(its if its > 0 else budget_iterations, 1)
    step_s = t_spmv + t_gmres * iterations_per_step / its
    return {"value": 1.0 / step_s, "unit": "time steps/s", "cores": O.max_threads(), "kind": "port",
            "sample": "one 2x2 SpMV (P c) and %d block-Jacobi GMRES(50) iterations (CPU restatement, including "
                      "its block-inverse build) on the full C3 transport system, scaled to %.1f iterations "
                      "per step" % (budget_iterations, iterations_per_step)}


def run_transport(args, world, rank, local):
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    from tubularflowiga_b200 import api
    tube, desc, wave = workload(args.transport_mesh)
    n = tube.mesh.nodes
    mesh = api.Mesh(tube.mesh)
    if args.transport_mesh == "c3":
        velocity = flow_velocity(api, mesh, tube, wave)
    else:
        # Poiseuille flow of the straight tube: peak 2 x mean along the axis
        velocity = 0.3 * tube.profile
        desc += "; Poiseuille velocity, mean 0.15 m/s"
    fp32 = args.transport_precision == "fp32"
    total_steps = args.warmup + args.steps

    def make_params(precision):
        return api.transport_params(steps=total_steps, restart=args.transport_restart, precision=precision,
                                    preconditioner=(api.TRANSPORT_FLOW_LINES if args.transport_preconditioner
                                                    == "flow-lines" else api.TRANSPORT_BLOCK_JACOBI),
                                    **TRANSPORT)

    params = make_params(api.MIXED if fp32 else api.FP64)
    mask, n0, nplus = api.resolve_transport_boundaries(tube.labels, velocity, params)
    velocity_pinned = torch.tensor(velocity.ravel()).pin_memory()
    mask_pinned = torch.tensor(mask).pin_memory()
    n0_pinned = torch.tensor(n0).pin_memory()
    nplus_pinned = torch.tensor(nplus).pin_memory()
    out_pinned = torch.empty(2 * n, dtype=torch.float64).pin_memory()
    lib = api.lib()

    def create(p):
        h = api.C.c_void_p()
        api.check(lib.tfiga_transport_create(mesh._h, api.C.byref(p), api.C.c_void_p(velocity_pinned.data_ptr()),
                                             api.C.c_void_p(mask_pinned.data_ptr()),
                                             api.C.c_void_p(n0_pinned.data_ptr()),
                                             api.C.c_void_p(nplus_pinned.data_ptr()), api.C.byref(h)))
        return h

    def timed(p, profile, clocks_index=None):
        """W untimed steps, then K steps between CUDA events on the handle's stream."""
        h = create(p)
        report = api.TransportReport()
        assembly_ms = api.C.c_double()
        api.check(lib.tfiga_transport_info(h, api.C.byref(assembly_ms), None, None))
        stream_ptr = api.C.c_void_p()
        api.check(lib.tfiga_transport_stream(h, api.C.byref(stream_ptr)))
        stream = torch.cuda.ExternalStream(stream_ptr.value)
        api.check(lib.tfiga_transport_step(h, args.warmup, api.C.byref(report)))
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        l0 = api.C.c_int64()
        api.check(lib.tfiga_transport_info(h, None, None, api.C.byref(l0)))
        if profile:
            api.check(lib.tfiga_transport_set_profiling(h, 1))
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local if clocks_index is None else clocks_index) as clocks:
            torch.cuda.synchronize()
            ev0.record(stream)
            api.check(lib.tfiga_transport_step(h, args.steps, api.C.byref(report)))
            ev1.record(stream)
            torch.cuda.synchronize()
        l1 = api.C.c_int64()
        api.check(lib.tfiga_transport_info(h, None, None, api.C.byref(l1)))
        fam_ms, fam_n = np.zeros(5), np.zeros(5, np.int64)
        if profile:
            api.check(lib.tfiga_transport_profile(h, api.C.c_void_p(fam_ms.ctypes.data),
                                                  api.C.c_void_p(fam_n.ctypes.data), 1))
            api.check(lib.tfiga_transport_set_profiling(h, 0))
        state = np.zeros(2 * n)
        api.check(lib.tfiga_transport_get_state(h, api.C.c_void_p(state.ctypes.data)))
        return {"h": h, "ms": ev0.elapsed_time(ev1), "report": report.as_dict(), "launches": l1.value - l0.value,
                "fam_ms": fam_ms, "fam_n": fam_n, "clocks": clocks.summary(), "state": state,
                "assembly_ms": assembly_ms.value}

    run = timed(params, profile=True)
    left = previous = None
    if not args.no_cpu_baseline and world == 1 and rank == 0:
        left = np.zeros(4 * mesh.blocks)
        previous = np.zeros(4 * mesh.blocks)
        api.check(lib.tfiga_transport_matrices(run["h"], api.C.c_void_p(left.ctypes.data),
                                               api.C.c_void_p(previous.ctypes.data)))
    api.check(lib.tfiga_transport_destroy(run["h"]))
    fp64_leg = None
    if fp32 and not args.no_fp64_leg:
        ref = timed(make_params(api.FP64), profile=False)
        api.check(lib.tfiga_transport_destroy(ref["h"]))
        diff = [float(np.linalg.norm(run["state"][f::2] - ref["state"][f::2]) / np.linalg.norm(ref["state"][f::2]))
                for f in (0, 1)]
        fp64_leg = {"value": replica_throughput(1, args.steps, ref["ms"]), "unit": "time steps/s",
                    "ms_per_step": ref["ms"] / args.steps,
                    "gmres_iterations_per_step": ref["report"]["total_iterations"] / args.steps,
                    "difference_after_%d_steps" % total_steps: {"N0": diff[0], "Nplus": diff[1]}}
    # e2e: the whole job through the C ABI from pinned host buffers, final state read back
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h = create(params)
    api.check(lib.tfiga_transport_step(h, total_steps, None))
    api.check(lib.tfiga_transport_get_state(h, api.C.c_void_p(out_pinned.data_ptr())))
    e2e_s = time.perf_counter() - t0
    api.check(lib.tfiga_transport_destroy(h))
    ms, e2e_ms = max_over_ranks(dist, [run["ms"], e2e_s * 1e3], "cuda")
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0
    hbm, _, peak_kind = peaks()
    timed_report = run["report"]
    its_per_step = timed_report["total_iterations"] / max(args.steps, 1)
    spmv_ms, spmv_n = float(run["fam_ms"][1]), int(run["fam_n"][1])
    orth_ms, orth_n = float(run["fam_ms"][2]), int(run["fam_n"][2])
    # one block-Jacobi SpMV launch: 2x2 values (32 B FP64, 16 B FP32) + column index (4 B) per block, row
    # offsets, the input vector and the output once (16 B per node each), the 2x2 inverse (32 B per node)
    spmv_bytes = mesh.blocks * (20 if fp32 else 36) + 4 * (n + 1) + 16 * n * 2 + 32 * n
    kernels = {}
    if spmv_n:
        a = spmv_bytes / (spmv_ms / spmv_n * 1e-3) / 1e9
        traffic = TRANSPORT_SPMV_FP32_DRAM_BYTES_PER_BLOCK * mesh.blocks if fp32 else None
        kernels["spmv_block_jacobi_2x2"] = {"bound": "hbm", "achieved": a, "peak": hbm, "unit": "GB/s",
                                            "frac": a / hbm, "traffic": traffic, "launches": spmv_n,
                                            "avg_ms": spmv_ms / spmv_n, "share": spmv_ms / ms,
                                            "algorithmic_bytes": spmv_bytes}
    if orth_n:
        kernels["krylov_orthogonalisation"] = {"launches": orth_n, "avg_ms": orth_ms / orth_n,
                                               "share": orth_ms / ms}
    roof = dict(kernels.get("spmv_block_jacobi_2x2", {}))
    roof["kernel"] = "spmv_block_jacobi_2x2"
    roof["peak_kind"] = f"{peak_kind} hbm_gbs"
    line = {
        "metric": TRANSPORT_METRIC, "value": replica_throughput(world, args.steps, ms), "unit": "time steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64" if fp32 else "f64",
        "data": "synthetic (seeded generator; velocity from one Navier-Stokes step of the same mesh)"
                if args.transport_mesh == "c3" else "synthetic (seeded generator; Poiseuille velocity)",
        "config": {"workload": "two-species transport on the " + desc, "elements": tube.mesh.elements, "nodes": n,
                   "block_nonzeros": mesh.blocks, "coefficients": TRANSPORT,
                   "solver": ("backward Euler, constant L and P assembled once; %s GMRES(%d) rtol 1e-8 "
                              "warm-started; %s" % (args.transport_preconditioner, args.transport_restart,
                                                    "FP32 copy of L in the Arnoldi SpMV, FP64 vectors, block "
                                                    "inverse and true residual" if fp32 else "FP64")),
                   "l2": "inputs larger than L2 (L %.2f GB)" % (mesh.blocks * 32 / 1e9),
                   "parallelism": "replicas only" if world > 1 else "single GPU"},
        "gmres_iterations_per_step": its_per_step, "final_l2": timed_report["final_l2"],
        "assembly_ms": run["assembly_ms"], "roofline": roof, "kernels": kernels, "fp64_gpu": fp64_leg,
        "gpu_launches": int(run["launches"]), "clocks": run["clocks"],
        "e2e": {"value": replica_throughput(world, total_steps, e2e_ms), "unit": "time steps/s",
                "h2d_bytes_per_step": (velocity.nbytes + mask.nbytes + n0.nbytes + nplus.nbytes) / total_steps,
                "d2h_bytes_per_step": 16 * n / total_steps,
                "includes": "create (uploads and assembly) + %d steps + final state read back" % total_steps},
    }
    if left is not None:
        try:
            line["cpu_baseline"] = transport_cpu_reference(mesh, left, previous, run["state"], its_per_step)
        except Exception as exc:  # noqa: BLE001 -- reported, not hidden
            line["cpu_baseline"] = {"value": None, "error": str(exc)}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c3", "c2", "c1", "c2-100", "c4", "c5", "transport"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--preconditioner", default="amg", choices=["amg", "block-jacobi"])
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "mixed", "tf32", "fp64"],
                    help="bf16x3: split-BF16 tensor-core tangent (hi + lo, three products); mixed: plain BF16; "
                         "tf32: TF32 operands; fp64: the FP64 solver alone")
    ap.add_argument("--no-fp64-leg", action="store_true")
    ap.add_argument("--tangent-kernel", default="auto", choices=["auto", "coefficients", "fused", "element"],
                    help="tensor-core tangent organisation (auto: the autotuner times both on the first tangent)")
    ap.add_argument("--learned", type=int, default=0,
                    help="time the learned FGMRES stage too, trained on pairs from this many further steps")
    ap.add_argument("--learned-pairs", type=int, default=256, help="pair store of the learned leg")
    ap.add_argument("--learned-adam", type=int, default=2000, help="Adam steps of the learned leg")
    ap.add_argument("--record-reference-counts", action="store_true",
                    help="print the Newton and GMRES counts of the reference's solver algorithm on the workload")
    ap.add_argument("--outlet-coupling", default="newton", choices=["newton", "outer"])
    ap.add_argument("--krylov-fp64-basis", action="store_true")
    ap.add_argument("--restart", type=int, default=64, help="FGMRES restart length")
    ap.add_argument("--tangent-reuse", type=float, default=100.0,
                    help="tensor-core modes: keep the previous Newton iteration's tangent while its contraction "
                         "is within this factor of its linear tolerance (0: off)")
    ap.add_argument("--forcing", default="ew", choices=["fixed", "ew"],
                    help="linear tolerance per Newton solve: fixed 1e-8, or Eisenstat-Walker forcing")
    ap.add_argument("--transport-precision", default="fp32", choices=["fp64", "fp32"],
                    help="transport workload: FP32 copy of L for the Arnoldi SpMV (FP64 true residual); with fp32 "
                         "the FP64 solver is timed too (fp64_gpu) unless --no-fp64-leg")
    ap.add_argument("--transport-restart", type=int, default=50, help="transport workload: GMRES restart")
    ap.add_argument("--transport-preconditioner", default="block-jacobi", choices=["block-jacobi", "flow-lines"],
                    help="transport workload: the reference's block-Jacobi or the flow-line factors")
    ap.add_argument("--transport-mesh", default="c3", choices=["c3", "c2-100"],
                    help="transport workload mesh: c3 with the velocity of one Navier-Stokes step, or the "
                         "12,800-element tube section with its Poiseuille profile at 0.15 m/s mean (profiling case)")
    ap.add_argument("--ref-budget", type=float, default=20.0,
                    help="seconds of CPU work per sample of the CPU reference path")
    ap.add_argument("--newton-rtol", type=float, default=None,
                    help="Newton test ||r|| <= rtol ||r_0|| of every arm (FP64 residual); default 1e-10, 1e-11 "
                         "for the binary tree")
    ap.add_argument("--amg-coarse-period", type=int, default=None,
                    help="AMG refreshes per rebuild of the dense coarse inverse; default 3, 9 for the binary "
                         "tree (a 7k-unknown coarse level)")
    args = ap.parse_args()
    if args.newton_rtol is None:
        args.newton_rtol = NEWTON_RTOL.get(args.workload, 1e-10)
    if args.amg_coarse_period is None:
        args.amg_coarse_period = COARSE_PERIOD.get(args.workload, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, world, rank)
    if args.record_reference_counts:
        return record_reference_counts(args)
    if args.workload == "transport":
        return run_transport(args, world, rank, local)

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    from tubularflowiga_b200 import api

    tube, desc, wave = workload(args.workload, world, rank)
    n = tube.mesh.nodes
    mesh = api.Mesh(tube.mesh)
    amg = args.preconditioner == "amg"
    mixed = args.precision in ("mixed", "bf16x3", "tf32")
    if mixed and not amg:
        raise SystemExit("--precision mixed needs --preconditioner amg")
    solver_kw = dict(density=RHO, viscosity=MU, dt=step_dt(args.workload),
                     nonlinear_rtol=args.newton_rtol, nonlinear_atol=1e-300,
                     mass_rtol=1e-3,
                     gmres_restart=args.restart, gmres_max_iterations=5000, gmres_rtol=1e-8,
                     preconditioner=api.AMG if amg else api.BLOCK_JACOBI,
                     amg_coarse_period=args.amg_coarse_period, krylov_fp64_basis=int(args.krylov_fp64_basis),
                     newton_forcing=int(args.forcing == "ew"), tangent_reuse_factor=args.tangent_reuse,
                     tangent_kernel={"auto": api.TANGENT_AUTO, "coefficients": api.TANGENT_COEFFICIENTS,
                                     "fused": api.TANGENT_FUSED, "element": api.TANGENT_ELEMENT}[args.tangent_kernel])
    precision = {"mixed": api.MIXED, "bf16x3": api.MIXED_BF16X3, "tf32": api.MIXED_TF32,
                 "fp64": api.FP64}[args.precision]
    ns = api.NavierStokes(mesh, precision=precision, **solver_kw)
    batched = args.workload == "c5"
    if batched:
        ns.set_segments(tube.node_offset)
    dt = ns.params.dt
    vmask, pmask, velocity_at = boundary(tube, wave)

    def bc(step):
        return velocity_at((step + 1) * dt).ravel()

    ns.set_dirichlet(vmask, pmask, velocity_at(0.0))
    models = outlet_models(args.workload)
    fixed_tractions = {} if models else {label: 0.0 for label in getattr(tube, "outlet_labels", (2,))}
    ns.set_tractions(fixed_tractions)
    s0 = api.initial_state(vmask, velocity_at(0.0))
    ns.set_state(s0, s0)
    outlets = [api.Outlet(**m.as_dict()) for m in models] if models else None
    stream = torch.cuda.ExternalStream(ns.stream())
    total = args.warmup + args.steps
    # every step's Dirichlet values resident in HBM before timing (value leg)
    bc_dev = torch.tensor(np.stack([bc(k) for k in range(total)]), dtype=torch.float64, device="cuda")
    bc_host = torch.tensor(np.stack([bc(k) for k in range(total)]), dtype=torch.float64).pin_memory()
    out_host = torch.empty(4 * n, dtype=torch.float64).pin_memory()

    reports = []

    def do_step(solver, solver_outlets, k, host=False, record=None):
        if host:
            api.check(api.lib().tfiga_ns_set_dirichlet_values(solver._h, api.C.c_void_p(bc_host[k].data_ptr()),
                                                              None))
        else:
            api.check(api.lib().tfiga_ns_set_dirichlet_values(solver._h, api.C.c_void_p(bc_dev[k].data_ptr()),
                                                              None))
        solver.commit_step()
        r = outlet_step(solver, solver_outlets, args.outlet_coupling) if solver_outlets else solver.step()
        if record is not None:
            record.append(r)
        if host:
            api.check(api.lib().tfiga_ns_get_state(solver._h, api.C.c_void_p(out_host.data_ptr())))

    states = []                                   # the arm's state after every step (error legs)
    for k in range(args.warmup):
        do_step(ns, outlets, k)
        states.append(ns.get_state())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    timed_start = ns.get_state()
    timed_outlets = [o.as_dict() for o in outlets] if outlets else None

    def restart():
        ns.set_state(timed_start, timed_start)
        if outlets:
            for o, d in zip(outlets, timed_outlets):
                for key, v in d.items():
                    setattr(o, key, v)

    # value leg: CUDA events on the solver stream, every input resident in HBM, no instrumentation
    ns.set_profiling(False)
    launches0 = ns.launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clocks:
        torch.cuda.synchronize()
        ev0.record(stream)
        for k in range(args.warmup, total):
            do_step(ns, outlets, k, record=reports)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = ns.launches() - launches0
    timed_reports = list(reports)
    tangents = None

    # profile leg: the same steps again from the same state with per-family CUDA events on the solver
    # stream (kernel rooflines and step shares, against this pass's own duration); the state after
    # every step is kept for the error legs
    restart()
    ns.set_profiling(True)
    ns.profile(reset=True)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    prof_ms = 0.0
    for k in range(args.warmup, total):
        torch.cuda.synchronize()
        p0.record(stream)
        do_step(ns, outlets, k)
        p1.record(stream)
        torch.cuda.synchronize()
        prof_ms += p0.elapsed_time(p1)
        states.append(ns.get_state())
    prof_bytes = ns.profile_bytes()
    orth_algo, orth_moved = prof_bytes["krylov_orthogonalisation"]
    spmv_counted = prof_bytes["spmv"][0]     # the per-tube solver counts the rows of open tubes only
    prof = ns.profile(reset=True)
    ns.set_profiling(False)

    # e2e leg: same steps from the same state through the C ABI, inputs from pinned host memory, the
    # state read back every step
    if dist:
        dist.barrier()
    restart()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for k in range(args.warmup, total):
        do_step(ns, outlets, k, host=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)

    # learned leg (--learned N): the learned FGMRES stage in the timed path.  Training pairs from N further
    # untimed steps after the timed ones (flexible-GMRES pairs w = A z and Newton pairs), the residual loss
    # through the bound Jacobian, --learned-adam Adam steps, the fitted output gain; then the timed steps
    # again from the same starting state with the stage attached, between CUDA events.
    learned_leg = None
    if args.learned > 0 and amg and not batched:
        net = api.Learned(ns, layers=3, seed=0, linear=False)
        net.set_capacity(args.learned_pairs)
        net.set_loss(False)
        net.attach(use=False, collect=True)
        t_train = time.perf_counter()
        for k in range(args.learned):
            ns.set_dirichlet_values(bc(total + k))
            ns.commit_step()
            outlet_step(ns, outlets, args.outlet_coupling) if outlets else ns.step()
        net.fit_scales()
        loss0 = net.evaluate()
        net.train(args.learned_adam, 1e-3)
        loss1 = net.evaluate()
        gain = net.fit_gain()
        train_s = time.perf_counter() - t_train
        restart()
        net.attach(use=True, collect=False)
        learned_reports = []
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        l0.record(stream)
        for k in range(args.warmup, total):
            do_step(ns, outlets, k, record=learned_reports)
        l1.record(stream)
        torch.cuda.synchronize()
        learned_ms = l0.elapsed_time(l1)
        fallbacks = net.fallbacks()
        net.detach()
        net.close()
        newton_l = sum(r["newton_iterations"] for r in learned_reports)
        learned_leg = {"value": replica_throughput(world, args.steps, learned_ms), "unit": "time steps/s",
                       "ms_per_step": learned_ms / args.steps, "newton_per_step": newton_l / args.steps,
                       "linear_iterations_per_newton": sum(r["linear_iterations"] for r in learned_reports)
                       / max(1, newton_l),
                       "linear_iterations_per_step": [r["linear_iterations"] for r in learned_reports],
                       "amg_only_linear_iterations_per_step": [r["linear_iterations"] for r in timed_reports],
                       "fallbacks": fallbacks,
                       "training": {"steps": args.learned, "pairs": args.learned_pairs, "adam_steps": args.learned_adam,
                                    "loss": [loss0, loss1], "output_gain": gain, "seconds": train_s},
                       "note": "same timed steps and starting state as the mixed arm, AMG + learned stage "
                               "(3-layer message passing, width 64, BF16 weights) in the flexible GMRES"}

    tube_metrics = None
    amg_levels = ns.amg_info() if amg else None
    tangent_info = ns.tangent_kernel() if mixed else None
    if batched:
        done, residuals = ns.segment_status()
        specs = c5_specs()
        tube_metrics = [{"tube": int(tube.tube_ids[k]), "rank": rank,
                         "elements": int(tube.element_offset[k + 1] - tube.element_offset[k]),
                         "helical": bool(specs[tube.tube_ids[k]].curvature_radius > 0),
                         "final_residual": float(residuals[k]), "passed": bool(done[k])}
                        for k in range(len(tube.tubes))]
    if batched or args.workload == "c4":
        ns.close()              # the FP64 arm below needs the memory; its errors use the saved states

    # plain FP64 GPU solver on the same steps: the same Dirichlet sequence and starting state, the same
    # Newton test, residual-first check, tangent-reuse rule, outlet coupling and restart; the warm-up
    # steps untimed, the timed steps between CUDA events.  Run with the mixed arm's linear-tolerance mode
    # and with the fixed tolerance 1e-8 of the reference; the faster is the baseline.  The mixed state
    # after every step is compared with the FP64 run of the same mode.
    fp64_leg = None
    if mixed and not args.no_fp64_leg:
        def fp64_run(forcing):
            kw = dict(solver_kw, newton_forcing=int(forcing == "ew"))
            ref = api.NavierStokes(mesh, precision=api.FP64, **kw)
            if batched:
                ref.set_segments(tube.node_offset)          # per-tube Newton tests and FGMRES, as the mixed arm
            ref.set_dirichlet(vmask, pmask, velocity_at(0.0))
            ref.set_tractions(fixed_tractions)
            ref.set_state(s0, s0)
            ref_outlets = [api.Outlet(**m.as_dict()) for m in models] if models else None
            rstream = torch.cuda.ExternalStream(ref.stream())
            errors, fp64_reports = [], []
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            fp64_ms = 0.0
            for k in range(total):
                torch.cuda.synchronize()
                a0.record(rstream)
                do_step(ref, ref_outlets, k, record=fp64_reports if k >= args.warmup else None)
                a1.record(rstream)
                torch.cuda.synchronize()
                if k >= args.warmup:
                    fp64_ms += a0.elapsed_time(a1)
                r64 = ref.get_state().reshape(-1, 4)
                mx = states[k].reshape(-1, 4)
                errors.append({"step": k,
                               "velocity": float(np.linalg.norm(mx[:, :3] - r64[:, :3]) / np.linalg.norm(r64[:, :3])),
                               "pressure": float(np.linalg.norm(mx[:, 3] - r64[:, 3]) / np.linalg.norm(r64[:, 3]))})
            if batched:
                # per-tube relative L2 error of the mixed state against this run after the last step
                r64 = ref.get_state().reshape(-1, 4)
                mx = states[total - 1].reshape(-1, 4)
                per_tube = []
                for k in range(len(tube.tubes)):
                    lo, hi = tube.node_offset[k], tube.node_offset[k + 1]
                    per_tube.append({"velocity": float(np.linalg.norm(mx[lo:hi, :3] - r64[lo:hi, :3])
                                                       / np.linalg.norm(r64[lo:hi, :3])),
                                     "pressure": float(np.linalg.norm(mx[lo:hi, 3] - r64[lo:hi, 3])
                                                       / max(np.linalg.norm(r64[lo:hi, 3]), 1e-300))})
            ref.close()
            newton_n = np.sum([r["newton_iterations"] for r in fp64_reports])
            return {"value": args.steps / (fp64_ms / 1e3), "unit": "time steps/s", "forcing": forcing,
                    "steps": args.steps, "timed_steps": [args.warmup, total - 1],
                    "ms_per_step": fp64_ms / args.steps,
                    "newton_per_step": float(newton_n / args.steps),
                    "linear_iterations_per_newton": float(np.sum([r["linear_iterations"] for r in fp64_reports])
                                                          / max(1, newton_n)),
                    "error_vs_fp64_per_step": errors,
                    "per_tube_error": per_tube if batched else None,
                    "max_error": {"velocity": max(e["velocity"] for e in errors),
                                  "pressure": max(e["pressure"] for e in errors)}}

        runs = {mode: fp64_run(mode) for mode in dict.fromkeys([args.forcing, "fixed"])}
        best = max(runs.values(), key=lambda r: r["value"] or 0.0)
        same = runs[args.forcing]
        fp64_leg = {k: v for k, v in best.items() if k not in ("error_vs_fp64_per_step", "max_error",
                                                               "per_tube_error")}
        if batched and tube_metrics is not None:
            for m, err in zip(tube_metrics, same["per_tube_error"]):
                m["error_vs_fp64"] = err
        fp64_leg["variants"] = {m: {k: r[k] for k in ("value", "ms_per_step", "newton_per_step",
                                                       "linear_iterations_per_newton", "max_error")}
                                for m, r in runs.items()}
        fp64_leg["error_vs_fp64_per_step"] = same["error_vs_fp64_per_step"]
        fp64_leg["max_error"] = same["max_error"]
        fp64_leg["error_reference"] = ("the FP64 run with the mixed arm's own settings (%s linear tolerance, "
                                       "Newton rel.res %g), every step from the same initial state"
                                       % (args.forcing, args.newton_rtol))
        fp64_leg["same_as_mixed"] = ("same steps (warm-up %d untimed, %d timed), Dirichlet sequence, outlet "
                                     "coupling, Newton test%s, residual-first check, tangent-reuse factor %g and "
                                     "FGMRES restart; precision FP64 everywhere" % (args.warmup, args.steps,
                                                                                    " and FGMRES per tube" if batched
                                                                                    else "", args.tangent_reuse))

    ms, e2e_ms = max_over_ranks(dist, [ms, e2e_ms], "cuda")
    if batched:
        tube_metrics = gather_tube_metrics(dist, tube.tube_ids, tube_metrics)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    hbm, bf16, peak_kind = peaks()
    bf16_sustained = sustained_bf16()
    b_spmv, b_bjac, f_asm = algorithmic_counts(tube, mesh.blocks)
    spmv_ms, spmv_n = prof["spmv"]
    asm_ms, asm_n = prof["assembly"]
    orth_ms, orth_n = prof["krylov_orthogonalisation"]
    amg_ms, amg_n = prof["amg_vcycle"]
    res_ms, res_n = prof.get("residual", (0.0, 0))
    kernels = {}
    if mixed:
        # FP32 Jacobian: 4-byte values in every pass over the matrix
        b_spmv -= mesh.blocks * 16 * 4
    spmv_bytes = b_spmv if amg else b_spmv + b_bjac
    spmv_name = "spmv" if amg else "spmv_block_jacobi"
    masked = spmv_counted > 0 and spmv_n > 0
    if masked:
        # tube batch: each Arnoldi SpMV skips the block rows of tubes that have stopped, so its bytes are
        # those of the open tubes' rows (counted by the solver at its host waits, a lower bound)
        spmv_bytes = spmv_counted / spmv_n
    if spmv_n:
        a = spmv_bytes / (spmv_ms / spmv_n * 1e-3) / 1e9
        traffic = (SPMV_FP32_DRAM_BYTES_PER_BLOCK * mesh.blocks if (mixed and amg) else None) if not masked else None
        kernels[spmv_name] = {"bound": "hbm", "achieved": a, "peak": hbm, "unit": "GB/s",
                              "frac": a / hbm, "traffic": traffic, "launches": spmv_n,
                              "avg_ms": spmv_ms / spmv_n, "share": spmv_ms / prof_ms,
                              "algorithmic_bytes": spmv_bytes}
    if amg_n:
        # one two-level application: restriction (b, mask, aggregate order), the dense coarse inverse
        # (dn^2 doubles), and the fused fine-level correction, which reads b, the mask, the aggregate
        # map, the A P blocks with their column indices and row offsets, the block-Jacobi inverse
        # (128 B per node), and writes z.  The smoother's residual goes through A P, so no pass over A.
        info = amg_levels
        dn = 4 * info["nodes"][-1]
        ap = info["transfer_blocks"]
        ap_entry = 4 if mixed else 8        # A P is stored in the fine matrix's precision
        vbytes = (2 * 4 * n * 8 + 4 * n) + dn * dn * 8 + (3 * 4 * n * 8 + 2 * 4 * n + ap * (16 * ap_entry + 4)
                                                          + n * 128)
        a = vbytes / (amg_ms / amg_n * 1e-3) / 1e9
        kernels["amg_vcycle"] = {"bound": "hbm", "achieved": a, "peak": hbm, "unit": "GB/s", "frac": a / hbm,
                                 "traffic": None, "launches": amg_n, "avg_ms": amg_ms / amg_n,
                                 "share": amg_ms / prof_ms, "algorithmic_bytes": vbytes,
                                 "levels": amg_levels}
    asm_name = "assembly_tc" if mixed else "assembly_fp64"
    if asm_n and mixed:
        # tensor-core element contraction: F_e = 8192 nen^2 MMA flops per element, timed inside the long
        # Newton step, so against the sustained bf16 peak
        a = f_asm / (asm_ms / asm_n * 1e-3) / 1e12
        kernels[asm_name] = {"bound": "tensor", "achieved": a, "peak": bf16_sustained, "unit": "TFLOP/s",
                             "frac": a / bf16_sustained, "traffic": None, "launches": asm_n,
                             "avg_ms": asm_ms / asm_n, "share": asm_ms / prof_ms,
                             "peak_kind": f"{peak_kind} bf16_tflops_sustained"}
    elif asm_n:
        a = f_asm / (asm_ms / asm_n * 1e-3) / 1e12
        kernels[asm_name] = {"bound": "fp64", "achieved": a, "peak": 37.0, "unit": "TFLOP/s",
                             "frac": a / 37.0, "traffic": None, "launches": asm_n,
                             "avg_ms": asm_ms / asm_n, "share": asm_ms / prof_ms,
                             "peak_note": "nominal B200 FP64 (no measured FP64 peak on this pool)"}
    if res_n:
        # FP64 residual (+ point coefficients in the tensor-core modes): per element it reads the FP64
        # basis tables (5 x 64 x 64 doubles) and the point data (64 x 11 doubles) and, in the tensor-core
        # modes, writes the coefficients of four row fields (4 x 80 x 64 floats)
        rbytes = tube.mesh.elements * (5 * 64 * 64 * 8 + 64 * 11 * 8 + (4 * 80 * 64 * 4 if mixed else 0))
        a = rbytes / (res_ms / res_n * 1e-3) / 1e9
        kernels["residual_point"] = {"bound": "hbm", "achieved": a, "peak": hbm, "unit": "GB/s", "frac": a / hbm,
                                     "traffic": None, "launches": res_n, "avg_ms": res_ms / res_n,
                                     "share": res_ms / prof_ms, "algorithmic_bytes": rbytes}
    if orth_n:
        # algorithmic bytes of Arnoldi step j as the solver accounts them: s_v N (2j + 7) (one dot
        # pass, one update pass, the normalisation; s_v = 4 for the FP32 basis of the mixed solver)
        # + 8 N for the stored preconditioned vector.  Classical Gram-Schmidt twice moves about twice
        # that (moved_*); achieved uses the algorithmic count.
        algo = orth_algo
        a = algo / (orth_ms * 1e-3) / 1e9
        kernels["krylov_orthogonalisation"] = {"bound": "hbm", "achieved": a, "peak": hbm, "unit": "GB/s",
                                               "frac": a / hbm, "traffic": None, "launches": orth_n,
                                               "avg_ms": orth_ms / orth_n, "share": orth_ms / prof_ms,
                                               "algorithmic_bytes_per_launch": algo / orth_n,
                                               "moved_bytes_per_launch": orth_moved / orth_n,
                                               "moved_gbs": orth_moved / (orth_ms * 1e-3) / 1e9}
    # the rest of the step: AMG set-up for each new Jacobian and the Newton / FGMRES vector bookkeeping
    # (zeroing, traction, diagnostics, Dirichlet rows, norms, restarts, state updates, outlet coupling)
    for name in ("amg_setup", "newton_vectors"):
        ms_f, n_f = prof.get(name, (0.0, 0))
        if n_f:
            kernels[name] = {"bound": None, "launches": n_f, "ms_per_step": ms_f / args.steps,
                             "share": ms_f / prof_ms}
    attributed = sum(k.get("share", 0.0) for k in kernels.values())
    dominant = max((spmv_name, asm_name, "amg_vcycle", "krylov_orthogonalisation", "residual_point"),
                   key=lambda k: kernels.get(k, {}).get("share", 0))
    roof = dict(kernels[dominant])
    roof["kernel"] = dominant
    roof["timing"] = "per-launch CUDA events of an instrumented repeat of the timed steps"
    if roof["bound"] == "hbm":
        roof["peak_kind"] = f"{peak_kind} hbm_gbs"
    steps_per_s = replica_throughput(world, args.steps, ms)
    newton = np.mean([r["newton_iterations"] for r in timed_reports])
    linear = np.sum([r["linear_iterations"] for r in timed_reports]) / max(1, np.sum(
        [r["newton_iterations"] for r in timed_reports]))
    line = {
        "metric": METRIC, "value": steps_per_s, "unit": "time steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": ("tf32-tc/f32/f64" if args.precision == "tf32" else "bf16-tc/f32/f64") if mixed else "f64",
        "data": "synthetic (seeded generator; the reference publishes no dataset for this metric)",
        "config": {"workload": desc, "elements": tube.mesh.elements, "nodes": n, "block_nonzeros": mesh.blocks,
                   "solver": (("mixed: tcgen05 %s tangent (FP32 accumulate), FP32 Jacobian, FP64 residual and "
                               "refinement; " % {"bf16x3": "split-BF16 (hi + lo, 3 products)", "tf32": "TF32",
                                                 "mixed": "BF16"}.get(args.precision, "") if mixed
                               else "plain FP64: ") +
                              "exact-tangent Newton to rel.res %g (FP64 residual, tested before the tangent is "
                              "assembled), " % args.newton_rtol +
                              ("inexact Newton (Eisenstat-Walker forcing tolerances, Dirichlet values lifted "
                               "into the state at step start), " if args.forcing == "ew" else "") +
                              ("tangent reused while Newton contracts within %g x the linear tolerance, "
                               % args.tangent_reuse if args.tangent_reuse > 0 else "") +
                              ("RCR outlets coupled by the relaxed fixed point (relaxation %g, tolerance "
                               "1e-8 + 1e-6 |P|; %s), " % (OUTLET_RELAXATION,
                                                          "pressures updated inside the Newton loop"
                                                          if args.outlet_coupling == "newton" else
                                                          "the reference's outer loop") if models else "") +
                              ("point-block two-level AMG-preconditioned FGMRES(%d)%s" % (args.restart, " rtol 1e-8" if args.forcing == "fixed"
                                                                                   else "") if amg else
                               "block-Jacobi GMRES(%d) rtol 1e-8" % args.restart)),
                   "newton_rtol": args.newton_rtol, "amg_coarse_period": args.amg_coarse_period,
                   "l2": "inputs larger than L2 (matrix %.2f GB)" % (mesh.blocks * 128 / 1e9),
                   "parallelism": "replicas only" if world > 1 else "single GPU"},
        "newton_per_step": float(newton), "linear_iterations_per_newton": float(linear),
        "outlets": ([{k: o.as_dict()[k] for k in ("label", "flow", "pressure", "capacitor_pressure")}
                     for o in outlets] if outlets else None),
        "outlet_iterations_per_step": (float(np.mean([r.get("outlet_iterations", r.get("pressure_updates", 0))
                                                      for r in timed_reports])) if outlets else None),
        "roofline": roof, "kernels": kernels,
        "profile_pass": {"ms_per_step": prof_ms / args.steps, "attributed_share": attributed,
                         "note": "kernel families timed in a repeat of the timed steps; shares are of that "
                                 "pass's duration"},
        "fp64_gpu": fp64_leg,
        "spmv_gbs": kernels.get(spmv_name, {}).get("achieved"),
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "e2e": {"value": replica_throughput(world, args.steps, e2e_ms), "unit": "time steps/s",
                "h2d_bytes_per_step": 3 * n * 8, "d2h_bytes_per_step": 4 * n * 8},
    }
    if fp64_leg:
        line["mixed_over_fp64"] = {m: steps_per_s / v["value"] for m, v in fp64_leg["variants"].items()}
    if tangent_info is not None:
        line["tangent_kernel"] = tangent_info
    if learned_leg is not None:
        learned_leg["over_mixed"] = learned_leg["value"] / steps_per_s
        line["learned"] = learned_leg
    if batched:
        line["tubes"] = tube_metrics
    if not args.no_cpu_baseline and world == 1:
        st = states[-1]
        try:
            rn, rl = reference_counts(args.workload) if args.workload in REFERENCE_COUNTS else (newton, linear)
            cpu = CpuReference(tube, st, st)
            cpu.calibrate(args.ref_budget)
            cb = cpu.sample(rn, rl)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as exc:  # noqa: BLE001 -- reported, not hidden
            line["cpu_baseline"] = {"value": None, "error": str(exc)}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0

if __name__ == "__main__":
    sys.exit(main())
