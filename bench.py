"""Benchmark of the B200 Z4c path: FP64 Z4c zone-updates/s.

Workload (one GPU): one Schwarzschild puncture (M = 1, precollapsed lapse) on
a uniform mesh of 128^3 cells split into 512 MeshBlocks of 16^3 (nghost 4),
domain [-16, 16]^3, extrapolate_outflow boundaries, 1+log slicing and
Gamma-driver shift (eta = 2), kappa1 = 0.02, KO dissipation 0.02, low-storage
RK4, Courant 0.25.  One step = one full RK4 step of the whole mesh (four
stages: fused RHS+KO+stage update, ghost exchange, boundary conditions,
AlgConstr; Z4cToADM after the last stage, as the task list runs it every
step), replayed from a captured CUDA graph.  A zone-update is one cell
advanced one full step (the reference's zone-cycle, main.cpp:239).

At N = 1 the line also carries "bbh_smr": the refined binary-puncture mesh
below (3,424 MeshBlocks on seven levels), its own zone-updates/s and the time
of one multilevel ghost fill (--no-smr skips it); and "bbh_amr": the adaptive
binary run (the same punctures on 8^3 root MeshBlocks, seven levels refined
by the reference's Linf_box_in_box criterion around the puncture trackers,
200 cycles with the block list changing), timed whole, regrids included, with
the block count after every regrid (--no-amr skips it).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank evolves its own replica of the mesh
("replicas only": the path has no cross-GPU exchange on one-GPU meshes); the
value is the total over ranks divided by the slowest rank's time.

  python bench.py --workload bbh_smr [--steps K] [--warmup W]
  python bench.py --workload bbh_amr [--steps K] [--warmup W]

print those measurements alone as a line of their own; one GPU.

The CPU baseline and --impl reference time the reference's own OpenMP build
(oracle/_ref/athena_ref_native: the reference's g++ flags with -march=native
of the machine that built it) on all host cores; a host whose cores lack one
of that machine's CPU flags times the portable build (-march=x86-64-v3)
instead, and the line says which.
"""
import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gr-athena_b200"))

METRIC = "FP64 Z4c zone-updates/s"
WORKLOAD = dict(workload="single puncture M=1, 128^3 cells as 512 MeshBlocks of 16^3, "
                         "nghost=4, [-16,16]^3, extrapolate_outflow, 1+log + Gamma-driver "
                         "(eta=2), kappa1=0.02, diss=0.02, rk4 (2S), cfl 0.25",
                nb=[8, 8, 8], nx=[16, 16, 16], xmin=[-16.0] * 3, xmax=[16.0] * 3)
PARAMS = dict(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, damp_kappa2=0.0,
              shift_eta=2.0, r_max_con=1e300)
CFL = 0.25
# jobs (one RK4 step each, from and to host memory) of the end-to-end measurement
E2E_JOBS = 16
# RK4 steps of the reference CPU build in the cpu_baseline leg (about 2 s of
# work per step on 16 cores)
CPU_SAMPLE_STEPS = 8
# timed RK4 steps of the refined-mesh measurement inside the headline run
# (about 150 ms each)
SMR_STEPS = 10
# timed RK4 steps of the robust-stability measurement in the headline run
RS_STEPS = 20
# cycles of the adaptive binary run (200 as the benchmark states; about 160 ms each),
# and of its shifted-gauge variant
AMR_STEPS = 200
AMR_SHIFTED_STEPS = 60
# initial shift of the shifted-gauge variant: the same data in a gauge whose
# constant beta^x carries both trackers about 0.25 along +x (the Gamma-driver
# damps it with eta = 2), past the first refinement boundaries at 0.094
AMR_SHIFT = (-0.5, 0.0, 0.0)
# Algorithmic HBM bytes of one fused stage per interior vertex: read u and u1,
# write u' and u1' (22 FP64 variables each).
STAGE_BYTES_PER_POINT = 4 * 22 * 8
# FP64 operations of the reference algorithm per interior vertex per stage on
# 16^3 MeshBlocks: 7697 for PrepareZ4cDerivatives + Z4cRHS with KO, counted by
# running the oracle with a counting number type (oracle/opcount), plus 154
# for the low-storage stage update (7 per variable).
FP64_OPS_PER_POINT_STAGE = 7697 + 154
# The launches of one fused stage and their measured DRAM traffic per interior
# vertex (ncu dram__bytes_read.sum + dram__bytes_write.sum summed over them,
# 64-block capture scaled by the vertex count; see profiles/).
STAGE_KERNELS = {0: "k_prep, k_ricci, k_adv, k_main, k_ko_stage_ls",
                 1: "k_prep, k_ricci_fast, k_main_fast, k_col_fast"}
# FP64 operations of PrepareZ4cDerivatives + Z4cWeyl per interior vertex
# (oracle/opcount), for the psi4 diagnostics line.
FP64_OPS_PER_POINT_WEYL = 7409
# psi4 extraction spheres of the diagnostics: (radius, nlev, lmax) inside
# the [-16,16]^3 domain
WAVE_SPHERES = ((6.0, 30, 8), (12.0, 30, 8))
STAGE_TRAFFIC_PER_POINT = {0: 1350.0e6 / (64 * 17 ** 3), 1: 1025.6e6 / (64 * 17 ** 3),
                           # the contracted stage on a merged grid: ncu on the 97^3-vertex
                           # grid of 6^3 blocks (registers 204 MB), per vertex
                           "merged": 2153.4e6 / 97 ** 3}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint-step measurements of the headline line")
    ap.add_argument("--no-smr", action="store_true",
                    help="skip the refined binary-puncture measurement of the headline line")
    ap.add_argument("--no-amr", action="store_true",
                    help="skip the adaptive binary-puncture run of the headline line")
    ap.add_argument("--contract", type=int, default=1, choices=[0, 1],
                    help="1: the contracted path (fused multiply-adds, four launches per "
                         "stage; the headline); 0: the exact path, bit for bit the "
                         "reference's arithmetic (also measured in the headline line)")
    ap.add_argument("--nb", type=int, default=8,
                    help="MeshBlocks per axis (8 = the 128^3 workload; smaller for profiling)")
    ap.add_argument("--profile-run", action="store_true",
                    help="graph-captured steps and the stage kernel only (for ncu)")
    ap.add_argument("--stage-profile", action="store_true",
                    help="profiling aid: only the contracted stage sequence, three times, on "
                         "the merged grid of --nb^3 MeshBlocks (one block of 16 nb cells)")
    ap.add_argument("--shape", default=None,
                    help="launch shape point_threads,column_threads,column_slabs instead of "
                         "the autotuner's pick (profiling under ncu, whose serialised launches "
                         "would mislead the autotuner)")
    ap.add_argument("--workload", default="uniform",
                    choices=["uniform", "bbh_smr", "bbh_amr", "bbh_adjoint"],
                    help="bbh_smr: binary punctures on a statically refined mesh of 7 levels; "
                         "bbh_amr: the adaptive run (separate measurements, not the headline "
                         "line)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region


class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baselines


def reference_deck(nlim, threads):
    nb, nx = WORKLOAD["nb"], WORKLOAD["nx"]
    lines = ["<job>", "problem_id = bench", "<z4c>"]
    lines += [f"{k} = {v!r}" for k, v in PARAMS.items()]
    lines += ["<task_triggers>", "adjust_mesh_dt = false", "<time>", f"cfl_number = {CFL}",
              "tlim = 1e10", f"nlim = {nlim}", "integrator = rk4", "ncycle_out = 1000000",
              "<mesh>"]
    for a in range(3):
        d = a + 1
        lines += [f"nx{d} = {nb[a] * nx[a]}", f"x{d}min = {WORKLOAD['xmin'][a]!r}",
                  f"x{d}max = {WORKLOAD['xmax'][a]!r}", f"ix{d}_bc = extrapolate_outflow",
                  f"ox{d}_bc = extrapolate_outflow"]
    lines += ["refinement = none", f"num_threads = {threads}", "<meshblock>"]
    lines += [f"nx{a + 1} = {nx[a]}" for a in range(3)]
    lines += ["<problem>", "test = one_puncture", "punc_ADM_mass = 1.0"]
    return "\n".join(lines) + "\n"


def reference_binary():
    """The reference build to time and how it was built: athena_ref_native
    (the reference's own g++ flags, -march=native of the machine that built
    it) when this host's cores have every CPU flag of that machine, else the
    portable athena_ref (-O3 -march=x86-64-v3)."""
    ref = os.path.join(ROOT, "oracle", "_ref")
    native = os.path.join(ref, "athena_ref_native")
    if os.path.exists(native) and os.path.exists(native + ".isa"):
        with open(native + ".isa") as f:
            need = set(f.read().split())
        have = set()
        try:
            with open("/proc/cpuinfo") as f:
                for line in f:
                    if line.startswith("flags"):
                        have = set(line.split(":", 1)[1].split())
                        break
        except OSError:
            pass
        if need and need <= have:
            return native, ("reference g++ flags (-O3 -fwhole-program -flto=auto "
                            "-fprefetch-loop-arrays -march=native -ffp-contract=off)")
        missing = sorted(need - have)[:5]
        note = f"portable build: this host lacks CPU flags of the native build ({missing})"
    else:
        note = "portable build (-O3 -march=x86-64-v3): no native build present"
    exe = os.path.join(ref, "athena_ref")
    return (exe if os.path.exists(exe) else None), note


def run_reference_cpu(nlim, threads):
    """Times the reference's own OpenMP CPU build (oracle/_ref, compiled from
    the reference sources) on the benchmark workload and returns its printed
    zone-cycles/omp_wsecond (main.hpp:739-742) and the build used."""
    exe, build = reference_binary()
    if exe is None:
        return None, build
    with tempfile.TemporaryDirectory() as tmp:
        inp = os.path.join(tmp, "bench.inp")
        with open(inp, "w") as f:
            f.write(reference_deck(nlim, threads))
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        out = subprocess.run([exe, "-i", inp], cwd=tmp, capture_output=True, text=True,
                             env=env, timeout=1800)
    m = re.search(r"zone-cycles/omp_wsecond\s*=\s*([0-9.eE+-]+)", out.stdout)
    if not m:
        return None, build
    return float(m.group(1)), build


def run_oracle_cpu(max_seconds=20.0):
    """Fallback CPU baseline: the C restatement (oracle/, single thread) on
    whole MeshBlocks of the workload until max_seconds of work."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import z4c_oracle as O
    from z4c_b200 import Mesh
    from z4c_b200 import initial_data as ID
    mesh = Mesh(WORKLOAD["nb"], WORKLOAD["nx"], WORKLOAD["xmin"], WORKLOAD["xmax"], "outflow")
    p = O.default_params(**PARAMS)
    xs, dxs = mesh.block_coords(0)
    blk = O.Block(mesh.nx, dxs, xs)
    u = np.ones((22,) + tuple(reversed(mesh.nn)))
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < max_seconds and n < 64:
        O.rhs(blk, p, u)
        n += 1
    el = time.perf_counter() - t0
    zones = 16 ** 3
    # one zone-update = 4 RHS evaluations (the stage updates are negligible)
    return n * zones / el / 4.0, n


def psi4_diagnostics(Z, ctx, stream, npts, nblocks, with_cpu):
    """Times Z4cWeyl alone (k_prep + k_weyl on every block) and the whole
    extraction sequence of the main loop (Z4cToADM, Z4cWeyl, Weyl ghost
    exchange, interpolation and (l, m) projection on WAVE_SPHERES, psi on
    the host) with CUDA events, median of 5; the oracle's Z4cWeyl on one
    MeshBlock, single thread, as the CPU figure."""
    import torch
    spheres = [Z.WaveExtract(ctx, r, nlev, lmax) for r, nlev, lmax in WAVE_SPHERES]

    def timed(fn, reps=5):
        out = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                fn()
                e1.record(stream)
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1))
        return sorted(out)[len(out) // 2]

    with torch.cuda.stream(stream):
        ctx.psi4_multipoles(spheres)  # warm-up
    torch.cuda.synchronize()
    weyl_ms = timed(lambda: ctx.Z4cWeyl())
    extract_ms = timed(lambda: ctx.psi4_multipoles(spheres))
    tf = FP64_OPS_PER_POINT_WEYL * npts / (weyl_ms * 1e-3) / 1e12
    out = {"weyl_ms": weyl_ms, "extraction_ms": extract_ms,
           "weyl_tflops": tf, "fp64_ops_per_vertex": FP64_OPS_PER_POINT_WEYL,
           "spheres": [{"radius": w.radius, "nlev": w.nlev, "lmax": w.lmax,
                        "points": w.num_points()} for w in spheres],
           "psi22_re_r6": float(spheres[0].psi[0, 4, 0]),
           "note": "weyl_ms: k_prep + k_weyl on all MeshBlocks; extraction_ms: Z4cToADM, "
                   "Z4cWeyl, Weyl ghost exchange and both spheres' multipoles to the host"}
    if with_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import z4c_oracle as O
        mesh = ctx.mesh
        xs, dxs = mesh.block_coords(0)
        blk = O.Block(mesh.nx, dxs, xs)
        u = ctx.download(Z.REG_U, block=0)
        adm = ctx.download(Z.REG_ADM, block=0)
        t0 = time.perf_counter()
        O.weyl(blk, O.default_params(**PARAMS), adm, u)
        per_block = time.perf_counter() - t0
        out["cpu_port_ms_all_blocks"] = per_block * nblocks * 1e3
        out["cpu_sample"] = "C oracle Z4cWeyl on one MeshBlock, single thread, times the block count"
    return out


def time_on(stream, fn, reps):
    """Device time of fn() per call: CUDA events on the context's stream
    around reps calls, after one untimed call."""
    import torch
    with torch.cuda.stream(stream):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    with torch.cuda.stream(stream):
        for _ in range(reps):
            fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


# The adjoint benchmark: the 48^3 gauge-wave benchmark's physics on 64^3 cells in one periodic
# MeshBlock, A = 0.05, seeded U(-1e-6, 1e-6) on the conformal metric, 100 rk4
# steps, objective = H-norm after the last step; eps_floor < 0 keeps
# AlgConstr's determinant normalisation on every vertex (differentiable)
ADJ_PARAMS = dict(lapse_harmonic=1.0, lapse_harmonicf=0.0, lapse_oplog=0.0, lapse_advect=0.0,
                  shift_Gamma=0.0, shift_eta=0.0, shift_advect=0.0, diss=0.02,
                  damp_kappa1=0.02, r_max_con=1e300, eps_floor=-1.0)
ADJ_STEPS, ADJ_SNAPSHOTS = 100, 9


def adjoint_diagnostics(Z, ID, head_ctx, head_stream, head_dt, exact_shape=None):
    """The differentiated step: one adjoint step (recomputation of the step
    included) against one forward step, on the 64^3 adjoint block and on the
    headline mesh, and the revolve-checkpointed gradient of the 64^3 adjoint benchmark."""
    import torch
    out = {}
    mesh = Z.Mesh((1, 1, 1), (64, 64, 64), (-0.5,) * 3, (0.5,) * 3, "periodic")
    ctx = Z.Z4c(mesh, Z.default_params(**ADJ_PARAMS), "rk4")
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.adj_setup()
    ID.load_adm(ctx, ID.gauge_wave1(mesh, amplitude=0.05))
    u = ctx.download(Z.REG_U)
    rng = np.random.default_rng(2024)
    u[:, Z.GXX:Z.GZZ + 1] += rng.uniform(-1e-6, 1e-6, size=u[:, Z.GXX:Z.GZZ + 1].shape)
    ctx.upload(Z.REG_U, u)
    ctx.init_finalize()
    u0 = ctx.download(Z.REG_U)
    dt = 0.25 / 64
    fwd = time_on(stream, lambda: ctx.evolve(dt, 1), 20)
    ctx.upload(Z.REG_U, u0)
    adj = time_on(stream, lambda: ctx.adj_step(dt), 10)
    ctx.upload(Z.REG_U, u0)
    with torch.cuda.stream(stream):
        J, pb, st = ctx.gradient(dt, ADJ_STEPS, ADJ_SNAPSHOTS)
    torch.cuda.synchronize()
    out["gw64_adjoint"] = {
        "workload": "gauge wave A=0.05 + U(-1e-6,1e-6) on g~, 64^3 cells, one periodic MeshBlock, "
                    "rk4, 100 steps, objective vol*sum H^2 after the last step",
        "forward_step_ms": fwd, "adjoint_step_ms": adj, "adjoint_over_forward": adj / fwd,
        "gradient_seconds": st["seconds"], "gradient_forward_steps": st["forward_steps"],
        "gradient_adjoint_steps": st["adjoint_steps"], "snapshots": ADJ_SNAPSHOTS,
        "objective": J, "d_shift_eta": float(pb[0]), "d_damp_kappa1": float(pb[1])}
    ctx.close()
    # the headline mesh (512 MeshBlocks, outflow faces), on the exact path the
    # adjoint differentiates
    contract, tile, regs = head_ctx.get_contract(), head_ctx.get_tile(), head_ctx.get_point_regs()
    head_ctx.set_contract(False)
    if exact_shape:  # the exact path's own autotuned shape
        head_ctx.set_tile(*exact_shape[0])
        head_ctx.set_point_regs(exact_shape[1])
    head_ctx.adj_setup()
    fwd = time_on(head_stream, lambda: head_ctx.evolve(head_dt, 1), 5)
    adj = time_on(head_stream, lambda: head_ctx.adj_step(head_dt), 3)
    head_ctx.set_contract(contract)
    head_ctx.set_tile(*tile)
    head_ctx.set_point_regs(regs)
    out["puncture_512"] = {"forward_step_ms": fwd, "adjoint_step_ms": adj,
                           "adjoint_over_forward": adj / fwd}
    out["note"] = ("adjoint_step_ms: the step recomputed stage by stage from its start state, then "
                   "the reverse of its four stages (AlgConstr, exchange, boundary conditions, "
                   "stage algebra, right-hand side); device time, CUDA events")
    return out


# ---------------------------------------------------------------------------


class Ranks:
    """Rank bookkeeping of the replica benchmark: every rank evolves its own
    copy of the mesh, and the timed region ends at the slowest rank.  dist is
    torch.distributed with an initialised process group (NCCL on the GPUs;
    the tests use gloo on the CPU), or None for one rank."""

    def __init__(self, dist, world, device):
        self.dist, self.world, self.device = dist, world, device

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x):
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())


def whole_job_rate(units_per_rank, world, max_seconds):
    """Units processed by all ranks divided by the slowest rank's time."""
    return units_per_rank * world / max_seconds


# Binary Brill-Lindquist punctures (masses 0.5 near (+-3, 0, 0)) on
# [-512, 512]^3 with 4^3 root MeshBlocks of 16^3 cells and seven nested
# static refinement boxes around them (level L reaches 3 + 6 * 2^(7-L), half
# as far along y and z from level 3 on): 3,424 MeshBlocks, finest spacing
# 1/8.  The punctures sit a fraction of a cell off the vertices that every
# level puts at (+-3, 0, 0), where psi diverges.
SMR_REGIONS = [dict(x1min=-r, x1max=r, x2min=-r * f, x2max=r * f, x3min=-r * f, x3max=r * f,
                    level=lv)
               for lv in range(1, 8)
               for r, f in [(min(3.0 + 6.0 * 2 ** (7 - lv), 511.0), 0.5 if lv > 2 else 1.0)]]
SMR_CENTRES = ((3.0, 0.0625 * 0.37, 0.0625 * 0.21), (-3.0, -0.0625 * 0.37, -0.0625 * 0.21))


# The adaptive binary: the punctures of SMR_CENTRES on [-512, 512]^3 with 8^3
# root MeshBlocks of 16^3 cells (dx 8) and 7 levels (finest dx 1/8), refined
# by Linf_box_in_box with par_b = 3 around the two puncture trackers, the
# reference's default derefinement count of 10 cycles.
AMR_MESH = dict(nb=(8, 8, 8), nx=(16, 16, 16), xmin=(-512.0,) * 3, xmax=(512.0,) * 3,
                numlevel=7, derefine_count=10, par_b=3.0)


def amr_measure(steps, warmup, shift=(0.0, 0.0, 0.0), contract=1):
    """The adaptive binary run: `warmup` cycles, then `steps` cycles timed
    whole on the device stream (RK steps, the host's refinement flags, which
    overlap the step, and every regrid: new context, state transfer, ghost
    finalisation, graph capture), with zone-updates counted per cycle on the
    mesh that cycle stepped.  `shift`: the initial shift (zero in the
    configuration as written); `contract`: the right-hand-side path."""
    import torch
    import z4c_b200 as Z
    from z4c_b200 import amr as A
    from z4c_b200 import initial_data as ID
    torch.cuda.set_device(0)
    m = AMR_MESH
    params = Z.default_params(**PARAMS)
    stream = torch.cuda.Stream()
    ref = A.Refinement(m["nb"], m["nx"], m["xmin"], m["xmax"], Z.Mesh(
        m["nb"], m["nx"], m["xmin"], m["xmax"], "outflow").bc, m["numlevel"],
        m["derefine_count"], m["par_b"])
    t0 = time.time()
    with torch.cuda.stream(stream):
        run = A.AdaptiveEvolution(
            ref, params, "rk4",
            lambda mesh: ID.punctures(mesh, params, masses=(0.5, 0.5), centres=SMR_CENTRES,
                                      shift=shift),
            SMR_CENTRES, cfl=CFL, history=False, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        setup_s = time.time() - t0
        run.contract = bool(contract)
        run.ctx.set_contract(run.contract)
        run.ctx.autotune(reps=2)
        run.tile = run.ctx.get_tile()
        run.point_regs = run.ctx.get_point_regs()
        initial_blocks = run.mesh.nblocks
        for _ in range(warmup):
            run.step()
        torch.cuda.synchronize()
        sampler = ClockSampler(0)
        sampler.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        zones, regrids, regrid_s = 0, [], []
        p0 = np.array(run.trackers())
        ev0.record(stream)
        w0 = time.time()
        for _ in range(steps):
            zones += run.mesh.zones()
            t = time.time()
            if run.step():
                regrids.append([run.ncycle, run.mesh.nblocks])
                regrid_s.append(time.time() - t)
        ev1.record(stream)
        torch.cuda.synchronize()
        wall = time.time() - w0
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    moved = float(np.abs(np.array(run.trackers()) - p0).max())
    finite = bool(run.ctx.check_finite())
    final_blocks = run.mesh.nblocks
    run.close()
    return {
        "metric": "zone-updates/s", "value": zones / (ms * 1e-3), "unit": "zone-updates/s",
        "n_gpus": 1, "steps": steps, "warmup": warmup, "ms_per_step": ms / steps,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "binary Brill-Lindquist punctures (m=0.5 each near (+-3,0,0)), "
                               "[-512,512]^3, 8^3 root MeshBlocks of 16^3 cells, 7 levels "
                               "refined by Linf_box_in_box (par_b 3) around the puncture "
                               "trackers, derefine_count 10, extrapolate_outflow, rk4 (2S), "
                               "cfl 0.25", "initial_shift": list(shift),
                   "path": "contracted" if contract else "exact",
                   "l2": "inputs larger than L2"},
        "initial_meshblocks": initial_blocks, "final_meshblocks": final_blocks,
        "regrids": regrids, "regrid_cycle_s": regrid_s, "tracker_displacement": moved,
        "wall_s": wall, "setup_s": setup_s, "finite": finite, "clocks": clocks,
    }


# The adjoint at scale: the binary of the adaptive runs on the same domain
# and finest spacing, with 4^3 root MeshBlocks (dx 16) and 8 levels, refined
# by Linf_box_in_box around the punctures at t = 0: 848 MeshBlocks.  (The
# 3,424-block mesh of 8^3 roots does not fit: its context holds ~72 GB and
# the adjoint's buffers ~13 state-sized registers of 9.4 GB more.)  The
# gradient over 400 steps of the time-integrated H-norm plus the Weyl-scalar
# proxy on the sphere of radius 50 (the weighted |psi4|^2 over its vertices,
# weighted so that both terms are equal at t = 0) with respect to the
# masses, the separation and eta, revolve snapshots sized to the free HBM.
ADJ_BBH = dict(nb=(4, 4, 4), nx=(16, 16, 16), xmin=(-512.0,) * 3, xmax=(512.0,) * 3,
               numlevel=8, par_b=3.0, masses=(0.5, 0.5), separation=6.0, steps=400,
               weyl_radius=50.0, weyl_nlev=30)


def bbh_adjoint_measure(steps=None, fd=True):
    """The revolve-checkpointed gradient on the refined binary mesh: J, the
    four parameter derivatives (the state's adjoint chained through
    ADMToZ4c and the host data's derivative), timings, snapshots; with fd a
    central difference of the full forward run in eta as a check."""
    import torch
    import z4c_b200 as Z
    from z4c_b200 import amr as A
    from z4c_b200 import initial_data as ID
    torch.cuda.set_device(0)
    c = ADJ_BBH
    steps = steps or c["steps"]
    bc = Z.Mesh(c["nb"], c["nx"], c["xmin"], c["xmax"], "outflow").bc
    ref = A.Refinement(c["nb"], c["nx"], c["xmin"], c["xmax"], bc, c["numlevel"], 10, c["par_b"])
    off = (0.0625 * 0.37, 0.0625 * 0.21)

    def centres(d):
        return ((0.5 * d, off[0], off[1]), (-0.5 * d, -off[0], -off[1]))

    ref.build_initial(centres(c["separation"]))
    mesh = ref.mesh()
    pdict = dict(PARAMS, eps_floor=-1.0)

    def data(m, th):
        return ID.punctures(m, Z.default_params(**pdict), masses=tuple(th[:2]),
                            centres=centres(th[2]))

    theta = np.array([c["masses"][0], c["masses"][1], c["separation"]])
    ctx = Z.Z4c(mesh, Z.default_params(**pdict), "rk4")
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.adj_setup()
    adm = data(mesh, theta)
    dt = mesh.new_dt(CFL)
    with torch.cuda.stream(stream):
        ctx.upload(Z.REG_ADM, adm)
        ctx.ADMToZ4c()
        ctx.init_finalize()
        u0 = ctx.download(Z.REG_U)
        # the Weyl term, normalised to the H-norm term at t = 0
        sphere = Z.WaveExtract(ctx, radius=c["weyl_radius"], nlev=c["weyl_nlev"], lmax=2)
        JH0 = ctx.objective()[0]
        ctx.adj_set_weyl(sphere, 1.0)
        JW0 = ctx.objective()[0] - JH0
        weyl_weight = JH0 / JW0
        ctx.adj_set_weyl(sphere, weyl_weight)
        fwd = time_on(stream, lambda: ctx.evolve(dt, 1), 3)
        ctx.upload(Z.REG_U, u0)
        adj = time_on(stream, lambda: ctx.adj_step(dt), 2)
        ctx.upload(Z.REG_U, u0)
        nsnap = ctx.snapshots(steps)
        J, pb, st = ctx.gradient(dt, steps, nsnap, w_final=0.0, w_step=dt)
        ctx.upload(Z.REG_ADM, adm)
        ctx.adj_adm_to_z4c()
        ab = ctx.download(Z.REG_ADM_ADJ)
    torch.cuda.synchronize()
    grads = {}
    for j, name in enumerate(("m1", "m2", "separation")):
        e = np.zeros(3)
        e[j] = 1e-6
        dadm = (data(mesh, theta + e) - data(mesh, theta - e)) / 2e-6
        grads[name] = float(np.sum(ab * dadm))
    grads["eta"] = float(pb[0])
    out = {"workload": "binary Brill-Lindquist punctures (m=0.5 each near (+-3,0,0)), "
                       "[-512,512]^3, 4^3 root MeshBlocks of 16^3 cells, 8 levels refined by "
                       "Linf_box_in_box (par_b 3) around the punctures at t=0, finest dx 1/8, "
                       f"outflow, rk4, {steps} steps, objective dt * sum_k (vol * sum H^2 "
                       f"+ w * sum_p w_p |psi4(p)|^2 on the r = {c['weyl_radius']:g} sphere)",
           "meshblocks": mesh.nblocks, "steps": steps, "snapshots": nsnap,
           "forward_step_ms": fwd, "adjoint_step_ms": adj, "adjoint_over_forward": adj / fwd,
           "gradient_seconds": st["seconds"], "gradient_forward_steps": st["forward_steps"],
           "gradient_adjoint_steps": st["adjoint_steps"], "objective": J, "gradient": grads,
           "weyl_term": {"radius": c["weyl_radius"], "sphere_vertices": sphere.num_points(),
                         "weight": weyl_weight, "J_H_t0": JH0, "J_W_t0": JW0}}
    ctx.close()
    if fd:
        # the full forward run at eta +- h (the objective reads the adjoint
        # buffers' scratch, hence adj_setup)
        def run_ctx(eta):
            cr = Z.Z4c(mesh, Z.default_params(**dict(pdict, shift_eta=eta)), "rk4")
            cr.set_stream(stream.cuda_stream)
            cr.adj_setup()
            cr.adj_set_weyl(Z.WaveExtract(cr, radius=c["weyl_radius"], nlev=c["weyl_nlev"],
                                          lmax=2), weyl_weight)
            with torch.cuda.stream(stream):
                cr.upload(Z.REG_U, u0)
                tot = 0.0
                for _ in range(steps):
                    cr.evolve(dt, 1)
                    tot += dt * cr.objective()[0]
            cr.close()
            return tot
        h = 1e-3
        eta0 = pdict["shift_eta"]
        fd_eta = (run_ctx(eta0 + h) - run_ctx(eta0 - h)) / (2 * h)
        out["fd_eta"] = fd_eta
        out["fd_eta_rel"] = abs(grads["eta"] - fd_eta) / abs(fd_eta)
    return out


def main_amr(args):
    print(json.dumps(amr_measure(args.steps, args.warmup, contract=args.contract)), flush=True)
    print(json.dumps(amr_measure(AMR_SHIFTED_STEPS, args.warmup, AMR_SHIFT,
                                 contract=args.contract)), flush=True)


def main_smr(args):
    print(json.dumps(smr_measure(args.steps, args.warmup, args.shape, args.contract)),
          flush=True)


def rs_measure(steps, warmup, contract=1):
    """The robust-stability workload of the same batched mesh: Minkowski plus
    seeded uniform noise of amplitude 1e-10 on every Z4c variable, 512
    MeshBlocks of 16^3, periodic, the puncture run's gauge and damping;
    graph-captured steps timed with CUDA events."""
    import torch
    import z4c_b200 as Z
    from z4c_b200 import initial_data as ID
    mesh = Z.Mesh([8] * 3, [16] * 3, [-16.0] * 3, [16.0] * 3, "periodic")
    params = Z.default_params(**PARAMS)
    ctx = Z.Z4c(mesh, params, "rk4")
    ctx.set_contract(bool(contract))
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ID.load_z4c(ctx, ID.noise_state(mesh))
    dt = CFL * float(np.min(ctx.dx()))
    with torch.cuda.stream(stream):
        ctx.evolve(dt, warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    with torch.cuda.stream(stream):
        ctx.evolve(dt, steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"value": mesh.zones() * steps / (ms * 1e-3), "unit": "zone-updates/s",
           "ms_per_step": ms / steps, "steps": steps, "merged_grid": ctx.get_merged(),
           "finite": ctx.check_finite(),
           "config": "robust stability: Minkowski + uniform noise 1e-10 (seeded) on all Z4c "
                     "variables, 128^3 cells as 512 MeshBlocks of 16^3, periodic, 1+log + "
                     "Gamma-driver (eta=2), kappa1=0.02, diss=0.02, rk4 (2S), cfl 0.25"}
    ctx.close()
    return out


def smr_measure(steps, warmup, shape=None, contract=1):
    """Steps of the refined binary-puncture mesh: zone-updates/s through
    the graph-captured step, and the multilevel ghost exchange alone."""
    import torch
    import z4c_b200 as Z
    from z4c_b200 import initial_data as ID
    torch.cuda.set_device(0)
    mesh = Z.Mesh((4, 4, 4), (16, 16, 16), (-512.0,) * 3, (512.0,) * 3, "outflow",
                  refinement=SMR_REGIONS)
    params = Z.default_params(**PARAMS)
    ctx = Z.Z4c(mesh, params, "rk4")
    ctx.set_contract(bool(contract))
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    t0 = time.time()
    ID.load_adm(ctx, ID.punctures(mesh, params, masses=(0.5, 0.5), centres=SMR_CENTRES))
    ctx.sync()
    setup_s = time.time() - t0
    if shape:
        ctx.set_tile(*(int(v) for v in shape.split(",")))
    else:
        with torch.cuda.stream(stream):
            ctx.autotune(reps=2)
    dt = mesh.new_dt(CFL)
    with torch.cuda.stream(stream):
        ctx.evolve(dt, warmup)
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    with torch.cuda.stream(stream):
        ctx.evolve(dt, steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1) / steps
    # the multilevel exchange alone (ghost fill of the 22-variable state)
    reps = 10
    with torch.cuda.stream(stream):
        ctx.ghost_fill(Z.REG_U)
    torch.cuda.synchronize()
    ev0.record(stream)
    with torch.cuda.stream(stream):
        for _ in range(reps):
            ctx.ghost_fill(Z.REG_U)
    ev1.record(stream)
    torch.cuda.synchronize()
    exch_ms = ev0.elapsed_time(ev1) / reps
    levels = np.bincount(mesh.locs[:, 0] - mesh.root_level).tolist()
    line = {
        "metric": "zone-updates/s", "value": mesh.zones() / (ms * 1e-3), "unit": "zone-updates/s",
        "n_gpus": 1, "steps": steps, "warmup": warmup, "ms_per_step": ms,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "binary punctures (m=0.5 each near (+-3,0,0)), [-512,512]^3, "
                               "4^3 root MeshBlocks of 16^3 cells, 7 nested static refinement "
                               "levels, extrapolate_outflow, rk4 (2S), cfl 0.25",
                   "path": "contracted" if contract else "exact",
                   "meshblocks": mesh.nblocks, "blocks_per_level": levels,
                   "finest_dx": float(min(min(mesh.block_coords(b)[1])
                                          for b in range(mesh.nblocks) if mesh.locs[b, 0] ==
                                          mesh.locs[:, 0].max())),
                   "l2": "inputs larger than L2"},
        "exchange_ms": exch_ms, "exchange_share": 4 * exch_ms / ms,
        "setup_s": setup_s, "finite": bool(ctx.check_finite()),
        "clocks": clocks,
    }
    ctx.close()
    return line


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return main_reference(args, rank, world)
    if args.workload == "bbh_smr":
        return main_smr(args)
    if args.workload == "bbh_amr":
        return main_amr(args)
    if args.workload == "bbh_adjoint":
        print(json.dumps(bbh_adjoint_measure(args.steps if args.steps != 60 else None)),
              flush=True)
        return

    import torch
    import torch.distributed as dist
    import z4c_b200 as Z
    from z4c_b200 import initial_data as ID

    torch.cuda.set_device(local_rank)
    if args.stage_profile:
        n_m, lim = 16 * args.nb, 2.0 * args.nb
        mmesh = Z.Mesh([1] * 3, [n_m] * 3, [-lim] * 3, [lim] * 3, "outflow")
        params = Z.default_params(**PARAMS)
        sctx = Z.Z4c(mmesh, params, "rk4")
        sctx.set_contract(True)
        if args.shape:
            sctx.set_tile(*(int(v) for v in args.shape.split(",")))
        ID.load_adm(sctx, ID.punctures(mmesh, params, masses=(1.0,), centres=((0.0, 0.0, 0.0),)))
        sctx.init_finalize()
        dt = CFL * float(np.min(sctx.dx()))
        for _ in range(3):
            sctx.rhs_stage(2, dt)
        sctx.sync()
        print(json.dumps({"stage_profile": True, "cells": n_m}), flush=True)
        sctx.close()
        return
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    nb = [args.nb] * 3
    lim = 2.0 * args.nb
    mesh = Z.Mesh(nb, WORKLOAD["nx"], [-lim] * 3, [lim] * 3, "outflow")
    params = Z.default_params(**PARAMS)
    ctx = Z.Z4c(mesh, params, "rk4")
    ctx.set_contract(bool(args.contract))
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    adm = ID.punctures(mesh, params, masses=(1.0,), centres=((0.0, 0.0, 0.0),))
    ID.load_adm(ctx, adm)
    ctx.sync()
    u_init = ctx.download(Z.REG_U)
    # launch shape of the right-hand-side passes, picked on this mesh
    if args.shape:
        tile = tuple(int(v) for v in args.shape.split(","))
        ctx.set_tile(*tile)
    else:
        with torch.cuda.stream(stream):
            tile, _ = ctx.autotune(reps=3)
    point_regs = ctx.get_point_regs()
    dt = CFL * float(np.min(ctx.dx()))
    zones = mesh.zones()
    npts = mesh.nblocks * 17 ** 3
    if args.nb != 8:
        WORKLOAD["workload"] = WORKLOAD["workload"].replace(
            "128^3 cells as 512", f"{16 * args.nb}^3 cells as {mesh.nblocks}").replace(
            "[-16,16]^3", f"[-{lim:g},{lim:g}]^3")

    ranks = Ranks(dist if world > 1 else None, world, "cuda")
    barrier, max_over_ranks = ranks.barrier, ranks.max

    # ---- device-resident throughput: graph-captured steps -------------------
    with torch.cuda.stream(stream):
        ctx.evolve(dt, args.warmup)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    sampler.start()
    launches0 = Z.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    with torch.cuda.stream(stream):
        ctx.evolve(dt, args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = Z.kernel_launches() - launches0
    barrier()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = whole_job_rate(zones * args.steps, world, ms * 1e-3)
    finite = ctx.check_finite()

    # ---- dominant kernel: the fused RHS+KO+stage kernel, timed alone -------
    def time_stage_seq(c=ctx, u0=u_init):
        with torch.cuda.stream(stream):
            c.upload(Z.REG_U, u0)
            c.init_finalize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            times = []
            for _ in range(5):
                e0.record(stream)
                c.rhs_stage(2, dt)
                e1.record(stream)
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1))
        return sorted(times)[len(times) // 2]
    # where the timed step runs it: on the merged vertex grid of the blocks
    # (one block of 16 nb cells per axis, the same kernels and launch shape)
    # when z4c_evolve merges them, else on the blocks
    merged = ctx.get_merged()
    stage_npts = npts
    if merged:
        n_m = 16 * args.nb
        mmesh = Z.Mesh([1] * 3, [n_m] * 3, [-lim] * 3, [lim] * 3, "outflow")
        sctx = Z.Z4c(mmesh, params, "rk4")
        sctx.set_contract(True)
        sctx.set_stream(stream.cuda_stream)
        sctx.set_tile(*tile)
        sctx.set_point_regs(point_regs)
        ID.load_adm(sctx, ID.punctures(mmesh, params, masses=(1.0,), centres=((0.0, 0.0, 0.0),)))
        sctx.sync()
        stage_ms = time_stage_seq(sctx, sctx.download(Z.REG_U))
        sctx.close()
        stage_npts = (n_m + 1) ** 3
    else:
        stage_ms = time_stage_seq()

    # ---- the exact path (bit for bit the reference's arithmetic) -----------
    exact = None
    if args.contract and not args.profile_run:
        ctx.set_contract(False)
        with torch.cuda.stream(stream):
            ctx.upload(Z.REG_U, u_init)
            ctx.init_finalize()
            etile, _ = ctx.autotune(reps=3)
            ctx.evolve(dt, args.warmup)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.evolve(dt, args.steps)
            e1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1))
        estage = time_stage_seq()
        exact = {"value": whole_job_rate(zones * args.steps, world, ems * 1e-3),
                 "ms_per_step": ems / args.steps, "stage_ms": estage, "launch_shape": etile,
                 "stage_kernels": STAGE_KERNELS[0],
                 "stage_traffic": STAGE_TRAFFIC_PER_POINT[0] * npts}
        exact["point_regs"] = ctx.get_point_regs()
        ctx.set_contract(True)
        ctx.set_tile(*tile)
        ctx.set_point_regs(point_regs)

    if args.profile_run:
        if rank == 0:
            print(json.dumps({"profile_run": True, "value": value, "stage_ms": stage_ms,
                              "gpu_launches": launches}), flush=True)
        ctx.close()
        return

    # ---- per-block plain path (one RHS launch per MeshBlock) ---------------
    pb_steps = max(2, min(5, args.steps))
    ctx.upload(Z.REG_U, u_init)
    ctx.init_finalize()
    ctx.set_per_block(True)
    with torch.cuda.stream(stream):
        ctx.evolve(dt, 1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.evolve(dt, pb_steps)
        e1.record(stream)
    torch.cuda.synchronize()
    pb_value = zones * pb_steps / (e0.elapsed_time(e1) * 1e-3)
    ctx.set_per_block(False)

    # ---- end to end through the public API with host buffers ----------------
    # Every step (one job of z4c_evolve_jobs): the pinned host state to the
    # device, one RK4 step, the constraints and the history norms (the step's
    # result metric) back to the host.  The library overlaps the copies of one
    # job with the evolution of the next.  The same with the final state
    # downloaded too is reported beside it.
    host = torch.from_numpy(u_init).pin_memory()
    host_np = host.numpy()
    outs = [torch.empty_like(host).pin_memory().numpy() for _ in range(2)]
    e2e_steps = E2E_JOBS
    ctx.evolve_jobs([host_np], [outs[0]], dt, 1)  # staging allocated, step captured
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    hst_jobs = ctx.evolve_jobs([host_np] * e2e_steps, None, dt, 1)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = whole_job_rate(zones * e2e_steps, world, e2e_s)
    barrier()
    t0 = time.perf_counter()
    ctx.evolve_jobs([host_np] * e2e_steps, [outs[j % 2] for j in range(e2e_steps)], dt, 1)
    torch.cuda.synchronize()
    e2e_state = {"value": whole_job_rate(zones * e2e_steps, world,
                                         max_over_ranks(time.perf_counter() - t0)),
                 "steps": e2e_steps, "h2d_bytes_per_step": host_np.nbytes,
                 "d2h_bytes_per_step": host_np.nbytes + 8 * 8 * mesh.nblocks,
                 "note": "the same jobs with each final state downloaded too"}
    state_bytes = host_np.nbytes
    hst_bytes = 8 * 8 * mesh.nblocks  # per-block history partials
    # norms-only jobs on the merged grid upload, of the blocks off the z faces,
    # only the vertex planes the merged grid reads (NG .. NG + nx)
    up_bytes = state_bytes
    if ctx.get_merged() and nb[2] > 2:
        per_block = host_np.nbytes // mesh.nblocks
        layer = nb[0] * nb[1]
        nn = [16 + 1 + 8] * 3
        up_bytes = (2 * layer * per_block +
                    (mesh.nblocks - 2 * layer) * 22 * nn[0] * nn[1] * 17 * 8)
    # the same sequence as separate calls, each waiting for the last
    seq_steps = max(2, min(args.steps, 5))
    out_host = outs[0]
    with torch.cuda.stream(stream):
        ctx.upload(Z.REG_U, host_np)
        ctx.evolve(dt, 1, with_constraints=True)
        ctx.hst_norms()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(seq_steps):
        ctx.upload(Z.REG_U, host_np)
        ctx.evolve(dt, 1, with_constraints=True)
        seq_hst = ctx.hst_norms()
        ctx.download(Z.REG_U, out=out_host)
    torch.cuda.synchronize()
    seq_s = max_over_ranks(time.perf_counter() - t0)
    e2e_seq = {"value": whole_job_rate(zones * seq_steps, world, seq_s), "steps": seq_steps,
               "note": "z4c_upload, z4c_evolve (1 step, constraints), z4c_hst_norms, "
                       "z4c_download per step, no overlap",
               "same_result": bool(np.array_equal(seq_hst, hst_jobs[-1]))}

    # ---- psi4 diagnostics: Z4cWeyl, then the extraction sequence ------------
    psi4 = psi4_diagnostics(Z, ctx, stream, npts, mesh.nblocks, rank == 0 and world == 1
                            and not args.no_cpu_baseline)

    # ---- differentiated step (N = 1) -----------------------------------------
    adjoint = None
    if world == 1 and not args.no_adjoint:
        adjoint = adjoint_diagnostics(
            Z, ID, ctx, stream, dt,
            (tuple(exact["launch_shape"]), exact["point_regs"]) if exact else None)

    # ---- CPU baseline (rank 0, N = 1) ---------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, build = run_reference_cpu(CPU_SAMPLE_STEPS, threads)
        if v is not None:
            cpu = {"value": v, "unit": "zone-updates/s", "cores": threads, "kind": "reference",
                   "sample": f"reference OpenMP build on the full workload, {CPU_SAMPLE_STEPS} "
                             f"RK4 steps, zone-cycles/omp_wsecond; {build}"}
        else:
            v, n = run_oracle_cpu()
            cpu = {"value": v, "unit": "zone-updates/s", "cores": 1, "kind": "port",
                   "sample": f"C oracle RHS on {n} MeshBlocks of 16^3, single thread"}

    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    fp64_peak_tf = ctx.fp64_probe()  # measured here: DFMA chains, 2 flops each
    stage_s = stage_ms * 1e-3
    achieved_gbs = STAGE_BYTES_PER_POINT * stage_npts / stage_s / 1e9
    achieved_tf = FP64_OPS_PER_POINT_STAGE * stage_npts / stage_s / 1e12
    path_key = "merged" if merged else args.contract
    traffic = STAGE_TRAFFIC_PER_POINT.get(path_key)
    roof = {"bound": "fp64", "achieved": achieved_tf, "peak": fp64_peak_tf, "unit": "TFLOP/s",
            "frac": achieved_tf / fp64_peak_tf,
            "peak_source": "measured in this run: dependent DFMA chains on every SM "
                           "(2 flops per DFMA); MEASURED_PEAKS.json has no FP64 figure",
            "frac_of_unfused_ceiling": achieved_tf / (0.5 * fp64_peak_tf),
            "traffic": traffic * stage_npts if traffic else None,
            "algorithmic_bytes": STAGE_BYTES_PER_POINT * stage_npts,
            "hbm_achieved_gbs": achieved_gbs, "hbm_peak_gbs": hbm_peak,
            "hbm_frac": achieved_gbs / hbm_peak, "hbm_peak_source": "MEASURED_PEAKS.json",
            "kernel": ("contracted" if args.contract else "exact") +
                      " RHS+KO+stage launch sequence (" + STAGE_KERNELS[args.contract] +
                      (f"), one stage on the merged {16 * args.nb + 1}^3-vertex grid of the "
                       f"{mesh.nblocks} MeshBlocks, where z4c_evolve runs it" if merged else
                       f"), one stage, all {mesh.nblocks} MeshBlocks"),
            "vertices": stage_npts,
            "kernel_ms": stage_ms, "fp64_ops_per_vertex": FP64_OPS_PER_POINT_STAGE}

    line = {
        "metric": METRIC, "value": value, "unit": "zone-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (analytic puncture initial data)",
        "config": dict(WORKLOAD, nb=nb, parallelism=f"replicas{world}", launch_shape=tile,
                       point_regs=point_regs,
                       path="contracted (fused multiply-adds; RHS within 1e-12 of the "
                            "reference's)" if args.contract else "exact (bit for bit)",
                       l2="inputs larger than L2 (1.4 GB per register)",
                       execution=("z4c_evolve runs the steps on the merged vertex grid of the "
                                  "MeshBlocks (z4c_set_merged)" if merged else "per MeshBlock"),
                       per_block_value=pb_value, batched_over_per_block=value / world / pb_value,
                       state_finite=finite),
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "zone-updates/s",
                "h2d_bytes_per_step": up_bytes, "d2h_bytes_per_step": hst_bytes,
                "steps": e2e_steps,
                "note": "per step, one job of z4c_evolve_jobs: pinned host state to device "
                        "(of the blocks off the mesh's z faces the vertex planes the merged "
                        "grid reads), one RK4 step, constraints, history norms (the result "
                        "metric) to host; the upload of one job overlaps the evolution of "
                        "the last",
                "with_state_download": e2e_state, "sequential": e2e_seq},
        "gpu_launches": launches,
        "clocks": clocks,
        "psi4": psi4,
        "adjoint": adjoint,
        "exact_path": exact,
    }
    ctx.close()
    if world == 1 and not args.no_smr:
        # the configuration's other workload on the same batched mesh
        line["robust_stability"] = rs_measure(RS_STEPS, 3, contract=args.contract)
        # the refined binary-puncture mesh (the adaptive benchmark's 7 levels,
        # static): its own context after this one is released
        smr = smr_measure(SMR_STEPS, 3, contract=args.contract)
        line["bbh_smr"] = {k: smr[k] for k in ("value", "unit", "ms_per_step", "steps",
                                               "exchange_ms", "exchange_share", "setup_s",
                                               "finite", "clocks")}
        line["bbh_smr"]["config"] = smr["config"]
    if world == 1 and not args.no_adjoint:
        # the gradient at scale on the refined binary mesh (40 of its 400 steps
        # here; bench.py --workload bbh_adjoint runs all 400), with the check
        # against differences of the full forward run in eta
        line["adjoint"]["bbh_refined"] = bbh_adjoint_measure(40)
    if world == 1 and not args.no_amr:
        # the adaptive binary-puncture run: 200 cycles, block list changing
        keys = ("value", "unit", "ms_per_step", "steps", "initial_meshblocks",
                "final_meshblocks", "regrids", "regrid_cycle_s", "tracker_displacement",
                "wall_s", "setup_s", "finite", "clocks", "config")
        amr = amr_measure(AMR_STEPS, 3, contract=args.contract)
        line["bbh_amr"] = {k: amr[k] for k in keys}
        # the same data in a shifted gauge: the trackers cross refinement
        # boundaries, so the regrid path runs at this size
        amr = amr_measure(AMR_SHIFTED_STEPS, 3, AMR_SHIFT, contract=args.contract)
        line["bbh_amr_shifted"] = {k: amr[k] for k in keys}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main_reference(args, rank, world):
    """The reference's own CPU implementation (the OpenMP build compiled from
    the reference sources) on the same workload and metric; rank 0 only."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    nlim = max(1, args.steps)
    v, build = run_reference_cpu(nlim, threads)
    kind = "reference"
    sample = f"reference OpenMP build, full workload, {nlim} RK4 steps; {build}"
    if v is None:
        v, n = run_oracle_cpu()
        kind, threads = "port", 1
        sample = f"C oracle RHS on {n} MeshBlocks of 16^3, single thread"
    line = {"metric": METRIC, "value": v, "unit": "zone-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (analytic puncture initial data)",
            "config": dict(WORKLOAD, parallelism="cpu"), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "zone-updates/s", "cores": threads,
                             "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
