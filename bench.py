#!/usr/bin/env python
"""solves/s of the self-consistent dipole solve on a B200.

Workload (one "step"): the N=4000 hexagonal monolayer of radius-5 nm spheres
(nearest-neighbour spacing 12 nm, rows of 128, periodic in-plane box with a
vacuum gap along z: 1542.0 x 332.6 x 1000 nm), Drude spheres
(eps_inf 4.0, omega_p 1.8 eV, gamma 0.1 eV) in eps_m = 1.77, 10 frequencies
evenly spaced over 0.2-1.0 eV x 3 incident polarisations = 30 right-hand
sides, Ewald accuracy = tol = 1e-6, GMRES(50) with Jacobi preconditioning.
A step is the per-frame precalculation plus the solve of all 30 right-hand
sides to a true fp64 relative residual |b - A x| / |b| <= 1e-6; a solve is
one converged right-hand side.

This arm: all 30 right-hand sides in one batch, fp32 operator inside fp64
iterative refinement.  `value` is device-timed with device-resident inputs;
`e2e` runs the same workload through the public drop-in API
(cumpm_b200.dipole_solver) with host inputs and outputs.  Beside it the line
carries: the plain per-system fp64 solve on this build's kernels, every
dipole's error against an fp64 solve of the same system, the reference
build's own GPU solve of the same workload (when it was compiled into
oracle/_ref), the CPU port's full solve, and the other benchmark workloads
(BiCGSTAB on the monolayer, the polydisperse packing, the small random
packing) as extra keys.

`--impl reference` times full single-right-hand-side GMRES solves of the CPU
port of the reference algorithm (oracle/) on the host cores.

Multi-GPU (torchrun): every rank solves an independent replica (the same
geometry at its own frequency set); no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_PART = 4000
SPACING = 12.0
RADIUS = 5.0
EPS_M = 1.77
TOL = 1e-6
XI = 0.5
N_FREQ = 10
K_POL = 3
# the fp64 solve every dipole is compared with (same operator, GMRES to this
# preconditioned residual)
REF_SOLVE_TOL = 1e-11
# true fp64 residual at which every monolayer dipole is within 1e-6 of that
# solution (at 1e-6 the per-dipole error is about nine times the residual)
DIPOLE_TOL_RESID = 5e-8


def hex_lattice(n, spacing):
    """Rows of 2*ceil(sqrt(n)) sites, odd rows shifted by half a spacing."""
    lim = int(np.ceil(np.sqrt(n))) * 2
    j, i = np.divmod(np.arange(n), lim)
    return np.stack([(i + 0.5 * (j % 2)) * spacing, j * (np.sqrt(3) / 2) * spacing, np.zeros(n)], axis=1)


def workload(rank=0):
    """The N=4000 monolayer (positions and box in nm, eps per frequency)."""
    pos = hex_lattice(N_PART, SPACING)
    rc = 5.256522
    mn = 2.1 * rc * RADIUS
    box = np.array([max(pos[:, 0].max() + SPACING, mn), max(pos[:, 1].max() + SPACING * np.sqrt(3) / 2, mn), 1000.0])
    lo, hi = 0.2, 1.0
    if rank:  # independent replica per rank: shifted frequency set
        lo, hi = 0.2 + 0.01 * rank, 1.0 + 0.01 * rank
    omega = np.linspace(lo, hi, N_FREQ)
    eps = 4.0 - 1.8 ** 2 / (omega ** 2 + 1j * omega * 0.1)
    return pos, box, eps


def rsa_packing(n, radii, phi, seed):
    """Random sequential addition of non-overlapping spheres in a periodic
    cube at volume fraction phi (seeded)."""
    rng = np.random.default_rng(seed)
    L = (np.sum(4.0 / 3.0 * np.pi * radii ** 3) / phi) ** (1.0 / 3.0)
    pos = np.zeros((n, 3))
    k = 0
    while k < n:
        p = rng.uniform(0, L, 3)
        d = pos[:k] - p
        d -= L * np.round(d / L)
        if k == 0 or np.all(np.sqrt(np.sum(d * d, axis=1)) >= radii[:k] + radii[k]):
            pos[k] = p
            k += 1
    return pos, np.array([L, L, L])


class Workload:
    """A benchmark system in the solver's units (lengths / smallest radius,
    permittivities / eps_m)."""

    def __init__(self, name, rank=0):
        self.name = name
        self.restart = 50
        if name == "monolayer":
            pos, box, eps = workload(rank)
            self.radius_nm = np.full(len(pos), RADIUS)
            self.K = K_POL
            self.label = WORKLOAD_LABEL
        elif name == "poly3d":
            rng = np.random.default_rng(1234)
            rad = rng.uniform(1.0, 4.0, 1000)
            pos, box = rsa_packing(1000, rad, 0.15, 1235)
            omega = np.linspace(0.2 + 0.01 * rank, 1.2 + 0.01 * rank, 64)
            eps = 4.0 - 1.8 ** 2 / (omega ** 2 + 1j * omega * 0.1)
            self.radius_nm = rad
            self.K = 3
            self.label = ("N=1000 polydisperse 3D packing, radii U[1,4] nm (seeded), phi 0.15, periodic box "
                          f"{box[0]:.1f} nm, Drude (eps_inf 4, wp 1.8 eV, gamma 0.1 eV), eps_m 1.77, 64 freqs "
                          "0.2-1.2 eV x 3 pols = 192 RHS, tol 1e-6, GMRES(50)+Jacobi, fp32 inner + fp64 refinement")
        elif name == "c1":
            rad = np.full(500, RADIUS)
            pos, box = rsa_packing(500, rad, 0.10, 500 + rank)
            omega = np.array([0.5 + 0.01 * rank])
            eps = 4.0 - 1.8 ** 2 / (omega ** 2 + 1j * omega * 0.1)
            self.radius_nm = rad
            self.K = 1
            self.restart = 30
            self.label = (f"N=500 random packing a=5nm, phi 0.10, periodic cube {box[0]:.1f} nm, Drude "
                          "(eps_inf 4, wp 1.8 eV, gamma 0.1 eV) at 0.5 eV, eps_m 1.77, x-polarised (1 RHS), "
                          "tol 1e-6, GMRES(30)+Jacobi")
        else:
            raise ValueError(f"unknown workload {name}")
        self.unit = float(self.radius_nm.min())
        self.pos_nm, self.box_nm, self.eps = pos, box, eps
        self.pos = pos / self.unit
        self.box = box / self.unit
        self.radius = self.radius_nm / self.unit
        self.mono = bool(np.all(self.radius == self.radius[0]))
        self.M = len(eps) * self.K

    def field(self, capi, tuning=None):
        if self.mono:
            return capi.Field(capi.FIELD_MONO, self.box, TOL, XI, tuning=tuning)
        return capi.Field(capi.FIELD_POLY, self.box, TOL, XI, radius=self.radius, tuning=tuning)

    def autotune(self, capi):
        """The field autotuner's pick for this workload (batch of M columns,
        fp32 reciprocal space as the inner solves run it)."""
        kind = capi.FIELD_MONO if self.mono else capi.FIELD_POLY
        return capi.autotune(kind, self.box, TOL, XI, self.pos, self.M, radius=None if self.mono else self.radius,
                             recip_fp32=True, real_fp32=False)


METRIC = "solves/s at N=4000, res 1e-6: batched mixed-prec vs plain; matvec % HBM peak"
METRICS = {"monolayer": METRIC,
           "poly3d": "solves/s, polydisperse N=1000, 192 RHS, res 1e-6: batched mixed-prec vs plain; matvec % HBM peak",
           "c1": "solves/s, N=500 random packing, 1 RHS, res 1e-6"}
DATA = {"monolayer": "synthetic (hexagonal monolayer generated as in the reference benchmark)",
        "poly3d": "synthetic (seeded random sequential addition of polydisperse spheres)",
        "c1": "synthetic (seeded random sequential addition of equal spheres)"}
WORKLOAD_LABEL = ("N=4000 hex monolayer a=5nm spacing 12nm, box 1542.0x332.6x1000nm, Drude "
                  "(eps_inf 4, wp 1.8 eV, gamma 0.1 eV), eps_m 1.77, 10 freqs 0.2-1.0 eV x 3 pols = 30 RHS, "
                  "tol 1e-6 (Ewald and true fp64 residual), GMRES(50)+Jacobi, fp32 inner + fp64 refinement")


def problem_arrays(wl):
    """Right-hand sides, mean-field initial guesses and self coefficients in
    the [row][M] layout (dipole_solver.cu:233-257, 438-489), host arrays.
    Column m is frequency m // K, polarisation m % K."""
    N = len(wl.pos)
    M = wl.M
    K = wl.K
    e = np.repeat(wl.eps / EPS_M, K)                          # per column
    a3 = wl.radius ** 3
    sc = 3.0 / (4 * np.pi * (e[None, :] - 1.0)) / a3[:, None]  # self coefficient s_i
    B = np.zeros((3 * N, M), complex)
    for m in range(M):
        B[m % K::3, m] = 1.0
    phi = np.sum(4.0 / 3.0 * np.pi * a3) / np.prod(wl.box)
    beta = (e - 1) / (e + 2)
    g = 4 * np.pi * beta / (1 - beta * phi)                   # per column, radius 1
    X0 = B * g[None, :] * np.repeat(a3, 3)[:, None]
    return B, X0, sc


def device_problem(wl, torch, dev):
    B, X0, sc = problem_arrays(wl)
    t = lambda a: torch.tensor(a, dtype=torch.complex128, device=dev)
    return t(B), t(X0), t(sc)


def fp64_reference_solution(F, B, X0, S, capi, tol=REF_SOLVE_TOL):
    """The fp64 solution every dipole is compared with: GMRES(50)+Jacobi on
    the fp64 operator (fp64 spread/FFT/contraction and real space) from X0,
    to a preconditioned residual of `tol`, all columns in one batch."""
    X = X0.clone()
    F.batch_solve(B, X, S, tol=tol, method=capi.METHOD_GMRES, restart=50, maxiter=4000, recip_fp32=False,
                  real_fp32=False, refine=False)
    return X


def dipole_errors(X, Xref, N):
    """Per-dipole error of X against Xref ([3N][M] complex): the largest
    |p_i - p_i^ref| / |p_i^ref| over particles and columns (3-vector norms),
    and the largest column-normwise |X - Xref| / |Xref|."""
    import torch
    D = (X - Xref)[:3 * N].reshape(N, 3, -1)
    R = Xref[:3 * N].reshape(N, 3, -1)
    dn = torch.linalg.vector_norm(D, dim=1)
    rn = torch.linalg.vector_norm(R, dim=1)
    per = (dn / rn.clamp_min(1e-300)).max().item()
    col = (torch.linalg.vector_norm(X - Xref, dim=0) / torch.linalg.vector_norm(Xref, dim=0)).max().item()
    return {"max_dipole_rel_err": per, "max_normwise_rel_err": col}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.th.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 9 for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per algorithmic
# byte of a stage's kernels, from ncu captures of one launch of each kernel
# on the same workload (monolayer: the x transform of a 9-column seed apply,
# 2.164 MB of DRAM traffic for 4.216 MB algorithmic, the grid's writes
# absorbed by L2; polydisperse packing: spread 1892 MB for 1962 MB, plain
# axis pass 3811 MB for 3870 MB).  Traffic scales with the columns a launch
# carries, so a stage's traffic per launch is this ratio times its
# algorithmic bytes per launch.  Below 1: the last writes of a launch are
# still in L2 when the kernel ends.
TRAFFIC_PER_ALG_BYTE = {
    ("monolayer", "fft_fwd"): 2.164 / 4.216,
    ("monolayer", "fft_inv"): 2.164 / 4.216,
    ("poly3d", "spread"): 1892.0 / 1962.0,
    ("poly3d", "fft_fwd"): 3811.0 / 3870.0,
    ("poly3d", "fft_inv"): 3811.0 / 3870.0,
}


def algorithmic_bytes(info, M, n_pairs, fp64, mono=True):
    """Minimum DRAM bytes of one launch of each stage of the batched matvec,
    for the kernels that run it.

    Grid G = stored voxels x C x M complex (C = 3 vector components for the
    monodisperse field, 1 scalar for the polydisperse one).  Spread writes
    it once; a 3-D transform counts as two read+write sweeps (4G) whatever
    number of axis passes it uses; the k-space step reads and writes it once
    plus its coefficients; contraction reads it once.  Fused slab layout
    (monodisperse monolayers): the forward and inverse stages are the x
    transforms alone (one sweep, 2G each) and the k-space stage is the y
    transforms with the Green tensor between them, one sweep (2G) plus three
    Toeplitz kernels per (kx, ky) column.  Moments and fields are [3N][M]
    complex128; the support weights are 3 x S values per particle
    (monodisperse, separable) or 3 x S^3 (polydisperse).
    """
    s = 16 if fp64 else 8
    nx, ny, nz = info["grid"]
    zs = info["z_slots"] if info["pruned"] else nz
    N = info["num_particles"]
    C = 3 if mono else 1
    G = nx * ny * zs * C * M * s
    mom = 3 * N * M * 16
    S = info["stencil"]
    w = N * 3 * (S if mono else S ** 3) * (8 if fp64 else 4)
    if info.get("slab_fused"):
        fwd = inv = 2 * G
        ksp = 2 * G + nx * ny * 3 * (2 * zs - 1) * s
    else:
        fwd = inv = 4 * G
        ksp = 2 * G + (nx * ny * 6 * (2 * zs - 1) * s if info["pruned"] else nx * ny * nz * (8 if fp64 else 4))
    return {
        "spread": G + mom + w,
        "fft_fwd": fwd,
        "kspace": ksp,
        "fft_inv": inv,
        "contract": G + mom + w,
        "real": n_pairs * (4 + (64 if fp64 else 32)) + 3 * mom,
    }


def matvec_bytes(info, M, n_pairs, fp64, mono=True):
    """Algorithmic bytes of one batched matvec, independent of how the
    stages are split into kernels: G_w + 2 n_pass 2G + G_scale + G_r +
    B_real + B_part with n_pass = 2 sweeps per 3-D transform and G_scale = 0
    when the k-space step is fused into a transform (else 2G + coefficients)."""
    b = algorithmic_bytes(info, M, n_pairs, fp64, mono)
    s = 16 if fp64 else 8
    nx, ny, nz = info["grid"]
    zs = info["z_slots"] if info["pruned"] else nz
    G = nx * ny * zs * (3 if mono else 1) * M * s
    g_scale = 0 if info.get("slab_fused") else b["kspace"]
    return b["spread"] + 8 * G + g_scale + b["contract"] + b["real"]


def replica_throughput(t_ms, units, dist=None, device="cpu"):
    """Whole-job throughput of independent replicas: (slowest rank's time in
    ms, units summed over the ranks, units per second over that time).
    Every rank takes the same two collectives; without a process group the
    rank's own figures."""
    import torch

    t_max, total = float(t_ms), int(units)
    if dist is not None:
        tt = torch.tensor([t_ms], device=device, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        cc = torch.tensor([units], device=device, dtype=torch.float64)
        dist.all_reduce(cc)
        t_max, total = float(tt.item()), int(round(cc.item()))
    return t_max, total, total / (t_max / 1e3)


class Timed:
    """The batched mixed-precision solve of one workload, its steps timed
    with CUDA events after an L2 flush (a 256 MB write outside the timed
    interval)."""

    def __init__(self, wl, capi, torch, dev, args, method, flush, dist=None, field=None):
        self.wl, self.capi, self.torch, self.dist, self.flush = wl, capi, torch, dist, flush
        self.F = wl.field(capi) if field is None else field
        self.B, self.X0, self.S = device_problem(wl, torch, dev)
        self.X = torch.empty_like(self.X0)
        self.M = self.B.shape[1]
        self.opts = dict(tol=TOL, method=method, restart=wl.restart, maxiter=1000, refine=True,
                         inner_tol=args.inner_tol, compact=not args.no_compact)
        self.reports = []

    def step(self):
        self.F.set_positions(self.wl.pos)
        self.X.copy_(self.X0)
        self.reports.append(self.F.batch_solve(self.B, self.X, self.S, **self.opts))

    def timed(self, nsteps):
        torch = self.torch
        if self.dist:
            self.dist.barrier()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
        for k in range(nsteps):
            self.flush.fill_(float(k))  # L2 flush outside the timed interval
            ev[k][0].record()
            self.step()
            ev[k][1].record()
        torch.cuda.synchronize()
        if self.dist:
            self.dist.barrier()
        return sum(a.elapsed_time(b) for a, b in ev)

    def warm(self, n):
        for _ in range(n):
            self.step()
        self.torch.cuda.synchronize()

    def true_residuals(self):
        torch = self.torch
        R = self.B - self.F.apply(self.X, self_coef=self.S)
        return (torch.linalg.vector_norm(R, dim=0) / torch.linalg.vector_norm(self.B, dim=0)).cpu().numpy()

    def accuracy(self):
        Xref = fp64_reference_solution(self.F, self.B, self.X0, self.S, self.capi)
        e = dipole_errors(self.X, Xref, len(self.wl.pos))
        e["reference"] = (f"fp64 GMRES(50)+Jacobi on the same fp64 operator to preconditioned residual "
                          f"{REF_SOLVE_TOL:g}, every column")
        return e, Xref


def run_ours(args, rank, world, local_rank):
    import torch

    from cumpm_b200 import capi

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    wl = Workload(args.workload, rank)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    method = capi.METHOD_BICGSTAB if args.method == "bicgstab" else capi.METHOD_GMRES
    T = Timed(wl, capi, torch, dev, args, method, flush, dist)
    F, B, X0, S, M = T.F, T.B, T.X0, T.S, T.M
    T.warm(args.warmup)
    info = F.info()

    # 1) the timed region: no stage timers
    T.reports.clear()
    launches0 = capi.kernel_launches()
    clocks = ClockSampler(local_rank)
    clocks.start()
    t_ms = T.timed(args.steps)
    clk = clocks.stop()
    launches = capi.kernel_launches() - launches0
    timed_reports = list(T.reports)
    # correctness of the timed result: fp64 true residual of every column
    rel = T.true_residuals()
    converged = int(np.sum(rel <= TOL))
    t_max, conv_total, value = replica_throughput(t_ms, converged * args.steps, dist, dev)
    ms_per_step = t_max / args.steps

    # 2) the same steps again with per-stage CUDA events on the launching
    #    stream: stage breakdown and the roofline of the dominant stage
    T.reports.clear()
    capi.profile_reset()
    capi.profile_enable(not args.no_profile)
    t_prof = T.timed(args.steps)
    capi.profile_enable(False)
    stages = capi.profile_read()
    rl, mv_frac = stage_roofline(wl, info, M, T.reports, stages, args.steps)

    out = None
    if rank == 0:
        # every dipole of the timed solve against an fp64 solve of the same system
        acc, Xref = T.accuracy() if world == 1 and not args.no_accuracy else (None, None)
        if acc is not None:
            acc["dipole_tol_run"] = dipole_tol_run(T, args, Xref)
        # 3) the plain per-system fp64 solve on the same operator: one
        #    right-hand side per solve, fp64 reciprocal and real space
        plain = run_plain(args, F, B, X0, S, M, torch, capi, wl) if not args.no_plain else None
        iters = [r["total_iterations"] / M for r in timed_reports]
        mv_per_step = sum(r["matvecs"] for r in timed_reports) / max(1, len(timed_reports))
        colmv_per_step = sum(r["column_matvecs"] for r in timed_reports) / max(1, len(timed_reports))
        solo = world == 1
        e2e = run_e2e(args, torch, wl) if solo and not args.no_e2e else None
        extras = run_extras(args, capi, torch, dev, flush) if solo and not args.no_extras else None
        ref_gpu = reference_gpu_leg(args, wl, F, B, S, Xref, torch) if solo and not args.no_reference_gpu else None
        cpu = cpu_baseline(args, wl) if solo and not args.no_cpu else None
        out = {
            "metric": METRICS[wl.name],
            "value": round(value, 3),
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_per_step, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "c64 operator / c128 refinement",
            "data": DATA[wl.name],
            "config": {
                "workload": wl.label,
                "method": args.method,
                "rhs_per_step": M,
                "converged_per_step": converged,
                "max_true_rel_resid": float(rel.max()),
                "krylov_steps_per_rhs": round(float(np.mean(iters)), 2),
                "matvecs_per_step": mv_per_step,
                "column_matvecs_per_step": colmv_per_step,
                "shifted_seed_columns": timed_reports[-1]["shift_seeds"] if timed_reports else 0,
                "inner_tol": f"max({args.inner_tol:g}, 0.5 tol |b_m| / |r_m|) per column",
                "compact_batch": not args.no_compact,
                "grid": info["grid"], "pruned_z_slots": info["z_slots"] if info["pruned"] else None,
                "single_layer": bool(info.get("single_layer")), "slab_fused": bool(info.get("slab_fused")),
                "support": info["stencil"],
                "real_space_pairs": info["num_pairs"],
                "l2": "inputs larger than L2 (grid + Krylov basis > 126 MB) and a 256 MB L2 flush before each step",
                "parallelism": f"replicas x{world}",
                "profiled_ms_per_step": round(t_prof / args.steps, 3),
                "stage_ms_per_step": {k: round(v[0] / args.steps, 3) for k, v in stages.items()},
                "stage_launches_per_step": {k: v[1] / args.steps for k, v in stages.items()},
            },
            "accuracy": acc,
            "matvec_hbm_frac": mv_frac,
            "plain_fp64": plain,
            "batched_vs_plain": round(value / plain["value"], 2) if plain else None,
            "roofline": rl,
            "reference_gpu": ref_gpu,
            "extra_workloads": extras,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return out


def dipole_tol_run(T, args, Xref):
    """The same steps with the true-residual target at which every dipole is
    within 1e-6 of the fp64 solution (DIPOLE_TOL_RESID), timed the same way:
    the throughput of the accuracy target, beside the residual-1e-6 headline."""
    tol0 = T.opts["tol"]
    T.opts["tol"] = DIPOLE_TOL_RESID
    try:
        T.warm(1)
        T.reports.clear()
        steps = max(2, min(args.steps, 5))
        t = T.timed(steps)
        rel = T.true_residuals()
        conv = int(np.sum(rel <= DIPOLE_TOL_RESID))
        e = dipole_errors(T.X, Xref, len(T.wl.pos))
        return {"true_resid_target": DIPOLE_TOL_RESID, "value": round(conv * steps / (t / 1e3), 3),
                "unit": "solves/s", "ms_per_step": round(t / steps, 3), "steps": steps,
                "converged_per_step": conv, "max_true_rel_resid": float(rel.max()), **e}
    finally:
        T.opts["tol"] = tol0


def stage_roofline(wl, info, M, reports, stages, nsteps):
    """Roofline of the dominant operator stage and the whole matvec's HBM
    fraction, from the per-stage CUDA-event times of a profiled pass."""
    matvecs = sum(r["matvecs"] for r in reports)
    mv64 = sum(r["fp64_matvecs"] for r in reports)  # fp64 true-residual matvecs (at most M columns each)
    mv32 = matvecs - mv64
    col64 = mv64 * M
    col32 = max(0, sum(r["column_matvecs"] for r in reports) - col64)
    op_stages = ["spread", "fft_fwd", "kspace", "fft_inv", "contract", "real"]

    def stage_bytes(k):
        """Algorithmic bytes of stage k over the pass: per-column part x columns + fixed part x launches."""
        tot = 0.0
        for fp64, mv, cols in ((False, mv32, col32), (True, mv64, col64)):
            b0 = algorithmic_bytes(info, 0, info["num_pairs"], fp64, wl.mono)[k]
            b1 = algorithmic_bytes(info, 1, info["num_pairs"], fp64, wl.mono)[k]
            tot += b0 * mv + (b1 - b0) * cols
        return tot

    b32 = algorithmic_bytes(info, M, info["num_pairs"], False, wl.mono)
    dom = max(op_stages, key=lambda k: stages[k][0])
    dom_ms, dom_n = stages[dom]
    if dom_ms <= 0:   # --no-profile: no stage timings, no roofline
        return None, None
    bytes_total = stage_bytes(dom)
    peak, peak_kind = measured_peaks()
    achieved = bytes_total / (dom_ms / 1e3) / 1e9
    ratio = TRAFFIC_PER_ALG_BYTE.get((wl.name, dom))
    traffic = round(ratio * bytes_total / max(1, dom_n)) if ratio else None
    mv_bytes = 0.0
    for fp64, mv, cols in ((False, mv32, col32), (True, mv64, col64)):
        b0 = matvec_bytes(info, 0, info["num_pairs"], fp64, wl.mono)
        b1 = matvec_bytes(info, 1, info["num_pairs"], fp64, wl.mono)
        mv_bytes += b0 * mv + (b1 - b0) * cols
    mv_ms = sum(stages[k][0] for k in op_stages)
    mv_frac = round(mv_bytes / (mv_ms / 1e3) / 1e9 / peak, 4) if mv_ms > 0 else None
    rl = {
        "kernel": dom,
        "bound": "hbm",
        "achieved": round(achieved, 1),
        "peak": peak,
        "peak_source": peak_kind,
        "unit": "GB/s",
        "frac": round(achieved / peak, 4),
        "traffic": traffic,
        "traffic_source": ("ncu DRAM bytes per algorithmic byte of this stage's kernels (one captured launch each)"
                           " x algorithmic bytes per launch") if traffic is not None else None,
        "algorithmic_bytes_per_launch": round(bytes_total / max(1, dom_n)),
        "algorithmic_bytes_full_batch_fp32": b32[dom],
        "launches": dom_n,
        "timing": "per-stage CUDA events on the launching stream over a second pass of the timed steps",
    }
    return rl, mv_frac


def run_plain(args, F, B, X0, S, M, torch, capi, wl):
    """Plain per-system fp64 solves: one right-hand side at a time.

    Right-hand sides are solved one by one with GMRES+Jacobi on the fp64
    operator (the reference's plain method), each timed with CUDA events;
    their count over the summed time gives plain solves/s.  All columns up to
    32; every 8th of the 192 polydisperse columns.
    """
    cols = list(range(0, M, 1 if M <= 32 else 8))
    Xp = torch.empty((B.shape[0], 1), dtype=B.dtype, device=B.device)
    o = dict(tol=TOL, method=capi.METHOD_GMRES, restart=wl.restart, maxiter=1000, recip_fp32=False, refine=False)
    # warm-up: plans and buffers for M=1
    Xp.copy_(X0[:, :1])
    F.batch_solve(B[:, :1].contiguous(), Xp, S[:, :1].contiguous(), **o)
    torch.cuda.synchronize()
    tot_ms, mvs, ok = 0.0, 0, 0
    for c in cols:
        b = B[:, c:c + 1].contiguous()
        sc = S[:, c:c + 1].contiguous()
        Xp.copy_(X0[:, c:c + 1])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        r = F.batch_solve(b, Xp, sc, **o)
        e1.record()
        torch.cuda.synchronize()
        tot_ms += e0.elapsed_time(e1)
        mvs += r["matvecs"]
        rr = b - F.apply(Xp, self_coef=sc)
        ok += int(float(torch.linalg.vector_norm(rr) / torch.linalg.vector_norm(b)) <= TOL * 1.0001)
    n = len(cols)
    return {"value": round(n / (tot_ms / 1e3), 3), "unit": "solves/s", "rhs_sampled": n, "converged": ok,
            "ms_per_solve": round(tot_ms / n, 3), "matvecs_per_solve": mvs / n,
            "method": f"GMRES({wl.restart})+Jacobi, fp64 operator, 1 RHS per solve, no refinement, "
                      f"{len(cols)} of {M} RHS"}


def run_extras(args, capi, torch, dev, flush):
    """The other benchmark workloads, each timed like the headline step
    (warm-up, CUDA events after an L2 flush): BiCGSTAB on the monolayer, the
    N=1000 polydisperse packing (192 RHS) and the N=500 random packing
    (1 RHS); with the plain fp64 leg and per-dipole accuracy."""
    out = {}
    steps = max(2, min(args.steps, 5))
    warm = max(1, min(args.warmup, 3))
    todo = [("monolayer_bicgstab", "monolayer", capi.METHOD_BICGSTAB), ("poly3d", "poly3d", capi.METHOD_GMRES),
            ("c1", "c1", capi.METHOD_GMRES)]
    for key, name, method in todo:
        if name == args.workload and (method == capi.METHOD_GMRES) == (args.method == "gmres"):
            continue
        wl = Workload(name)
        T = Timed(wl, capi, torch, dev, args, method, flush)
        T.warm(warm)
        T.reports.clear()
        t = T.timed(steps)
        rel = T.true_residuals()
        conv = int(np.sum(rel <= TOL))
        acc, _ = T.accuracy()
        plain = run_plain(args, T.F, T.B, T.X0, T.S, T.M, torch, capi, wl)
        value = conv * steps / (t / 1e3)
        info = T.F.info()
        out[key] = {
            "workload": wl.label, "method": "bicgstab" if method == capi.METHOD_BICGSTAB else "gmres",
            "value": round(value, 3), "unit": "solves/s", "ms_per_step": round(t / steps, 3), "steps": steps,
            "rhs_per_step": T.M, "converged_per_step": conv, "max_true_rel_resid": float(rel.max()),
            "krylov_steps_per_rhs": round(float(np.mean([r["total_iterations"] / T.M for r in T.reports])), 2),
            "grid": info["grid"], "accuracy": acc, "plain_fp64": plain,
            "batched_vs_plain": round(value / plain["value"], 2),
        }
        del T
        torch.cuda.empty_cache()
    out["c4_adjoint"] = run_c4(args, torch)
    out["autotuned"] = {name: run_autotuned(args, capi, torch, dev, flush, name) for name in ("monolayer", "poly3d")}
    if not args.no_c5:
        out["c5_systems"] = run_c5(args, torch)
    return out


def run_autotuned(args, capi, torch, dev, flush, name):
    """The workload with the field autotuner's pick (xi, grid, support,
    spread tile measured on this GPU) in place of the reference's rule:
    tuning time, the pick, the batched solve timed like the headline, and
    per-dipole errors against the fp64 solutions of both the tuned operator
    and the rule's operator."""
    wl = Workload(name)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pick = wl.autotune(capi)
    torch.cuda.synchronize()
    tune_s = time.perf_counter() - t0
    steps = max(2, min(args.steps, 5))
    T = Timed(wl, capi, torch, dev, args, capi.METHOD_GMRES, flush, field=wl.field(capi, tuning=pick))
    T.warm(max(1, min(args.warmup, 3)))
    T.reports.clear()
    t = T.timed(steps)
    rel = T.true_residuals()
    conv = int(np.sum(rel <= TOL))
    acc, _ = T.accuracy()
    rule = wl.field(capi)
    rule.set_positions(wl.pos)
    Xrule = fp64_reference_solution(rule, T.B, T.X0, T.S, capi)
    vs_rule = dipole_errors(T.X, Xrule, len(wl.pos))
    info = T.F.info()
    out = {
        "workload": wl.label, "tune_s": round(tune_s, 3),
        "pick": {"xi": pick["xi"], "grid": list(info["grid"]), "support": info["stencil"], "tile": list(pick["tile"])},
        "rule": {"xi": XI, "grid": list(rule.info()["grid"]), "support": rule.info()["stencil"], "tile": [8, 8]},
        "apply_ms": round(pick["apply_ms"], 4), "apply_ms_rule": round(pick["apply_ms_rule"], 4),
        "operator_error": pick["error"], "operator_error_rule": pick["error_rule"],
        "error_bound": pick["error_bound"], "candidates": pick["candidates"], "accepted": pick["accepted"],
        "value": round(conv * steps / (t / 1e3), 3), "unit": "solves/s", "ms_per_step": round(t / steps, 3),
        "converged_per_step": conv, "rhs_per_step": T.M, "max_true_rel_resid": float(rel.max()),
        "accuracy": acc, "vs_rule_fp64": vs_rule,
    }
    del T, rule
    torch.cuda.empty_cache()
    return out


C5_FREQS = np.linspace(0.2, 1.0, 8)


def c5_systems(seed=5, total=250_000, lo=1000, hi=64000):
    """The uneven multi-system workload: 16 periodic systems, N log-uniform
    in [1k, 64k] (seeded) scaled to about 250k particles in all; even
    systems hexagonal monolayers (a = 5 nm, spacing 12 nm, 80 nm box height),
    odd ones random packings at phi in [0.05, 0.2] (a jittered simple-cubic
    lattice: spacing (4 pi a^3 / 3 phi)^(1/3), each particle displaced
    uniformly by less than half the gap, so none overlap); Drude spheres in
    eps_m 1.77, 8 frequencies 0.2-1.0 eV x 3 polarisations, dipoles and
    quadrupoles, tol 1e-6.  Returns cumpm_b200.systems.System objects (nm)."""
    from cumpm_b200.systems import System

    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(math.log(lo), math.log(hi), 16))
    n = np.clip(np.round(n * total / n.sum()), lo, hi).astype(int)
    eps = 4.0 - 1.8 ** 2 / (C5_FREQS ** 2 + 1j * C5_FREQS * 0.1)
    out = []
    for i, N in enumerate(n):
        if i % 2 == 0:
            cols = max(2, int(round(math.sqrt(N / (math.sqrt(3) / 2)))))
            rows = max(2, int(math.ceil(N / cols)))
            rows += rows % 2
            pos = np.array([[(c + 0.5 * (r % 2)) * 12.0, r * math.sqrt(3) / 2 * 12.0, 0.0]
                            for r in range(rows) for c in range(cols)])[:N]
            box = [cols * 12.0, rows * math.sqrt(3) / 2 * 12.0, 80.0]
        else:
            phi = rng.uniform(0.05, 0.2)
            sp = (4.0 * math.pi * RADIUS ** 3 / (3.0 * phi)) ** (1.0 / 3.0)
            m = int(math.ceil(N ** (1.0 / 3.0)))
            g = np.stack(np.meshgrid(*(np.arange(m),) * 3, indexing="ij"), axis=-1).reshape(-1, 3)
            g = g[rng.permutation(len(g))[:N]]
            jit = (sp - 2.0 * RADIUS) / 2.0 * 0.98
            pos = (g + 0.5) * sp + rng.uniform(-jit, jit, (N, 3))
            box = [m * sp] * 3
        out.append(System(box=box, positions=pos, eps_p=eps, radius=RADIUS, eps_m=EPS_M, tol=TOL, xi=XI,
                          quadrupoles=True, field_type="monodisperse",
                          options={"batch_all": True, "refine": True}))
    return out


def run_c5(args, torch):
    """The 16 uneven systems solved on this GPU through
    cumpm_b200.systems.solve_systems: one after another, and two at a time
    from host threads (each system its own device stream); wall clock with
    the device synchronised on both sides."""
    from cumpm_b200 import systems as S

    syst = c5_systems()
    out = {"workload": ("16 periodic systems, N log-uniform [1k, 64k] (seeded), sum N = "
                        f"{sum(s.num_particles for s in syst)}; hex monolayers and random packings "
                        "phi U[0.05, 0.2]; a = 5 nm Drude spheres, eps_m 1.77; dipoles + quadrupoles; "
                        "8 freqs 0.2-1.0 eV x 3 pols; tol 1e-6; batched mixed precision per system"),
           "sizes": [s.num_particles for s in syst], "rhs": 24 * len(syst)}
    for conc in (1, 2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = S.solve_systems(syst, concurrency=conc)
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        ok = all(np.all(np.isfinite(r["dipoles"])) for r in res)
        out[f"concurrency_{conc}"] = {"s": round(t, 3), "solves_per_s": round(out["rhs"] / t, 2),
                                      "systems_per_s": round(len(syst) / t, 3), "finite": bool(ok)}
        del res
        torch.cuda.empty_cache()
    return out


def rocksalt_lattice(spacing=7.0):
    """The differentiation workload: a 20 x 10 x 10 simple-cubic lattice
    (10 x 10 x 10 cells of two sites) with the two species alternating on
    it (rock-salt order), nearest-neighbour spacing `spacing` nm.  Species A
    (index 0): radius 3 nm, Drude; species B (-1): radius 2 nm, eps 2.5."""
    i, j, k = np.meshgrid(np.arange(20), np.arange(10), np.arange(10), indexing="ij")
    pos = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64) * spacing
    species = np.where((i + j + k).ravel() % 2 == 0, 0, -1)
    radii = np.where(species == 0, 3.0, 2.0)
    box = np.array([20.0, 10.0, 10.0]) * spacing
    return pos, radii, species, box


def run_c4(args, torch):
    """Adjoint gradients of the summed extinction cross-section (32
    frequencies over 0.3-1.0 eV, x-polarised) of the N=2000 rock-salt
    lattice with respect to every position and radius and the Drude omega_p
    and gamma: forward + adjoint solve + derivative contraction timed with
    CUDA events, and central finite differences (step 1e-4 relative) of the
    loss for omega_p, gamma and two coordinates checked against it."""
    from cumpm_b200.adjoint import extinction_loss, wavenumber_from_ev

    pos, radii, species, box = rocksalt_lattice()
    omega = np.linspace(0.3, 1.0, 32)
    cfg = dict(box=box, omega=omega, species=species, eps_inf=[4.0], eps_m=EPS_M,
               eps_const=np.where(species < 0, 2.5, 0.0).astype(complex),
               wavenumber=wavenumber_from_ev(omega, EPS_M), tol=TOL, length_scale=2.0)

    def leaves(p=pos, r=radii, wp=1.8, g=0.1):
        return (torch.tensor(p, dtype=torch.float64, requires_grad=True),
                torch.tensor(r, dtype=torch.float64, requires_grad=True),
                torch.tensor([wp], dtype=torch.float64, requires_grad=True),
                torch.tensor([g], dtype=torch.float64, requires_grad=True))

    def grad_once():
        P, R, W, G = leaves()
        L = extinction_loss(P, R, W, G, **cfg)
        L.backward()
        return float(L), P.grad.numpy(), R.grad.numpy(), float(W.grad[0]), float(G.grad[0])

    grad_once()   # warm-up: plans and buffers
    steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        L, gp, gr, gw, gg = grad_once()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps

    def loss_at(**kw):
        with torch.no_grad():
            return float(extinction_loss(*leaves(**kw), **cfg))

    checks = {}
    h = 1e-4
    for name, base, an in (("omega_p", 1.8, gw), ("gamma", 0.1, gg)):
        d = h * base
        fd = (loss_at(**{("wp" if name == "omega_p" else "g"): base + d})
              - loss_at(**{("wp" if name == "omega_p" else "g"): base - d})) / (2 * d)
        checks[name] = {"adjoint": an, "fd": fd, "rel_err": abs(an - fd) / max(abs(fd), 1e-300)}
    # the radius of a species-A particle (the length unit, the smallest
    # radius, is held fixed); positions are checked in the tests, where the
    # step can be kept inside one linear segment of the pair tables (a
    # lattice puts every neighbour distance on a table node)
    for idx in (0, 2):
        d = h * radii[idx]
        rp, rm = radii.copy(), radii.copy()
        rp[idx] += d
        rm[idx] -= d
        fd = (loss_at(r=rp) - loss_at(r=rm)) / (2 * d)
        checks[f"radius[{idx}]"] = {"adjoint": float(gr[idx]), "fd": fd,
                                    "rel_err": abs(float(gr[idx]) - fd) / max(abs(fd), 1e-300)}
    return {"workload": "N=2000 rock-salt lattice (20x10x10 sites, spacing 7 nm): A radius 3 nm Drude (eps_inf 4, "
                        "wp 1.8 eV, gamma 0.1 eV), B radius 2 nm eps 2.5, eps_m 1.77; loss = extinction summed over "
                        "32 freqs 0.3-1.0 eV (x-polarised); gradients w.r.t. all positions, radii, wp, gamma",
            "value": round(1e3 / ms, 3), "unit": "gradients/s", "ms_per_gradient": round(ms, 2), "steps": steps,
            "loss": L, "fd_checks": checks,
            "method": "forward batched fp64 solve (32 RHS) + adjoint solve with the same operator + derivative "
                      "contraction on the GPU; FD step 1e-4 relative"}


def run_e2e(args, torch, wl):
    """Same workload through the public drop-in API with host buffers."""
    import cumpm_b200 as cuMPM

    rad = wl.radius_nm if not wl.mono else float(wl.radius_nm[0])
    E0 = None if wl.K == 3 else [[1.0, 0.0, 0.0]]
    mk = lambda: cuMPM.dipole_solver(wl.box_nm, wl.eps, radius=rad, eps_m=EPS_M, tol=TOL, quiet=True, E0=E0,
                                     solver_type=args.method)
    s = mk()
    s.set_solver_options(batch_all=True, refine=True, inner_tol=args.inner_tol)
    s.compute(wl.pos_nm)  # warm-up (plans, precalc buffers)
    # compute() takes host positions, copies the batch's inputs to the device,
    # solves, and copies this step's dipoles back into host memory before it
    # returns; it is timed alone, as the reference's own benchmark times it
    # (benchmarks/benchmark_cumpm_vs_pympm.py:77-79).  get_dipoles() (a host
    # copy of every frame so far) is read once after the loop.
    times = []
    for k in range(max(2, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.compute(wl.pos_nm)
        t1 = time.perf_counter()
        times.append(t1 - t0)
    d = s._solver.get_dipoles(True)
    if d.shape[0] != max(2, args.steps) + 1 or not np.all(np.isfinite(d[-1])):
        raise RuntimeError("e2e: unexpected dipoles from get_dipoles()")
    N = len(wl.pos)
    M = wl.M
    # per step: positions and the batch's initial guesses (the right-hand
    # sides and self terms depend only on the frequencies and stay on the
    # device from the warm-up frame on)
    h2d = 3 * N * 8 + 3 * N * M * 16
    d2h = 3 * N * M * 16
    t = float(np.median(times))
    return {"value": round(M / t, 3), "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "timing": "wall clock around dipole_solver.compute() (host positions in, this step's dipoles in host "
                      "memory out), median of steps; get_dipoles() read once after the loop"}


# ---------------------------------------------------------------- baselines

REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def reference_gpu_child(args):
    """Runs in a child process (an error exit of the reference build cannot
    take the benchmark down): the reference build's own Dipole_Solver on the
    monolayer workload, timed as the reference's benchmark times it
    (benchmarks/benchmark_cumpm_vs_pympm.py:35-89: a small warm-up solve,
    then wall clock around one compute() of all frequencies and
    polarisations), for fp64 ("double") and the default AUTO precision, with
    GMRES and BiCGSTAB.  Writes the dipoles of each run to args.ref_out and
    prints one JSON line."""
    import glob

    if not glob.glob(os.path.join(REF_DIR, "_cuMPM*.so")):
        print(json.dumps({"unavailable": "reference build oracle/_ref not present"}))
        return
    sys.path.insert(0, REF_DIR)
    import _cuMPM as R

    wl = Workload("monolayer")
    pos, box = wl.pos_nm, wl.box_nm
    eps = [complex(e) for e in wl.eps]

    def solver(prec, method, e, tol):
        return R.Dipole_Solver(list(map(float, box)), e, radius=[RADIUS], eps_m=EPS_M, xi=XI, tol=tol, quiet=True,
                               guess_type="derivative", solver_type=method, field_type="monodisperse", E0=[],
                               solve_quadrupoles=False, quad_idxs=[], precision=prec)

    w = solver(R.PrecisionMode.AUTO, "gmres", eps[:2], 1e-3)   # warm-up: context, cuFFT
    w.compute(list(pos[:100, 0]), list(pos[:100, 1]), list(pos[:100, 2]))
    res = {}
    dips = {}
    for pname, prec in (("double", R.PrecisionMode.DOUBLE), ("auto", R.PrecisionMode.AUTO)):
        for method in ("gmres", "bicgstab"):
            s = solver(prec, method, eps, TOL)
            t0 = time.perf_counter()
            s.compute(list(pos[:, 0]), list(pos[:, 1]), list(pos[:, 2]))
            t = time.perf_counter() - t0
            d = np.asarray(s.get_dipoles(True))
            key = f"{pname}_{method}"
            dips[key] = d.reshape(-1)
            res[key] = {"s_per_compute": round(t, 4), "rhs": wl.M, "rhs_per_s": round(wl.M / t, 3)}
            del s
    np.savez(args.ref_out, **dips)
    print(json.dumps(res), flush=True)


def reference_gpu_leg(args, wl, F, B, S, Xref, torch):
    """The reference build (oracle/_ref) solving the same monolayer on this
    GPU, in a child process; its dipoles are checked here with this build's
    fp64 operator (true residual) and against the fp64 solution."""
    if wl.name != "monolayer" or wl.K != 3:
        return None
    with tempfile.TemporaryDirectory() as td:
        outp = os.path.join(td, "ref_dipoles.npz")
        cmd = [sys.executable, os.path.abspath(__file__), "--_reference-gpu-child", "--ref-out", outp]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
        except subprocess.TimeoutExpired:
            return {"unavailable": "reference build run exceeded 600 s"}
        lines = [ln for ln in r.stdout.strip().splitlines() if ln.startswith("{")]
        if r.returncode != 0 or not lines:
            return {"unavailable": f"reference build run failed (rc {r.returncode}): {r.stderr.strip()[-300:]}"}
        res = json.loads(lines[-1])
        if "unavailable" in res:
            return res
        dz = np.load(outp)
        N, K, W = len(wl.pos), wl.K, len(wl.eps)
        scale = EPS_M * wl.unit ** 3
        for key, v in res.items():
            d = dz[key].reshape(-1, W, N, K, 3)[-1] / scale           # (W, N, K, 3), solver units
            X = np.transpose(d, (1, 3, 0, 2)).reshape(3 * N, W * K)  # row 3i+c, column w*K+k
            X = np.ascontiguousarray(X)
            Xt = torch.tensor(X, dtype=torch.complex128, device=B.device)
            R = B - F.apply(Xt, self_coef=S)
            rel = (torch.linalg.vector_norm(R, dim=0) / torch.linalg.vector_norm(B, dim=0)).cpu().numpy()
            v["max_true_rel_resid"] = float(rel.max())
            v["rhs_within_true_resid_tol"] = int(np.sum(rel <= TOL))
            if Xref is not None:
                v.update(dipole_errors(Xt, Xref, N))
    return {"runs": res,
            "protocol": "reference build (oracle/_ref, compiled from the reference sources for sm_100a) Dipole_Solver "
                        "on the same workload: wall clock around one compute() of 10 freqs x 3 pols after a small "
                        "warm-up solve, as benchmarks/benchmark_cumpm_vs_pympm.py times it; one RHS at a time, "
                        "its own stop rule |D^-1 r| < tol |b|; residuals and errors computed here with this "
                        "build's fp64 operator"}


def _cpu_operator(wl, threads):
    from oracle import mpm_oracle as O

    if wl.mono:
        op = O.MonoEwaldOperator(wl.box, TOL, XI, True, fft_workers=threads)
    else:
        op = O.PolyEwaldOperator(wl.box, TOL, XI, wl.radius, True)
    op.set_positions(wl.pos)
    return op


def cpu_solve(op, wl, B, X0, S, m):
    """One full fp64 GMRES+Jacobi solve of column m on the CPU port (the
    reference's plain method: restart 50, stop rule |D^-1 r| < tol |b|);
    (seconds, matvecs)."""
    from oracle import mpm_oracle as O

    N = len(wl.pos)
    count = [0]

    def A(v):
        count[0] += 1
        return op.apply(v, S[:, m])

    Mj = O.jacobi_inverse(S[:, m], N)
    t0 = time.perf_counter()
    O.gmres(A, B[:, m], X0[:, m], TOL, Mj, restart=wl.restart)
    return time.perf_counter() - t0, count[0]


def cpu_baseline(args, wl, min_s=10.0):
    """Full fp64 single-right-hand-side solves of the CPU port (oracle/) on
    the full workload, on all host threads (FFTs), until about min_s seconds
    of CPU work: solves/s = solves / time."""
    threads = os.cpu_count() or 1
    op = _cpu_operator(wl, threads)
    B, X0, S = problem_arrays(wl)
    ts, mvs = [], []
    while not ts or (sum(ts) < min_s and len(ts) < wl.M):
        t, n = cpu_solve(op, wl, B, X0, S, len(ts))
        ts.append(t)
        mvs.append(n)
    return {"value": round(len(ts) / sum(ts), 5), "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"{len(ts)} full fp64 GMRES({wl.restart})+Jacobi solves (columns 0..{len(ts) - 1}) of the CPU "
                      f"port (oracle/) on the full workload, {np.mean(ts):.2f} s and {np.mean(mvs):.1f} matvecs "
                      f"each, FFTs on {threads} threads"}


def run_reference(args, rank):
    """CPU port of the reference solve on the host cores (rank 0 only): each
    timed step is one full fp64 single-right-hand-side GMRES solve (column
    step mod M of the workload); warm-up steps are one operator application
    each."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    wl = Workload(args.workload)
    op = _cpu_operator(wl, threads)
    B, X0, S = problem_arrays(wl)
    for _ in range(max(1, args.warmup)):
        op.apply(X0[:, 0], S[:, 0])
    ts, mvs = [], []
    for k in range(max(1, args.steps)):
        t, n = cpu_solve(op, wl, B, X0, S, k % wl.M)
        ts.append(t)
        mvs.append(n)
    t = float(np.median(ts))
    v = 1.0 / t
    line = {
        "impl": "reference",
        "metric": METRICS[wl.name],
        "value": round(v, 5), "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t * 1e3, 1), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128", "data": DATA[wl.name],
        "config": {"workload": wl.label,
                   "step": f"one full fp64 GMRES({wl.restart})+Jacobi solve of one right-hand side (column step mod "
                           f"{wl.M}) with the CPU port of the reference algorithm, stop rule |D^-1 r| < tol |b|; "
                           f"{np.mean(mvs):.1f} matvecs per solve"},
        "cpu_baseline": {"value": round(v, 5), "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{len(ts)} full solves, median {t:.2f} s each, FFTs on {threads} threads"},
        "e2e": {"value": round(v, 5), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_apply_only(args):
    """Operator applications only (for profiler captures): the workload's
    field at all its right-hand sides, fp32 reciprocal and real space (the
    inner solves' operator), args.apply_only times after one untimed
    application of each precision; prints the mean time per application."""
    import torch

    from cumpm_b200 import capi

    torch.cuda.set_device(0)
    wl = Workload(args.workload)
    F = wl.field(capi)
    F.set_positions(wl.pos)
    B, X0, S = device_problem(wl, torch, torch.device("cuda", 0))
    Y = torch.empty_like(X0)
    F.apply(X0, Y, self_coef=S, recip_fp32=False)
    F.apply(X0, Y, self_coef=S, recip_fp32=True, real_fp32=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.apply_only):
        F.apply(X0, Y, self_coef=S, recip_fp32=True, real_fp32=True)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"workload": wl.name, "M": wl.M, "applications": args.apply_only,
                      "ms_per_apply": round(e0.elapsed_time(e1) / max(1, args.apply_only), 4),
                      "info": F.info()}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--method", default="gmres", choices=["gmres", "bicgstab"])
    ap.add_argument("--inner-tol", type=float, default=1e-4, help="floor of one inner solve's reduction")
    ap.add_argument("--no-compact", action="store_true", help="idle columns still go through the operator")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-profile", action="store_true", help="skip the stage-timer pass")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-system fp64 leg")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the per-dipole fp64 comparison")
    ap.add_argument("--no-extras", action="store_true", help="skip the other workloads")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip the reference build's GPU solve")
    ap.add_argument("--no-c5", action="store_true", help="skip the 16-system workload")
    ap.add_argument("--c5-only", action="store_true", help="run only the 16-system workload and print its line")
    ap.add_argument("--workload", default="monolayer", choices=["monolayer", "poly3d", "c1"],
                    help="monolayer: the headline N=4000 case; poly3d: the N=1000 polydisperse 192-RHS case; "
                         "c1: the N=500 single-RHS case")
    ap.add_argument("--apply-only", type=int, default=0, metavar="K",
                    help="only apply the workload's operator K times (fp32, all right-hand sides): profiler runs")
    ap.add_argument("--_reference-gpu-child", dest="ref_child", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--ref-out", default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.ref_child:
        reference_gpu_child(args)
        return
    if args.apply_only:
        run_apply_only(args)
        return
    if args.c5_only:
        import torch

        print(json.dumps({"c5_systems": run_c5(args, torch)}))
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
