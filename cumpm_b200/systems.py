"""Many independent periodic systems across the ranks of one job, and one
system's frequencies across the ranks (``solve_sharded``).

Systems (different sizes, boxes, materials, with or without quadrupoles)
share nothing but the code: each is a ``dipole_solver`` of its own.  Across
GPUs they are whole units: every rank solves the systems assigned to it,
one process per GPU, and the moments are gathered once at the end; there is
no collective inside a solve.

Assignment is longest-processing-time first by the cost of one operator
application, which the grid transforms dominate: cost(N) = N log2 N.  The
largest remaining system goes to the least-loaded rank (lowest rank on a
tie), so the result is deterministic and every rank computes the same
assignment without communicating.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np


@dataclass
class System:
    """One periodic system: the arguments of ``dipole_solver`` plus its
    positions (N, 3) or frames (F, N, 3)."""
    box: Sequence[float]
    positions: np.ndarray
    eps_p: object
    radius: object = 1.0
    eps_m: float = 1.0
    xi: float = 0.5
    tol: float = 1e-3
    quadrupoles: object = False
    solver_type: str = "gmres"
    field_type: str = "auto"
    E0: object = None
    precision: Optional[str] = None
    extra: Dict[str, object] = field(default_factory=dict)
    options: Dict[str, object] = field(default_factory=dict)   # set_solver_options keywords

    @property
    def num_particles(self) -> int:
        return int(np.asarray(self.positions).shape[-2])


def system_cost(n: int) -> float:
    """Relative cost of one operator application of an N-particle system."""
    n = max(int(n), 2)
    return n * math.log2(n)


def partition(sizes: Sequence[int], world_size: int) -> List[List[int]]:
    """Indices of the systems each rank solves (longest first, to the
    least-loaded rank).  Every index appears exactly once; each rank's list
    is in increasing index order."""
    if world_size < 1:
        raise ValueError("world_size must be at least 1")
    order = sorted(range(len(sizes)), key=lambda i: (-system_cost(sizes[i]), i))
    load = [0.0] * world_size
    out: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += system_cost(sizes[i])
    return [sorted(s) for s in out]


def _solver_for(system: System):
    from .solver import dipole_solver

    s = dipole_solver(system.box, system.eps_p, radius=system.radius, eps_m=system.eps_m, xi=system.xi,
                      tol=system.tol, quiet=True, solver_type=system.solver_type, field_type=system.field_type,
                      E0=system.E0, quadrupoles=system.quadrupoles, precision=system.precision, **system.extra)
    if system.options:
        s.set_solver_options(**system.options)
    s.compute(np.asarray(system.positions, dtype=np.float64))
    return s


def _has_quads(system: System) -> bool:
    return system.quadrupoles is not False and system.quadrupoles is not None


def solve_one(system: System) -> Dict[str, np.ndarray]:
    """Solve one system with ``dipole_solver``; its physical results."""
    s = _solver_for(system)
    out = {"eff_polarizability": np.asarray(s.get_eff_polarizability()),
           "dipoles": np.asarray(s.get_dipoles())}
    if _has_quads(system):
        out["quadrupoles"] = np.asarray(s.get_quadrupoles())
    return out


def solve_one_unsqueezed(system: System) -> Dict[str, np.ndarray]:
    """``solve_one`` with every axis kept: eff_polarizability (W, K, 3),
    dipoles (frames, W, N, K, 3), quadrupoles (frames, W, Nq, K, 5)."""
    s = _solver_for(system)
    raw = s._solver
    out = {"eff_polarizability": np.asarray(raw.get_eff_polarizability(True)),
           "dipoles": np.asarray(raw.get_dipoles(True))}
    if _has_quads(system):
        out["quadrupoles"] = np.asarray(raw.get_quadrupoles(True))
    return out


# the frequency axis of each unsqueezed result
_FREQ_AXIS = {"eff_polarizability": 0, "dipoles": 1, "quadrupoles": 1}


def frequency_shards(num_freqs: int, world_size: int) -> List[List[int]]:
    """Contiguous, balanced blocks of frequency indices, one per rank (the
    first num_freqs % world_size ranks take one more; ranks beyond
    num_freqs take none)."""
    if world_size < 1:
        raise ValueError("world_size must be at least 1")
    return [list(map(int, b)) for b in np.array_split(np.arange(int(num_freqs)), world_size)]


def _eps_rows(eps_p) -> np.ndarray:
    """eps_p as (W, 1) or (W, N): a scalar is one frequency, a 1-D array one
    value per frequency, a 2-D array one row per frequency."""
    e = np.asarray(eps_p, dtype=np.complex128)
    if e.ndim == 0:
        return e.reshape(1, 1)
    if e.ndim == 1:
        return e.reshape(-1, 1)
    if e.ndim == 2:
        return e
    raise ValueError("eps_p must be a scalar, 1D array, or 2D array")


def local_device_ordinal(rank: int, env=None, device_count: Optional[int] = None) -> int:
    """The GPU a rank binds to: LOCAL_RANK when the launcher sets it
    (torchrun does), else the rank modulo the visible device count."""
    env = os.environ if env is None else env
    if "LOCAL_RANK" in env:
        return int(env["LOCAL_RANK"])
    if device_count is None:
        import torch

        device_count = torch.cuda.device_count()
    return rank % max(1, int(device_count))


def _bind_device(ordinal: int) -> None:
    import torch

    if torch.cuda.is_available():
        torch.cuda.set_device(ordinal)


class SystemSolveError(RuntimeError):
    """One or more systems failed on some rank; raised on every rank after
    the results have been exchanged, so no rank is left waiting."""


def _solve_share(systems: Sequence[System], idx: Sequence[int], solve_fn, concurrency: int,
                 bind: Optional[Callable[[], None]], rank: int):
    """(index, ok, result or message) for each system of idx, solved one
    after another or, with concurrency > 1, by that many host threads at
    once (each solve has its own device stream, so small systems overlap on
    the GPU; the native solve releases the interpreter lock)."""
    def one(i):
        try:
            return (i, True, solve_fn(systems[i]))
        except Exception as e:  # reported on every rank after the gather
            return (i, False, f"rank {rank}: {type(e).__name__}: {e}")

    if concurrency <= 1 or len(idx) <= 1:
        return [one(i) for i in idx]
    from concurrent.futures import ThreadPoolExecutor

    # largest first, so that the long solves start early; results in idx order
    order = sorted(idx, key=lambda i: -system_cost(systems[i].num_particles))
    with ThreadPoolExecutor(max_workers=int(concurrency), initializer=bind) as ex:
        done = dict(zip(order, ex.map(one, order)))
    return [done[i] for i in idx]


def solve_systems(systems: Sequence[System], *, dist=None,
                  solve_fn: Callable[[System], Dict[str, np.ndarray]] = solve_one,
                  bind_device: Optional[Callable[[int], None]] = _bind_device,
                  concurrency: int = 1) -> List[Dict[str, np.ndarray]]:
    """Solve every system once across the ranks of ``dist`` (an initialised
    ``torch.distributed``, or None for one process) and return all results,
    in system order, on every rank.

    Each rank first binds its own GPU (``local_device_ordinal``; pass
    ``bind_device=None`` when the caller has done so), then solves its
    share (:func:`partition`); the only exchange is one
    ``all_gather_object`` of the results at the end, which every rank joins,
    whether its share is empty or not and whether its solves succeeded or
    not.  A solve that raises is caught and its message travels in the
    gather; afterwards every rank raises :class:`SystemSolveError` naming the
    failed systems.

    ``concurrency`` > 1 solves up to that many of a rank's systems at once
    from host threads (each bound to the rank's GPU), so that systems too
    small to fill the GPU overlap; results do not depend on it.
    """
    sizes = [s.num_particles for s in systems]
    if dist is None or not dist.is_initialized():
        if concurrency <= 1:
            return [solve_fn(s) for s in systems]
        res = _solve_share(systems, range(len(systems)), solve_fn, concurrency, None, 0)
        bad = [f"system {i} ({r})" for i, ok, r in res if not ok]
        if bad:
            raise SystemSolveError("; ".join(bad))
        return [r for _, _, r in res]
    rank, world = dist.get_rank(), dist.get_world_size()
    ordinal = local_device_ordinal(rank)
    if bind_device is not None:
        bind_device(ordinal)
    mine = partition(sizes, world)[rank]
    bind = (lambda: bind_device(ordinal)) if bind_device is not None else None
    local = _solve_share(systems, mine, solve_fn, concurrency, bind, rank)
    gathered: List[object] = [None] * world
    dist.all_gather_object(gathered, local)
    out: List[Optional[Dict[str, np.ndarray]]] = [None] * len(systems)
    errors = []
    for part in gathered:
        for i, ok, res in part:
            if not ok:
                errors.append(f"system {i} ({res})")
                continue
            if out[i] is not None:
                raise RuntimeError(f"system {i} solved on two ranks")
            out[i] = res
    if errors:
        raise SystemSolveError("; ".join(errors))
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise RuntimeError(f"systems {missing} were not solved")
    return out  # type: ignore[return-value]


def solve_sharded(system: System, *, dist=None,
                  solve_fn: Callable[[System], Dict[str, np.ndarray]] = solve_one_unsqueezed,
                  bind_device: Optional[Callable[[int], None]] = _bind_device) -> Dict[str, np.ndarray]:
    """One system, its frequencies split across the ranks of ``dist``
    (strong scaling of one solve): every rank solves the same positions for
    its contiguous block of frequencies (:func:`frequency_shards`) with its
    own ``dipole_solver``, and one ``all_gather_object`` returns the results,
    concatenated along the frequency axis in frequency order and squeezed
    as ``dipole_solver``'s getters squeeze, on every rank.  The frequencies
    are independent solves (the warm start of each block begins from the
    mean-field guess).  A rank whose share is empty, or whose solve raises,
    still joins the gather; a failure raises :class:`SystemSolveError` on
    every rank."""
    rows = _eps_rows(system.eps_p)
    W = rows.shape[0]

    def part(idx):
        if not idx:
            return None
        sub = System(**{**system.__dict__, "eps_p": rows[idx] if rows.shape[1] > 1 else rows[idx, 0]})
        return solve_fn(sub)

    if dist is None or not dist.is_initialized():
        parts = [part(list(range(W)))]
    else:
        rank, world = dist.get_rank(), dist.get_world_size()
        if bind_device is not None:
            bind_device(local_device_ordinal(rank))
        mine = frequency_shards(W, world)[rank]
        try:
            local = (True, part(mine))
        except Exception as e:  # reported on every rank after the gather
            local = (False, f"rank {rank}: {type(e).__name__}: {e}")
        gathered: List[object] = [None] * world
        dist.all_gather_object(gathered, local)
        errors = [res for ok, res in gathered if not ok]
        if errors:
            raise SystemSolveError("; ".join(errors))
        parts = [res for ok, res in gathered]
    parts = [p for p in parts if p is not None]
    out = {}
    for key, axis in _FREQ_AXIS.items():
        if key in parts[0]:
            out[key] = np.squeeze(np.concatenate([p[key] for p in parts], axis=axis))
    return out
