"""Many independent periodic systems across the ranks of one job.

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


def solve_one(system: System) -> Dict[str, np.ndarray]:
    """Solve one system with ``dipole_solver``; its physical results."""
    from .solver import dipole_solver

    s = dipole_solver(system.box, system.eps_p, radius=system.radius, eps_m=system.eps_m, xi=system.xi,
                      tol=system.tol, quiet=True, solver_type=system.solver_type, field_type=system.field_type,
                      E0=system.E0, quadrupoles=system.quadrupoles, precision=system.precision, **system.extra)
    s.compute(np.asarray(system.positions, dtype=np.float64))
    out = {"eff_polarizability": np.asarray(s.get_eff_polarizability()),
           "dipoles": np.asarray(s.get_dipoles())}
    if system.quadrupoles is not False and system.quadrupoles is not None:
        out["quadrupoles"] = np.asarray(s.get_quadrupoles())
    return out


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


def solve_systems(systems: Sequence[System], *, dist=None,
                  solve_fn: Callable[[System], Dict[str, np.ndarray]] = solve_one,
                  bind_device: Optional[Callable[[int], None]] = _bind_device) -> List[Dict[str, np.ndarray]]:
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
    """
    sizes = [s.num_particles for s in systems]
    if dist is None or not dist.is_initialized():
        return [solve_fn(s) for s in systems]
    rank, world = dist.get_rank(), dist.get_world_size()
    if bind_device is not None:
        bind_device(local_device_ordinal(rank))
    mine = partition(sizes, world)[rank]
    local = []
    for i in mine:
        try:
            local.append((i, True, solve_fn(systems[i])))
        except Exception as e:  # reported on every rank after the gather
            local.append((i, False, f"rank {rank}: {type(e).__name__}: {e}"))
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
