"""Independent systems across ranks (cumpm_b200.systems): the assignment of
whole systems to ranks and the one gather at the end, on CPU with gloo ranks
and a stand-in solve (no GPU)."""
import math
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from cumpm_b200 import systems as S  # noqa: E402


def uneven_sizes(seed, n=16, lo=1000, hi=64000):
    """Particle counts drawn log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    return [int(round(math.exp(x))) for x in rng.uniform(math.log(lo), math.log(hi), n)]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8, 20])
def test_partition_covers_every_system_once(world):
    sizes = uneven_sizes(5)
    parts = S.partition(sizes, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(sizes)))
    assert all(p == sorted(p) for p in parts)
    assert S.partition(sizes, world) == parts   # deterministic


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
@pytest.mark.parametrize("world", [2, 4, 8])
def test_partition_is_balanced_within_the_lpt_bound(seed, world):
    sizes = uneven_sizes(seed)
    cost = [S.system_cost(n) for n in sizes]
    loads = [sum(cost[i] for i in p) for p in S.partition(sizes, world)]
    lower = max(sum(cost) / world, max(cost))   # no assignment does better
    assert max(loads) <= (4.0 / 3.0) * lower + 1e-9


def test_more_ranks_than_systems_leaves_ranks_empty():
    parts = S.partition([1000, 5000, 2000], 5)
    assert sorted(len(p) for p in parts) == [0, 0, 1, 1, 1]
    assert parts[0] == [1]   # the largest system goes to rank 0


def test_partition_rejects_no_ranks():
    with pytest.raises(ValueError):
        S.partition([10], 0)


def _fake_solve(system):
    return {"n": np.array([system.num_particles]), "sum": np.asarray(system.positions).sum(axis=-2)}


def _systems():
    rng = np.random.default_rng(9)
    out = []
    for n in (5, 17, 3, 11, 8, 2, 13):
        out.append(S.System(box=[10.0, 10.0, 10.0], positions=rng.uniform(0, 10, (n, 3)), eps_p=[2.0 + 0.1j]))
    return out


def test_single_process_solves_in_order():
    res = S.solve_systems(_systems(), solve_fn=_fake_solve)
    assert [int(r["n"][0]) for r in res] == [5, 17, 3, 11, 8, 2, 13]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    from cumpm_b200 import systems as S2

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        solved = []

        def solve(system):
            solved.append(system.num_particles)
            return _fake_solve(system)

        res = S2.solve_systems(_systems(), dist=dist, solve_fn=solve)
        q.put((rank, [int(r["n"][0]) for r in res], [r["sum"].tolist() for r in res], solved))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_share_the_systems_and_gather_once(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + world * 50 + (os.getpid() % 40)
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, ns, sums, solved = q.get(timeout=120)
        out[r] = (ns, sums, solved)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    serial = S.solve_systems(_systems(), solve_fn=_fake_solve)
    sizes = [s.num_particles for s in _systems()]
    parts = S.partition(sizes, world)
    for r in range(world):
        ns, sums, solved = out[r]
        assert ns == [int(x["n"][0]) for x in serial]
        np.testing.assert_array_equal(np.array(sums), np.array([x["sum"] for x in serial]))
        assert solved == [sizes[i] for i in parts[r]]   # each rank solved its own share only


def _rank_fail(rank, world, port, q):
    """Rank 1's solve of its first system raises; every rank must come back
    from the gather and raise the same error (none waits forever)."""
    sys.path.insert(0, ROOT)
    from cumpm_b200 import systems as S2

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bound = []
    try:
        calls = []

        def solve(system):
            calls.append(system.num_particles)
            if rank == 1 and len(calls) == 1:
                raise ValueError("injected failure")
            return _fake_solve(system)

        try:
            S2.solve_systems(_systems(), dist=dist, solve_fn=solve, bind_device=bound.append)
            q.put((rank, "no error", bound))
        except S2.SystemSolveError as e:
            q.put((rank, str(e), bound))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_a_failing_solve_raises_on_every_rank_without_a_hang():
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29950 + (os.getpid() % 40)
    procs = [ctx.Process(target=_rank_fail, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, msg, bound = q.get(timeout=120)
        out[r] = (msg, bound)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    first_of_rank1 = S.partition([s.num_particles for s in _systems()], world)[1][0]
    for r in range(world):
        msg, bound = out[r]
        assert f"system {first_of_rank1} (rank 1: ValueError: injected failure)" == msg
        assert bound == [r]   # each rank bound the GPU of its LOCAL_RANK before solving


def test_local_device_ordinal():
    assert S.local_device_ordinal(5, env={"LOCAL_RANK": "1"}) == 1
    assert S.local_device_ordinal(5, env={}, device_count=4) == 1
    assert S.local_device_ordinal(3, env={}, device_count=0) == 0


def test_solve_one_calls_dipole_solver_with_its_own_arguments(monkeypatch):
    """solve_one's call binds to the real dipole_solver signature and reads
    back the three results (quadrupoles only when asked for)."""
    import inspect

    from cumpm_b200 import solver

    sig = inspect.signature(solver.dipole_solver.__init__)
    seen = []

    class Recorder:
        def __init__(self, *a, **k):
            sig.bind(None, *a, **k)
            seen.append(k)

        def compute(self, pos):
            self.n = pos.shape[-2]

        def get_eff_polarizability(self):
            return np.zeros(3)

        def get_dipoles(self):
            return np.zeros((self.n, 3))

        def get_quadrupoles(self):
            return np.zeros((1, 5))

    monkeypatch.setattr(solver, "dipole_solver", Recorder)
    sysq = S.System(box=[20.0] * 3, positions=np.zeros((4, 3)), eps_p=[3.0], radius=1.0, eps_m=1.77, tol=1e-6,
                    quadrupoles=[0, 2], extra={"guess_type": "previous"})
    res = S.solve_one(sysq)
    assert set(res) == {"eff_polarizability", "dipoles", "quadrupoles"} and res["dipoles"].shape == (4, 3)
    assert seen[-1]["quadrupoles"] == [0, 2] and seen[-1]["guess_type"] == "previous" and seen[-1]["quiet"] is True
    res = S.solve_one(S.System(box=[20.0] * 3, positions=np.zeros((4, 3)), eps_p=[3.0]))
    assert set(res) == {"eff_polarizability", "dipoles"}


# ---- one system's frequencies across ranks (solve_sharded) -----------------

@pytest.mark.parametrize("W,world", [(10, 1), (10, 3), (10, 4), (2, 3), (64, 8)])
def test_frequency_shards_are_contiguous_and_balanced(W, world):
    sh = S.frequency_shards(W, world)
    assert len(sh) == world
    assert [i for b in sh for i in b] == list(range(W))
    sizes = [len(b) for b in sh]
    assert max(sizes) - min(sizes) <= 1
    assert sizes == sorted(sizes, reverse=True)


def _fake_unsqueezed(system):
    """Results whose values name their frequency: eff (W, K, 3) and dipoles
    (1, W, N, K, 3) filled with eps_p of each frequency."""
    e = np.atleast_1d(np.asarray(system.eps_p, dtype=np.complex128))
    W, N = len(e), system.num_particles
    return {"eff_polarizability": np.broadcast_to(e[:, None, None], (W, 3, 3)).copy(),
            "dipoles": np.broadcast_to(e[None, :, None, None, None], (1, W, N, 3, 3)).copy()}


def _sharded_system():
    rng = np.random.default_rng(4)
    return S.System(box=[10.0, 10.0, 10.0], positions=rng.uniform(0, 10, (6, 3)),
                    eps_p=np.arange(10) + 2.0 + 0.5j)


def test_sharded_single_process_is_the_whole_sweep():
    out = S.solve_sharded(_sharded_system(), solve_fn=_fake_unsqueezed)
    e = np.arange(10) + 2.0 + 0.5j
    np.testing.assert_array_equal(out["eff_polarizability"][:, 0, 0], e)
    assert out["dipoles"].shape == (10, 6, 3, 3)


def _rank_sharded(rank, world, port, q, fail):
    sys.path.insert(0, ROOT)
    from cumpm_b200 import systems as S2

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seen, bound = [], []

        def solve(system):
            seen.append(np.atleast_1d(system.eps_p).real.tolist())
            if fail and rank == 1:
                raise RuntimeError("injected")
            return _fake_unsqueezed(system)

        try:
            out = S2.solve_sharded(_sharded_system(), dist=dist, solve_fn=solve, bind_device=bound.append)
            q.put((rank, out["eff_polarizability"][:, 0, 0].tolist(), out["dipoles"].shape, seen, bound))
        except S2.SystemSolveError as e:
            q.put((rank, str(e), None, seen, bound))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,fail", [(3, False), (2, True)])
def test_gloo_ranks_shard_the_frequencies(world, fail):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30150 + world * 20 + int(fail) * 7 + (os.getpid() % 40)
    procs = [ctx.Process(target=_rank_sharded, args=(r, world, port, q, fail)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, *rest = q.get(timeout=120)
        out[r] = rest
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = S.frequency_shards(10, world)
    e = (np.arange(10) + 2.0 + 0.5j).tolist()
    for r in range(world):
        res, shape, seen, bound = out[r]
        assert bound == [r]
        assert seen == [[2.0 + i for i in shards[r]]]   # each rank solved its own block only
        if fail:
            assert res == "rank 1: RuntimeError: injected"
        else:
            assert res == e and shape == (10, 6, 3, 3)


def test_concurrent_share_gives_the_serial_results():
    """Threads within a rank: same results in the same order, a failing
    system raises SystemSolveError naming it, others still solved."""
    serial = S.solve_systems(_systems(), solve_fn=_fake_solve)
    conc = S.solve_systems(_systems(), solve_fn=_fake_solve, concurrency=3)
    assert [int(r["n"][0]) for r in conc] == [int(r["n"][0]) for r in serial]
    calls = []

    def solve(system):
        calls.append(system.num_particles)
        if system.num_particles == 11:
            raise ValueError("boom")
        return _fake_solve(system)

    with pytest.raises(S.SystemSolveError, match=r"system 3 \(rank 0: ValueError: boom\)"):
        S.solve_systems(_systems(), solve_fn=solve, concurrency=2)
    assert sorted(calls) == sorted(s.num_particles for s in _systems())
