"""Specimens sharded across GPUs, one process per GPU.

The hot path has no exchange between specimens: a set of specimens (a 64-disc batch, or
the (NParam + 1) x 2 finite-difference runs of one step of the reference's material
fitter, mp_determineconjgradient.cu:87-124) splits into whole specimens per rank. Each
rank advances its share in one batched engine (rf_engine_create_batch) with no per-step
collective; at the end one reduction assembles every specimen's scalars (steps, peak
stress and strain, final stress and strain, fracture flag, broken bonds) on every rank.
"""
import numpy as np

RESULT_FIELDS = ("steps", "FractureStress", "FractureStrain", "Stress", "Strain", "Fracture", "broken_bonds")


def assign(costs, world):
    """Whole specimens per rank, balanced by cost (particles x steps): longest first, each
    to the least-loaded rank (the lowest rank on a tie). Deterministic. Returns one list
    of specimen indices per rank, each in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    costs = [float(c) for c in costs]
    order = sorted(range(len(costs)), key=lambda q: (-costs[q], q))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for q in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(q)
        load[r] += costs[q]
    return [sorted(p) for p in parts]


def engine_runner(steps):
    """The default runner: the rank's specimens in one batched engine on its GPU, `steps`
    explicit steps (each specimen stops earlier at its own fracture or strain limit)."""
    def run(tasks, params, Rs, radii):
        from . import BatchEngine
        be = BatchEngine(tasks, params, Rs, radii)
        try:
            be.step(steps)
            rows = []
            for s in range(len(tasks)):
                _, r = be.sync_spec(s)
                rows.append([float(getattr(r, f)) for f in RESULT_FIELDS])
            return rows
        finally:
            be.close()
    return run


def gather_results(rows, index, n_total, dist=None, device="cpu"):
    """Every specimen's result row on every rank: this rank's rows (for specimens `index`)
    are placed in an [n_total, fields] table of zeros and the tables are summed over the
    ranks in one all-reduce (each specimen belongs to exactly one rank, so the sum is the
    table). Returns a float64 numpy array."""
    import torch
    t = torch.zeros((n_total, len(RESULT_FIELDS)), dtype=torch.float64, device=device)
    if len(index):
        t[torch.as_tensor(index, dtype=torch.long, device=device)] = torch.as_tensor(
            np.asarray(rows, np.float64).reshape(len(index), len(RESULT_FIELDS)), device=device)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def run_sharded(tasks, params, Rs, radii, steps, dist=None, runner=None):
    """Run the specimens sharded over the process group `dist` (None: this process alone)
    and return the [n, fields] result table (RESULT_FIELDS) on every rank. runner(tasks,
    params, Rs, radii) -> rows runs one rank's share (default: engine_runner(steps))."""
    rank, world = 0, 1
    if dist is not None and dist.is_initialized():
        rank, world = dist.get_rank(), dist.get_world_size()
    n = len(tasks)
    costs = [int(t.N) * int(steps) for t in tasks]
    mine = assign(costs, world)[rank]
    run = runner or engine_runner(steps)
    rows = run([tasks[q] for q in mine], [params[q] for q in mine], [Rs[q] for q in mine],
               [radii[q] for q in mine]) if mine else []
    device = "cpu"
    if dist is not None and dist.is_initialized() and dist.get_backend() == "nccl":
        import torch
        device = "cuda:%d" % torch.cuda.current_device()
    return gather_results(rows, mine, n, dist, device)
