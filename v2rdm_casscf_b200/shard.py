"""Sharding of independent active-space instances over ranks (one rank per GPU).

The batched solve has no exchange between instances, so a multi-GPU run deals
the instances to ranks and each rank solves its share on its own GPU; the job
time is the slowest rank's.  Instances are dealt by a greedy longest-first
bin-pack on a per-outer-iteration cost model, so that ranks finish together:

    cost = MAP_S * (dimx + nconstraints) + PROJ_S * sum_b n_b^3

MAP_S covers the maps and vector work of about 35 CG iterations per outer
iteration (they stream the primal and dual vectors), PROJ_S the projection (a
few FP64 GEMM-like passes over every PSD block).  Both were measured on B200 for
19 instances of n = 20 in lock step: 52 ms of CG and 53 ms of projection per
outer iteration, i.e. 0.9 ns per vector element and 3.2 ps per n_b^3.
"""

MAP_S = 0.9e-9
PROJ_S = 3.2e-12


def instance_cost(dimx, nconstraints, block_dims):
    """Modelled seconds per outer iteration of one instance."""
    return MAP_S * (dimx + nconstraints) + PROJ_S * sum(float(d) ** 3 for d in block_dims)


def partition(costs, world):
    """Instance indices per rank: longest first, each to the least-loaded rank.

    Deterministic (ties go to the lower instance index and the lower rank), so
    every rank computes the same assignment without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    for lst in out:
        lst.sort()
    return out


def workload_costs(spaces, options=None):
    """Cost of each hamiltonian.ActiveSpace, from its layout (one layout per distinct shape)."""
    from . import V2RDMSolver

    cache = {}
    out = []
    for a in spaces:
        key = (a.n, a.na, a.nb, a.multiplicity)
        if key not in cache:
            s = V2RDMSolver([a.n], a.na, a.nb, a.multiplicity, options=options)
            cache[key] = instance_cost(s.dimx, s.nconstraints, s.dimensions)
        out.append(cache[key])
    return out


def gather_results(mine, results, world, dist=None):
    """Per-instance results of every rank, on every rank, sorted by instance:
    [(instance, e_total, status, oiter), ...].  ``results`` are this rank's
    result dicts in the order of ``mine``; with world > 1 the lists travel by
    ``dist.all_gather_object`` (NCCL on GPUs, gloo in the CPU tests)."""
    local = [(int(i), float(r["e_total"]), int(r["status"]), int(r["oiter"])) for i, r in zip(mine, results)]
    if world <= 1 or dist is None:
        return sorted(local)
    got = [None] * world
    dist.all_gather_object(got, local)
    return sorted(x for part in got for x in part)
