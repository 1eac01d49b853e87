#!/usr/bin/env python3
"""Benchmark: time to a converged v2RDM boundary-point SDP solve on B200.

Metric: time to 1e-6 Eh (E_CONVERGENCE 1e-7, R_CONVERGENCE 1e-6) of the
solver's own stopping test, for three solvers on the same input:

  value           the product's solve (FP64 maps / CG, mixed-precision
                  adaptive projection on the tensor cores, least-norm feasible
                  warm start, Anderson acceleration of the outer iteration with
                  the extrapolated CG start), device seconds
                  with the inputs resident in HBM (CUDA events around the
                  iteration phase inside the C ABI call)
  plain_fp64_gpu  the reference's algorithm, options and random start
                  (srand(0)) run by the same GPU kernels, one solve
  cpu_baseline    the reference's own CPU code (oracle/_ref: the reference's
                  hot-path sources with OpenMP and OpenBLAS on every host core),
                  time per CG iteration and per outer iteration sampled on this
                  input and multiplied by the reference's own iteration counts
                  for it (a full CPU solve takes most of an hour)

Workload (default "h10", the metric's (10e,10o) case): linear H10, 0.9 A,
STO-3G RHF orbitals with Cholesky-decomposed integrals, all 10 orbitals active,
C1, DQG, CONSTRAIN_SPIN.  The integrals are those of
tests/golden/solve_h10_chain.npz, the input the reference solved for the
golden fixture, so the converged energies are compared with the reference's
(|E - E_ref| <= 1e-6 Eh, in the line as energy_check).

  step      one complete solve through the public C ABI (v2g_solve_batch),
            from host buffers: the inputs are copied to the device, the solve
            runs to the stopping test, x, y, z are copied back
  e2e       that whole call, copies included (seconds per step)
  L2        a 256 MiB buffer is written between steps (inputs of this size
            stay inside the 126 MB L2 otherwise)
  roofline  the CG's FP64 gather map (A / A^T): algorithmic bytes 8 (rows +
            columns) per launch over its CUDA-event duration (launches of the
            workload's instance replayed from a CUDA graph), against the
            measured HBM copy bandwidth; the same kernel on the batched
            workload's largest group (n = 20, 19 instances) is reported beside
            it (roofline_batch), and the tensor-core product of the
            mixed-precision projection on that group's G2 blocks
            (roofline_tensor, against half the measured BF16 peak)

Other workloads: batch256 (256 seeded synthetic active spaces, n ~ U{8..20},
singlets, DQG; instances bin-packed over ranks) with --warmup-outer capping the
warm-up solves; h20scan, h20t2 and h50 (--max-outer caps them).

Multi-GPU (torchrun): h10 is one instance and does not shard, so every rank
solves its own replica ("replicas only", weak scaling) and the time is the
maximum over ranks; batch256 deals instances to ranks with no exchange.
`--impl reference` times the reference CPU path instead (rank 0 only).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from v2rdm_casscf_b200.hamiltonian import ActiveSpace, batch_sizes, synthetic  # noqa: E402

METRIC = "time-to-1e-6Eh v2RDM solve: mixed+warm-start vs plain FP64 GPU vs ref CPU"
OPTIONS = dict(R_CONVERGENCE=1e-6, E_CONVERGENCE=1e-7)
GOLDEN_H10 = os.path.join(ROOT, "tests", "golden", "solve_h10_chain.npz")
ITER_FILE = os.path.join(ROOT, "profiles", "batch256_outer_iterations.json")
L2_FLUSH_BYTES = 256 << 20


def golden_h10():
    g = np.load(GOLDEN_H10)
    n = int(g["n"])
    return ActiveSpace(g["h"], g["L"], n // 2, n // 2, float(g["enuc"]), name="H10 0.9 A (golden input)"), g


def workload(name, count):
    if name == "h10":  # linear H10, 0.9 A, STO-3G RHF orbitals, all active (the golden input)
        return [golden_h10()[0]]
    if name == "batch256":
        ns = batch_sizes(count)
        return [synthetic(int(n), s) for s, n in enumerate(ns)]
    if name.startswith("uniform"):  # uniformN: count instances of n = N (experiments)
        n = int(name[len("uniform"):])
        return [synthetic(n, s) for s in range(count)]
    if name == "h20scan":  # symmetric H20 dissociation scan, spacings 0.6..3.0 A
        from v2rdm_casscf_b200.hchain import hydrogen_scan

        return hydrogen_scan(20, 0.6, 3.0, count if count != 256 else 64)
    if name == "h20t2":  # linear H20, 1.0 A, (20e,20o), DQGT2 (T2 blocks of 11,800 and 3,800)
        from v2rdm_casscf_b200.hchain import hydrogen_chain

        return [hydrogen_chain(20, 1.0)]
    if name == "h50":  # linear H50, 1.2 A, (50e,50o), DQG (G2aa blocks of 5,000)
        from v2rdm_casscf_b200.hchain import hydrogen_chain

        return [hydrogen_chain(50, 1.2)]
    raise SystemExit(f"unknown workload {name}")


def workload_positivity(name):
    """POSITIVITY of a workload (DQG unless it names T2)."""
    return "DQGT2" if name == "h20t2" else "DQG"


def workload_text(name, count):
    opts = "C1, DQG, CONSTRAIN_SPIN, E_CONVERGENCE 1e-7, R_CONVERGENCE 1e-6"
    if name == "h10":
        return "h10: linear H10, 0.9 A, STO-3G RHF orbitals (CD integrals), (10e,10o) all active, " + opts
    if name == "batch256":
        return f"batch256: {count} synthetic active spaces n~U{{8..20}}, singlet N=n (n-1 for odd n), " + opts
    if name == "h20scan":
        return f"h20scan: {count} linear H20 geometries, spacing 0.6..3.0 A, STO-3G RHF orbitals, (20e,20o), " + opts
    if name == "h20t2":
        return ("h20t2: linear H20, 1.0 A, STO-3G RHF orbitals, (20e,20o) all active, "
                + opts.replace("DQG", "DQGT2"))
    if name == "h50":
        return "h50: linear H50, 1.2 A, STO-3G RHF orbitals, (50e,50o) all active, " + opts
    return f"{name}: {count} synthetic active spaces, " + opts


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """Samples SM clocks and throttle reasons while the timed region runs."""

    def __init__(self, gpu_index, path):
        self.path = path
        self.proc = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [v.strip() for v in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm = float(p[1])
                mx = float(p[2])
            except ValueError:
                continue
            sms.append(sm)
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sms:
            return None
        loaded = [s for s in sms if mx and s > 0.5 * mx] or sms
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sms)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def product_kw(args):
    """Solver options of the product's mode (or of the plain reference algorithm with --plain)."""
    if args.plain:
        return dict(projection="exact", cg_tolerance_factor=0.01, start="state", cg_extrapolate=False,
                    anderson_memory=0), dict(MU_UPDATE_FREQUENCY=500, TAU_PARAMETER=1.0)
    return (dict(projection=args.projection, cg_tolerance_factor=args.cg_factor, start=args.start,
                 cg_extrapolate=args.cg_extrapolate, anderson_memory=args.anderson,
                 mixed_precision=args.mixed and args.projection == "adaptive"),
            dict(MU_UPDATE_FREQUENCY=args.mu_freq, TAU_PARAMETER=args.tau))


PLAIN_KW = (dict(projection="exact", cg_tolerance_factor=0.01, start="state", cg_extrapolate=False, anderson_memory=0,
                 mixed_precision=False),
            dict(MU_UPDATE_FREQUENCY=500, TAU_PARAMETER=1.0))


def mode_text(kw, opt):
    if kw == PLAIN_KW[0] and opt == PLAIN_KW[1]:
        return "plain FP64 (the reference's algorithm, options and random start)"
    return ("FP64 maps / CG / errors, "
            + ("mixed-precision projection (3xTF32 tcgen05 products while the projection tolerance is >= 1e-5, "
               "FP64 after), " if kw.get("mixed_precision") else "FP64 projection, ")
            + ("adaptive projection accuracy" if kw["projection"] == "adaptive" else "converged projections")
            + (", least-norm feasible warm start" if kw["start"] == "feasible" else ", the reference's random start")
            + (", extrapolated CG start" if kw["cg_extrapolate"] else "")
            + (f", Anderson acceleration (memory {kw['anderson_memory']})" if kw["anderson_memory"] else "")
            + (f", MU_UPDATE_FREQUENCY {opt['MU_UPDATE_FREQUENCY']}" if opt["MU_UPDATE_FREQUENCY"] != 500 else "")
            + (f", TAU_PARAMETER {opt['TAU_PARAMETER']}" if opt["TAU_PARAMETER"] != 1.0 else ""))


def run_gpu(args):
    import torch

    import v2rdm_casscf_b200 as V

    rank, world, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(minutes=20))
    dev = local
    all_spaces = workload(args.workload, args.count)
    replicas = len(all_spaces) == 1
    if replicas or world == 1:
        mine = list(range(len(all_spaces)))
    else:
        from v2rdm_casscf_b200.shard import partition, workload_costs

        mine = partition(workload_costs(all_spaces), world)[rank]
    kw, opt = product_kw(args)

    def make(kw, opt, maxiter, profile=False):
        o = dict(OPTIONS, POSITIVITY=workload_positivity(args.workload), **opt)
        if maxiter:
            o["MAXITER"] = maxiter
        return [V.V2RDMSolver.from_active_space(all_spaces[i], options=o, device=dev, profile=profile, **kw)
                for i in mine]

    solvers = make(kw, opt, args.max_outer)
    if args.gemm_only:
        if rank == 0:
            print(json.dumps({"gemm_only": True, "detail": roofline_tensor(V, torch, dev)}))
        if world > 1:
            dist.destroy_process_group()
        return
    if args.roofline_only:
        achieved, detail = roofline_alone(V, solvers, all_spaces, mine, dev, torch)
        if rank == 0:
            print(json.dumps({"roofline_only": True, "achieved_GBps": achieved, "detail": detail}))
        if world > 1:
            dist.destroy_process_group()
        return
    warm = make(kw, opt, args.warmup_outer) if args.warmup_outer else solvers
    # every step starts from the same host state (the reference's random start;
    # the feasible start replaces it inside the solve)
    starts = {}
    for s in solvers + warm:
        key = (s.dimx, s.nconstraints)
        if key not in starts:
            s.guess()
            starts[key] = s.get_state()

    def reset(group):
        for s in group:
            x, y, z, mu = starts[(s.dimx, s.nconstraints)]
            s.set_state(x, y, z, mu)

    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{dev}")

    def step(group):
        reset(group)
        flush.fill_(1.0)  # evicts the previous step's data from L2 (outside the C ABI call)
        torch.cuda.synchronize(dev)
        res = V.solve_batch(group)
        return res, V.last_batch_stats()

    for _ in range(args.warmup):
        step(warm)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk_dir = os.environ.get("V2G_CLOCKS_DIR", tempfile.gettempdir())
    clk = Clocks(dev, os.path.join(clk_dir, f"clocks_rank{rank}.csv")) if args.clocks else None
    t0 = time.time()
    stats, results = [], None
    for _ in range(args.steps):
        results, st = step(solvers)
        stats.append(st)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    wall = time.time() - t0
    clocks = clk.stop() if clk else None
    dev_s = [s["device_seconds"] for s in stats]
    e2e_s = [s["e2e_seconds"] for s in stats]
    value, e2e = float(np.mean(dev_s)), float(np.mean(e2e_s))
    launches = sum(s["kernel_launches"] for s in stats)
    h2d = float(np.mean([s["h2d_bytes"] for s in stats]))
    d2h = float(np.mean([s["d2h_bytes"] for s in stats]))
    n_conv = sum(int(r["status"] == 0) for r in results)
    if world > 1:
        t = torch.tensor([value, e2e], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        value, e2e = float(t[0]), float(t[1])
        t = torch.tensor([float(launches), h2d, d2h, float(n_conv)], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        launches, h2d, d2h, n_conv = int(t[0]), float(t[1]), float(t[2]), int(t[3])
    # per-instance results of every rank reach rank 0 (energies, statuses, iterations)
    from v2rdm_casscf_b200.shard import gather_results

    allres = gather_results(mine, results, world, dist if world > 1 else None)
    pk, pk_kind = peaks()
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": value * 1e3,
        "higher_is_better": False,
        "scaling": "weak" if replicas else "strong",
        "vs_baseline": None,
        "dtype": "f64",
        "data": ("generated: STO-3G hydrogen-chain integrals and RHF computed in the project (the golden input "
                 "for h10); no dataset involved" if args.workload.startswith("h") else
                 "synthetic: seeded Philox active spaces; no dataset involved"),
        "config": {
            "workload": workload_text(args.workload, len(all_spaces)),
            "instances": len(all_spaces),
            "mode": mode_text(kw, opt),
            "precision": "FP64 maps, CG and projection",
            "l2": f"flushed between steps ({L2_FLUSH_BYTES >> 20} MiB write)",
            "parallelism": ("replicas only: every rank solves the same instance" if replicas else
                            f"instances bin-packed over {world} rank(s) by modelled cost, no exchange"),
            "warmup_steps": (f"{args.warmup} solves capped at {args.warmup_outer} outer iterations"
                             if args.warmup_outer else f"{args.warmup} full solves"),
            "max_outer": args.max_outer or None,
        },
        "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": roofline_workload(solvers, pk, pk_kind),
        "converged": n_conv,
        "projection_work": {"refine_sweeps": int(sum(s["refine_sweeps"] for s in stats)),
                            "jacobi_sweeps": int(sum(s["jacobi_sweeps"] for s in stats)),
                            "jacobi_blocks": int(sum(s["jacobi_blocks"] for s in stats)),
                            "jacobi_unconverged": int(sum(s["jacobi_unconverged"] for s in stats)),
                            "steps": len(stats)},
        "phase_seconds": ({"cg": float(results[0]["t_cg"]), "projection": float(results[0]["t_xz"]),
                           "rest": value - float(results[0]["t_cg"]) - float(results[0]["t_xz"]),
                           "note": "last step, CUDA events on the solve's stream: the CG, the projection "
                                   "(A^T y, Update_xz), and the error norms, Anderson step and host "
                                   "synchronisation between them"}
                          if len(results) == 1 else None),
        "wall_s": wall,
    }
    if clocks:
        out["clocks"] = clocks
    if rank == 0:
        its = [int(r["oiter"]) for r in results]
        out["outer_iterations"] = {"max": max(its), "median": float(np.median(its)), "total": int(sum(its))}
        out["cg_iterations_total"] = int(sum(int(r["iiter"]) for r in results))
        out["unconverged"] = [{"instance": int(i), "status": int(s), "oiter": int(o)}
                              for i, e, s, o in allres if s != 0]
        if args.workload == "h10":
            out["e_total_Eh"] = float(results[0]["e_total"])
        # the timed part of the line, on stderr, in case a later leg fails
        print("timed part: " + json.dumps(out), file=sys.stderr, flush=True)
    # the other two solvers of the metric, after the timed steps
    if args.workload == "h10" and not args.plain and args.compare_plain:
        plain = make(*PLAIN_KW, 0, profile=False)
        reset(plain)
        pres = V.solve_batch(plain)
        pst = V.last_batch_stats()
        pval = pst["device_seconds"]
        if world > 1:
            t = torch.tensor([pval], dtype=torch.float64, device=f"cuda:{dev}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            pval = float(t[0])
        out["plain_fp64_gpu"] = {"value": pval, "unit": "s", "e2e": pst["e2e_seconds"],
                                 "oiter": int(pres[0]["oiter"]), "iiter": int(pres[0]["iiter"]),
                                 "status": int(pres[0]["status"]), "e_total_Eh": float(pres[0]["e_total"]),
                                 "mode": mode_text(*PLAIN_KW)}
        out["speedup_vs_plain_fp64_gpu"] = pval / value
    if args.workload == "h10":
        _, g = golden_h10()
        eref = float(g["e_primal"])
        chk = {"reference_Eh": eref, "reference": "the compiled reference's own solve of this input "
                                                  "(tests/golden/solve_h10_chain.npz)",
               "product_abs_err_Eh": abs(float(results[0]["e_total"]) - eref)}
        if "plain_fp64_gpu" in out:
            chk["plain_abs_err_Eh"] = abs(out["plain_fp64_gpu"]["e_total_Eh"] - eref)
        chk["within_1e-6"] = all(v <= 1e-6 for k, v in chk.items() if k.endswith("abs_err_Eh"))
        out["energy_check"] = chk
    # the same map kernel timed alone on the batched workload's largest group
    if args.roofline_batch:
        b20 = V.V2RDMSolver([20], 10, 10, device=dev)
        ta, tt = b20.time_maps(19, 20)
        nbytes = 8.0 * (b20.dimx + b20.nconstraints) * 19
        ach = 2 * nbytes / (ta + tt) / 1e9
        out["roofline_batch"] = {"kernel": "ell_kernel + long_kernel, A and A^T of n = 20 with 19 instances "
                                           "interleaved (the batched workload's largest group), graph replay",
                                 "bound": "hbm", "achieved": ach, "peak": pk, "peak_kind": pk_kind, "unit": "GB/s",
                                 "frac": ach / pk, "traffic": ROOFLINE_TRAFFIC.get((20, 19)),
                                 "bytes_per_launch": nbytes, "us_per_launch": {"A": ta * 1e6, "AT": tt * 1e6}}
    if args.roofline_batch:
        out["roofline_tensor"] = roofline_tensor(V, torch, dev)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        if args.cpu_baseline and world == 1:
            out["cpu_baseline"] = cpu_baseline(args, all_spaces)
        print(json.dumps(out), flush=True)


# DRAM bytes (read + write) per launch of the roofline kernels, from one ncu
# capture of the same launches (profiles/ell_kernel_*.md gives the command):
# key = (n, instances)
ROOFLINE_TRAFFIC = {
    # A 556.5 MB, A^T 763.3 MB (means of 23 launches each), ell_kernel<4, 1>
    (20, 19): 659.9e6,
    # H10: A 4.22 MB, A^T 4.15 MB read, nothing written back (ell_kernel<2, 0>);
    # ncu flushes the caches before each launch, so this is the tables and the
    # input read cold: inside the solve both stay in L2
    (10, 1): 4.18e6,
}


def bf16_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def roofline_tensor(V, torch, dev, dims=(800,) * 19, reps=20):
    """The projection's product on the tensor cores, timed alone: C_i = A_i B_i
    for the G2 blocks of the batched workload's largest group (19 blocks of 800,
    padded to 832), two TF32 split launches + the tcgen05 MMA launch per product,
    CUDA events over `reps` back-to-back products.  Three TF32 products per FP64
    product (hi.hi + hi.lo + lo.hi) run on the 128-row tiles (832 -> 896 rows);
    the TF32 peak is taken as half the measured dense BF16 figure (the B200's
    nominal TF32 : BF16 ratio)."""
    npad = [(n + 63) // 64 * 64 for n in dims]
    tot = sum(p * p for p in npad)
    g = torch.Generator(device=f"cuda:{dev}").manual_seed(0)
    a = torch.randn(tot, dtype=torch.float64, device=f"cuda:{dev}", generator=g)
    b = torch.randn(tot, dtype=torch.float64, device=f"cuda:{dev}", generator=g)
    c = torch.empty_like(a)
    t_tc = V.time_block_gemm(list(dims), a.data_ptr(), b.data_ptr(), c.data_ptr(), True, reps, dev)
    t_64 = V.time_block_gemm(list(dims), a.data_ptr(), b.data_ptr(), c.data_ptr(), False, reps, dev)
    fp64_flops = sum(2.0 * p ** 3 for p in npad)
    tf32_flops = sum(3 * 2.0 * (-(-p // 128) * 128) ** 2 * p for p in npad)
    pk, kind = bf16_peak()
    ach = tf32_flops / t_tc / 1e12
    return {"kernel": "tc_split_kernel x 2 + tc_gemm_kernel (3xTF32 tcgen05, TMEM accumulator), "
                      f"{len(dims)} blocks of {dims[0]}", "bound": "tensor", "achieved": ach,
            "peak": pk / 2, "peak_kind": f"half of the {kind} dense BF16 {pk} TFLOP/s", "unit": "TFLOP/s",
            "frac": ach / (pk / 2), "traffic": None, "us_per_product": t_tc * 1e6,
            "fp64_equivalent_tflops": fp64_flops / t_tc / 1e12,
            "fp64_kernel": {"us_per_product": t_64 * 1e6, "tflops": fp64_flops / t_64 / 1e12}}


def roofline_workload(solvers, pk, pk_kind):
    """The map kernels of the workload's largest instance layout: A and A^T on
    the instance's own vector size, `reps` launches replayed from a CUDA graph
    between CUDA events on their stream (the kernels' own duration; the host's
    launch rate, which bounds a single small instance inside the solve, is
    excluded), algorithmic bytes 8 (rows + columns) per launch."""
    s = max(solvers, key=lambda v: v.dimx)
    ta, tt = s.time_maps(1, 50)
    nbytes = 8.0 * (s.dimx + s.nconstraints)
    ach = 2 * nbytes / (ta + tt) / 1e9
    key = (int(s.active[0]), 1)
    return {"kernel": "ell_kernel + long_kernel (A and A^T of the CG), one instance of the workload, graph replay",
            "bound": "hbm", "achieved": ach, "peak": pk, "peak_kind": pk_kind, "unit": "GB/s", "frac": ach / pk,
            "traffic": ROOFLINE_TRAFFIC.get(key), "bytes_per_launch": nbytes,
            "us_per_launch": {"A": ta * 1e6, "AT": tt * 1e6},
            "note": "bytes per launch fit in L2 at this size: the kernel is bound by latency, not HBM"
                    if nbytes < 64e6 else ""}


def roofline_alone(V, solvers, spaces, mine, dev, torch, reps=20, force_B=None):
    """Algorithmic GB/s of A and A^T for the largest group (bytes 8*(rows+cols) per vector)."""
    if force_B:
        s, B, n = solvers[0], force_B, spaces[0].n
    else:
        by_n = {}
        for k, i in enumerate(mine):
            by_n.setdefault(spaces[i].n, []).append(solvers[k])
        n = max(by_n)
        grp = by_n[n]
        B, s = len(grp), grp[0]
    nx, nc = s.dimx, s.nconstraints
    g = torch.Generator(device=f"cuda:{dev}").manual_seed(0)
    x = torch.randn(nx * B, dtype=torch.float64, device=f"cuda:{dev}", generator=g)
    y = torch.randn(nc * B, dtype=torch.float64, device=f"cuda:{dev}", generator=g)
    ox = torch.empty_like(x)
    oy = torch.empty_like(y)
    stream = torch.cuda.current_stream(dev)
    out = {}
    total_b, total_t = 0.0, 0.0
    for name, tr, src, dst in (("A", False, x, oy), ("AT", True, y, ox)):
        for _ in range(3):
            s.map_batched_device(B, src.data_ptr(), dst.data_ptr(), stream.cuda_stream, transpose=tr)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(reps):
            s.map_batched_device(B, src.data_ptr(), dst.data_ptr(), stream.cuda_stream, transpose=tr)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        nbytes = 8.0 * (nx + nc) * B
        out[name] = {"us_per_launch": t * 1e6, "GBps": nbytes / t / 1e9}
        total_b += nbytes
        total_t += t
    out["group"] = f"n={n}, {B} instances interleaved"
    out["bytes_per_launch"] = 8.0 * (nx + nc) * B
    return total_b / total_t / 1e9, out


# ---- the reference's CPU path (oracle/_ref) ---------------------------------


def ref_sample(space, threads, positivity="DQG", outer=10):
    """Seconds per CG iteration and per outer iteration outside the CG of the
    reference on this input: one outer iteration to warm up, then `outer` more
    from that state, with the reference's own phase timers (omp_get_wtime
    around the CG, v2rdm_solver.cc:1781-1824)."""
    from oracle import ref as R

    R.set_threads(threads)
    r = R.RefSolver([space.n], [space.nb], soccpi=[space.na - space.nb], multiplicity=space.multiplicity,
                    positivity=positivity, r_convergence=OPTIONS["R_CONVERGENCE"],
                    e_convergence=OPTIONS["E_CONVERGENCE"])
    r.set_integrals(space.oei_packed, space.qmo, space.nq, space.enuc)
    r.guess()
    r.build_constraints()
    r.solve(max_outer=1, trace_cap=0)
    out = r.solve(max_outer=outer, trace_cap=0)
    return {"t_cg_iter": out["t_cg"] / max(out["iiter"], 1),
            "t_outer": (out["t_total"] - out["t_cg"]) / max(out["oiter"], 1),
            "t_per_outer_sampled": out["t_total"] / max(out["oiter"], 1),
            "sampled_outer": out["oiter"], "sampled_cg": out["iiter"]}


def reference_counts(name):
    """The reference's own outer / CG iteration counts to convergence for a workload."""
    if name == "h10":
        _, g = golden_h10()
        return int(g["oiter"]), int(g["iiter"]), float(g["t_total"]), (
            "the compiled reference's own solve of this input from its random start "
            "(tests/golden/solve_h10_chain.npz); the model was checked against a timed full solve of it: "
            "815 s on 4 idle cores of the build container against 763 s predicted (profiles/reference_h10_cpu.md)")
    return None


def cpu_baseline(args, spaces):
    """The reference's CPU time to solution for the workload (extrapolated from a timed sample)."""
    from oracle import ref as R

    if not R.available():
        return {"unavailable": "oracle/_ref not built"}
    threads = os.cpu_count() or 1
    t0 = time.time()
    if args.workload == "h10":
        smp = ref_sample(spaces[0], threads)
        oit, cgit, t_meas, src = reference_counts("h10")
        value = oit * smp["t_outer"] + cgit * smp["t_cg_iter"]
        return {"value": value, "unit": "s", "cores": threads, "kind": "reference",
                "sample": (f"reference oracle/_ref (OpenMP + OpenBLAS, {threads} threads) on this input: "
                           f"{smp['sampled_outer']} outer / {smp['sampled_cg']} CG iterations after one warm-up "
                           f"iteration give {smp['t_cg_iter'] * 1e3:.3f} ms per CG iteration and "
                           f"{smp['t_outer'] * 1e3:.2f} ms per outer iteration outside the CG; times the "
                           f"reference's own {oit} outer / {cgit} CG iterations to convergence ({src}); "
                           f"extrapolated, sampling took {time.time() - t0:.1f} s"),
                "extrapolated": True}
    # batched workloads: seconds per outer iteration sampled per size, power law
    # in n for the others, times the recorded outer-iteration counts
    by_n = {}
    for a in spaces:
        by_n.setdefault(a.n, a)
    sample = [n for n in args.cpu_sample if n in by_n] or sorted(by_n)[:4]
    per_it = {n: ref_sample(by_n[n], threads, workload_positivity(args.workload), outer=1)["t_per_outer_sampled"]
              for n in sample}
    xs = np.log(np.array(sample, dtype=float))
    ys = np.log(np.array([per_it[n] for n in sample]))
    p, lna = np.polyfit(xs, ys, 1) if len(sample) > 1 else (0.0, float(ys[0]))
    if args.workload == "batch256" and args.count == 256 and os.path.exists(ITER_FILE):
        oiters = json.load(open(ITER_FILE))["outer_iterations"]
        src = "outer-iteration counts of the same instances solved on the GPU from the reference's start (profiles/)"
    else:
        oiters = [2500] * len(spaces)
        src = "2500 outer iterations per instance (no recorded counts for this workload)"
    total = sum(per_it.get(a.n, float(np.exp(lna) * a.n ** p)) * k for a, k in zip(spaces, oiters))
    return {"value": total, "unit": "s", "cores": threads, "kind": "reference", "extrapolated": True,
            "sample": (f"reference oracle/_ref ({threads} threads) timed per outer iteration on one instance of n in "
                       f"{sample} ({', '.join(f'{n}: {per_it[n]:.3g} s' for n in sample)}), power law n^{p:.2f} "
                       f"for other sizes, times {src}; sampling took {time.time() - t0:.1f} s")}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import ref as R

    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built on this box"}))
        return
    spaces = workload(args.workload, args.count)
    vals, base = [], None
    t0 = time.time()
    for _ in range(args.warmup + args.steps):
        base = cpu_baseline(args, spaces)
        vals.append(base["value"])
    value = float(np.mean(vals[args.warmup:]))
    base["value"] = value
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
           "scaling": "weak" if len(spaces) == 1 else "strong", "vs_baseline": None, "dtype": "f64",
           "data": "generated (the golden H10 input)" if args.workload == "h10" else "synthetic",
           "config": {"workload": workload_text(args.workload, len(spaces)), "instances": len(spaces),
                      "mode": "the reference's own CPU code, loop and random start (oracle/_ref)",
                      "note": ("each step samples the reference's time per CG iteration and per outer iteration "
                               "on this input and multiplies them by the reference's own iteration counts to "
                               "convergence (a full CPU solve takes most of an hour); the value is that "
                               "extrapolated time to solution, the mean over the timed steps"),
                      "wall_s": time.time() - t0},
           "cpu_baseline": base,
           "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--workload", default="h10")
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--max-outer", type=int, default=0, help="cap outer iterations (experiments only)")
    ap.add_argument("--warmup-outer", type=int, default=None,
                    help="cap the warm-up solves at this many outer iterations (default: full solves for h10, "
                         "3 otherwise)")
    ap.add_argument("--projection", default="adaptive", choices=["exact", "adaptive"])
    ap.add_argument("--cg-factor", type=float, default=0.01, help="CG tolerance factor (0.01 = the reference's rule)")
    ap.add_argument("--mu-update-frequency", dest="mu_freq", type=int, default=250,
                    help="MU_UPDATE_FREQUENCY (the reference's default is 500)")
    ap.add_argument("--start", default="feasible", choices=["feasible", "state"],
                    help="feasible: least-norm feasible warm start; state: the reference's random start")
    ap.add_argument("--tau", type=float, default=1.0, help="TAU_PARAMETER (the plugin's default 1.0)")
    ap.add_argument("--anderson", type=int, default=10,
                    help="Anderson acceleration of the outer iteration with this memory (0 = off)")
    ap.add_argument("--no-mixed", dest="mixed", action="store_false",
                    help="FP64 projection products throughout (no tensor-core phase)")
    ap.add_argument("--no-cg-extrapolate", dest="cg_extrapolate", action="store_false",
                    help="start each CG from y_k (the reference's) instead of y_k + (y_k - y_k-1)")
    ap.add_argument("--plain", action="store_true",
                    help="time the reference's algorithm, options and random start instead of the product's mode")
    ap.add_argument("--no-compare-plain", dest="compare_plain", action="store_false",
                    help="skip the plain FP64 GPU solve that is reported beside the value")
    ap.add_argument("--no-roofline-batch", dest="roofline_batch", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-sample", type=lambda s: [int(v) for v in s.split(",")], default=[8, 12, 16, 20])
    ap.add_argument("--no-clocks", dest="clocks", action="store_false")
    ap.add_argument("--gemm-only", action="store_true",
                    help="run only the timed block products of the mixed-precision projection (for profilers)")
    ap.add_argument("--roofline-only", action="store_true",
                    help="run only the timed A / A^T launches of the roofline (for profilers)")
    args = ap.parse_args()
    if args.warmup_outer is None:
        args.warmup_outer = 0 if args.workload == "h10" else 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
