#!/usr/bin/env python3
"""Benchmark: time to a converged (E_CONVERGENCE 1e-7, R_CONVERGENCE 1e-6) v2RDM
boundary-point SDP solve of a batch of active spaces on B200.

Workload (default "batch256"): 256 seeded synthetic active spaces, n ~ U{8..20}
orbitals, singlets with N = n electrons (N = n - 1 for odd n), C1, DQG
with CONSTRAIN_SPIN, all solved in one batched call of the C ABI
(v2g_solve_batch).  By default every instance starts from the least-norm
feasible point of A x = b with zero duals (computed on the GPU inside the
timed solve); --start state / --plain use the reference's random start.  One step = one
full batched solve.  Inputs are far larger than L2 (the primal/dual vectors of
the batch take several GB), so no L2 flush is needed between steps.

  step      one complete batched solve, from the reference's start to every
            instance passing the stopping test (the metric is a time to
            solution).  Warm-up steps make the same batched call capped at
            --warmup-outer outer iterations: they run every kernel, table
            build and allocation of the step without repeating a
            many-minute solve.
  value     device seconds of the batched solve, inputs resident in HBM
            (CUDA events around the iteration phase, max over ranks)
  e2e       the same solve through the public C ABI from host buffers,
            host-to-device and device-to-host copies inside the timed region
  roofline  the dominant kernel, the FP64 gather map (A / A^T) of the CG:
            algorithmic bytes 8*(rows+cols) per instance per launch over its
            CUDA-event duration, against the measured HBM copy bandwidth
  cpu_baseline  the reference's own hot-path code (oracle/_ref, OpenMP + the
            OpenBLAS of scipy on all host cores) timed per outer iteration on a
            sample of sizes and extrapolated to the batch with the iteration
            counts of the same instances

Loop options: --accelerated runs the solver's Anderson acceleration (memory 10)
with the extrapolated CG start and MU_UPDATE_FREQUENCY 250 (each also on its
own: --anderson, --cg-extrapolate, --mu-update-frequency, --tau); the line's
config names the options used, and the default is the reference's loop from
the feasible start with the adaptive projection.

Multi-GPU (torchrun): instances are dealt to ranks by a longest-first bin-pack
on a per-iteration cost model (v2rdm_casscf_b200/shard.py), with no exchange
during the solve; value is the max over ranks.  `--impl reference` times the
reference CPU path instead (rank 0 only).
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

from v2rdm_casscf_b200.hamiltonian import batch_sizes, synthetic  # noqa: E402

METRIC = "time-to-1e-6Eh v2RDM solve: mixed+warm-start vs plain FP64 GPU vs ref CPU"
OPTIONS = dict(R_CONVERGENCE=1e-6, E_CONVERGENCE=1e-7)
ITER_FILE = os.path.join(ROOT, "profiles", "batch256_outer_iterations.json")
# DRAM bytes (read + write) per launch of the roofline launches, averaged over A and A^T,
# from one ncu capture of exactly those launches (cold caches, as ncu replays them):
#   ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum
#       --clock-control none -k regex:ell_kernel -c 46 --csv python bench.py --roofline-only
# A: 442.8 MB read + 203.6 MB written; A^T: 528.1 MB + 237.4 MB (B200, 20 launches each).
ROOFLINE_TRAFFIC = {
    "n=20, 19 instances interleaved": {
        "bytes_per_launch": 0.5 * ((442.8 + 203.6) + (528.1 + 237.4)) * 1e6,
        "source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the same launches "
                  "(python bench.py --roofline-only), mean of A and A^T",
    },
}


def workload(name, count):
    if name == "batch256":
        ns = batch_sizes(count)
        return [synthetic(int(n), s) for s, n in enumerate(ns)]
    if name.startswith("uniform"):  # uniformN: count instances of n = N (experiments)
        n = int(name[len("uniform"):])
        return [synthetic(n, s) for s in range(count)]
    if name == "h10":  # linear H10, 0.9 A, STO-3G RHF orbitals, all active
        from v2rdm_casscf_b200.hchain import hydrogen_chain

        return [hydrogen_chain(10, 0.9)]
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


def workload_text(args, count):
    opts = "C1, DQG, CONSTRAIN_SPIN, E_CONVERGENCE 1e-7, R_CONVERGENCE 1e-6"
    if args.workload == "batch256":
        return f"batch256: {count} synthetic active spaces n~U{{8..20}}, singlet N=n (n-1 for odd n), " + opts
    if args.workload == "h10":
        return "h10: linear H10, 0.9 A, STO-3G RHF orbitals, (10e,10o) all active, " + opts
    if args.workload == "h20scan":
        return f"h20scan: {count} linear H20 geometries, spacing 0.6..3.0 A, STO-3G RHF orbitals, (20e,20o), " + opts
    if args.workload == "h20t2":
        return ("h20t2: linear H20, 1.0 A, STO-3G RHF orbitals, (20e,20o) all active, "
                + opts.replace("DQG", "DQGT2"))
    if args.workload == "h50":
        return "h50: linear H50, 1.2 A, STO-3G RHF orbitals, (50e,50o) all active, " + opts
    return f"{args.workload}: {count} synthetic active spaces, " + opts


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


def run_gpu(args):
    import torch

    import v2rdm_casscf_b200 as V

    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(minutes=30))
    dev = local
    all_spaces = workload(args.workload, args.count)
    # instances dealt to ranks by a longest-first bin-pack on the modelled cost
    from v2rdm_casscf_b200.shard import partition, workload_costs

    mine = partition(workload_costs(all_spaces), world)[rank] if world > 1 else list(range(len(all_spaces)))
    def make(maxiter):
        opts = dict(OPTIONS, MU_UPDATE_FREQUENCY=args.mu_freq, TAU_PARAMETER=args.tau,
                    POSITIVITY=workload_positivity(args.workload))
        if maxiter:
            opts["MAXITER"] = maxiter
        return [V.V2RDMSolver.from_active_space(all_spaces[i], options=opts, device=dev, profile=True,
                                                projection=args.projection, cg_tolerance_factor=args.cg_factor,
                                                start=args.start, cg_extrapolate=args.cg_extrapolate,
                                                anderson_memory=args.anderson)
                for i in mine]

    solvers = make(args.max_outer)
    if args.roofline_only:
        # the roofline launches alone (A and A^T of the largest group), for profilers
        achieved, detail = roofline_pass(V, solvers, all_spaces, mine, dev, torch)
        if rank == 0:
            print(json.dumps({"roofline_only": True, "achieved_GBps": achieved, "detail": detail}))
        if world > 1:
            dist.destroy_process_group()
        return
    warm_solvers = make(args.warmup_outer) if args.warmup else []
    # the random start of the reference depends only on the layout: compute once per size
    starts = {}
    for s in solvers:
        key = (s.dimx, s.nconstraints)
        if key not in starts:
            s.guess()
            starts[key] = s.get_state()
    def reset(group):
        for s in group:
            x, y, z, mu = starts[(s.dimx, s.nconstraints)]
            s.set_state(x, y, z, mu)

    def step(group=None):
        group = solvers if group is None else group
        reset(group)
        res = V.solve_batch(group)
        st = V.last_batch_stats()
        return res, st

    for _ in range(args.warmup):
        step(warm_solvers)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    # the raw clock samples go to $V2G_CLOCKS_DIR (default: the temporary directory)
    clk_dir = os.environ.get("V2G_CLOCKS_DIR", tempfile.gettempdir())
    clk = Clocks(dev, os.path.join(clk_dir, f"clocks_rank{rank}.csv")) if args.clocks else None
    t0 = time.time()
    dev_s, e2e_s, stats, results = [], [], [], None
    for _ in range(args.steps):
        results, st = step()
        dev_s.append(st["device_seconds"])
        e2e_s.append(st["e2e_seconds"])
        stats.append(st)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    wall = time.time() - t0
    clocks = clk.stop() if clk else None
    value = float(np.mean(dev_s))
    e2e = float(np.mean(e2e_s))
    map_s = sum(s["map_seconds"] for s in stats)
    map_n = sum(s["map_launches"] for s in stats)
    map_b = sum(s["map_bytes"] for s in stats)
    launches = sum(s["kernel_launches"] for s in stats)
    h2d = float(np.mean([s["h2d_bytes"] for s in stats]))
    d2h = float(np.mean([s["d2h_bytes"] for s in stats]))
    if world > 1:
        t = torch.tensor([value, e2e], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        value, e2e = float(t[0]), float(t[1])
        t = torch.tensor([float(launches), h2d, d2h], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        launches, h2d, d2h = int(t[0]), float(t[1]), float(t[2])
    conv = [r["status"] == 0 for r in results]
    n_conv = int(sum(conv))
    n_stall = int(sum(r["cg_stalls"] for r in results))
    if world > 1:  # instances converged and CG stops on all ranks
        t = torch.tensor([float(n_conv), float(n_stall)], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        n_conv, n_stall = int(t[0]), int(t[1])
    if rank == 0:
        oiters = {}
        for i, r in zip(mine, results):
            oiters.setdefault(int(all_spaces[i].n), []).append(int(r["oiter"]))
    # Roofline of the dominant kernel, timed alone: inside the solve every
    # layout group runs on its own stream, so per-kernel events there also
    # cover other groups' kernels.  The largest group's maps are applied to
    # interleaved vectors of its own size on one stream, CUDA events around them.
    pk, pk_kind = peaks()
    achieved, map_detail = roofline_pass(V, solvers, all_spaces, mine, dev, torch)
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": value * 1e3,
        "higher_is_better": False,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f64",
        "data": ("generated (STO-3G hydrogen-chain integrals and RHF computed in the project; no dataset involved)"
                 if args.workload.startswith("h") else
                 "synthetic (seeded Philox active spaces; no public dataset involved)"),
        "config": {
            "workload": workload_text(args, len(all_spaces)),
            "instances": len(all_spaces),
            "precision": "FP64 (maps, CG, projection)",
            "projection": args.projection,
            "cg_tolerance_factor": args.cg_factor,
            "cg_start": "extrapolated y_k + (y_k - y_k-1)" if args.cg_extrapolate else "previous y (the reference's)",
            "mu_update_frequency": args.mu_freq,
            "tau_parameter": args.tau,
            "anderson_memory": args.anderson,
            "start": ("least-norm feasible point of A x = b, zero duals, mu 1 (computed on the GPU inside "
                      "the timed solve)") if args.start == "feasible" else "the reference's random start (srand(0))",
            "mode": "plain FP64 (reference algorithm, options and start)"
                    if (args.projection == "exact" and args.cg_factor == 0.01 and args.mu_freq == 500
                        and args.start == "state" and not args.cg_extrapolate and args.tau == 1.0
                        and args.anderson == 0)
                    else "FP64 maps/CG/projection, adaptive projection accuracy"
                         + (", feasible warm start" if args.start == "feasible" else "")
                         + (", extrapolated CG start" if args.cg_extrapolate else "")
                         + (f", mu update every {args.mu_freq}" if args.mu_freq != 500 else "")
                         + (f", TAU_PARAMETER {args.tau}" if args.tau != 1.0 else "")
                         + (f", Anderson acceleration (memory {args.anderson})" if args.anderson else ""),
            "warmup_steps": f"{args.warmup} batched calls capped at {args.warmup_outer} outer iterations",
            "l2": "inputs larger than L2 (no flush needed)",
            "parallelism": f"instances bin-packed over {world} rank(s) by modelled cost, no exchange",
            "max_outer": args.max_outer or None,
        },
        "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": {
            "kernel": "ell_kernel + long_kernel (A and A^T gathers of the CG), largest layout group, timed alone",
            "bound": "hbm",
            "detail": map_detail,
            "in_solve_event_timing_gbs": (map_b / map_s / 1e9) if map_s > 0 else None,
            "achieved": achieved,
            "peak": pk,
            "peak_kind": pk_kind,
            "unit": "GB/s",
            "frac": (achieved / pk) if achieved else None,
            "traffic": ROOFLINE_TRAFFIC.get(map_detail["group"], {}).get("bytes_per_launch"),
            "traffic_source": ROOFLINE_TRAFFIC.get(map_detail["group"], {}).get("source"),
            "launches_timed": map_n,
        },
        "converged": n_conv,
        "cg_stalls": n_stall,
        "unconverged": [{"instance": int(mine[k]), "n": int(all_spaces[mine[k]].n), "status": int(r["status"]),
                         "oiter": int(r["oiter"])} for k, r in enumerate(results) if r["status"] != 0],
        "wall_s": wall,
    }
    # energies against a recorded solve of the same instances from the reference's
    # start (the metric asks for |E - E_FP64| <= 1e-6 Eh per instance)
    if world == 1 and args.workload == "batch256" and args.count == 256 and os.path.exists(ITER_FILE):
        rec = json.load(open(ITER_FILE))
        if "energies" in rec:
            d = [abs(results[k]["e_total"] - rec["energies"][mine[k]]) for k in range(len(results))
                 if results[k]["status"] == 0 and rec["status"][mine[k]] == 0]
            out["energy_check"] = {"against": "recorded FP64 solve from the reference's random start",
                                   "instances": len(d), "max_abs_diff_Eh": max(d) if d else None,
                                   "within_1e-6": int(sum(x <= 1e-6 for x in d))}
    if clocks:
        out["clocks"] = clocks
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank == 0:
        out["outer_iterations"] = {str(k): v for k, v in sorted(oiters.items())}
        allit = [int(r["oiter"]) for r in results]
        if allit:
            # the slowest instance sets the time to solution; seconds per outer
            # iteration of the batch while it runs
            out["time_per_outer_iteration_s"] = value / max(allit)
            out["outer_iterations_summary"] = {"max": max(allit), "median": float(np.median(allit)),
                                               "total": int(sum(allit))}
        if args.cpu_baseline and world == 1:
            # the reference runs from its own random start: its iteration counts are
            # those of a solve from that start (recorded), else this run's
            oiters, src = reference_iterations(args, [results[k]["oiter"] for k in range(len(results))])
            out["cpu_baseline"] = cpu_baseline(all_spaces, oiters, args.cpu_sample,
                                               workload_positivity(args.workload))
            out["cpu_baseline"]["sample"] += "; iteration counts: " + src
        if args.save_iterations and world == 1 and not args.max_outer and args.start == "state":
            os.makedirs(os.path.dirname(ITER_FILE), exist_ok=True)
            json.dump({"workload": args.workload, "count": args.count,
                       "outer_iterations": [int(r["oiter"]) for r in results],
                       "energies": [float(r["e_total"]) for r in results],
                       "status": [int(r["status"]) for r in results],
                       "n": [int(a.n) for a in all_spaces]}, open(ITER_FILE, "w"))
        print(json.dumps(out))


def roofline_pass(V, solvers, spaces, mine, dev, torch, reps=20):
    """Algorithmic GB/s of A and A^T for the largest group (bytes 8*(rows+cols) per vector)."""
    by_n = {}
    for k, i in enumerate(mine):
        by_n.setdefault(spaces[i].n, []).append(solvers[k])
    n = max(by_n)
    grp = by_n[n]
    B = len(grp)
    s = grp[0]
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


def ref_time_per_iteration(space, iters, threads, positivity="DQG"):
    """Seconds per outer iteration of the reference on one instance (after one warm-up iteration)."""
    from oracle import ref as R

    R.set_threads(threads)
    r = R.RefSolver([space.n], [space.nb], soccpi=[space.na - space.nb], multiplicity=space.multiplicity,
                    positivity=positivity, r_convergence=OPTIONS["R_CONVERGENCE"],
                    e_convergence=OPTIONS["E_CONVERGENCE"])
    r.set_integrals(space.oei_packed, space.qmo, space.nq)
    r.guess()
    r.build_constraints()
    out = r.solve(max_outer=iters + 1, trace_cap=0)
    t1 = out["t_total"]
    r2 = R.RefSolver([space.n], [space.nb], soccpi=[space.na - space.nb], multiplicity=space.multiplicity,
                     positivity=positivity, r_convergence=OPTIONS["R_CONVERGENCE"],
                     e_convergence=OPTIONS["E_CONVERGENCE"])
    r2.set_integrals(space.oei_packed, space.qmo, space.nq)
    r2.guess()
    r2.build_constraints()
    t0 = r2.solve(max_outer=1, trace_cap=0)["t_total"]
    return max(t1 - t0, 1e-9) / iters


def reference_iterations(args, fallback):
    """Outer-iteration counts of the reference's own start for this workload."""
    if args.workload == "batch256" and args.count == 256 and os.path.exists(ITER_FILE):
        d = json.load(open(ITER_FILE))
        return d["outer_iterations"], ("outer-iteration counts of the same instances solved on the GPU from the "
                                       "reference's random start with its loop options (profiles/)")
    golden = os.path.join(ROOT, "tests", "golden", "solve_h10_chain.npz")
    if args.workload == "h10" and os.path.exists(golden):
        return [int(np.load(golden)["oiter"])], ("the outer-iteration count of the compiled reference's own solve of "
                                                 "this input from its random start (tests/golden/solve_h10_chain.npz)")
    plain = (args.start == "state" and args.anderson == 0 and not args.cg_extrapolate and args.tau == 1.0
             and args.mu_freq == 500)
    if plain:
        return fallback, "outer-iteration counts of this run (the reference's loop and start)"
    return fallback, ("outer-iteration counts of this run, whose start or loop options need fewer iterations than "
                      "the reference's own loop: the CPU time is an underestimate")


def cpu_baseline(spaces, oiters, sample_sizes, positivity="DQG"):
    """Reference CPU time for the batch, extrapolated from a timed sample."""
    from oracle import ref as R

    if not R.available():
        return {"unavailable": "oracle/_ref not built"}
    threads = os.cpu_count() or 1
    by_n = {}
    for a in spaces:
        by_n.setdefault(a.n, a)
    sample = [n for n in sample_sizes if n in by_n] or sorted(by_n)[:4]
    t0 = time.time()
    per_it = {}
    for n in sample:
        iters = 1 if n >= 16 else (2 if n >= 12 else 3)
        per_it[n] = ref_time_per_iteration(by_n[n], iters, threads, positivity)
    # power-law fit t(n) = a n^p over the sampled sizes for the others
    xs = np.log(np.array(sample, dtype=float))
    ys = np.log(np.array([per_it[n] for n in sample]))
    if len(sample) > 1:
        p, lna = np.polyfit(xs, ys, 1)
    else:  # one size only: every instance has it
        p, lna = 0.0, float(ys[0])
    total = 0.0
    for a, k in zip(spaces, oiters):
        t = per_it.get(a.n, float(np.exp(lna) * a.n ** p))
        total += t * k
    return {"value": total, "unit": "s", "cores": threads, "kind": "reference",
            "sample": f"reference oracle/_ref (OpenMP, {threads} threads) timed per outer iteration on one "
                      f"instance of n in {sample} ({', '.join(f'{n}: {per_it[n]:.3g} s' for n in sample)}), "
                      f"power law n^{p:.2f} for other sizes, times the outer-iteration counts of the same "
                      f"instances; extrapolated, sampling took {time.time() - t0:.1f} s"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import ref as R

    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built on this box"}))
        return
    spaces = workload(args.workload, args.count)
    oiters, src = reference_iterations(args, [2500] * len(spaces))
    if not (args.workload == "batch256" and args.count == 256 and os.path.exists(ITER_FILE)) and args.workload != "h10":
        src = "2500 outer iterations per instance (no recorded counts for this workload)"
    vals = []
    base = None
    for _ in range(args.warmup + args.steps):
        base = cpu_baseline(spaces, oiters, args.cpu_sample, workload_positivity(args.workload))
        vals.append(base["value"])
    value = float(np.mean(vals[args.warmup:]))
    base["value"] = value
    base["sample"] += "; iteration counts: " + src
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
           "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": workload_text(args, len(spaces)),
                      "instances": len(spaces), "mu_update_frequency": args.mu_freq,
                      "note": "reference CPU path (oracle/_ref) with the same options; time per outer iteration "
                              "sampled, times the outer-iteration counts the GPU solve needed with those options"},
           "cpu_baseline": base,
           "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--workload", default="batch256")
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--max-outer", type=int, default=0, help="cap outer iterations (experiments only)")
    ap.add_argument("--projection", default="adaptive", choices=["exact", "adaptive"])
    ap.add_argument("--cg-factor", type=float, default=0.01,
                    help="CG tolerance factor (0.01 = the reference's rule)")
    ap.add_argument("--mu-update-frequency", dest="mu_freq", type=int, default=500,
                    help="MU_UPDATE_FREQUENCY (the reference's default is 500)")
    ap.add_argument("--start", default="feasible", choices=["feasible", "state"],
                    help="feasible: least-norm feasible warm start; state: the reference's random start")
    ap.add_argument("--tau", type=float, default=1.0,
                    help="TAU_PARAMETER (the plugin's default 1.0; its documented range is [1.0, 1.6])")
    ap.add_argument("--anderson", type=int, default=0,
                    help="Anderson acceleration of the outer iteration with this memory (0 = off)")
    ap.add_argument("--cg-extrapolate", action="store_true",
                    help="start each CG from y_k + (y_k - y_k-1) instead of y_k (same stopping test)")
    ap.add_argument("--accelerated", action="store_true",
                    help="Anderson acceleration (memory 10), extrapolated CG start, MU_UPDATE_FREQUENCY 250")
    ap.add_argument("--plain", action="store_true",
                    help="reference algorithm, options and start: exact projection, CG factor 0.01, "
                         "mu update every 500, random start")
    ap.add_argument("--warmup-outer", type=int, default=3, help="outer iterations per warm-up step")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-sample", type=lambda s: [int(v) for v in s.split(",")], default=[8, 12, 16, 20])
    ap.add_argument("--no-clocks", dest="clocks", action="store_false")
    ap.add_argument("--save-iterations", action="store_true")
    ap.add_argument("--roofline-only", action="store_true",
                    help="run only the timed A / A^T launches of the roofline (for profiling)")
    args = ap.parse_args()
    if args.accelerated and args.plain:
        ap.error("--accelerated and --plain exclude each other")
    if args.accelerated:
        args.anderson, args.cg_extrapolate, args.mu_freq = 10, True, 250
    if args.plain:
        args.projection, args.cg_factor, args.mu_freq, args.start = "exact", 0.01, 500, "state"
        args.cg_extrapolate, args.tau, args.anderson = False, 1.0, 0
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
