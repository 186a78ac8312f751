"""Benchmark of the explicit MHD hot path: cell-updates/s on the 3D
Orszag-Tang workload (256^3 cells = 32768 blocks of 8^3, Linde HLL + Koren,
CFL 0.8, 2-stage), FP64 and FP32-bulk.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full time step (2 fused stage launches plus the device-side
time-step update) over all blocks.  ``value`` is device-resident throughput
(state in HBM before the timed region, CUDA events on the library's stream,
max over ranks); ``e2e`` runs the same steps through the C ABI from pinned
host State_VGB (upload + K steps + download inside the timed region).
``--impl reference`` times the CPU restatement of the reference's orig path
(oracle/) on the host cores.  N > 1: one process per GPU, each rank advances
its own 256^3 Orszag-Tang domain (independent replicas of the workload,
weak scaling; the single-GPU path has no inter-rank exchange).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s FP64 vs FP32 bulk; JFNK s/step learned vs BILU precond at 1e-3"
UNIT = "cell-updates/s"
BYTES_PER_CELL_STEP = {"fp64": 320, "fp32": 256}  # algorithmic HBM bytes per cell and step
WORKLOAD = "orszag_tang_3d_256cubed_linde_koren"


def dist_env():
    r = int(os.environ.get("RANK", "0"))
    w = int(os.environ.get("WORLD_SIZE", "1"))
    lr = int(os.environ.get("LOCAL_RANK", "0"))
    return r, w, lr


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per cell of one
# stage8_kernel launch, the mean of a stage-1 and a stage-2 launch, from ncu
# captures of the 160^3 Orszag-Tang case (20^3 blocks, 0.26 GB of state,
# larger than L2):
#   python bench.py --nroot 20 --precisions <p> --steps 2 --warmup 3 --no-e2e --no-cpu \
#       --no-amr --jfnk-precond= --heat-precond= --no-autotune
#   ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum \
#       --clock-control none -k regex:stage8 -s 2 -c 2 --csv <same command>
# FP64: 135.8 and 200.1 B; FP32-bulk: 111.8 and 159.0 B.  Traffic grows in
# proportion to the blocks, so the bench scales it by the cells of its grid.
DRAM_BYTES_PER_CELL_LAUNCH = {"fp64": 168.0, "fp32": 135.4}


def profile_traffic(prec):
    return DRAM_BYTES_PER_CELL_LAUNCH.get(prec)


class ClockSampler:
    def __init__(self, gpu):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def allreduce_max(x, world):
    """the maximum of x over the ranks (NCCL on the GPUs, or gloo)"""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def replica_rate(timed, units, world):
    """One timed region of replicas: a barrier, this rank's timed() (it
    returns milliseconds measured on its device), a barrier, the maximum over
    the ranks.  Returns (whole-job units per second = world x units / the
    slowest rank's time, that time in ms)."""
    barrier(world)
    ms = timed()
    barrier(world)
    ms = allreduce_max(ms, world)
    return world * units / (ms * 1e-3), ms


def run_ours(args):
    rank, world, lrank = dist_env()
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(lrank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from batsrus_b200 import configs
    from batsrus_b200.explicit import ExplicitSolver

    hbm_peak, peak_kind = peaks()
    if args.stage_ctas:
        from batsrus_b200 import capi
        capi.tune_set("stage_ctas_per_sm", args.stage_ctas)
    out = {}
    st = None
    for prec in args.precisions.split(","):
        g, s, st0, _ = configs.orszag_tang_3d(nRoot=args.nroot, precision=prec, flux=args.flux,
                                              with_state=st is None)
        st = st0 if st is None else st
        nCell = g.nCell
        x = ExplicitSolver(g, s, device=lrank)
        # ---- device-resident throughput ----------------------------------
        x.set_state(st)
        x.advance(max(args.warmup, 3))  # includes the first Dt = 0 step
        tuned = x.autotune() if args.autotune else None
        x.synchronize()
        x.timing(True)
        x.timing_reset()
        clk = ClockSampler(lrank)

        def timed():
            with clk:
                x.region_begin()
                x.advance(args.steps)
                return x.region_end()
        value, ms = replica_rate(timed, nCell * args.steps, world)
        kern_ms, n_launch, n_total = x.timing_get()
        x.timing(False)
        launch_bytes = BYTES_PER_CELL_STEP[prec] / 2 * nCell  # average over the 2 stages
        achieved = launch_bytes / (kern_ms * 1e-3) / 1e9
        t_per_cell = profile_traffic(prec)
        res = {"value": value, "ms_per_step": ms / args.steps, "kernel_ms": kern_ms,
               "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak,
                            "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                            "traffic": (t_per_cell * nCell if t_per_cell else None),
                            "peak_source": peak_kind},
               "clocks": clk.summary(), "gpu_launches": 4 * args.steps,
               "autotune": ({k: v["value"] for k, v in tuned.items()} if tuned else None)}
        # ---- end to end through the C ABI with pinned host buffers ----------
        if args.e2e:
            import torch
            host = torch.empty(g.state_shape_fortran(), dtype=torch.float64).pin_memory()
            host.numpy()[...] = st
            back = torch.empty(g.state_shape_fortran(), dtype=torch.float64).pin_memory()
            x2 = ExplicitSolver(g, s, device=lrank)
            x2.set_state(host.numpy())
            x2.advance(1)
            x2.synchronize()

            def timed_e2e():
                x2.region_begin()
                x2.set_state(host.numpy())
                x2.set_time(0.0, 1)  # first Dt = 0 step already taken: time the K full steps
                x2.advance(args.steps)
                x2.get_state(back.numpy())
                return x2.region_end()
            # one untimed pass: the download's staging buffer (all of
            # State_VGB, ghost cells included) and the K-step graph are
            # created here, not in the timed region
            timed_e2e()
            evalue, ems = replica_rate(timed_e2e, nCell * args.steps, world)
            # bx_download_state returns all of State_VGB, ghost cells included;
            # bx_upload_state moves the interior cells only (strided copies of
            # the interior x runs: nI x nJ x nK of nIg x nJg x nKg per block)
            sh = g.state_shape_fortran()  # (8, nIg, nJg, nKg, nBlock)
            d2h = host.numel() * 8
            h2d = d2h * (g.nI * g.nJ * g.nK) // (sh[1] * sh[2] * sh[3])
            res["e2e"] = {"value": evalue, "unit": UNIT,
                          "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                          "ms": ems}
            x2.close()
        else:
            x.close()
        out[prec] = res
    return out


def run_sharded(args):
    """One Orszag-Tang domain (nroot^3 blocks of 8^3) partitioned over the
    ranks by shard.GpuRank: halo copies exchanged over NCCL before every
    stage, the time step a MIN over the ranks (strong scaling).  Device time
    of the steps, max over ranks."""
    import datetime
    import torch
    import torch.distributed as dist
    from batsrus_b200 import configs, shard
    rank, world, lrank = dist_env()
    torch.cuda.set_device(lrank)
    if world > 1 and not dist.is_initialized():
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    g, s, st, _ = configs.orszag_tang_3d(nRoot=args.nroot, precision=args.precisions.split(",")[0], flux=args.flux)
    r = shard.GpuRank(g, s, max(world, 1), rank, device=lrank)
    r.set_state(st)
    del st
    r.advance(max(args.warmup, 3))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    ev0.record()
    r.advance(args.steps)
    ev1.record()
    torch.cuda.synchronize()
    ms = allreduce_max(ev0.elapsed_time(ev1), world)
    barrier(world)
    out = {"value": g.nCell * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps, "ranks": world,
           "owned_blocks": r.dom.nOwned, "halo_blocks": len(r.dom.glob) - r.dom.nOwned,
           "timing": "torch CUDA events on the current stream around whole steps (host-synchronised halo "
                     "exchanges included), max over ranks", "scaling": "strong"}
    r.close()
    return out


def run_jfnk(args, lrank):
    """Implicit JFNK steps on the perturbed Orszag-Tang workload, wall time
    per implicit step (CUDA events around whole steps, the host-side Krylov
    control included) and Krylov matrix-vector products per step, for each
    preconditioner."""
    from batsrus_b200 import configs
    from batsrus_b200.explicit import ExplicitSolver
    from batsrus_b200.implicit import ImplicitSolver
    g, s, _, st = configs.jfnk_ot(nRoot=args.jfnk_nroot)
    out = {"workload": "perturbed_orszag_tang_%dcubed_bdf2_cfl20_gmres30_1e-3" % (8 * args.jfnk_nroot),
           "bilu_factors": args.bilu_factors,
           "cells": g.nCell, "blocks": g.nBlock, "steps": args.jfnk_steps, "warmup": args.jfnk_warmup,
           "unit": "s/step", "higher_is_better": False}
    net = None
    for prec in args.jfnk_precond.split(","):
        p = configs.jfnk_ot(nRoot=args.jfnk_nroot, precond=prec, with_state=False,
                            precondPrecision=args.bilu_factors)[2]
        if prec.upper() == "LEARNED" and net is None:
            net, out["learned_training"] = train_learned(args, g, s, lrank)
        x = ExplicitSolver(g, s, device=lrank)
        x.set_state(st)
        im = ImplicitSolver(x, p)
        from batsrus_b200.capi import BxError
        try:
            for _ in range(1 + args.jfnk_warmup):  # the first step only sets the time step
                im.advance_part_impl()
            if args.autotune:
                x.autotune()
            x.synchronize()
            x.region_begin()
            stats = [im.advance_part_impl() for _ in range(args.jfnk_steps)]
            ms = x.region_end()
        except BxError as e:
            out[prec.lower()] = {"failed": str(e)}
            x.close()
            continue
        out[prec.lower()] = {
            "s_per_step": ms * 1e-3 / args.jfnk_steps,
            "s_per_step_per_mcell": ms * 1e-3 / args.jfnk_steps / (g.nCell / 1e6),
            "matvec_per_step": float(np.mean([q["nMatvec"] for q in stats])),
            "matvec": [q["nMatvec"] for q in stats],
            "krylov_error": [q["Error"] for q in stats],
            "ms_precond_setup": float(np.mean([q["msPrecondSetup"] for q in stats])),
            "converged": all(q["iError"] == 0 for q in stats)}
        x.close()
    if net is not None:
        net.close()
    return out


def train_learned(args, g, s, lrank, nPair=2000, blocksPerPair=32):
    """Training data and training of the learned preconditioner: (v, BILU(v))
    pairs, half of them the Krylov vectors of the BILU-preconditioned FGMRES
    of implicit steps, half seeded probe vectors (noise smoothed inside the
    blocks to several degrees) at the last step's state; the steps start from
    a differently seeded perturbation (seed 2025) than the timed steps,
    blocksPerPair random blocks of each of nPair pairs; then Adam."""
    from batsrus_b200 import configs
    from batsrus_b200.explicit import ExplicitSolver
    from batsrus_b200.implicit import ImplicitSolver
    from batsrus_b200.learned import LearnedPreconditioner
    net = LearnedPreconditioner(nSampleMax=nPair * blocksPerPair, seed=2024)
    # the training targets BILU(v) from FP32 factors (closer to the exact block ILU)
    _, _, p, st2 = configs.jfnk_ot(nRoot=args.jfnk_nroot, precond="BILU", seed=2025, precondPrecision="fp32")
    x = ExplicitSolver(g, s, device=lrank)
    x.set_state(st2)
    im = ImplicitSolver(x, p)
    t0 = time.perf_counter()
    # half of the pairs from the Krylov vectors of BILU-preconditioned
    # implicit steps, half from seeded probe vectors at the last step's state
    net.collect(blocksPerPair)
    nStep = 0
    from batsrus_b200.capi import BxError
    while net.num_samples() < (nPair // 2) * blocksPerPair and nStep < 100:
        try:
            im.advance_part_impl()
        except BxError:  # a failed solve ends the collection
            break
        nStep += 1
    net.collect(0)
    nKrylov = net.num_samples() // blocksPerPair
    net.collect_probes(nPair - nKrylov, blocksPerPair, seed=2025)
    x.close()
    t1 = time.perf_counter()
    first, last = net.train(nEpoch=args.learned_epochs, batch=256, lr=1e-3)
    net.set_blend(args.learned_blend)
    t2 = time.perf_counter()
    return net, {"pairs": net.num_samples() // blocksPerPair, "krylov_pairs": nKrylov,
                 "probe_pairs": net.num_samples() // blocksPerPair - nKrylov, "block_samples": net.num_samples(),
                 "collect_steps": nStep, "collect_s": t1 - t0, "epochs": args.learned_epochs,
                 "train_s": t2 - t1, "mse_first_epoch": first, "mse_last_epoch": last,
                 "seed_data": 2025, "seed_timed": 2024, "mode": "linear, identity part + learned remainder",
                 "blend": args.learned_blend}


def run_amr(args, lrank):
    """The block-adaptive blast workload: all levels in one persistent stage
    kernel per stage, resolution-change ghost cells and flux correction,
    args.amr_steps time steps captured in one CUDA graph; FP32-bulk (the
    configuration's precision) and FP64, cell-updates/s (cells of all levels
    x steps / device time of the graph launch)."""
    from batsrus_b200 import configs
    from batsrus_b200.explicit import ExplicitSolver
    out = {}
    st = None
    for prec in ("fp32", "fp64"):
        g, s, st0, _ = configs.amr_blast(nRoot=args.amr_nroot, maxLevel=3, precision=prec, with_state=st is None)
        st = st0 if st is None else st
        x = ExplicitSolver(g, s, device=lrank)
        x.set_state(st)
        x.advance(1)  # Dt = 0 step
        tuned = x.autotune() if args.autotune else None
        x.set_graph_steps(args.amr_steps)
        x.advance(1 + args.amr_steps)  # one uncaptured step, capture, one graph launch
        x.synchronize()
        x.region_begin()
        x.advance(args.amr_steps)  # one graph launch
        ms = x.region_end()
        lev = np.bincount(g.iLevelCoord[:, 0])
        out[prec] = {"value": g.nCell * args.amr_steps / (ms * 1e-3), "ms_per_step": ms / args.amr_steps,
                     "autotune": ({k: v["value"] for k, v in tuned.items() if k.startswith("stage")}
                                  if tuned else None)}
        x.close()
    out.update({"workload": "amr_blast_levels0-3_nroot%d_hlld_mc" % args.amr_nroot, "unit": UNIT,
                "blocks": int(g.nBlock), "cells": int(g.nCell), "blocks_per_level": [int(v) for v in lev],
                "steps_per_graph": args.amr_steps, "value_is": "fp32 bulk (FP64 accumulation)"})
    return out


def run_amr_dynamic(args, lrank):
    """The blast with dynamic AMR (#DOAMR every args.amr_dyn_dn steps,
    #AMRCRITERIA pjumpratio refining above 1.3 and coarsening below 1.02,
    #AMRLEVELS 0..4, MaxTotalBlocks 3x the initial grid): FP32-bulk steps plus the regrids
    (criteria on the GPU, the tree in the library's host code, the state
    remapped on the GPU, tables and graph rebuilt).  Reports the steps'
    cell-updates/s without and with the regrid time, and the time per regrid
    (host wall clock around bx_do_amr, synchronised)."""
    from batsrus_b200 import amr, configs
    from batsrus_b200.explicit import ExplicitSolver
    g, s, st, _ = configs.amr_blast(nRoot=args.amr_nroot, maxLevel=3, precision="fp32")
    x = ExplicitSolver(g, s, device=lrank)
    x.set_state(st)
    x.advance(2)  # Dt = 0 step, then one step
    if args.autotune:
        x.autotune()
    p = amr.AmrParams(dnRefine=args.amr_dyn_dn, criteria=[amr.AmrCriterion("pjumpratio", 1.02, 1.3)],
                      minBlockLevel=0, maxBlockLevel=4, maxTotalBlocks=3 * g.nBlock)
    blocks0 = g.nBlock
    stepMs, cellSteps, regridMs, blocks = 0.0, 0, [], [g.nBlock]
    done = 0
    while done < args.amr_dyn_steps:
        k = min(args.amr_dyn_dn, args.amr_dyn_steps - done)
        x.synchronize()
        x.region_begin()
        x.advance(k)
        stepMs += x.region_end()
        cellSteps += x.grid.nCell * k
        done += k
        t0 = time.perf_counter()
        x.do_amr(p)
        x.synchronize()
        regridMs.append(1e3 * (time.perf_counter() - t0))
        blocks.append(x.grid.nBlock)
    x.close()
    tot = stepMs + sum(regridMs)
    return {"workload": "amr_blast_dynamic_nroot%d_levels0-4_doamr%d_pjumpratio" % (args.amr_nroot, args.amr_dyn_dn),
            "unit": UNIT, "precision": "fp32", "steps": args.amr_dyn_steps, "regrids": len(regridMs),
            "blocks_initial": blocks0, "blocks_after_each_regrid": blocks,
            "steps_value": cellSteps / (stepMs * 1e-3), "value_with_regrids": cellSteps / (tot * 1e-3),
            "ms_per_regrid": regridMs, "steps_ms": stepMs,
            "criteria": "pjumpratio coarsen < 1.02, refine > 1.3",
            "regrid_timing": "host wall clock around bx_do_amr, synchronised"}


def run_heat(args, lrank):
    """Semi-implicit field-aligned heat conduction on the dipole workload:
    device time per solve (CUDA events around bx_advance_semi_impl, the
    host-side Krylov control included) and matrix-vector products per solve,
    for each preconditioner; every solve advances the temperature."""
    from batsrus_b200.capi import BxError
    from batsrus_b200.explicit import ExplicitSolver
    from batsrus_b200.heat import HeatSolver
    from batsrus_b200.heat_params import HeatParams, heat_dipole, global_to_blocks
    from batsrus_b200.param import Scheme
    nR = args.heat_nroot
    n = 8 * nR
    g, Te, b, used, dx = heat_dipole(nRoot=nR)
    tb = lambda a: global_to_blocks(a.reshape((n, n, n) + a.shape[1:]), nR)
    Te, b, used = tb(Te), tb(b), tb(used)
    out = {"workload": "dipole_heat_conduction_%dcubed_kpar_kperp_1e6_gmres30_1e-6" % n, "cells": g.nCell,
           "blocks": g.nBlock, "used_fraction": float(used.mean()), "solves": args.heat_steps,
           "warmup": args.heat_warmup, "unit": "s/solve", "higher_is_better": False,
           "bilu_sweeps": args.heat_ilu, "operator_tensor": args.heat_operator}
    net = None
    for prec in args.heat_precond.split(","):
        x = None
        try:
            if prec.upper() == "LEARNED" and net is None:
                net, out["learned_training"] = train_learned_heat(args, g, lrank)
            x = ExplicitSolver(g, Scheme(), device=lrank)
            h = HeatSolver(x, HeatParams(typePrecond=prec, precondPrecision=args.heat_ilu,
                                         operatorPrecision=args.heat_operator), Te, b, used)
            if args.autotune:
                x.autotune()
            for _ in range(args.heat_warmup):
                h.advance_semi_impl()
            x.synchronize()
            x.region_begin()
            stats = [h.advance_semi_impl() for _ in range(args.heat_steps)]
            ms = x.region_end()
        except BxError as e:
            out[prec.lower()] = {"failed": str(e)}
            if x is not None:
                x.close()
            continue
        nmv = float(np.mean([q["nMatvec"] for q in stats]))
        out[prec.lower()] = {"s_per_solve": ms * 1e-3 / args.heat_steps,
                             "matvec_per_solve": nmv,
                             "s_per_matvec_per_mcell": ms * 1e-3 / args.heat_steps / nmv / (g.nCell / 1e6),
                             "matvec": [q["nMatvec"] for q in stats],
                             "krylov_error": [q["Error"] for q in stats],
                             "criterion": ("true residual (flexible GMRES)" if prec.upper() in ("LEARNED", "NONE")
                                           else "preconditioned residual (left GMRES)")}
        x.close()
    if net is not None:
        net.close()
    return out


def train_learned_heat(args, g, lrank, nPair=2000, blocksPerPair=16):
    """The learned preconditioner of the heat solve: (t, BILU(t)) block pairs
    with the blocks' ILU factors from BILU solves of a differently seeded
    field (seed 2025), training on the residual-space loss, blend 0.05 (the
    largest weight of the learned remainder that keeps flexible GMRES
    convergent at 256^3)."""
    from batsrus_b200.explicit import ExplicitSolver
    from batsrus_b200.heat import HeatSolver
    from batsrus_b200.heat_params import HeatParams, heat_dipole, global_to_blocks
    from batsrus_b200.learned import LearnedPreconditioner
    from batsrus_b200.param import Scheme
    nR = args.heat_nroot
    n = 8 * nR
    _, Te, b, used, _ = heat_dipole(nRoot=nR, seed=2025)
    tb = lambda a: global_to_blocks(a.reshape((n, n, n) + a.shape[1:]), nR)
    net = LearnedPreconditioner(nSampleMax=nPair * blocksPerPair, seed=2024)
    x = ExplicitSolver(g, Scheme(), device=lrank)
    h = HeatSolver(x, HeatParams(), tb(Te), tb(b), tb(used))
    t0 = time.perf_counter()
    net.collect(blocksPerPair)
    nSolve = 0
    while net.num_samples() < nPair * blocksPerPair and nSolve < 60:
        h.advance_semi_impl()
        nSolve += 1
    net.collect(0)
    x.close()
    t1 = time.perf_counter()
    first, last = net.train(nEpoch=12, batch=256, lr=1e-3)
    net.set_blend(0.05)
    t2 = time.perf_counter()
    return net, {"pairs": net.num_samples() // blocksPerPair, "collect_solves": nSolve, "collect_s": t1 - t0,
                 "train_s": t2 - t1, "loss_first_epoch": first, "loss_last_epoch": last,
                 "loss": "residual space |M N(t) - t|^2 with the blocks' ILU factors", "seed_data": 2025,
                 "seed_timed": 2024, "blend": 0.05}


def cpu_baseline_heat(args, seconds=20.0):
    """The oracle's heat conduction solve (BILU) on a 64^3 sample of the
    dipole workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from batsrus_b200.heat_params import HeatParams, heat_dipole
    from oracle import HeatOracle
    nR = 8
    _, Te, b, used, dx = heat_dipole(nRoot=nR)
    o = HeatOracle(8 * nR, dx, Te, b, used, HeatParams())
    n, t0, nm = 0, time.perf_counter(), 0
    while True:
        r, _, m, _ = o.solve()
        n, nm = n + 1, nm + m
        el = time.perf_counter() - t0
        if el > seconds or n >= 5:
            break
    o.close()
    return {"value": el / n, "unit": "s/solve", "cores": os.cpu_count(), "kind": "port",
            "matvec_per_solve": nm / n,
            "cells": (8 * nR) ** 3,
            "s_per_matvec_per_mcell": el / nm / ((8 * nR) ** 3 / 1e6),
            "sample": "oracle/ C++ restatement of advance_semi_impl with BILU, 64^3 (512 blocks) of the "
                      "dipole workload, %d solves (residual, block ILU and vector updates on all threads, "
                      "inner products on one)" % n}


def cpu_baseline_jfnk(args, seconds=20.0):
    """The oracle's implicit step (BILU) on a 32^3 sample of the JFNK workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from batsrus_b200 import configs
    from oracle import Oracle
    cores = os.cpu_count()
    g, s, p, st = configs.jfnk_ot(nRoot=4)
    o = Oracle(g, s, n_thread=cores)
    o.set_state(st)
    o.exchange_messages()
    o.set_implicit(p)
    o.advance_implicit()  # sets the time step
    n, t0, nm = 0, time.perf_counter(), 0
    while True:
        r, m, _ = o.advance_implicit()
        n, nm = n + 1, nm + m
        el = time.perf_counter() - t0
        if el > seconds or n >= 10:
            break
    return {"value": el / n, "unit": "s/step", "cores": cores, "kind": "port",
            "matvec_per_step": nm / n, "cells": g.nCell, "s_per_step_per_mcell": el / n / (g.nCell / 1e6),
            "sample": "oracle/ C++ restatement of advance_part_impl with BILU, 32^3 (64 blocks) of the "
                      "perturbed Orszag-Tang workload, %d steps on %d threads" % (n, cores)}


def cpu_baseline(args, seconds=12.0):
    """The oracle (C++ restatement of the orig path, OpenMP over blocks) on a
    64^3 Orszag-Tang sample, on all host cores, timed until ~seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from batsrus_b200 import configs
    from oracle import Oracle
    cores = os.cpu_count()
    g, s, st, _ = configs.orszag_tang_3d(nRoot=8, flux=args.flux)
    o = Oracle(g, s, n_thread=cores)
    o.set_state(st)
    o.exchange_messages()
    o.advance(1)  # Dt = 0 step
    n, t0 = 0, time.perf_counter()
    while True:
        o.advance(1)
        n += 1
        el = time.perf_counter() - t0
        if el > seconds or n >= 40:
            break
    return {"value": g.nCell * n / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "oracle/ C++ restatement, 64^3 Orszag-Tang (512 blocks of 8^3), " + args.flux + "+Koren, "
                      "FP64, %d full steps in %.1f s on %d threads" % (n, el, cores)}


def run_reference(args):
    """The reference arm: the oracle (C++ restatement of the orig path,
    OpenMP over blocks, all host threads) on the bench's own workload, the
    full Orszag-Tang domain of --nroot^3 blocks (256^3 by default: about 2 s
    per step on 16 threads, 11 GB of host memory), W untimed steps after the
    Dt = 0 step, then K timed steps."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from batsrus_b200 import configs
    from oracle import Oracle
    cores = os.cpu_count()
    g, s, st, _ = configs.orszag_tang_3d(nRoot=args.nroot, flux=args.flux)
    o = Oracle(g, s, n_thread=cores)
    o.set_state(st)
    del st
    o.exchange_messages()
    o.advance(1 + args.warmup)
    t0 = time.perf_counter()
    o.advance(args.steps)
    el = time.perf_counter() - t0
    v = g.nCell * args.steps / el
    n = 8 * args.nroot
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": (WORKLOAD if args.flux == "Linde" else
                                    "orszag_tang_3d_256cubed_%s_koren" % args.flux.lower())
                       if args.nroot == 32 else "orszag_tang_3d_%dcubed_%s_koren" % (n, args.flux.lower()),
                       "cells": g.nCell, "blocks": g.nBlock, "block_cells": "8x8x8", "flux": args.flux,
                       "limiter": "mc3 beta=1.2", "cfl": 0.8, "stages": 2},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "oracle/ C++ restatement of the orig path, the whole %d^3 Orszag-Tang "
                                       "domain, %d steps, %d threads" % (n, args.steps, cores)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nroot", type=int, default=32, help="root blocks per dimension (32 -> 256^3)")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu", dest="cpu", action="store_false")
    ap.add_argument("--precisions", default="fp64,fp32")
    ap.add_argument("--flux", default="Linde", choices=["Rusanov", "Linde", "HLLD", "Roe"],
                    help="TypeFlux of the explicit Orszag-Tang workload (Linde is the headline)")
    ap.add_argument("--jfnk-precond", default="BILU,NONE,LEARNED", help="'' to skip the implicit workload")
    ap.add_argument("--learned-epochs", type=int, default=64)
    ap.add_argument("--learned-blend", type=float, default=0.6)
    ap.add_argument("--amr", dest="amr", action="store_true", default=True)
    ap.add_argument("--no-amr", dest="amr", action="store_false")
    ap.add_argument("--amr-nroot", type=int, default=19,
                    help="root blocks per dimension of the blast grid (19: 20,544 blocks, 10.5 M cells)")
    ap.add_argument("--amr-steps", type=int, default=50)
    ap.add_argument("--amr-dyn-steps", type=int, default=50, help="steps of the dynamic-AMR blast (0: skip)")
    ap.add_argument("--amr-dyn-dn", type=int, default=10, help="steps between regrids (#DOAMR DnAmr)")
    ap.add_argument("--jfnk-nroot", type=int, default=16, help="16 -> 128^3 cells")
    ap.add_argument("--jfnk-steps", type=int, default=5)
    ap.add_argument("--bilu-factors", default="bf16", choices=["fp64", "fp32", "bf16"],
                    help="storage of the BILU factors of the implicit workload")
    ap.add_argument("--heat-ilu", default="fp32", choices=["fp64", "fp32"],
                    help="precision of the BILU sweeps of the heat conduction workload")
    ap.add_argument("--heat-operator", default="fp32", choices=["fp64", "fp32"],
                    help="storage of the face conduction tensor in the heat solve's matrix-free product")
    ap.add_argument("--jfnk-warmup", type=int, default=2)
    ap.add_argument("--sharded", action="store_true",
                    help="one domain partitioned over the ranks (shard.GpuRank) instead of replicas")
    ap.add_argument("--stage-ctas", type=int, default=0,
                    help="pin stage_ctas_per_sm (FP32-bulk stage 2: 2 -> two 256-thread CTAs per SM)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default launch shapes instead of bx_autotune")
    ap.add_argument("--heat-precond", default="BILU,NONE,LEARNED", help="'' to skip the heat conduction workload")
    ap.add_argument("--heat-nroot", type=int, default=32, help="32 -> 256^3 cells")
    ap.add_argument("--heat-steps", type=int, default=3)
    ap.add_argument("--heat-warmup", type=int, default=1)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, _ = dist_env()
    if args.sharded:
        res = run_sharded(args)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": max(world, 1),
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                              "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                              "dtype": "f64" if args.precisions.startswith("fp64") else "f32/f64",
                              "data": "synthetic",
                              "config": {"workload": "orszag_tang_3d_%dcubed_%s_koren_partitioned" %
                                                     (8 * args.nroot, args.flux.lower()),
                                         "parallelism": "blocks partitioned over ranks (Morton ranges)"},
                              "sharded": res}))
        return
    res = run_ours(args)
    if rank != 0:
        return
    r64, r32 = res.get("fp64", res.get("fp32")), res.get("fp32", {})
    line = {"metric": METRIC, "value": r64["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r64["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD if args.flux == "Linde" else
                       "orszag_tang_3d_%dcubed_%s_koren" % (8 * args.nroot, args.flux.lower()),
                       "cells": (8 * args.nroot) ** 3, "blocks": args.nroot ** 3,
                       "block_cells": "8x8x8", "flux": "Linde", "limiter": "mc3 beta=1.2", "cfl": 0.8,
                       "stages": 2, "l2": "inputs larger than L2 (state %.2f GB)" % ((8 * args.nroot) ** 3 * 64 / 1e9),
                       "parallelism": "one domain per GPU"},
            "roofline": r64["roofline"], "clocks": r64["clocks"], "gpu_launches": r64["gpu_launches"],
            "autotune": r64.get("autotune"),
            "fp32_bulk": ({"value": r32["value"], "ms_per_step": r32["ms_per_step"], "dtype": "f32/f64",
                           "roofline": r32["roofline"], "e2e": r32.get("e2e")} if r32 else None)}
    if "e2e" in r64:
        line["e2e"] = r64["e2e"]
    if args.jfnk_precond:
        line["jfnk"] = run_jfnk(args, 0)
    if args.amr:
        line["amr"] = run_amr(args, 0)
        if args.amr_dyn_steps > 0:
            line["amr"]["dynamic"] = run_amr_dynamic(args, 0)
    if args.heat_precond:
        line["heat"] = run_heat(args, 0)
    if args.cpu and world == 1:
        line["cpu_baseline"] = cpu_baseline(args)
        if args.jfnk_precond:
            line["jfnk"]["cpu_baseline"] = cpu_baseline_jfnk(args)
        if args.heat_precond:
            line["heat"]["cpu_baseline"] = cpu_baseline_heat(args)
    line["summary"] = summary(line)  # last key: the end of the line shows every leg
    print(json.dumps(line))


def summary(line):
    """The key figure of every leg, compactly (rounded to 4 digits)."""
    r = lambda v: None if v is None else float("%.4g" % v)
    out = {"fp64": r(line["value"]), "fp64_frac": line["roofline"]["frac"],
           "fp64_e2e": r(line.get("e2e", {}).get("value"))}
    fb = line.get("fp32_bulk")
    if fb:
        out.update({"fp32_bulk": r(fb["value"]), "fp32_bulk_frac": fb["roofline"]["frac"],
                    "fp32_bulk_e2e": r((fb.get("e2e") or {}).get("value"))})
    j = line.get("jfnk")
    if j:
        sp = {k: r(j[k]["s_per_step"]) for k in ("bilu", "none", "learned") if "s_per_step" in j.get(k, {})}
        mv = {k: r(j[k]["matvec_per_step"]) for k in sp}
        out["jfnk_s_per_step"] = sp
        out["jfnk_matvec_per_step"] = mv
        if "learned" in sp:  # time per step of the learned preconditioner / of BILU, of NONE
            for k in ("bilu", "none"):
                if k in sp:
                    out["jfnk_learned_over_%s" % k] = r(sp["learned"] / sp[k])
        if "cpu_baseline" in j:
            out["jfnk_cpu_s_per_step"] = r(j["cpu_baseline"]["value"])
            if "bilu" in sp:  # per cell: the CPU sample is 32^3, the GPU workload 128^3
                out["jfnk_cpu_over_gpu_bilu_per_cell"] = r(j["cpu_baseline"]["s_per_step_per_mcell"] /
                                                           j["bilu"]["s_per_step_per_mcell"])
    a = line.get("amr")
    if a:
        out["amr"] = {"blocks": a["blocks"], "cells": a["cells"], "fp32": r(a["fp32"]["value"]),
                      "fp64": r(a["fp64"]["value"])}
        if "dynamic" in a:
            out["amr"]["dynamic_steps"] = r(a["dynamic"]["steps_value"])
            out["amr"]["dynamic_with_regrids"] = r(a["dynamic"]["value_with_regrids"])
    h = line.get("heat")
    if h:
        sp = {k: r(h[k]["s_per_solve"]) for k in ("bilu", "none", "learned") if "s_per_solve" in h.get(k, {})}
        out["heat_s_per_solve"] = sp
        out["heat_matvec_per_solve"] = {k: r(h[k]["matvec_per_solve"]) for k in sp}
        if "cpu_baseline" in h:
            out["heat_cpu_s_per_solve"] = r(h["cpu_baseline"]["value"])
            if "bilu" in sp:  # per matrix-vector product and cell: the CPU sample is 64^3
                out["heat_cpu_over_gpu_bilu_per_matvec_cell"] = r(h["cpu_baseline"]["s_per_matvec_per_mcell"] /
                                                                  h["bilu"]["s_per_matvec_per_mcell"])
    if "cpu_baseline" in line:
        out["cpu"] = r(line["cpu_baseline"]["value"])
    return out


if __name__ == "__main__":
    main()
