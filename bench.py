"""Benchmark: Gcell-updates/s of the composite-grid time loop on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--small]

Workload (one step = one pass of main.cpp's time loop over the whole composite):
the three-grid ratio-3 composite 1081x1081x121 @ 5 m / 361x361x161 @ 15 m /
121x121x101 @ 45 m (163,856,303 points), FP32 fields, tilted-VTI medium with
all 21 Cij (Thomsen eps 0.10, delta 0.05, gamma 0.08, seeded smooth dip <= 30
deg and azimuth), free surface, Ricker vz source at the surface centre, 1081 vz
surface receivers, energy every 100 steps.  Inputs are seeded synthetic media
(no dataset exists for this path).  --medium iso runs the isotropic twin.
N > 1 runs N independent replicas (one per GPU, launched by torchrun): the
path has no exchange step, so there is no collective on the data path.

The line printed by rank 0 carries the device-timed throughput (`value`), the
end-to-end throughput through the C ABI with host buffers (`e2e`), the HBM
roofline of the dominant kernel (`roofline`), the reference's OpenMP CPU path
timed on this host (`cpu_baseline`), SM clocks sampled during the timed
region, and the number of kernels launched.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_CELL = {"iso": 132, "ortho9": 148, "tti": 196}    # compulsory FP32 traffic per cell-update
STRESS_BYTES = {"iso": 80, "ortho9": 96, "tti": 144}        # stress kernel: 3v + 6 sigma (rmw) + N_C words
VEL_BYTES = 52                                              # velocity kernel: 6 sigma + 3 v (rmw) + buoyancy
DISP_BYTES = 24                                             # 21-Cij energy: 3 displacement sums (rmw)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling (200 ms) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
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
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_reference(steps_sample=None, warm=2):
    """The reference's own OpenMP time loop (oracle/_ref/libecsg_ref64.so, the
    unmodified sources compiled with -O3 -fopenmp) on its own experiment
    tests/test1-cmp-eci-ii/eci (two grids at ratio 2, 13,055,365 points; the
    reference cannot run ratio 3), check_energy off, all host threads."""
    from ecsg_b200.workloads import eci_test_case
    from oracle.ref import RefRun
    cores = len(os.sched_getaffinity(0))
    case = eci_test_case(1)
    r = RefRun(case, energy=False, threads=cores)
    try:
        r.run(warm, 0)
        # size the sample to roughly 10-20 s of CPU work
        t1 = r.run(2, warm)
        n = steps_sample or max(2, min(200, int(15.0 / max(t1 / 2, 1e-3))))
        t = r.run(n, warm + 2)
    finally:
        r.close()
    pts = case.points()
    return {"value": pts * n / t / 1e9, "unit": "Gcell/s", "cores": cores, "kind": "reference",
            "sample": "%d steps of the reference experiment test1-cmp-eci-ii/eci (2 grids, ratio 2, %d points, "
                      "FP64 as shipped, energy off) on %d host threads; wall clock" % (n, pts, cores)}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    try:
        base = cpu_reference()
    except Exception as e:  # the reference build did not travel
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build not runnable: %s" % e}))
        return
    line = {"impl": "reference", "metric": "Gcell-updates/s", "value": base["value"], "unit": "Gcell/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "reference experiment test1-cmp-eci-ii/eci (CPU twin of the three-grid "
                                   "benchmark: the reference implements ratio 2 and isotropic media only)"},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "Gcell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# geometries of the shot-gradient leg: the benchmark's (None: the workload
# default, 361x361x61 @ 10 m over 121x121x81 @ 30 m) and a medium one for
# profiling captures (1/8 of the volume: 181x181x31 over 61x61x41)
GRAD_GRIDS = {"full": None, "medium": [((180, 180, 30), 10.0), ((60, 60, 40), 30.0)]}


def shot_gradients(args, local, world, max_over_ranks, barrier):
    """Misfit gradients on the two-grid adjoint workload: 361x361x61 @ 10 m
    over 121x121x81 @ 30 m (9,135,502 points), smooth orthorhombic model,
    121 x 121 surface vz receivers, checkpoints every 50 steps; observed data
    from the same model with a 3 % vs blob.

    Plain: one shot at a time (ecsg_misfit_gradient: forward with
    checkpoints, recomputation, adjoint) on each GPU.  Batched (--grad-batch
    B > 1): B shots of the same model sharing one medium allocation
    (ecsg_create_shot), advanced in lockstep (ecsg_shots_misfit_gradient: the
    medium adjoints and the interface solves once for all shots, the gradient
    of the shots' summed misfit).  Both legs are device-timed with CUDA events
    on the library stream (the lockstep call runs on the first instance's
    stream); on several GPUs the plain leg includes the FP64 all-reduce of the
    gradient volumes (NCCL, on the same stream)."""
    import ecsg_b200
    from ecsg_b200.workloads import two_grid_adjoint_case
    n = args.grad_steps
    shot = local % 16
    G = GRAD_GRIDS[args.grad_size]
    with ecsg_b200.Simulation(two_grid_adjoint_case(0, shot, n, blob=True, grids=G), precision="f32", device=local) as s:
        obs = s.run(n)["rec"].T.copy()
    case = two_grid_adjoint_case(0, shot, n, blob=False, grids=G)
    with ecsg_b200.Simulation(case, precision="f32", device=local) as s:
        s.misfit_gradient(obs[: min(n, 60)], ckpt_every=50)   # warm-up (allocations, tensor maps)
        if world > 1:
            from ecsg_b200.distributed import allreduce_gradients
            allreduce_gradients(s)   # warm-up of the collective
        barrier()
        s.timer_start()
        loss = s.misfit_gradient(obs, ckpt_every=50)
        if world > 1:
            allreduce_gradients(s)
        ms = s.timer_stop()
        gmax = float(np.abs(s.gradient(0, 0)).max())
        status = s.status()
    ms = max_over_ranks(ms)
    batched = None
    nb = args.grad_batch
    if nb > 1:
        shots = [(local * nb + k) % 16 for k in range(nb)]
        obs_b = []
        for k in shots:
            with ecsg_b200.Simulation(two_grid_adjoint_case(0, k, n, blob=True, grids=G), precision="f32", device=local) as s:
                obs_b.append(s.run(n)["rec"].T.copy())
        model = ecsg_b200.Simulation(two_grid_adjoint_case(0, shots[0], n, blob=False, grids=G), precision="f32", device=local)
        sims = [model] + [ecsg_b200.Simulation.shot(model, two_grid_adjoint_case(0, k, n, blob=False, grids=G)) for k in shots[1:]]
        try:
            ecsg_b200.shots_misfit_gradient(sims, [o[: min(n, 60)] for o in obs_b], ckpt_every=50)   # warm-up
            barrier()
            model.timer_start()
            losses = ecsg_b200.shots_misfit_gradient(sims, obs_b, ckpt_every=50)
            bms = model.timer_stop()
            bstatus = max(x.status() for x in sims)
            bgmax = float(np.abs(model.gradient(0, 0)).max())
        finally:
            for x in sims[1:]:
                x.close()
            model.close()
        bms = max_over_ranks(bms)
        batched = {"shots": nb, "value": world * nb / (bms * 1e-3), "ms_per_batch": bms,
                   "ms_per_shot_gradient": bms / nb, "speedup_vs_plain": (nb / bms) / (1.0 / ms),
                   "finite": bool(np.isfinite(losses).all() and np.isfinite(bgmax)), "status": bstatus,
                   "mode": "lockstep shots sharing the medium (ecsg_shots_misfit_gradient), gradient of the summed "
                           "misfit", "timing": "CUDA events on the library stream, both legs"}
    return {"metric": "shot-gradients/s", "value": world / (ms * 1e-3), "unit": "shot-gradients/s",
            "mode": "plain (one shot per GPU at a time)" + (", FP64 NCCL all-reduce of the gradients" if world > 1 else ""),
            "ms_per_shot_gradient": ms, "steps": n,
            "ckpt_every": 50, "points": case.points(), "receivers": len(case.rec), "dtype": "f32",
            "loss": loss, "finite": bool(np.isfinite(loss) and np.isfinite(gmax)), "status": status,
            "workload": "two-grid %s, smooth orthorhombic, shot %d of 4x4" % (
                " / ".join("%dx%dx%d@%gm" % (g["n"][0] + 1, g["n"][1] + 1, g["n"][2] + 1, g["h"][0]) for g in case.grids), shot),
            "batched": batched}


def config5_subset(args, local, world, max_over_ranks, barrier):
    """Batched shot gradients with the structure of the benchmark's batched
    configuration (shots on an 8 x 8 surface grid of the three-grid tilted-VTI
    model, 8 shots per lockstep call sharing the medium, 2000 steps,
    checkpoints every 100 steps) on the 1/27-volume copy of the model
    (361x361x41 @ 5 m / 121x121x55 @ 15 m / 41x41x35 @ 45 m): at full size one
    shot's 21 checkpoints alone (6.5 GB each) exceed a GPU's memory.  Observed
    data: the model built from seed 1 (other perturbations, dips and
    azimuths).  The first args.c5_shots shots of the 8 x 8 grid in lockstep
    against plain runs of the first args.c5_plain of them, device-timed."""
    import ecsg_b200
    from ecsg_b200.workloads import three_grid_case
    n, k = args.c5_steps, 100
    grids = [((360, 360, 40), 5.0), ((120, 120, 54), 15.0), ((40, 40, 34), 45.0)]

    def shot_case(j, seed):
        c = three_grid_case(seed=seed, grids=grids, nsteps=n, medium="tti")
        n0, h0 = grids[0]
        c.src = dict(c.src, xyz=((j % 8 + 0.5) / 8 * n0[0] * h0, (j // 8 + 0.5) / 8 * n0[1] * h0, 0.0))
        return c
    S = args.c5_shots
    obs = []
    for j in range(S):
        with ecsg_b200.Simulation(shot_case(j, 1), precision="f32", device=local) as s:
            obs.append(s.run(n)["rec"].T.copy())
    plain_ms = []
    for j in range(args.c5_plain):
        with ecsg_b200.Simulation(shot_case(j, 0), precision="f32", device=local) as s:
            s.misfit_gradient(obs[j][:min(n, 120)], ckpt_every=k)
            s.timer_start()
            s.misfit_gradient(obs[j], ckpt_every=k)
            plain_ms.append(s.timer_stop())
    model = ecsg_b200.Simulation(shot_case(0, 0), precision="f32", device=local)
    sims = [model] + [ecsg_b200.Simulation.shot(model, shot_case(j, 0)) for j in range(1, S)]
    try:
        ecsg_b200.shots_misfit_gradient(sims, [o[:min(n, 120)] for o in obs], ckpt_every=k)
        barrier()
        model.timer_start()
        losses = ecsg_b200.shots_misfit_gradient(sims, obs, ckpt_every=k)
        bms = model.timer_stop()
        status = max(x.status() for x in sims)
    finally:
        for x in sims[1:]:
            x.close()
        model.close()
    bms = max_over_ranks(bms)
    pms = max_over_ranks(float(np.mean(plain_ms)))
    return {"metric": "shot-gradients/s", "workload": "batched-configuration subset: %d shots of the 8 x 8 surface "
                                                      "grid, three-grid tilted VTI at 1/27 volume (6,207,251 points), "
                                                      "%d steps, checkpoints every %d" % (S, n, k),
            "shots": S, "value": world * S / (bms * 1e-3), "ms_per_batch": bms,
            "plain_value": world / (pms * 1e-3), "plain_ms_per_shot_gradient": pms, "plain_shots_timed": args.c5_plain,
            "speedup_vs_plain": (S / bms) / (1.0 / pms), "finite": bool(np.isfinite(losses).all()), "status": status,
            "timing": "CUDA events on the library stream"}


def accuracy(args, local):
    """FP32 production path against an FP64 shadow run of a reduced copy of the
    benchmark case (three grids at ratio 3, 181x181x25 @ 5 m / 61x61x19 @ 15 m
    / 21x21x13 @ 45 m, the same seeded tilted-VTI construction, free surface,
    vz source and surface vz receivers), over args.accuracy_steps steps with
    energy every 10 steps: rel-L2 of the traces and of the final fields (the
    largest over the 27 components), and the energy: the largest relative
    difference FP32 / FP64, and the drift (max - min) / mean of each after the
    source has stopped."""
    import ecsg_b200
    from ecsg_b200.workloads import three_grid_case
    n = args.accuracy_steps
    grids = [((180, 180, 24), 5.0), ((60, 60, 18), 15.0), ((20, 20, 12), 45.0)]
    case = three_grid_case(seed=0, grids=grids, nsteps=n, medium="tti")
    runs = {}
    for prec in ("f64", "f32"):
        with ecsg_b200.Simulation(case, precision=prec, energy=True, device=local) as s:
            out = s.run(n, energy_every=10)
            e = out["energy"]
            runs[prec] = (out["rec"].astype(np.float64), e[~np.isnan(e)],
                          [s.field(g, k)[1:-1, 1:-1, 1:-1] for g in range(3) for k in range(9)])
    (r64, e64, f64), (r32, e32, f32) = runs["f64"], runs["f32"]
    rel = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    src_end = len(case.src["trace"])
    post = [i for i in range(len(e64)) if 10 * i > src_end + 10]   # energy on steps 0, 10, 20, ...
    drift = lambda e: float((e.max() - e.min()) / e.mean()) if len(e) > 1 else None
    return {"workload": "three-grid ratio-3 tilted VTI 181x181x25@5m / 61x61x19@15m / 21x21x13@45m, %d steps" % n,
            "reference": "FP64 device path (bitwise equal to the FP64 CPU oracle per operator)",
            "traces_rel_l2": rel(r32, r64), "final_fields_rel_l2_max": max(rel(a, b) for a, b in zip(f32, f64)),
            "energy_rel_diff_max": float(np.abs(e32 - e64).max() / np.abs(e64).max()),
            "energy_drift_post_source_f32": drift(e32[post]) if post else None,
            "energy_drift_post_source_f64": drift(e64[post]) if post else None,
            "mirror_fix": False}


def batched_forward(args, local, world, max_over_ranks, barrier):
    """48 independent two-grid composites of uneven size (fine nx, ny in
    {61, ..., 301} x 31 @ 10 m over the matching coarse grid with 31..81 z
    points @ 30 m, seeded 3-layer tilted-VTI media, one Ricker each), FP32:
    one CUDA graph launch per step advances all of them (ecsg_batch_run),
    against the same instances run one after another (each its own graph
    replay).  Device time with CUDA events."""
    import ecsg_b200
    from ecsg_b200.workloads import batch_instance_case
    n = args.batch_steps
    cases = [batch_instance_case(k + 48 * local, n + 6) for k in range(48)]
    pts = sum(c.points() for c in cases)
    sims = [ecsg_b200.Simulation(c, precision="f32", device=local) for c in cases]
    try:
        for s in sims:
            s.run(3)
        plain = 0.0
        for s in sims:
            s.run(n)
            plain += s.last_run()[0]
        ecsg_b200.batch_run(sims, 3, n0=n + 3)
        barrier()
        _, ms = ecsg_b200.batch_run(sims, n, n0=0)
    finally:
        for s in sims:
            s.close()
    ms = max_over_ranks(ms)
    plain = max_over_ranks(plain)
    return {"metric": "Gcell-updates/s", "instances": 48, "points": pts, "steps": n, "dtype": "f32",
            "value": pts * n * world / (ms * 1e-3) / 1e9, "plain_value": pts * n * world / (plain * 1e-3) / 1e9,
            "ms_per_step": ms / n, "plain_ms_per_step": plain / n, "speedup_vs_plain": plain / ms,
            "workload": "48 uneven two-grid composites (ratio 3), 3-layer tilted VTI, one graph launch per step"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)   # the configured run length
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="1/27-volume case (profiling); same as --size small")
    ap.add_argument("--size", default="full", choices=["full", "medium", "small"],
                    help="medium: 541x541x61 / 181x181x55 / 61x61x35 (2.9 GB, for ncu captures)")
    ap.add_argument("--energy-every", type=int, default=100)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the sweeps' built-in z-march depth (default: ecsg_autotune before the warm-up)")
    ap.add_argument("--medium", default="tti", choices=["tti", "iso"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grad-batch", type=int, default=8,
                    help="shots per batched shot-gradient run (0 or 1: no batched leg)")
    ap.add_argument("--grad-size", choices=sorted(GRAD_GRIDS), default="full",
                    help="geometry of the shot-gradient leg (medium: for profiling captures)")
    ap.add_argument("--grad-steps", type=int, default=1500,
                    help="steps of the shot-gradient measurement (0: skip it)")
    ap.add_argument("--c5-steps", type=int, default=2000,
                    help="steps of the batched-configuration subset (0: skip it)")
    ap.add_argument("--c5-shots", type=int, default=8)
    ap.add_argument("--c5-plain", type=int, default=1, help="plain shots timed for the subset's comparison")
    ap.add_argument("--accuracy-steps", type=int, default=600,
                    help="steps of the FP32-vs-FP64 accuracy run (0: skip it)")
    ap.add_argument("--batch-steps", type=int, default=1000,
                    help="steps of the batched-forward measurement (0: skip it)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import ecsg_b200
    from ecsg_b200.workloads import three_grid_case, THREE_GRID

    rank, world, local = dist_env()
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        pg = dist

    grids = THREE_GRID
    if args.small or args.size == "small":
        grids = [((360, 360, 40), 5.0), ((120, 120, 54), 15.0), ((40, 40, 34), 45.0)]
    elif args.size == "medium":
        grids = [((540, 540, 60), 5.0), ((180, 180, 54), 15.0), ((60, 60, 34), 45.0)]
    medium = args.medium
    case = three_grid_case(seed=0, grids=grids, nsteps=args.steps, medium=medium)
    pts = case.points()
    ev = args.energy_every
    sim = ecsg_b200.Simulation(case, precision="f32", energy=ev > 0, device=local)
    # 21-Cij energy needs the displacement sums, updated by every stress sweep
    acc = DISP_BYTES if (medium == "tti" and ev > 0) else 0

    def barrier():
        if pg is not None:
            import torch
            t = torch.zeros(1, device="cuda:%d" % local)
            pg.all_reduce(t)
            torch.cuda.synchronize()

    def max_over_ranks(x):
        if pg is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device="cuda:%d" % local)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    # the library's own autotuner picks the z-march depth of the FP32 sweeps of
    # each grid (ecsg_autotune: trial sweeps, state restored), before the warm-up
    tuned = None if args.no_autotune else sim.autotune()
    # warm-up (untimed), then the device-timed region (inputs resident in HBM,
    # 20 GB of fields and media >> 126 MB L2)
    sim.run(max(args.warmup, 3), energy_every=ev)
    barrier()
    with Clocks(local) as clk:
        sim.run(args.steps, energy_every=ev)
        run_ms, launches = sim.last_run()
    barrier()
    run_ms = max_over_ranks(run_ms)
    value = pts * args.steps * world / (run_ms * 1e-3) / 1e9

    # end to end through the C ABI with host buffers: source trace H2D from
    # pinned memory, all steps, receiver traces D2H into pinned memory
    import torch
    trace_host = torch.empty((args.steps, len(sim.rec)), dtype=torch.float32).pin_memory().numpy()
    src_host = torch.from_numpy(np.ascontiguousarray(case.src["trace"], dtype=np.float32)).pin_memory().numpy()
    L = ecsg_b200.lib()
    barrier()
    sim.timer_start()
    g, ix, iy, iz = sim.src
    sim._ck(L.ecsg_set_source(sim.h, g, ix, iy, iz, case.src["comp"], src_host.ctypes.data_as(ecsg_b200.c_fp),
                              src_host.size, float(case.src["scale"])))
    sim.run(args.steps, energy_every=ev, traces_out=trace_host)
    e2e_ms = sim.timer_stop()
    barrier()
    e2e_ms = max_over_ranks(e2e_ms)
    e2e = pts * args.steps * world / (e2e_ms * 1e-3) / 1e9
    h2d = src_host.nbytes / args.steps
    d2h = trace_host.nbytes / args.steps
    ok_traces = bool(np.isfinite(trace_host).all())

    # roofline of the dominant kernel from per-kernel CUDA events
    kt = sim.time_kernels(3)
    peak, peak_kind = measured_peak()
    n0 = case.grids[0]["n"]
    cells0 = (n0[0] + 1) * (n0[1] + 1) * (n0[2] + 1)
    st_ms, ve_ms = kt["stress"][0], kt["vel"][0]
    # algorithmic bytes: the compulsory traffic of the stencil update alone
    # (stress: 3 v + 6 sigma rmw + N_C moduli); the displacement sums that the
    # 21-Cij sweep also updates for the energy (24 B per cell) are reported
    # beside it, not in the numerator
    if st_ms >= ve_ms:
        kname = "stress21_tma_kernel<%s>" % ("true" if acc else "false") if medium == "tti" else "stress_kernel_v4<ISO5>"
        dom, dom_ms, dom_bytes, dom_acc = kname + " (grid 0)", st_ms, STRESS_BYTES[medium] * cells0, acc
    else:
        dom, dom_ms, dom_bytes, dom_acc = "vel_tma_kernel (grid 0)", ve_ms, VEL_BYTES * cells0, 0
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    achieved_acc = (dom_bytes + dom_acc * cells0) / (dom_ms * 1e-3) / 1e9
    step_ms = run_ms / args.steps
    step_gbs = BYTES_PER_CELL[medium] * pts / (step_ms * 1e-3) / 1e9
    # DRAM bytes per cell of the dominant kernel from an ncu capture of the
    # medium case (profiles/traffic.json), scaled to this launch's cells
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            entry = json.load(open(tpath)).get(dom.split(" ")[0], {})
            # only a capture of the same kernel variant (same bytes moved)
            same = entry.get("algorithmic_bytes_per_cell") == dom_bytes / cells0 and \
                entry.get("accumulator_bytes_per_cell", 0) == dom_acc
            per_cell = entry.get("dram_bytes_per_cell") if same else None
            traffic = per_cell * cells0 if per_cell else None
        except Exception:
            traffic = None

    base = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            base = cpu_reference()
        except Exception as e:
            base = {"value": None, "unit": "Gcell/s", "cores": 0, "kind": "reference", "sample": "unavailable: %s" % e}

    dev_bytes = sim.device_bytes()
    sim.close()
    grad = shot_gradients(args, local, world, max_over_ranks, barrier) if args.grad_steps > 0 else None
    batched = batched_forward(args, local, world, max_over_ranks, barrier) if args.batch_steps > 0 else None
    c5 = config5_subset(args, local, world, max_over_ranks, barrier) if args.c5_steps > 0 else None
    acc_line = accuracy(args, local) if (rank == 0 and args.accuracy_steps > 0) else None
    if rank == 0:
        line = {
            "metric": "Gcell-updates/s", "value": value, "unit": "Gcell/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "three-grid ratio-3 composite %s, %d points, free surface, Ricker vz point "
                                   "force, %d vz receivers, energy every %d steps"
                                   % (" / ".join("%dx%dx%d@%gm" % (n[0] + 1, n[1] + 1, n[2] + 1, h)
                                                 for n, h in grids), pts, len(sim.rec), ev),
                       "medium": ("tilted VTI, all 21 Cij, built on the device from seeded node vp/vs/rho/dip/"
                                  "azimuth (Thomsen eps 0.10, delta 0.05, gamma 0.08)" if medium == "tti" else
                                  "isotropic stiffness from the seeded vp/vs/rho model (5 distinct moduli)"),
                       "points": pts, "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2: %.1f GB of fields and media resident" % (dev_bytes / 1e9),
                       "z_march_chunks": ({"autotuned": True, "per_grid_vel_stress": [list(t) for t in tuned]}
                                          if tuned is not None else {"autotuned": False})},
            "e2e": {"value": e2e, "unit": "Gcell/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "traces_finite": ok_traces},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": dom_bytes,
                         "algorithmic_bytes_per_cell": dom_bytes / cells0,
                         "step_achieved": step_gbs, "step_frac": step_gbs / peak,
                         "bytes_per_cell_update": BYTES_PER_CELL[medium],
                         "energy_accumulator": {"bytes_per_cell": dom_acc, "step_bytes_per_cell": acc,
                                                "achieved_with_accumulator": achieved_acc,
                                                "frac_with_accumulator": achieved_acc / peak}},
            "kernel_ms_per_step": kt,
            "cpu_baseline": base,
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "shot_gradients": grad,
            "batched_forward": batched,
            "shot_gradients_batched_config_subset": c5,
            "accuracy": acc_line,
        }
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
