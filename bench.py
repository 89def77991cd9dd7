"""Benchmark of the B200 ADMM substep: simulated steps/s to ADMM residual 1e-4, learned global
step against plain Jacobi, on one or more GPUs.

Metric: substeps per second, each substep iterating ADMM until both relative residuals
(primal and dual, FP64 reductions) are <= 1e-4, tested after every chunk of 5 iterations,
capped at the reference's admm_max_iter (30).  `value` is the learned global step
(global_solver 3: the trained network's per-vertex scaling and warm start, the trained
per-sweep schedule, judged per solve, plain Jacobi substep as the fallback); the plain
Jacobi path (the reference's algorithm) runs the same frames in the same process and sits
beside it in `config.plain_jacobi`, with iterations, converged fraction and fallback counts.
On frames with contact neither reaches 1e-4 within 30 iterations (the reference's contact
splitting plateaus near a 2e-2 primal residual), so both run to the cap there.

Workload (default, `--config batch`): 256 independent tet soft bodies (cubes and voxelised
ellipsoids, 500-20000 vertices log-uniform, 1.45 M vertices and 6.07 M tets in all, E
log-uniform in [1e4, 1e6], mu U(0.2, 0.6) per body), each released 6-20 mm above the
ground (contact thickness 12 mm), so ground and self contacts start in the first frames;
dt = 1/100, 30 ADMM iterations, DCD every 5.  The timed frames are start_frame ..
start_frame + steps - 1 of the run.  Synthetic, seeded scene (seed = rank).

One "step" is one full substep (IADMMBackend::step), replayed as one CUDA graph.  L2 is
flushed (a 256 MiB write) between timed steps.

Multi-GPU: independent bodies shard by whole batches with no collective in the data path:
--gpus N runs N batches, one per rank ("scaling": "weak"); value = total steps of all
ranks / max over ranks of the device time.

`--impl reference` times the CPU restatement of the reference's GPU-backend algorithm
(the oracle, OpenMP on all host threads, plain Jacobi) on a size-stratified sample of 16
of the 256 bodies over the same frames, scaled to the whole batch by its share of the
work (constraint rows + vertices).
"""
from __future__ import annotations

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

CONFIGS = {
    "cube": dict(fn="cube_on_ground", kw=dict(n=20, seed=0),
                 workload="tet cube 20^3 cells (9261 verts, 40000 tets), 1 m drop onto ground, "
                          "30 ADMM iters/step, DCD every 5, dt=1/100"),
    "cloth": dict(fn="cloth_on_box", kw=dict(nx=32, seed=0),
                  workload="cloth 32x32 (1024 verts, 1922 tris) over a unit box, 20 ADMM iters/step, dt=1/200"),
    "sheets": dict(fn="sheets_on_sphere", kw=dict(nx=512, layers=4, seed=0),
                   workload="4 x 512^2 cloth sheets on a sphere r=0.3, 40 ADMM iters/step, dt=1/300"),
    "batch": dict(fn="batch_bodies", kw=dict(n_bodies=256, seed=0), per_rank_seed=True,
                  workload="256 independent tet soft bodies (cubes and ellipsoids, 500-20000 verts log-uniform, "
                           "1.45 M verts, 6.07 M tets, E log-U[1e4,1e6], mu U(0.2,0.6) per body) released 6-20 mm "
                           "above the ground (contact from the first frames), self-contact, 30 ADMM iters/step, "
                           "DCD every 5, dt=1/100; each rank simulates its own batch (seed = rank)"),
    "batch_prof": dict(fn="batch_bodies", kw=dict(n_bodies=192, seed=0),
                       workload="192 bodies of the 256-body batch's distribution (about 1.1 M verts; the sweep's "
                                "algorithmic bytes exceed L2): profiling stand-in for the batch workload"),
    "sheets_small": dict(fn="sheets_on_sphere", kw=dict(nx=256, layers=2, seed=0),
                         workload="2 x 256^2 cloth sheets on a sphere r=0.3, 40 ADMM iters/step, dt=1/300 "
                                  "(profiling stand-in for the sheets workload)"),
}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


WEIGHTS_DIR = os.path.join(ROOT, "parallel_admm_b200", "weights")
# the trained learned step of each workload's family (train_learned.py --family ...)
WEIGHTS = {"batch": "learned_step.npz", "batch_prof": "learned_step.npz", "cube": "learned_step_cube.npz",
           "sheets": "learned_step_sheets.npz", "sheets_small": "learned_step_sheets.npz",
           "cloth": "learned_step_sheets.npz"}


def make_scene(args, rank=0, only=None):
    """The configured scene with the solver options of the command line applied."""
    from parallel_admm_b200 import scene
    c = CONFIGS[args.config]
    kw = dict(c["kw"])
    if c.get("per_rank_seed"):
        from parallel_admm_b200 import replicas as R
        kw["seed"] = R.rank_seed(kw.get("seed", 0), rank)
    if only is not None:
        kw["only"] = only
    sc = getattr(scene, c["fn"])(**kw)
    sc.params.jacobi_mode = args.jacobi_mode
    sc.params.ell_lanes = args.ell_lanes
    sc.params.pcg_iter = args.pcg_iter
    sc.params.query_lanes = args.query_lanes
    if args.semantics == "cpu":
        # the reference CPU backend's solver: damped system, exact global solve (the GPU arm:
        # PCG with --pcg-iter iterations), serial Gauss-Seidel contact, CPU contact predicates
        sc.params.backend_semantics = 1
        sc.params.contact_semantics = 1
    return sc


def metric_name(tol, cap, arm, semantics="gpu"):
    how = {"learned": "learned global step (Jacobi fallback)", "jacobi": "plain Jacobi",
           "pcg": "PCG diag(A)"}[arm]
    if semantics == "cpu":
        how = ("the CPU backend's solver (damped system, exact global solve, serial Gauss-Seidel contact)"
               if arm == "jacobi" else f"the CPU backend's solver with {how} as the global step")
    if tol > 0:
        return f"sim steps/s to ADMM residual {tol:g}: {how}, cap {cap} ADMM iterations = reference count"
    return f"sim steps/s: {how}, fixed {cap} ADMM iterations = reference count"


def pair_nnz(sc):
    """Off-diagonal non-zeros of A (ordered vertex pairs coupled by a constraint)."""
    keys = []
    n = np.int64(sc.n_vert)
    groups = [sc.tet_inds, sc.tri_inds]
    for t in groups:
        t = np.asarray(t, np.int64)
        if len(t) == 0:
            continue
        for a in range(t.shape[1]):
            for b in range(t.shape[1]):
                if a != b:
                    keys.append(t[:, a] * n + t[:, b])
    for c in range(len(sc.bend_w)):
        ids = np.asarray(sc.bend_inds[sc.bend_offsets[c]:sc.bend_offsets[c + 1]], np.int64)
        ii, jj = np.meshgrid(ids, ids)
        keep = ii != jj
        keys.append(ii[keep] * n + jj[keep])
    if not keys:
        return 0
    return int(len(np.unique(np.concatenate(keys))))


def algorithmic_bytes(sc, kernel, nnz=None):
    """Bytes one launch must move at minimum (each array touched once, FP32, gathers once per element)."""
    n, nd, m = sc.n_vert, sc.n_dyn, sc.n_rows
    if kernel == "local":
        # per row: Ue r+w, z r+w, y w (12 B each); per tet: inds 16 + Binv 36; per tri: 12 + 16;
        # bending: (ring+1)*(4 idx + 4 coef); pins: 4 + 12; x gathered once per vertex
        ring = int(sc.bend_offsets[-1]) if len(sc.bend_w) else 0
        return (60 * m + 52 * len(sc.tet_inds) + 28 * len(sc.tri_inds) + 8 * ring +
                16 * len(sc.pin_inds) + 12 * nd)
    if kernel in ("jacobi", "learned"):
        nnz = pair_nnz(sc) if nnz is None else nnz
        # Jacobi: diag 4 + b 12 + x_out 12 per row, (4 val + 4 col) per off-diagonal, x_in gathered once;
        # learned sweep: + m 4 and the previous iterate 12 per row
        return (28 + 12 + (16 if kernel == "learned" else 0)) * nd + 8 * nnz
    if kernel == "rhs":
        nnz_d = 4 * 3 * len(sc.tet_inds) + 3 * 2 * len(sc.tri_inds) + int(
            sc.bend_offsets[-1] if len(sc.bend_w) else 0) + len(sc.pin_inds)
        return 8 * nnz_d + 12 * m + 12 * nd * 5
    raise ValueError(kernel)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.f.flush()
        rows = []
        with open(self.f.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def stratified_bodies(sc_meta, k=16):
    """k bodies of the batch spread evenly over its size distribution (by vertex count)."""
    counts = np.array([c[0] for c in sc_meta["all_body_counts"]])
    order = np.argsort(counts, kind="stable")
    step = len(order) / k
    return sorted(int(order[int(step * j + step / 2)]) for j in range(k))


def work_of(counts):
    """Per-substep CPU work proxy of bodies: constraint rows (3 per tet) + vertices."""
    return float(sum(3 * t + v for v, t in counts))


def oracle_sample_rate(args, rank, frames, budget_s):
    """The oracle (FP32 restatement of the reference GPU-backend algorithm, plain Jacobi, all
    host threads) over frames 0.. of the workload, stopping once budget_s of CPU time is spent;
    for the batch a size-stratified 16-body sample scaled to the whole batch by its work share.
    Returns (steps/s, threads, description, ADMM iteration cap)."""
    from oracle import oracle as O
    from parallel_admm_b200 import backend as B
    frac = 1.0
    what = "the whole workload"
    if args.config == "batch":
        from parallel_admm_b200 import scene
        c = CONFIGS["batch"]["kw"]
        seed = c["seed"] + rank
        meta = scene.batch_bodies(c["n_bodies"], seed, only=[]).meta
        sel = stratified_bodies(meta)
        sc = make_scene(args, rank, only=sel)
        allc = meta["all_body_counts"]
        frac = work_of([allc[b] for b in sel]) / work_of(allc)
        what = (f"bodies {sel} (16 of {len(allc)}, size-stratified: {sc.n_dyn} verts, {len(sc.tet_inds)} tets), "
                f"time scaled by their work share {frac:.4f} (constraint rows + vertices)")
    else:
        sc = make_scene(args, rank)
    holder = B.DescHolder(sc, residual_tol=args.tol, global_solver=0)
    o = O.Oracle(holder, double=False)
    if args.semantics == "cpu":
        what += "; the CPU backend's semantics (damped system solved exactly by an FP64 Cholesky, serial Gauss-Seidel contact)"
    secs, k, iters = 0.0, 0, 0
    for _ in range(frames):
        t = time.perf_counter()
        iters += o.step(1)["iters"]
        secs += time.perf_counter() - t
        k += 1
        if secs >= budget_s:
            break
    rate = k / (secs / frac)
    desc = (f"{what}; frames 0..{k - 1} ({secs:.1f} s of CPU time), mean {iters / max(k, 1):.1f} ADMM iterations "
            f"per step, oracle FP32, OpenMP")
    return rate, O.num_threads(), desc, sc.params.admm_max_iter


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    frames = args.start_frame + min(args.steps, args.ref_steps)
    rate, cores, desc, cap = oracle_sample_rate(args, 0, frames, budget_s=args.ref_budget)
    line = {
        "impl": "reference", "metric": metric_name(args.tol, cap, "jacobi", args.semantics),
        "value": rate, "unit": "steps/s", "n_gpus": args.gpus, "steps": min(args.steps, args.ref_steps),
        "warmup": 0, "ms_per_step": 1e3 / rate, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": CONFIGS[args.config]["workload"]},
        "cpu_baseline": {"value": rate, "unit": "steps/s", "cores": cores, "kind": "port", "sample": desc},
        "e2e": {"value": rate, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def learned_model(args, h, sc):
    """The trained learned global step applied to handle h (global_solver 3); without the
    weights file, the untrained model (zero head = Jacobi scaling, Chebyshev schedule)."""
    from parallel_admm_b200 import gnn
    sysm = gnn.system(h)
    x, ef = gnn.scene_features(sc, sysm)
    if args.weights and os.path.exists(args.weights):
        model = gnn.LearnedGlobalStep.load(args.weights)
        source = os.path.relpath(args.weights, ROOT)
    else:
        model = gnn.LearnedGlobalStep(K=args.learned_sweeps)
        model.init_chebyshev(gnn.jacobi_spectrum_top(sysm))
        source = "untrained (Chebyshev schedule, Jacobi scaling)"
    model.apply(h, sysm, x, ef)
    info = {"weights": source, "sweeps": int(model.K)}
    model.net.close()
    return info


def run_arm(args, B, R, sc, local, world, arm, flush, nnz):
    """Warm-up, then the timed frames of one arm; returns its handle and numbers."""
    import torch
    import torch.distributed as dist
    gs = {"learned": 3, "jacobi": 0, "pcg": 1}[arm]
    h = B.Handle(sc, device=local, residual_tol=args.tol, global_solver=gs)
    info = learned_model(args, h, sc) if arm == "learned" else {}
    allow = (B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW)
    for _ in range(args.warmup):
        h.step(1, allow=allow)
    h.reset()
    for _ in range(args.start_frame):
        h.step(1, allow=allow)
    st0 = h.learned_stats() if arm == "learned" else None
    dev_ms, contacts, iters, conv = [], [], [], []
    launches, peak, status = 0, 0, 0

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    with ClockSampler(local) as clk:
        barrier()
        for k in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            if args.profile_steps and k == 0:
                torch.cuda.cudart().cudaProfilerStart()
            st = h.step(1, allow=allow)
            if args.profile_steps and k + 1 == args.profile_steps:
                torch.cuda.cudart().cudaProfilerStop()
            dev_ms.append(h.last_step_device_ms())
            contacts.append(st["n_contacts"])
            iters.append(st["iters"])
            launches += h.kernels_per_step()
            conv.append(st["primal"] <= args.tol and st["dual"] <= args.tol)
            peak = max(peak, st["peak"])
            status = status or st["status"]
        barrier()
    total_ms = float(np.sum(dev_ms))
    max_total_ms = R.max_over_ranks(total_ms, f"cuda:{local}")
    out = {"h": h, "value": R.job_throughput(args.steps, world, max_total_ms / 1e3),
           "ms_per_step": max_total_ms / args.steps, "max_total_ms": max_total_ms, "clocks": clk.summary(),
           "contacts": contacts, "iters": iters, "conv": conv, "peak": peak, "status": status,
           "launches": launches, "info": info}
    if arm == "learned":
        st1 = h.learned_stats()
        d = {k: st1[k] - st0[k] for k in st1}
        out["learned"] = d
        # every failed learned solve ran the plain solve in its IF node: count those kernels
        out["launches"] += d["fallbacks"] * h.kernels_fallback()
    return out


def arm_summary(args, r, sc, world):
    return {"steps_per_s": r["value"], "ms_per_step": r["ms_per_step"],
            "admm_iters_mean": float(np.mean(r["iters"])),
            "converged_fraction": float(np.mean(r["conv"])) if args.tol > 0 else None,
            "contacts_mean": float(np.mean(r["contacts"])), "contacts_peak": int(r["peak"]),
            "contacts_per_s": world * float(np.sum(r["contacts"])) / (r["max_total_ms"] / 1e3),
            "kernels_launched": r["launches"]}


def profile_only(args):
    """The substeps an ncu capture looks at (ncu --profile-from-start off): the arm's handle as
    the bench builds it, warm-up and start-frame substeps outside the range, then
    --profile-steps substeps inside it, launched eagerly (the same kernels as the step graph:
    ncu does not profile the kernel nodes of a graph that holds conditional nodes, which the
    learned step's fallback and the residual test use)."""
    import torch
    from parallel_admm_b200 import backend as B
    torch.cuda.set_device(0)
    sc = make_scene(args)
    gs = {"learned": 3, "jacobi": 0, "pcg": 1}[args.solver]
    h = B.Handle(sc, residual_tol=args.tol, global_solver=gs)
    info = learned_model(args, h, sc) if args.solver == "learned" else {}
    allow = (B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW)
    for _ in range(args.warmup + args.start_frame):
        h.step(1, allow=allow)
    h.set_profiling(True)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    for _ in range(max(1, args.profile_steps)):
        st = h.step(1, allow=allow)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    print("profiled", args.config, args.solver, info, st, "kernels per substep", h.kernels_per_step(), flush=True)
    h.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="batch", choices=sorted(CONFIGS))
    ap.add_argument("--solver", default="learned", choices=["learned", "jacobi", "pcg"],
                    help="the arm reported as value; with learned, plain Jacobi runs beside it")
    ap.add_argument("--weights", default=None,
                    help="trained learned-step weights (npz; default: the model of the workload's family)")
    ap.add_argument("--learned-sweeps", type=int, default=10, help="sweeps of the untrained learned step")
    ap.add_argument("--probe", default="jacobi", choices=["local", "jacobi", "rhs"])
    ap.add_argument("--tol", type=float, default=1e-4, help="ADMM residual tolerance (0 = fixed iteration count)")
    ap.add_argument("--ell-lanes", type=int, default=0, choices=[0, 1, 2, 4, 8],
                    help="pin the lanes per row of both sliced-ELL matrices (0 = autotuned; pin it under a profiler, "
                         "whose serialised launches mislead the autotuner)")
    ap.add_argument("--jacobi-mode", type=int, default=0, choices=[0, 1, 2, 3],
                    help="global step: 0 autotuned, 1 one kernel per sweep, 2 persistent kernel, 3 two sweeps per launch")
    ap.add_argument("--pcg-iter", type=int, default=0, help="PCG iterations per global step (0 = jacobi_iter / 2)")
    ap.add_argument("--query-lanes", type=int, default=0, choices=[0, 8, 16, 32],
                    help="lanes per grid DCD query (0 = chosen from the number of queries)")
    ap.add_argument("--ref-steps", type=int, default=20, help="cap on steps timed by --impl reference")
    ap.add_argument("--ref-budget", type=float, default=60.0, help="CPU seconds the reference arm may spend")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="CPU seconds of the cpu_baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--start-frame", type=int, default=0,
                    help="advance this many substeps (untimed) before the timed region")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="open a CUDA profiler range (cudaProfilerStart/Stop) around the first N timed steps, "
                         "for ncu --profile-from-start off")
    ap.add_argument("--phase-steps", type=int, default=10, help="substeps of the phase-probe pass (roofline)")
    ap.add_argument("--semantics", default="gpu", choices=["gpu", "cpu"],
                    help="the reference backend whose solver runs: the GPU backend's (default) or the CPU "
                         "backend's (damping, exact global solve, serial Gauss-Seidel contact; with "
                         "--solver pcg --pcg-iter N on the GPU)")
    ap.add_argument("--profile-only", action="store_true",
                    help="profiling run: the --solver arm's warm-up and --start-frame substeps, then --profile-steps "
                         "substeps inside a CUDA profiler range; no timing, no JSON line")
    args = ap.parse_args()
    if args.weights is None:
        args.weights = os.path.join(WEIGHTS_DIR, WEIGHTS[args.config])
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_only:
        return profile_only(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    from parallel_admm_b200 import backend as B
    from parallel_admm_b200 import replicas as R

    sc = make_scene(args, rank)
    nnz = pair_nnz(sc)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    arms = [args.solver] + (["jacobi"] if args.solver == "learned" else [])
    res = {}
    for arm in arms:
        res[arm] = run_arm(args, B, R, sc, local, world, arm, flush, nnz)
        if arm != args.solver:
            res[arm]["h"].close()
            res[arm]["h"] = None
    main_r = res[args.solver]
    h = main_r["h"]

    # end to end through the public C ABI: pinned host buffers in, one substep, host buffers out,
    # over the same frames as the timed region
    allow = (B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW)
    h.reset()
    for _ in range(args.start_frame):
        h.step(1, allow=allow)
    x0, v0 = h.get_state()
    x_in = torch.from_numpy(x0.copy()).pin_memory().numpy()
    v_in = torch.from_numpy(v0.copy()).pin_memory().numpy()
    x_out = torch.zeros((sc.n_vert, 3), dtype=torch.float32).pin_memory().numpy()
    v_out = torch.zeros((sc.n_vert, 3), dtype=torch.float32).pin_memory().numpy()
    e2e_s = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h.step_host(x_in, v_in, x_out, v_out)
        e2e_s += time.perf_counter() - t0
        x_in[:] = x_out
        v_in[:] = v_out
    e2e_value = R.job_throughput(args.steps, world, R.max_over_ranks(e2e_s, f"cuda:{local}"))
    bytes_io = 2 * sc.n_vert * 3 * 4

    # Device time per phase inside the step graph (events at phase changes), over the first
    # --phase-steps timed frames, on a handle with the same solver and tuning that runs all
    # admm_max_iter iterations (no conditional node, whose body holds no events; the
    # contact frames run to the cap anyway); the roofline divides the probed kernel's bytes by
    # its phase's time per launch.  Then an event pair around each of the first launches of the
    # probed class (a pass of its own: the events break the overlap).
    phases = None
    probe_ms, probe_n = 0.0, 0
    if rank == 0:
        nph = min(args.steps, args.phase_steps)
        tn0 = h.tuning()
        sc_ph = sc
        sc_ph.params.ell_lanes = tn0["jacobi_lanes"] if tn0["jacobi_lanes"] == tn0["rhs_lanes"] else sc.params.ell_lanes
        hp = B.Handle(sc_ph, device=local, residual_tol=0.0,
                      global_solver={"learned": 3, "jacobi": 0, "pcg": 1}[args.solver])
        if args.solver == "learned":
            learned_model(args, hp, sc_ph)
        for _ in range(args.start_frame):
            hp.step(1, allow=allow)
        hp.set_probe("phases")
        hp.phase_times()
        ls0 = hp.learned_stats() if args.solver == "learned" else None
        for _ in range(nph):
            hp.step(1, allow=allow)
        raw = hp.phase_times()
        phases = {k: {"ms_per_step": v["ms"] / nph, "launches_per_step": v["launches"] / nph} for k, v in raw.items()}
        if ls0 is not None:
            # the plain solves that replaced failed learned ones run inside the global step's phase
            # (the IF node's body holds no event nodes): count their kernels with the phase's
            replaced = hp.learned_stats()["fallbacks"] - ls0["fallbacks"]
            phases["jacobi"]["replaced_solves_per_step"] = replaced / nph
            phases["jacobi"]["launches_per_step"] += replaced * hp.kernels_fallback() / nph
        phases["scope"] = (f"frames {args.start_frame}..{args.start_frame + nph - 1}, whole step, "
                           f"{sc.params.admm_max_iter} ADMM iterations (no residual test)")
        hp.close()
        h.reset()
        for _ in range(args.start_frame):
            h.step(1, allow=allow)
        h.set_probe(args.probe)
        h.probe_time()
        for _ in range(nph):
            h.step(1, allow=allow)
        probe_ms, probe_n = h.probe_time()
        h.set_probe("none")

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    peak_gbs, peak_kind = load_peaks()
    pk = "learned" if (args.probe == "jacobi" and args.solver == "learned") else args.probe
    alg = algorithmic_bytes(sc, pk, nnz)
    ph = phases.get(args.probe, {}) if phases else {}
    if args.probe == "jacobi" and args.solver == "learned":
        ph = phases.get("jacobi", {})
    phase_ms = ph["ms_per_step"] / ph["launches_per_step"] if ph.get("launches_per_step") else 0.0
    achieved = alg / (phase_ms * 1e-3) / 1e9 if phase_ms > 0 else None
    traffic = None
    tp = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(args.config, {}).get(pk)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        rate, cores, desc, _ = oracle_sample_rate(args, rank, args.start_frame + args.steps, args.cpu_budget)
        cpu = {"value": rate, "unit": "steps/s", "cores": cores, "kind": "port", "sample": desc}
    tn, gm = h.tuning(), h.global_mode()
    tuned = {"jacobi_lanes": tn["jacobi_lanes"], "rhs_lanes": tn["rhs_lanes"], "global_mode": gm["mode"]}
    cfg = {"workload": CONFIGS[args.config]["workload"], "frames": f"{args.start_frame}..{args.start_frame + args.steps - 1}",
           "n_vert": sc.n_vert, "n_rows": sc.n_rows, "parallelism": f"replicas x{world}",
           "l2": "flushed (256 MiB write) between timed steps", "residual_tol": args.tol,
           "admm_iter_cap": sc.params.admm_max_iter, "solver": args.solver, "tuned": tuned}
    cfg.update(arm_summary(args, main_r, sc, world))
    if args.solver == "learned":
        cfg["learned"] = dict(main_r["info"], **main_r["learned"])
        pj = arm_summary(args, res["jacobi"], sc, world)
        cfg["plain_jacobi"] = pj
        cfg["learned_over_plain"] = main_r["value"] / pj["steps_per_s"] if pj["steps_per_s"] else None
    line = {
        "metric": metric_name(args.tol, sc.params.admm_max_iter, args.solver, args.semantics),
        "value": main_r["value"], "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": main_r["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": cfg,
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io},
        "gpu_launches": main_r["launches"] + (res["jacobi"]["launches"] if args.solver == "learned" else 0),
        "roofline": {"bound": "hbm", "kernel": {"learned": "k_lsweep (learned sweep)"}.get(pk, args.probe),
                     "achieved": achieved, "peak": peak_gbs,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": (achieved / peak_gbs) if achieved else None, "traffic": traffic,
                     "algorithmic_bytes_per_launch": alg, "mean_launch_ms": phase_ms,
                     "mean_launch_ms_how": "device time of the kernel's phase in the step graph / the kernels it ran "
                                           "(with the learned step: its sweeps, judge and decision, and the plain "
                                           "solves that replaced failed ones)",
                     "isolated_launch_ms": probe_ms, "isolated_launches": probe_n,
                     "isolated_how": "event pair around each of the first launches of the class (adds the "
                                     "event overhead, breaks the programmatic overlap)"},
        "cpu_baseline": cpu,
        "clocks": main_r["clocks"],
        "status": main_r["status"],
    }
    if phases is not None:
        line["phases"] = phases
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
