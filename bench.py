"""Benchmark of the B200 ADMM substep: simulated steps/s to ADMM residual 1e-4, on one or more GPUs.

Metric: substeps per second, each substep iterating ADMM until both relative residuals
(primal and dual, FP64 reductions) are <= 1e-4, tested after every chunk of 5 iterations,
capped at the reference's own admm_max_iter (30).  With the reference algorithm (Jacobi
global solve, Jacobi friction-cone contact, DCD every 5 iterations) contact-free frames
converge within the first chunk and contact frames run to the cap, exactly like the
reference's fixed-count step; the line reports the converged fraction and the mean
iteration count.  `--tol 0` measures the fixed-count step.

Workload (default): the tetrahedralised cube, 20^3 cells (9261 vertices, 40000
tets, 5 tets/cell, edge 0.5 m), dropped 1 m onto a ground quad, 30 ADMM
iterations per substep, dt = 1/100 s, frames 0..K-1 of the drop (K = 200 by
default: the whole 200-frame run, free fall, impact with thousands of contacts,
rebound).  Synthetic, seeded scene (seed 0: E = 1.88e5, nu = 0.4).

One "step" is one full substep (IADMMBackend::step): pre-integration, 30 ADMM
iterations with a DCD (LBVH build + traversal) every 5 iterations, contact
projection (10 Jacobi passes), 20 Jacobi sweeps of the global solve, dual
updates, post-process -- replayed as one CUDA graph.  The scene's working set
(~30 MB) fits in L2, so L2 is flushed (a 256 MiB write) between timed steps.

Multi-GPU: the substep of one coupled body does not shard (contacts and the
global solve couple every vertex every iteration), so --gpus N runs N
independent replicas, one per rank, with no collective in the data path
("scaling": "weak"); value = total steps of all ranks / max over ranks of the
device time.

`--impl reference` times the CPU restatement of the reference's GPU-backend
algorithm (the oracle, OpenMP on all host threads) on the same workload.
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
                           "E log-U[1e4,1e6], mu U(0.2,0.6) per body) dropped onto the ground, 30 ADMM iters/step, "
                           "dt=1/100; each rank simulates its own batch (seed = rank)"),
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


def make_scene(args, rank=0):
    """The configured scene with the solver options of the command line applied."""
    from parallel_admm_b200 import scene
    c = CONFIGS[args.config]
    kw = dict(c["kw"])
    if c.get("per_rank_seed"):
        from parallel_admm_b200 import replicas as R
        kw["seed"] = R.rank_seed(kw.get("seed", 0), rank)
    sc = getattr(scene, c["fn"])(**kw)
    sc.params.jacobi_mode = args.jacobi_mode
    sc.params.ell_lanes = args.ell_lanes
    sc.params.global_solver = args.global_solver
    sc.params.pcg_iter = args.pcg_iter
    sc.params.query_lanes = args.query_lanes
    return sc


def metric_name(tol, cap, solver=0, pcg_iter=0):
    how = {0: "plain Jacobi", 1: f"PCG diag(A) x{pcg_iter}", 2: f"PCG learned blocks x{pcg_iter}"}[solver]
    if tol > 0:
        return f"sim steps/s to ADMM residual {tol:g} ({how}, cap {cap} ADMM iterations = reference count)"
    return f"sim steps/s ({how}, fixed {cap} ADMM iterations = reference count)"


def pair_nnz(sc):
    """Off-diagonal non-zeros of A (vertex pairs coupled by a constraint)."""
    pairs = set()

    def add(ids):
        ids = [int(i) for i in ids]
        for a in ids:
            for b in ids:
                if a != b:
                    pairs.add((a, b))
    for t in sc.tet_inds:
        add(t)
    for t in sc.tri_inds:
        add(t)
    for c in range(len(sc.bend_w)):
        add(sc.bend_inds[sc.bend_offsets[c]:sc.bend_offsets[c + 1]])
    return len(pairs)


def algorithmic_bytes(sc, kernel):
    """Bytes one launch must move at minimum (each array touched once, FP32, gathers once per element)."""
    n, nd, m = sc.n_vert, sc.n_dyn, sc.n_rows
    if kernel == "local":
        # per row: Ue r+w, z r+w, y w (12 B each); per tet: inds 16 + Binv 36; per tri: 12 + 16;
        # bending: (ring+1)*(4 idx + 4 coef); pins: 4 + 12; x gathered once per vertex
        ring = int(sc.bend_offsets[-1]) if len(sc.bend_w) else 0
        return (60 * m + 52 * len(sc.tet_inds) + 28 * len(sc.tri_inds) + 8 * ring +
                16 * len(sc.pin_inds) + 12 * nd)
    if kernel == "jacobi":
        nnz = pair_nnz(sc)
        # diag 4 + b 12 + x_out 12 per row, (4 val + 4 col) per off-diagonal, x_in gathered once
        return 28 * nd + 8 * nnz + 12 * nd
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


def cpu_baseline(sc, h, frames, stride):
    """The oracle (FP32 restatement of the reference GPU-backend algorithm) on the host cores.

    Stratified sample of the workload: the GPU replays frames 0..frames-1; at every
    `stride`-th frame its full state (x, v, both duals) is copied into the oracle, which
    is timed for one substep.  Returns steps/s over the sampled substeps.
    """
    from oracle import oracle as O
    from parallel_admm_b200 import backend as B
    o = O.Oracle(h.holder, double=False)
    h.reset()
    secs = 0.0
    n = 0
    iters = 0
    for f in range(frames):
        if f % stride == 0:
            x, v = h.get_state()
            for buf, a in ((B.BUF_X0, x), (B.BUF_X, x), (B.BUF_V, v), (B.BUF_UE, h.read(B.BUF_UE)),
                           (B.BUF_UC, h.read(B.BUF_UC))):
                o.write(buf, a.astype(np.float64))
            t = time.perf_counter()
            iters += o.step(1)["iters"]
            secs += time.perf_counter() - t
            n += 1
        h.step(1, allow=(B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW))
    return n / secs, O.num_threads(), secs, n, iters / max(n, 1)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sc = make_scene(args)
    from oracle import oracle as O
    from parallel_admm_b200 import backend as B
    holder = B.DescHolder(sc, residual_tol=args.tol)
    o = O.Oracle(holder, double=False)
    o.step(min(args.warmup, 3))
    o.reset()
    k = min(args.steps, args.ref_steps)
    t = time.perf_counter()
    iters = 0
    for _ in range(k):
        iters += o.step(1)["iters"]
    dt = time.perf_counter() - t
    value = k / dt
    sample = (f"frames 0..{k - 1} of the workload ({k} of {args.steps} steps; CPU time bounded), "
              f"mean {iters / k:.1f} ADMM iterations per step")
    line = {
        "impl": "reference", "metric": metric_name(args.tol, sc.params.admm_max_iter, args.global_solver,
                              args.pcg_iter or max(1, sc.params.jacobi_iter // 2)),
        "value": value, "unit": "steps/s", "n_gpus": args.gpus, "steps": k, "warmup": min(args.warmup, 3),
        "ms_per_step": 1e3 * dt / k, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": {"workload": CONFIGS[args.config]["workload"]},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": O.num_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cube", choices=sorted(CONFIGS))
    ap.add_argument("--probe", default="jacobi", choices=["local", "jacobi", "rhs"])
    ap.add_argument("--cpu-stride", type=int, default=3,
                    help="CPU-baseline sample: one substep every N frames (3: 67 of the cube's 200, ~13 s on 16 cores)")
    ap.add_argument("--tol", type=float, default=1e-4, help="ADMM residual tolerance (0 = fixed iteration count)")
    ap.add_argument("--ell-lanes", type=int, default=0, choices=[0, 1, 2, 4, 8],
                    help="pin the lanes per row of both sliced-ELL matrices (0 = autotuned; pin it under a profiler, "
                         "whose serialised launches mislead the autotuner)")
    ap.add_argument("--jacobi-mode", type=int, default=0, choices=[0, 1, 2, 3],
                    help="global step: 0 autotuned, 1 one kernel per sweep, 2 persistent kernel, 3 two sweeps per launch")
    ap.add_argument("--global-solver", type=int, default=0, choices=[0, 1, 2],
                    help="global step: 0 Jacobi sweeps (the reference's), 1 PCG with diag(A), 2 PCG with blocks")
    ap.add_argument("--pcg-iter", type=int, default=0, help="PCG iterations per global step (0 = jacobi_iter / 2)")
    ap.add_argument("--query-lanes", type=int, default=0, choices=[0, 8, 16, 32],
                    help="lanes per grid DCD query (0 = chosen from the number of queries)")
    ap.add_argument("--ref-steps", type=int, default=200, help="cap on steps timed by --impl reference")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--start-frame", type=int, default=0,
                    help="advance this many substeps (untimed) before the timed region, e.g. to time contact frames")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="open a CUDA profiler range (cudaProfilerStart/Stop) around the first N timed steps, "
                         "for ncu --profile-from-start off")
    ap.add_argument("--profile", action="store_true", help="phase pass over all timed frames (default: the first 50)")
    ap.add_argument("--phase-steps", type=int, default=50, help="substeps of the phase-probe pass (roofline)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)

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
    h = B.Handle(sc, device=local, residual_tol=args.tol)
    for _ in range(args.warmup):
        h.step(1, allow=(B.ERR_CONTACT_OVERFLOW,))
    h.reset()

    for _ in range(args.start_frame):
        h.step(1, allow=(B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    dev_ms = []
    contacts = []
    iters = []
    conv = []
    launches = 0
    peak = 0
    status = 0

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
            st = h.step(1, allow=(B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW))
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
    clocks = clk.summary()
    total_ms = float(np.sum(dev_ms))
    max_total_ms = R.max_over_ranks(total_ms, f"cuda:{local}")
    ms_per_step = max_total_ms / args.steps
    value = R.job_throughput(args.steps, world, max_total_ms / 1e3)

    # end to end through the public C ABI: pinned host buffers in, one substep, host buffers out
    h.reset()
    x_in = torch.from_numpy(sc.verts.copy()).pin_memory().numpy()
    v_in = torch.zeros((sc.n_vert, 3), dtype=torch.float32).pin_memory().numpy()
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

    # Device time per phase inside the step graph (events at phase changes, so the launch gaps
    # inside a phase are included), over the same frames as the timed region (the first
    # --phase-steps of them); with a residual tolerance only the first chunk of each step is
    # covered.  The roofline below divides the probed kernel's bytes by its phase's time per launch.
    phases = None
    probe_ms, probe_n = 0.0, 0
    if rank == 0:
        nph = args.steps if args.profile else min(args.steps, args.phase_steps)
        h.reset()
        for _ in range(args.start_frame):
            h.step(1, allow=(B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW))
        h.set_probe("phases")
        h.phase_times()
        for _ in range(nph):
            h.step(1, allow=(B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW))
        raw = h.phase_times()
        phases = {k: {"ms_per_step": v["ms"] / nph, "launches_per_step": v["launches"] / nph} for k, v in raw.items()}
        phases["scope"] = (f"frames {args.start_frame}..{args.start_frame + nph - 1}, "
                           + ("first chunk of each step" if args.tol > 0 else "whole step"))
        # Isolated launches of the probed kernel class: an event pair around each of its first
        # launches in the step graph (this breaks their programmatic overlap, so it runs in a
        # pass of its own, never in the timed region).
        h.reset()
        for _ in range(args.start_frame):
            h.step(1, allow=(B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW))
        h.set_probe(args.probe)
        h.probe_time()
        for _ in range(nph):
            h.step(1, allow=(B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW))
        probe_ms, probe_n = h.probe_time()
        h.set_probe("none")

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    peak_gbs, peak_kind = load_peaks()
    alg = algorithmic_bytes(sc, args.probe)
    ph = phases.get(args.probe, {}) if phases else {}
    phase_ms = ph["ms_per_step"] / ph["launches_per_step"] if ph.get("launches_per_step") else 0.0
    achieved = alg / (phase_ms * 1e-3) / 1e9 if phase_ms > 0 else None
    traffic = None
    tp = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(args.config, {}).get(args.probe)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        v, cores, secs, n, it_mean = cpu_baseline(sc, h, args.steps, args.cpu_stride)
        cpu = {"value": v, "unit": "steps/s", "cores": cores, "kind": "port",
               "sample": f"{n} substeps, one every {args.cpu_stride} frames of frames 0..{args.steps - 1}, "
                         f"each from the GPU run's state; {secs:.1f} s of CPU time (oracle FP32, OpenMP), "
                         f"mean {it_mean:.1f} ADMM iterations per step"}
    tn, gm = h.tuning(), h.global_mode()
    tuned = {"jacobi_lanes": tn["jacobi_lanes"], "rhs_lanes": tn["rhs_lanes"], "global_mode": gm["mode"]}
    line = {
        "metric": metric_name(args.tol, sc.params.admm_max_iter, args.global_solver,
                              args.pcg_iter or max(1, sc.params.jacobi_iter // 2)),
        "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": CONFIGS[args.config]["workload"], "n_vert": sc.n_vert, "n_rows": sc.n_rows,
                   "parallelism": f"replicas x{world}", "l2": "flushed (256 MiB write) between timed steps",
                   "contacts_mean": float(np.mean(contacts)), "contacts_peak": int(peak),
                   # contacts projected per second of substep device time (rank 0's count x ranks)
                   "contacts_per_s": world * float(np.sum(contacts)) / (max_total_ms / 1e3),
                   "residual_tol": args.tol, "admm_iter_cap": sc.params.admm_max_iter,
                   "admm_iters_mean": float(np.mean(iters)),
                   "converged_fraction": float(np.mean(conv)) if args.tol > 0 else None,
                   "tuned": tuned},
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": args.probe, "achieved": achieved, "peak": peak_gbs,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": (achieved / peak_gbs) if achieved else None, "traffic": traffic,
                     "algorithmic_bytes_per_launch": alg, "mean_launch_ms": phase_ms,
                     "mean_launch_ms_how": "device time of the kernel's phase in the step graph / its launches",
                     "isolated_launch_ms": probe_ms, "isolated_launches": probe_n,
                     "isolated_how": "event pair around each of the first launches of the class (adds the "
                                     "event overhead, breaks the programmatic overlap)"},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "status": status,
    }
    if phases is not None:
        line["phases"] = phases
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
