"""Benchmark of the ASOHF particle hot path on B200.

One step = one pass of the hot path over one synthetic snapshot: species
sort, kernel deposit (base grid + AMR patches) and renormalisation, x-slab
sort, then per level PRUNE_POOR_HALOES / HALOFIND_PARTICLES and per
substructure level SUBSTRUCTURE_PARTICLES, ending with the catalogue and the
bound-particle ID lists.  The workload is the 512^3-particle snapshot
(134M particles, 250 Mpc/h, 512^3 base grid, 6 AMR levels, ~2e5 haloes with
subhaloes); inputs (4.3 GB of particles) are far larger than L2.

  value  particles/s with the particles already in HBM (device timing);
  e2e    particles/s through the same public API from pinned host arrays,
         host->device copy of the particles and device->host copy of the
         catalogue and IDs inside the timed region.
Before the timed steps the size-tier thresholds of the per-halo kernels are
tuned on the workload itself (asohf_b200/autotune.py; --no-tune keeps the
defaults); the line names the setting used (launch_shape).
Multi-GPU: the path does not exchange data, so every rank runs a replica
on its own snapshot (weak scaling).

--impl reference times the CPU restatement of the reference routines (the
reference is Fortran and no Fortran compiler exists here) on a bounded
sample of the same workload (the 512^3 recipe at 1/64 of the volume: 128^3
particles), then once on the recipe at 1/8 of the volume (256^3 particles).
From the two measured points each stage's cost is fitted as a power of the
particle count and extrapolated to 512^3; the extrapolation is labelled as
such.  The CPU's particles/s falls as the snapshot grows (the patch deposit
scans every particle once per patch, the halo queries scan x-slabs that
span the box), so the measured 256^3 rate bounds the 512^3 rate from above.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CPU_SAMPLE = "cfg4s"
CPU_TREND = "cfg4m"   # the second point of the CPU scaling trend
# algorithmic bytes of one (particle, pass) of the per-halo kernels: the
# particle's position 12, velocity 12, mass 4 and ID 8 read, its distance and
# flag 8 written
BYTES_PER_ELEMENT_PASS = 44
# DRAM bytes (read + write) per element-pass of k_halo_main: 3.60 GB over
# 136.4M element-passes in one ncu capture of the 256^3 workload's 14 launches
# (`--config cfg2 --steps 1 --warmup 0 --no-cpu --no-layer --no-e2e --no-grid`)
DRAM_BYTES_PER_ELEMENT_PASS = 26.4


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def clock_sampler(device):
    f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                              "-lms", "200", "-i", str(device)], stdout=f, stderr=subprocess.DEVNULL)
    except Exception:
        p = None
    return p, f.name


def clock_summary(proc, path):
    if proc is None:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    proc.terminate()
    try:
        proc.wait(timeout=5)
    except Exception:
        proc.kill()
    sm, smax, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    with open(path) as f:
        for line in f:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
    os.unlink(path)
    return {"sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": float(max(smax)) if smax else None,
            "reasons": sorted(reasons), "samples": len(sm)}


def cpu_oracle_run(name, steps, warmup, nthreads):
    """The oracle pipeline (CPU restatement of the reference routines):
    particles, seconds per step and seconds per stage (mean over steps)."""
    from asohf_b200 import driver, synth
    from oracle import oracle as O
    snap = synth.generate(name)
    plan = driver.prepare(snap)
    b = O.OracleBackend(nthreads=nthreads)
    for _ in range(warmup):
        driver.execute(plan, b, download=False)
    stages = {}
    t0 = time.perf_counter()
    for _ in range(steps):
        r = driver.execute(plan, b, download=False)
        for k, v in r.stage_s.items():
            stages[k] = stages.get(k, 0.0) + v / steps
    dt = (time.perf_counter() - t0) / steps
    return snap.cfg.n, dt, stages


def cpu_trend(small, nthreads, target_n):
    """Measured CPU points at 128^3 (`small` = (n, dt, stages)) and 256^3
    particles of the 512^3 recipe, and each stage fitted as t = a n^k through
    the two points and extrapolated to target_n particles."""
    from asohf_b200 import synth
    n1, dt1, st1 = small
    n2, dt2, st2 = cpu_oracle_run(CPU_TREND, 1, 0, nthreads)
    pts = []
    for name, n, dt, st in ((CPU_SAMPLE, n1, dt1, st1), (CPU_TREND, n2, dt2, st2)):
        c = synth.CONFIGS[name]
        pts.append({"workload": f"{name}: {c.npart_side}^3 particles, {c.box_mpc_h} Mpc/h, NX={c.nx}",
                    "particles": n, "s_per_step": round(dt, 3), "particles_per_s": n / dt,
                    "stage_s": {k: round(v, 4) for k, v in st.items()}})
    ratio = n2 / n1
    ext, exps = {}, {}
    for k in st2:
        a, b = max(st1.get(k, 0.0), 1e-9), max(st2[k], 1e-9)
        kexp = math.log(b / a) / math.log(ratio)
        exps[k] = round(kexp, 3)
        ext[k] = b * (target_n / n2) ** kexp
    t_ext = sum(ext.values())
    return {"points": pts,
            "extrapolated": {"particles": target_n, "s_per_step": round(t_ext, 1),
                             "particles_per_s": target_n / t_ext, "stage_exponents": exps,
                             "stage_s": {k: round(v, 1) for k, v in ext.items()},
                             "note": "extrapolated, not measured: each stage fitted as a power of the particle "
                                     "count through the two measured points"}}


def layer_bench(iters=10, warmup=3):
    """Deposit+Poisson forward vs forward+adjoint: 8 jittered copies of the
    64^3-particle set (positions + N(0, 0.01 cell)) onto a periodic 256^3 grid."""
    import torch
    from asohf_b200 import synth
    from asohf_b200.autograd import DepositPoissonLayer
    s = synth.generate("cfg1")
    L = s.cfg.lado0
    nx = 256
    layer = DepositPoissonLayer(nx, L)
    B = 8
    rng = np.random.default_rng(3)
    cell = L / nx
    base = np.stack([s.x, s.y, s.z])
    pos = base[:, None, :] + rng.normal(0.0, 0.01 * cell, (3, B, base.shape[1]))
    pos = (np.mod(pos + L / 2, L) - L / 2).astype(np.float32)
    dev = torch.device("cuda", torch.cuda.current_device())
    x, y, z = (torch.tensor(pos[i], device=dev) for i in range(3))
    m = torch.tensor(np.broadcast_to(s.m, (B, s.m.shape[0])).copy(), device=dev)
    w = torch.randn((B, nx, nx, nx), generator=torch.Generator(device=dev).manual_seed(7), device=dev)
    st = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(iters):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / iters

    fwd = timed(lambda: layer.forward(x, y, z, m))
    both = timed(lambda: (layer.forward(x, y, z, m), layer.adjoint(x, y, z, m, w, need_m=False)))
    G = B * nx ** 3
    N = B * base.shape[1]
    # algorithmic bytes: deposit (read 16 B/particle, write rho), FFT pair
    # (read rho, write/read half spectrum, write phi); adjoint: FFT pair on w,
    # read 16 B/particle, write 12 B/particle of gradient
    fwd_bytes = 16 * N + 4 * G + 16 * G
    adj_bytes = 16 * G + 4 * G + 16 * N + 12 * N
    hbm, src = peaks()
    gbs = (fwd_bytes + adj_bytes) / (both * 1e-3) / 1e9
    return {"config": "8 x 262144 particles (64^3 set, jittered N(0,0.01 cell)) -> periodic 256^3, FFT Poisson",
            "fwd_ms": round(fwd, 4), "fwd_adj_ms": round(both, 4), "ratio": round(both / fwd, 4),
            "fwd_adj_GBps": round(gbs, 1), "hbm_frac": round(gbs / hbm, 4), "peak_source": src}


def grid_finder_bench(b, plan, iters=3):
    """HALOFIND_GRID at the base level on the device, on the renormalised
    base grid the benchmark step left on the device (512^3 cells), with the
    snapshot's cosmology; device time per call (CUDA events)."""
    import torch
    from asohf_b200 import abi
    cfg, cos = plan.snap.cfg, plan.cos
    u1 = b._u1
    args = (float(cos["contrastec"]), float(cos["rote"]), float(cos["rete"]), float(cos["rodo"]),
            float(cos["re0"]), float(cfg.lado0) / 4, 0.2)
    cat = abi.Catalogue(max(plan.capacity, 1 << 20))
    st = torch.cuda.current_stream()
    b.sync_outputs()
    n = b.a.halofind_grid_base(cfg.nx, float(plan.dx), u1, plan.radx, *args, cat)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(iters):
        n = b.a.halofind_grid_base(cfg.nx, float(plan.dx), u1, plan.radx, *args, cat)
    e1.record(st)
    torch.cuda.synchronize()
    return {"grid": f"{cfg.nx}^3 cells (the step's renormalised U1)", "haloes": int(n),
            "ms": round(e0.elapsed_time(e1) / iters, 3),
            "note": "HALOFIND_GRID base level (haloes_grids.f:287-582) and OVERLAPPING, catalogue to the host"}


def replica_config(cfg, rank):
    """The snapshot recipe of one replica: the same sizes, seed + rank (the
    ranks share nothing, so each runs the hot path on its own snapshot)."""
    from asohf_b200 import synth
    return synth.SnapshotConfig(**{**cfg.__dict__, "seed": cfg.seed + rank})


def max_over_ranks(ms, world, dist, device):
    """The slowest rank's step time (all ranks take this collective in the
    same order); whole-job throughput is world * particles / this time."""
    import torch
    t = torch.tensor([float(ms)], device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg4")
    ap.add_argument("--no-subs", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-cpu-trend", action="store_true",
                    help="skip the CPU run of the 256^3 sample and the extrapolation to the full size")
    ap.add_argument("--no-layer", action="store_true", help="skip the deposit+Poisson layer leg")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end leg (profiling runs: only the device-timed steps)")
    ap.add_argument("--no-grid", action="store_true", help="skip the grid halo finder leg")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default size-tier thresholds (no launch-shape tuning before the timed steps)")
    ap.add_argument("--layer-only", action="store_true",
                    help="only the deposit+Poisson layer leg (profiling runs of its kernels)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    metric = "particles/s (512^3 snapshot, hot path end to end)"

    if args.impl == "reference":
        if rank != 0:
            return
        from asohf_b200 import synth
        nth = os.cpu_count() or 1
        small = cpu_oracle_run(CPU_SAMPLE, args.steps, args.warmup, nth)
        n, dt, _ = small
        v = n / dt
        cb = {"value": v, "unit": "particles/s", "cores": nth, "kind": "port",
              "sample": "full hot path on the 128^3 sample of the 512^3 recipe (C restatement of the Fortran), "
                        f"{args.steps} steps"}
        if not args.no_cpu_trend:
            cb["trend"] = cpu_trend(small, nth, synth.CONFIGS[args.config].n)
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": v, "unit": "particles/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": f"{CPU_SAMPLE}: 128^3 particles, 62.5 Mpc/h, the 512^3 recipe at 1/64 volume",
                       "parallelism": "cpu"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    import torch
    import torch.distributed as dist
    from types import SimpleNamespace
    from asohf_b200 import api, autotune, driver, synth

    torch.cuda.set_device(local)
    # the hot path on a high-priority stream: the library's size-tier streams
    # take its priority, and the deferred AMR-patch deposit (least priority)
    # runs in the gaps the halo finder leaves
    torch.cuda.set_stream(torch.cuda.Stream(priority=-1))
    if args.layer_only:
        if rank == 0:
            print(json.dumps({"deposit_poisson": layer_bench()}))
        return
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    cfg = replica_config(synth.CONFIGS[args.config], rank)
    snap = synth.generate_fast(cfg, device=f"cuda:{local}", keep_on_device=True)
    plan = driver.prepare(snap)
    with_subs = not args.no_subs
    b = api.DeviceBackend(local)
    b.a.set_stream(torch.cuda.current_stream().cuda_stream)
    # the size-tier thresholds: tuned on this workload before the timed steps
    # (coordinate descent, 2 timed runs per setting, the chosen setting's
    # catalogue checked against the defaults'), or the defaults
    launch = {"setting": dict(autotune.DEFAULTS), "tuned": False}
    if not args.no_tune:
        best, ms_best, trials = autotune.tune_plan(plan, b, with_subs=with_subs, reps=2, rounds=1)
        launch = {"setting": best, "tuned": True, "settings_timed": len(trials),
                  "ms_chosen": round(ms_best, 2), "ms_defaults": round(trials[0][1], 2)}

    def step():
        return driver.execute(plan, b, with_subs=with_subs, download=False)

    for _ in range(args.warmup):
        r = step()
    st = torch.cuda.current_stream()
    clk, clk_path = clock_sampler(local)
    b.a.set_profiling(True)
    b.a.work_counters(reset=True)
    l0 = b.a.launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        r = step()
    e1.record(st)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    clocks = clock_summary(clk, clk_path)
    launches = (b.a.launch_count() - l0) // args.steps
    free_b, total_b = torch.cuda.mem_get_info(local)  # the library keeps its stores and arenas
    kstats = b.a.kernel_stats()
    work = b.a.work_counters()
    b.a.set_profiling(False)
    ms_max = max_over_ranks(ms, world, dist, "cuda")
    n = cfg.n
    value = world * n / (ms_max * 1e-3)

    e2e = None
    if not args.no_e2e:
        # e2e: pinned host particles in, catalogue and IDs out, through the API
        host = [a.cpu().pin_memory() for a in (snap.x, snap.y, snap.z, snap.vx, snap.vy, snap.vz, snap.m, snap.id)]
        parts_h = SimpleNamespace(x=host[0].numpy(), y=host[1].numpy(), z=host[2].numpy(), vx=host[3].numpy(),
                                  vy=host[4].numpy(), vz=host[5].numpy(), m=host[6].numpy(), id=host[7].numpy(), n=n)
        be = api.GpuBackend(local)
        be.a.set_stream(torch.cuda.current_stream().cuda_stream)
        autotune.apply(be.a, launch["setting"])

        def step_e2e():
            return driver.execute(plan, be, with_subs=with_subs, particles=parts_h, download=False)

        re = step_e2e()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(st)
        # snapshots back to back: each step's upload takes the particles
        # prefetched during the step before (the first step's copy is not
        # overlapped); every step still copies its particles from the host
        be.prefetch(parts_h)
        for k in range(args.steps):
            be.prefetch_next = parts_h if k + 1 < args.steps else None
            re = step_e2e()
        be.prefetch_next = None
        e1.record(st)
        torch.cuda.synchronize()
        ms_e2e = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3) / args.steps
        ms_e2e = max_over_ranks(ms_e2e, world, dist, "cuda")
        ncat = re.cat.nclus
        cat_bytes = ncat * 4 * (45 + 2 * 20 + 3 + 3 + 6 + 2)
        h2d = n * 32 + cat_bytes  # particles; the catalogue windows go both ways
        grid_bytes = 4 * (cfg.nx ** 3 + plan.mesh.total * 32 ** 3)  # U1 and U11 after RENORM_DENSITY
        d2h = int(re.pph.shape[0]) * 4 + cat_bytes + grid_bytes
        e2e = {"value": world * n / (ms_e2e * 1e-3), "unit": "particles/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e}

    # roofline of the dominant kernel (kernel names only: "host:" entries are
    # host phases, "idle:" entries gaps of the stream, "k_x/tier" entries split
    # a kernel's launches by size tier)
    hbm, src = peaks()
    kern = {k: v for k, v in kstats.items() if not k.startswith(("host:", "idle:")) and "/" not in k}
    # the deferred AMR-patch deposit runs at the least priority beside the
    # halo finder: its event span is mostly time spent waiting for SMs, so
    # the dominant kernel is taken among the hot path's own stream's kernels
    hot = {k: v for k, v in kern.items() if k != "density_patches"}
    top = max(hot.items(), key=lambda kv: kv[1][0]) if hot else ("none", (0.0, 1))
    name, (tot_ms, nl) = top
    roofline = None
    if name == "halo_main" and tot_ms > 0:
        alg = float(work[0]) * BYTES_PER_ELEMENT_PASS
        ach = alg / (tot_ms * 1e-3) / 1e9
        roofline = {"kernel": name, "bound": "hbm", "achieved": round(ach, 2), "peak": hbm, "unit": "GB/s",
                    "frac": round(ach / hbm, 5),
                    "traffic": round(float(work[0]) / nl * DRAM_BYTES_PER_ELEMENT_PASS),
                    "peak_source": src,
                    "algorithmic_bytes_per_launch": alg / nl, "avg_launch_ms": tot_ms / nl,
                    "note": (f"{BYTES_PER_ELEMENT_PASS} B per element-pass, element-passes counted on the device; "
                             f"traffic: {DRAM_BYTES_PER_ELEMENT_PASS} DRAM bytes per element-pass from an ncu "
                             "capture of every k_halo_main launch of the 256^3 workload, times this launch's "
                             "element-passes")}
    out = {
        "metric": metric, "value": value, "unit": "particles/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
        "config": {"workload": f"{cfg.name}: {cfg.npart_side}^3 particles, {cfg.box_mpc_h} Mpc/h box, "
                               f"NX={cfg.nx}, NL={cfg.nl}, {cfg.n_haloes} NFW haloes"
                               + (" + subhaloes" if with_subs else ""),
                   "global_batch": world * n, "parallelism": f"replicas x{world}",
                   "l2": "inputs > L2 (4.3 GB of particles per step)"},
        "e2e": e2e, "roofline": roofline, "clocks": clocks, "gpu_launches": int(launches),
        "launch_shape": launch,
        "device_memory_in_use_gb": round((total_b - free_b) / 1e9, 2),
        "kernels_ms_per_step": {k: round(v[0] / args.steps, 3) for k, v in
                                sorted(kstats.items(), key=lambda kv: -kv[1][0])
                                if not k.startswith(("host:", "idle:"))},
        "stream_idle_ms_per_step": {k[5:]: round(v[0] / args.steps, 3) for k, v in
                                    sorted(kstats.items(), key=lambda kv: -kv[1][0])
                                    if k.startswith("idle:") and v[0] / args.steps >= 0.1},
        "host_phases_ms_per_step": {k[5:]: round(v[0] / args.steps, 3) for k, v in
                                    sorted(kstats.items(), key=lambda kv: -kv[1][0])
                                    if k.startswith("host:")},
        "stage_s": {k: round(v, 4) for k, v in r.stage_s.items()},
        "halo_element_passes_per_step": int(work[0]) // args.steps,
        "catalogue": {"haloes": int((r.cat.realclus[: r.cat.nclus] == -1).sum()),
                      "subhaloes": int((r.cat.realclus[: r.cat.nclus] > 0).sum()),
                      "bound_ids": int(r.pph.shape[0])},
    }
    if rank == 0 and not args.no_layer:
        out["deposit_poisson"] = layer_bench()
    if rank == 0 and not args.no_grid:
        out["grid_finder"] = grid_finder_bench(b, plan)
    if rank == 0 and not args.no_cpu:
        nth = os.cpu_count() or 1
        small = cpu_oracle_run(CPU_SAMPLE, 1, 0, nth)
        n_s, dt, _ = small
        out["cpu_baseline"] = {"value": n_s / dt, "unit": "particles/s", "cores": nth, "kind": "port",
                               "sample": f"{CPU_SAMPLE}: 128^3 particles, the 512^3 recipe at 1/64 volume, "
                                         "full hot path, 1 step"}
        if not args.no_cpu_trend:
            out["cpu_baseline"]["trend"] = cpu_trend(small, nth, n)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
