"""Benchmark of the B200 QuickPIC slice engine (one JSON line on rank 0).

Workload (default, --config medium): the 512 x 512 x 512 plain-method case --
transverse grid 512^2 over 12 x 12 c/wp, 512 slices over 10 c/wp, uniform
plasma with 2 x 2 particles per cell (the reference loader gives
510 * 511 * 4 = 1,042,440 FP32 electrons), tri-Gaussian drive beam of
256 x 256 x 128 = 8,388,608 macro-particles, sigma_r = 0.3, sigma_z = 0.6 c/wp,
nb/np = 4, gamma = 20000 with 1% energy spread and normalised emittance 0.01.
A step is one 3D step: beam deposit, all 512 slices, the beam push with the
step's 3D fields (dt = 10 / omega_p), species renew.
Inputs are synthetic (seeded loaders of the reference, no dataset).

metric: plasma particle-slices/s = (plasma particles x slices) / device time.
value  = inputs resident on the GPU; e2e = the same through the public API with
the beam particles copied from pinned host memory each step and the on-axis
wake lineout read back.

--impl reference: the reference's algorithm on the host cores (the CPU oracle,
QuickPIC's routines restated in C++/OpenMP; the Fortran reference needs gfortran,
MPI, HDF5 and json-fortran, none of which exist in this image), timed over one
whole 3D step of the same workload.
The engine's line also carries the error of sampled slices against the FP64
oracle (fp64_error) and a CPU baseline timed on the same sampled slices.
Multi-GPU: the path does not shard (slices are a recurrence in xi); --gpus N
runs N independent replicas, one per GPU, and value is their aggregate.
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
for p in (os.path.join(ROOT, "quickpic-opensource_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

BOX = [[-6.0, 6.0], [-6.0, 6.0], [0.0, 10.0]]

CONFIGS = {
    # the plain-method medium case (512^3, 4 ppc, 8.4M beam particles), B iterated
    # per slice to a relative change of 1e-4 (at most 16 passes)
    "medium": dict(grid=dict(ind=[9, 9, 9], box=BOX), iter=16, tol=1e-4, dt=10.0,
                   species=dict(ppc=[2, 2], q=-1.0, m=1.0, density=1.0, xtras=0.2),
                   beams=[dict(np=[256, 256, 128], q=-1.0, m=1.0, gamma=20000.0,
                               peak_density=4.0, quiet_start=True, center=[0.0, 0.0, 3.0],
                               sigma=[0.3, 0.3, 0.6],
                               sigma_v=[0.01 / 0.3, 0.01 / 0.3, 200.0])]),
    # the medium case, B to 1e-4, each slice's B passes started from the quadratic
    # extrapolation of the three previous slices' B_perp (the predictor form)
    "medium_predict": dict(grid=dict(ind=[9, 9, 9], box=BOX), iter=16, tol=1e-4, predict=2,
                           dt=10.0,
                           species=dict(ppc=[2, 2], q=-1.0, m=1.0, density=1.0, xtras=0.2),
                           beams=[dict(np=[256, 256, 128], q=-1.0, m=1.0, gamma=20000.0,
                                       peak_density=4.0, quiet_start=True,
                                       center=[0.0, 0.0, 3.0], sigma=[0.3, 0.3, 0.6],
                                       sigma_v=[0.01 / 0.3, 0.01 / 0.3, 200.0])]),
    # the medium case, B to 1e-4, each slice's B passes started by the learned
    # network (trained over the parameter-scan ranges, weights in the package)
    "medium_learned": dict(grid=dict(ind=[9, 9, 9], box=BOX), iter=16, tol=1e-4, predict=3,
                           dt=10.0,
                           species=dict(ppc=[2, 2], q=-1.0, m=1.0, density=1.0, xtras=0.2),
                           beams=[dict(np=[256, 256, 128], q=-1.0, m=1.0, gamma=20000.0,
                                       peak_density=4.0, quiet_start=True,
                                       center=[0.0, 0.0, 3.0], sigma=[0.3, 0.3, 0.6],
                                       sigma_v=[0.01 / 0.3, 0.01 / 0.3, 200.0])]),
    # the medium case with the reference's fixed 2 B passes per slice (no tolerance)
    "medium_fixed2": dict(grid=dict(ind=[9, 9, 9], box=BOX), iter=2, dt=10.0,
                          species=dict(ppc=[2, 2], q=-1.0, m=1.0, density=1.0, xtras=0.2),
                          beams=[dict(np=[256, 256, 128], q=-1.0, m=1.0, gamma=20000.0,
                                      peak_density=4.0, quiet_start=True,
                                      center=[0.0, 0.0, 3.0], sigma=[0.3, 0.3, 0.6],
                                      sigma_v=[0.01 / 0.3, 0.01 / 0.3, 200.0])]),
    # the medium transverse grid with 64 slices: the profiling case (< 1 GB on the device)
    "prof": dict(grid=dict(ind=[9, 9, 6], box=BOX), iter=16, tol=1e-4, dt=10.0,
                 species=dict(ppc=[2, 2], q=-1.0, m=1.0, density=1.0, xtras=0.2),
                 beams=[dict(np=[256, 256, 16], q=-1.0, m=1.0, gamma=20000.0,
                             peak_density=4.0, quiet_start=True, center=[0.0, 0.0, 3.0],
                             sigma=[0.3, 0.3, 0.6],
                             sigma_v=[0.01 / 0.3, 0.01 / 0.3, 200.0])]),
    # the profiling case with the reference's fixed 2 passes
    "prof_fixed2": dict(grid=dict(ind=[9, 9, 6], box=BOX), iter=2, dt=10.0,
                        species=dict(ppc=[2, 2], q=-1.0, m=1.0, density=1.0, xtras=0.2),
                        beams=[dict(np=[256, 256, 16], q=-1.0, m=1.0, gamma=20000.0,
                                    peak_density=4.0, quiet_start=True, center=[0.0, 0.0, 3.0],
                                    sigma=[0.3, 0.3, 0.6],
                                    sigma_v=[0.01 / 0.3, 0.01 / 0.3, 200.0])]),
    # the nonlinear blow-out case: 1024^2 x 1024 slices, 2x2 ppc (4.2M
    # electrons), a narrow drive beam (sigma_r 0.1, sigma_z 0.4, nb/np 20,
    # 16.8M particles) and a witness bunch 4 c/wp behind it (nb/np 10, 2.1M
    # particles, the drive's sigmas), B to 1e-4
    "blowout": dict(grid=dict(ind=[10, 10, 10], box=BOX), iter=16, tol=1e-4, dt=10.0,
                    species=dict(ppc=[2, 2], q=-1.0, m=1.0, density=1.0, xtras=0.2),
                    beams=[dict(np=[256, 256, 256], q=-1.0, m=1.0, gamma=20000.0,
                                peak_density=20.0, quiet_start=True, center=[0.0, 0.0, 2.0],
                                sigma=[0.1, 0.1, 0.4], sigma_v=[0.0, 0.0, 0.0]),
                           dict(np=[128, 128, 128], q=-1.0, m=1.0, gamma=20000.0,
                                peak_density=10.0, quiet_start=True, center=[0.0, 0.0, 6.0],
                                sigma=[0.1, 0.1, 0.4], sigma_v=[0.0, 0.0, 0.0])]),
    # the small CPU-runnable case (128^3, 2x2 ppc, 262,144 beam particles)
    "small": dict(grid=dict(ind=[7, 7, 7], box=BOX), iter=2, dt=10.0,
                  species=dict(ppc=[2, 2], q=-1.0, m=1.0, density=1.0, xtras=0.2),
                  beams=[dict(np=[64, 64, 64], q=-1.0, m=1.0, gamma=20000.0,
                              peak_density=2.0, quiet_start=True, center=[0.0, 0.0, 2.5],
                              sigma=[0.3, 0.3, 0.5], sigma_v=[0.0, 0.0, 0.0])]),
}


def plasma_count(cfg):
    nx, ny = (1 << cfg["grid"]["ind"][0]), (1 << cfg["grid"]["ind"][1])
    ppc = cfg["species"]["ppc"]
    return (nx - 2) * (ny - 1) * ppc[0] * ppc[1]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms in a thread."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def l2_copy_gbs(device):
    """Copy bandwidth of a working set that stays in L2: a 16 MiB float buffer
    copied into another (32 MiB of the 126 MB L2), 100 copies captured in one
    CUDA graph so that launch gaps do not count, read + write bytes per
    second, best of 5 replays timed with CUDA events.  The roofline of a
    kernel whose data the slice keeps in L2."""
    import torch

    dev = torch.device("cuda", device)
    a = torch.ones(4 * 1024 * 1024, dtype=torch.float32, device=dev)
    b = torch.empty_like(a)
    s = torch.cuda.Stream(device=dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(s):
        for _ in range(10):
            b.copy_(a)
    torch.cuda.current_stream(dev).wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(100):
            b.copy_(a)
    g.replay()
    torch.cuda.synchronize(dev)
    best = None
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / 100
        best = ms if best is None else min(best, ms)
    del g
    return 2 * a.numel() * 4 / (best * 1e-3) / 1e9


def ncu_traffic(kernel, workload):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = dict(kv.split("=", 1) for kv in line.split() if "=" in kv)
        if f.get("kernel") == kernel and f.get("workload") == workload:
            return float(f["dram_bytes_per_launch"])
    return None


def make_engine(qpgpu, cfg, device, graphs=0):
    g = cfg["grid"]
    ctx = qpgpu.Context(g["ind"][0], g["ind"][1], g["ind"][2], g["box"], device=device)
    s = cfg["species"]
    sp = qpgpu.Species2d(ctx, ppc=tuple(s["ppc"]), q=s["q"], m=s["m"], density=s["density"],
                         xtras=s["xtras"])
    beams = []
    for b in cfg["beams"]:
        beams.append(qpgpu.Beam3d(ctx, b["np"], q=b["q"], m=b["m"], gamma=b["gamma"],
                                  peak_density=b["peak_density"], quiet_start=b["quiet_start"],
                                  center=b["center"], sigma=b["sigma"], sigma_v=b["sigma_v"]))
    sim = qpgpu.Simulation(ctx, [sp], beams, iter=cfg["iter"], store3d=True,
                           use_graphs=bool(graphs),
                           dt=cfg.get("dt", 0.0), tol=cfg.get("tol", 0.0),
                           predict=cfg.get("predict", False))
    if cfg.get("predict") == 3:
        w = os.path.join(ROOT, "quickpic-opensource_b200", "qpgpu", "predictor_weights.npy")
        if not os.path.exists(w):
            raise SystemExit(f"{w} is missing: train it with qpgpu/train_predictor.py")
        net = qpgpu.Predictor(device=device)
        net.set_params(np.load(w))
        sim.set_predictor(net)
        sim._net = net
    return ctx, sp, beams, sim


def run_engine(args, cfg, rank, world, local_rank, dist):
    import qpgpu

    ctx, sp, beams, sim = make_engine(qpgpu, cfg, local_rank, args.graphs)
    npl = sp.np()
    nz = ctx.nz
    for _ in range(args.warmup):
        st = sim.step3d()
    kernels_per_step = st.kernels if args.warmup else 0

    def barrier():
        ctx.sync()
        if dist is not None:
            import torch

            torch.cuda.synchronize()
            dist.barrier()

    # ---- value: inputs resident in HBM
    import torch

    clocks = ClockSampler(local_rank)
    barrier()
    clocks.start()
    # the timed steps are the capture range of `ncu --profile-from-start off`
    # (the start/stop calls do nothing without a profiler attached)
    torch.cuda.profiler.start()
    ctx.timer_start()
    regrow = passes = unconverged = 0
    for _ in range(args.steps):
        st = sim.step3d()
        regrow += st.regrowths
        passes += st.iterations
        unconverged += st.unconverged
        kernels_per_step = st.kernels
    t_ms = ctx.timer_stop()
    torch.cuda.profiler.stop()
    clocks.stop()
    barrier()
    value, t_ms = job_throughput(float(npl * nz * args.steps), t_ms, dist)

    # ---- e2e: beam in from pinned host memory, wake lineout out, every step
    bm = beams[0]
    host = bm.get_particles()
    pinned = torch.empty(host.size, dtype=torch.float32, pin_memory=True).numpy()
    pin2 = pinned.reshape(host.shape, order="F")
    pin2[...] = host
    line = torch.empty(nz + 1, dtype=torch.float32, pin_memory=True).numpy()
    barrier()
    ctx.timer_start()
    for _ in range(args.steps):
        bm.set_particles(pin2)
        sim.step3d()
        sim.lineout(3, out=line)
    e_ms = ctx.timer_stop()
    barrier()
    e_val, e_ms = job_throughput(float(npl * nz * args.steps), e_ms, dist)
    e2e = {"value": e_val, "unit": "particle-slices/s",
           "h2d_bytes_per_step": int(host.nbytes), "d2h_bytes_per_step": int(line.nbytes),
           "ms_per_step": e_ms / args.steps}

    # ---- roofline of the dominant kernel: a per-launch profile of one more 3D
    # step, with every launch of prof_slices slices spread over the box timed
    prof = sim.profile(min(args.prof_slices, nz))
    peak, peak_kind = load_peaks()
    # the dominant kernel with algorithmic bytes (the network's launches of the
    # learned start are FLOP-bound and reported under `kernels` only)
    top = max(((k, v) for k, v in prof.items() if not k.endswith(":skipped") and v[2] > 0),
              key=lambda kv: kv[1][0])
    name, (ms, cnt, byts) = top
    tot = sum(v[0] for v in prof.values())
    achieved = (byts / cnt) / (ms / cnt * 1e-3) / 1e9 if ms > 0 else 0.0
    traffic = ncu_traffic(name, args.config)
    l2 = l2_copy_gbs(local_rank)
    roofline = {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                "peak_source": peak_kind, "share": round(ms / tot, 4),
                "algorithmic_bytes_per_launch": byts / cnt,
                "avg_launch_us": round(ms / cnt * 1e3, 2),
                "l2_peak": round(l2, 1),
                "l2_peak_source": "measured in this run: L2-resident copy, 16 MiB -> 16 MiB, graph of 100",
                "l2_frac": round(achieved / l2, 4)}

    def gbps(v):
        return v[2] / (v[0] * 1e-3) / 1e9 if v[0] > 0 and v[2] > 0 else None

    kernels = {k: {"ms": round(v[0], 4), "launches": v[1],
                   "GBps": round(gbps(v), 1) if gbps(v) else None,
                   "of_hbm": round(gbps(v) / peak, 4) if gbps(v) else None,
                   "of_l2": round(gbps(v) / l2, 4) if gbps(v) else None}
               for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}
    # ---- error against the FP64 oracle, and the CPU baseline, on sampled slices
    errors = cpu = None
    if world == 1 and not args.no_cpu_baseline:
        errors, cpu = sampled_slices(cfg, ctx, sp, sim, args.error_samples,
                                     os.cpu_count() or 1)
    sim.close()
    for b in beams:
        b.close()
    sp.close()
    ctx.close()
    return dict(value=value, t_ms=t_ms, e2e=e2e, roofline=roofline, kernels=kernels,
                errors=errors, cpu=cpu, prof_slices=args.prof_slices,
                clocks=clocks.summary(), npl=npl, nz=nz, regrow=regrow,
                passes_per_slice=passes / (nz * args.steps), unconverged=unconverged,
                launches=kernels_per_step * args.steps,
                beam_np=int(sum(np.prod(b["np"]) for b in cfg["beams"])))


def scan_instances(n, seed=2024):
    """The batched parameter scan: n instances, transverse grids drawn
    log-uniform from 128^2, 256^2, 512^2 (powers of two), 256 slices each over a
    12 x 12 x 10 c/wp box, 2 x 2 ppc; beam nb/np log-uniform in [0.5, 20],
    sigma_r uniform in [0.1, 0.5] c/wp, sigma_z = 0.5 c/wp, beam particles in
    proportion to the grid area from 262,144 at 128^2, at most 2,097,152.
    Pairs with a normalised beam charge (nb/np) sigma_r^2 above 1 are drawn
    again: in that full blow-out some plasma electrons reach gamma - p_z -> 0,
    where the quasi-static push moves them across the box in one slice (the
    reference's push has no guard for it either; the engine stops with an
    error)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        it = int(rng.integers(7, 10))
        while True:
            peak = float(np.exp(rng.uniform(np.log(0.5), np.log(20.0))))
            sr = float(rng.uniform(0.1, 0.5))
            if peak * sr * sr <= 1.0:
                break
        nb = {7: [64, 64, 64], 8: [128, 128, 64], 9: [128, 128, 128]}[it]
        out.append(dict(grid=dict(ind=[it, it, 8], box=BOX), iter=2, dt=0.0,
                        species=dict(ppc=[2, 2], q=-1.0, m=1.0, density=1.0, xtras=0.2),
                        beams=[dict(np=nb, q=-1.0, m=1.0, gamma=20000.0, peak_density=peak,
                                    quiet_start=True, center=[0.0, 0.0, 2.5],
                                    sigma=[sr, sr, 0.5], sigma_v=[0.0, 0.0, 0.0])]))
    return out


def run_scan_case(args):
    """Aggregate throughput of the batched scan (instances stepped concurrently,
    the worker count from the autotuner) against the same instances stepped one
    after another."""
    import qpgpu

    insts = []
    for cfg in scan_instances(args.scan_n):
        g = cfg["grid"]
        ctx = qpgpu.Context(g["ind"][0], g["ind"][1], g["ind"][2], g["box"])
        s = cfg["species"]
        sp = qpgpu.Species2d(ctx, ppc=tuple(s["ppc"]), q=s["q"], m=s["m"], density=s["density"],
                             xtras=s["xtras"])
        b = cfg["beams"][0]
        bm = qpgpu.Beam3d(ctx, b["np"], q=b["q"], m=b["m"], gamma=b["gamma"],
                          peak_density=b["peak_density"], quiet_start=True, center=b["center"],
                          sigma=b["sigma"], sigma_v=b["sigma_v"])
        sim = qpgpu.Simulation(ctx, [sp], [bm], iter=cfg["iter"], store3d=False, dt=0.0,
                               use_graphs=bool(args.graphs))
        insts.append((ctx, sp, bm, sim))
    sims = [i[3] for i in insts]
    workers, _ = qpgpu.scan_tune(sims, probe_steps=1)
    for _ in range(args.warmup):
        qpgpu.scan_run(sims, steps=1, workers=workers)
    clocks = ClockSampler(0)
    clocks.start()
    st = qpgpu.scan_run(sims, steps=args.steps, workers=workers)
    clocks.stop()
    seq = qpgpu.scan_run(sims, steps=args.steps, workers=1)
    value = st.particle_slices / (st.gpu_ms * 1e-3)
    v_seq = seq.particle_slices / (seq.gpu_ms * 1e-3)
    grids = {}
    for cfg in scan_instances(args.scan_n):
        k = f"{1 << cfg['grid']['ind'][0]}^2"
        grids[k] = grids.get(k, 0) + 1
    line = {"metric": "plasma particle-slices/s (scan aggregate)", "value": value,
            "unit": "particle-slices/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": st.gpu_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded reference loaders)",
            "config": {"workload": f"scan: {args.scan_n} instances, grids {grids}, 256 slices, "
                                   "2x2 ppc, iter=2, no beam push, 3D fields not kept",
                       "instances": args.scan_n, "workers": st.workers,
                       "slice_graphs": bool(args.graphs),
                       "sequential_value": v_seq,
                       "speedup_vs_sequential": round(value / v_seq, 3),
                       "parallelism": "single"},
            "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)
    for ctx, sp, bm, sim in insts:
        sim.close()
        bm.close()
        sp.close()
        ctx.close()


def run_fft_case(args, cfg):
    """Kernel case: class-level fftrk + fftkr (kind 2) of a 3-component field on the
    workload's transverse grid; one step = one round trip.  Deterministic and
    free of particles, so the transform kernels can be profiled on their own."""
    import qpgpu

    g = cfg["grid"]
    ctx = qpgpu.Context(g["ind"][0], g["ind"][1], 1, g["box"])
    f = qpgpu.Field2d(ctx, 3)
    rng = np.random.default_rng(1)
    f.set_rs(rng.standard_normal(ctx.rs_shape(3)).astype(np.float32))
    for _ in range(args.warmup):
        f.fftrk(2)
        f.fftkr(2)
    ctx.sync()
    import torch

    torch.cuda.profiler.start()
    ctx.timer_start()
    for _ in range(args.steps):
        f.fftrk(2)
        f.fftkr(2)
    ms = ctx.timer_stop()
    torch.cuda.profiler.stop()
    nx, ny = 1 << g["ind"][0], 1 << g["ind"][1]
    byts = 3 * 4.0 * (nx + 1) * (ny + 1) * 2 * 2 * args.steps  # 3 comps, 2 passes each way
    print(json.dumps({"case": "fft", "grid": [nx, ny], "components": 3, "steps": args.steps,
                      "us_per_round_trip": 1e3 * ms / args.steps,
                      "algorithmic_GBps": byts / (ms * 1e-3) / 1e9}), flush=True)
    f.close()
    ctx.close()


def run_particle_case(args, cfg):
    """Kernel cases: one class-level particle routine of a 2 x 2 ppc plasma on the
    workload's transverse grid -- amjdp (the current and acceleration deposit
    with the half push, PPGRDCJPPOST2L_QP) or push (the full push with the
    re-bin, PPGRBPPUSHF23L_QP + PPPORDERF2LA/PPPORDER2LB).  The particles are
    moved by up to 2 cells, given thermal momenta and re-binned (which leaves
    each tile in cell order, as in the step); the fields are seeded random
    values.  One step = one call; the kernel can be profiled without the rest
    of the slice."""
    import qpgpu

    g = cfg["grid"]
    ctx = qpgpu.Context(g["ind"][0], g["ind"][1], 1, g["box"])
    sp = qpgpu.Species2d(ctx, ppc=(2, 2), xtras=0.5)
    pp, kp = sp.get_particles()
    rng = np.random.default_rng(3)
    for t in range(len(kp)):
        n = kp[t]
        pp[0, :n, t] += rng.uniform(-2.0, 2.0, n).astype(np.float32)
        pp[1, :n, t] += rng.uniform(-2.0, 2.0, n).astype(np.float32)
        for c in (2, 3, 4):
            pp[c, :n, t] = rng.normal(0.0, 0.1, n).astype(np.float32)
        for c in (5, 6):
            pp[c, :n, t] = (1.0 + 0.01 * rng.standard_normal(n)).astype(np.float32)
    np.clip(pp[0], 0.0, ctx.nx - 1e-3, out=pp[0])
    np.clip(pp[1], 0.0, ctx.ny - 1e-3, out=pp[1])
    sp.set_particles(pp, kp)
    sp.pmove()
    fxy, bxyz, psit = qpgpu.Field2d(ctx, 2), qpgpu.Field2d(ctx, 3), qpgpu.Field2d(ctx, 1)
    cu, amu, dcu = qpgpu.Field2d(ctx, 3), qpgpu.Field2d(ctx, 3), qpgpu.Field2d(ctx, 2)
    for f, d in ((fxy, 2), (bxyz, 3), (psit, 1)):
        f.set_rs((0.01 * rng.standard_normal(ctx.rs_shape(d))).astype(np.float32))
    dex = ctx.dex
    if args.case == "amjdp":
        def call():
            sp.amjdp(fxy, bxyz, psit, cu, amu, dcu, dex)
    else:
        def call():
            sp.push(fxy, bxyz, psit, dex)
    for _ in range(args.warmup):
        call()
    ctx.sync()
    import torch

    torch.cuda.profiler.start()
    ctx.timer_start()
    for _ in range(args.steps):
        call()
    ms = ctx.timer_stop()
    torch.cuda.profiler.stop()
    npart = sp.np()
    print(json.dumps({"case": args.case, "grid": [ctx.nx, ctx.ny], "particles": npart,
                      "steps": args.steps, "us_per_call": 1e3 * ms / args.steps,
                      "particles_per_s": npart * args.steps / (ms * 1e-3)}), flush=True)
    for f in (fxy, bxyz, psit, cu, amu, dcu):
        f.close()
    sp.close()
    ctx.close()


def run_nn_train_case(args):
    """Kernel case: training steps of the learned B start on pairs recorded
    from one 3D step of a 128^2 x 128-slice case (passes to 1e-4); one step =
    one Adam step on a minibatch of 32 pairs of 128 x 128 Fourier-mode images
    (the 5 forward, 4 data-gradient and 5 weight-gradient tensor-core kernels).
    FLOPs per step: 3 x 2 x MACs of the forward (the backward is twice the
    forward)."""
    import qpgpu

    c = qpgpu.Context(7, 7, 7, BOX)
    sp = qpgpu.Species2d(c, ppc=(2, 2))
    bm = qpgpu.Beam3d(c, [64, 64, 64], q=-1.0, m=1.0, gamma=20000.0, peak_density=3.0,
                      quiet_start=True, center=[0.0, 0.0, 2.5], sigma=[0.3, 0.3, 0.5])
    sim = qpgpu.Simulation(c, [sp], [bm], iter=16, tol=1e-4, store3d=False)
    data = qpgpu.TrainingSet(128)
    sim.record(data)
    sim.step3d()
    net = qpgpu.Predictor(seed=1)
    net.train(data, steps=max(1, args.warmup), batch=32, lr=1e-3)
    st = net.train(data, steps=args.steps, batch=32, lr=1e-3)
    macs_px = 9 * (16 * 32 + 3 * 32 * 32 + 32 * 16)
    flops = 3 * 2 * macs_px * 32 * 128 * 128 * args.steps
    print(json.dumps({"case": "nn_train", "steps": args.steps, "batch": 32,
                      "image": [128, 128], "ms_per_step": st.gpu_ms / args.steps,
                      "tflops": flops / (st.gpu_ms * 1e-3) / 1e12,
                      "first_loss": st.first_loss, "last_loss": st.last_loss}), flush=True)
    for o in (net, data, sim, bm, sp, c):
        o.close()


def _reduce(v, dist, op):
    if dist is None:
        return v
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op(dist))
    return float(t.item())


def max_over_ranks(v, dist):
    return _reduce(v, dist, lambda d: d.ReduceOp.MAX)


def sum_over_ranks(v, dist):
    return _reduce(v, dist, lambda d: d.ReduceOp.SUM)


def job_throughput(units_local, t_ms_local, dist):
    """Whole-job throughput of independent replicas: the units every rank
    processed over the slowest rank's device time.  Returns (units/s, max ms)."""
    t_ms = max_over_ranks(t_ms_local, dist)
    units = sum_over_ranks(units_local, dist)
    return units / (t_ms * 1e-3), t_ms


def _oracle_fields(o, nx, ny):
    """A slice's outputs held by the oracle after it: the stored force
    (fxy, psit), B (bxy, bz), psi, epw and the extrapolated current."""
    nxv, nyp = nx + 2, 2 * ny + 1
    fxy = o.get("fxy").reshape((2, nxv, nyp), order="F")[:, :, : ny + 1]
    bxyz = o.get("bxyz").reshape((3, nxv, nyp), order="F")[:, :, : ny + 1]
    return dict(fxy=fxy, psit=o.get("psit").reshape((nxv, nyp), order="F")[:, : ny + 1],
                bxy=bxyz[0:2], bz=bxyz[2],
                psi=o.get("psi").reshape((nxv, nyp), order="F")[:, : ny + 1],
                epw=o.get("epw_k").reshape((2, ny + 1, nx + 1), order="F"),
                cu_k=o.get("cu_k").reshape((3, ny + 1, nx + 1), order="F"))


def _engine_fields(sim, j, ny):
    be, bb = sim.get_plane("bexyz", j), sim.get_plane("bbxyz", j)
    return dict(fxy=be[0:2], psit=be[2], bxy=bb[0:2], bz=bb[2],
                psi=sim.get_field("psi")[0, :, : ny + 1], epw=sim.get_field("epw"),
                cu_k=sim.get_field("cu_k"))


def _err(a, b, ref_norm=None):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = ref_norm if ref_norm is not None else np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a))


def sampled_slices(cfg, ctx, sp, sim, nsamples, threads):
    """One more 3D step of the engine, stopped before each of `nsamples`
    slices spread evenly over the box (slice 1 + floor((2i+1) nz / (2 n))).
    Before a sampled slice j the engine's state -- tiled particles, the
    Fourier-space B_perp iterate, the extrapolated current and slice j's beam
    charge plane -- is handed to the oracle, the engine runs slice j, and the
    FP32 oracle (the reference's SGL build, timed: the CPU baseline) and the
    FP64 oracle (its DBL build: the error) run slice j from the same state.
    Returns (errors, cpu figures)."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle

    nx, ny, nz = ctx.nx, ctx.ny, ctx.nz
    # the oracle starts each slice's passes from epw(j-1), the reference's start;
    # under a tolerance the converged fields do not depend on the start
    ocfg = dict(cfg, beams=[], store3d=False, predict=0)
    o32, o64 = oracle.Sim(ocfg, np.float32), oracle.Sim(ocfg, np.float64)
    samples = sorted({1 + ((2 * i + 1) * nz) // (2 * nsamples) for i in range(nsamples)})
    names = ("fxy", "psit", "bxy", "bz", "psi", "epw", "cu_k")
    e64 = {k: [] for k in names}
    e32 = {k: [] for k in names}
    eref = {k: [] for k in names}
    sq = {k: [0.0, 0.0, 0.0] for k in names}  # sum |engine - fp64|^2, |fp32 - fp64|^2, |fp64|^2
    t32 = 0.0
    p0 = int(o32.get("passes")[0])
    sim.begin3d()
    for j in samples:
        if j > sim.next_slice:
            sim.slices(j - sim.next_slice)
        pp, kp = sp.get_particles()
        st = dict(ppart=pp, kpic=kp, epw_k=sim.get_field("epw"), cu_k=sim.get_field("cu_k"),
                  qb=sim.get_plane("qb", j))
        sim.slices(1)
        got = _engine_fields(sim, j, ny)
        for o in (o32, o64):
            o.set_state(**st)
        t0 = time.perf_counter()
        o32.slice(j)
        t32 += time.perf_counter() - t0
        o64.slice(j)
        r32, r64 = _oracle_fields(o32, nx, ny), _oracle_fields(o64, nx, ny)
        bnorm = float(np.linalg.norm(np.asarray(r64["bxy"], dtype=np.float64)))
        for k in names:
            ref = bnorm if k == "bz" else None
            e64[k].append(_err(got[k], r64[k], ref))
            e32[k].append(_err(got[k], r32[k], ref))
            eref[k].append(_err(r32[k], r64[k], ref))
            a64 = np.asarray(r64[k], dtype=np.float64)
            sq[k][0] += float(np.sum((np.asarray(got[k], np.float64) - a64) ** 2))
            sq[k][1] += float(np.sum((np.asarray(r32[k], np.float64) - a64) ** 2))
            sq[k][2] += bnorm ** 2 if k == "bz" else float(np.sum(a64 ** 2))
    passes32 = int(o32.get("passes")[0]) - p0
    if sim.next_slice <= nz:
        sim.slices(nz - sim.next_slice + 1)
    sim.end3d()
    o32.close()
    o64.close()
    npl = sp.np()
    errors = {"samples": samples,
              "vs_fp64_oracle": {k: float(np.sqrt(v[0] / v[2])) for k, v in sq.items()},
              "fp32_oracle_vs_fp64_oracle": {k: float(np.sqrt(v[1] / v[2]))
                                             for k, v in sq.items()},
              "vs_fp64_oracle_max_slice": {k: float(max(v)) for k, v in e64.items()},
              "fp32_oracle_vs_fp64_max_slice": {k: float(max(v)) for k, v in eref.items()},
              "vs_fp32_oracle_max_slice": {k: float(max(v)) for k, v in e32.items()},
              "note": "relative L2 from identical inputs (the engine's state before each "
                      "sampled slice): vs_fp64_oracle pools all samples, *_max_slice is the "
                      "worst single slice; bz against |B_perp| (roundoff-level in an "
                      "axisymmetric wake); the FP32 oracle (the reference's SGL arithmetic) "
                      "is shown against the FP64 oracle for scale"}
    cpu = {"value": npl * len(samples) / t32, "seconds": t32, "slices": len(samples),
           "passes_per_slice": passes32 / len(samples) if cfg.get("tol", 0.0) > 0 else cfg["iter"]}
    return errors, cpu


def workload_desc(cfg, name):
    g = cfg["grid"]["ind"]
    beams = "; ".join(
        f"beam {int(np.prod(b['np']))} particles sigma_r={b['sigma'][0]} "
        f"sigma_z={b['sigma'][2]} nb/np={b['peak_density']} at z={b['center'][2]}"
        for b in cfg["beams"])
    return (f"{name}: {1 << g[0]}x{1 << g[1]} transverse, {1 << g[2]} slices, "
            f"{cfg['species']['ppc'][0]}x{cfg['species']['ppc'][1]} ppc, {beams}, "
            f"{passes_desc(cfg)}, beam push dt={cfg.get('dt', 0.0)}")


def passes_desc(cfg):
    start = {1: ", started from the linear extrapolation of B_perp",
             2: ", started from the quadratic extrapolation of B_perp",
             3: ", started by the learned network (BF16 tcgen05 convolutions)"}.get(
        cfg.get("predict", 0), "")
    if cfg.get("tol", 0.0) > 0:
        return (f"B predictor-corrector passes per slice until the relative change of B_perp "
                f"<= {cfg['tol']:g} (at most {cfg['iter']}){start}")
    return f"iter={cfg['iter']} (fixed predictor-corrector passes)"


def run_reference(args, cfg):
    """The reference's algorithm on the host cores: the CPU oracle (QuickPIC's
    routines restated in C++, FP32 like the reference's SGL build, OpenMP on
    every host core) runs one whole 3D step of the same workload -- the beam
    deposit, every slice with the same B passes and tolerance, the beam push,
    the species renew -- timed end to end.  The particles are loaded before the
    timer, as the engine's are.  One medium step takes minutes on the host, so
    the step is not repeated K times: the line reports the one step it timed
    (timed_3d_steps), after W slices of the small case as warm-up."""
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle

    warm = oracle.Sim(dict(CONFIGS["small"], store3d=False), np.float32)
    warm.begin3d()
    for j in range(1, max(1, args.warmup) + 1):
        warm.slice(j)
    warm.close()
    c = dict(cfg)
    c["store3d"] = True  # the beam push reads the stored 3D fields
    c["predict"] = 0  # the reference's start of the passes
    sim = oracle.Sim(c, np.float32)
    npl = int(sim.get("np")[0])
    nz = 1 << cfg["grid"]["ind"][2]
    t0 = time.perf_counter()
    sim.step3d()
    secs = time.perf_counter() - t0
    passes = int(sim.get("passes")[0]) if cfg.get("tol", 0.0) > 0 else nz * cfg["iter"]
    unconv = int(sim.get("unconverged")[0])
    sim.close()
    value = npl * nz / secs
    sample = (f"one whole {args.config} 3D step (beam deposit, {nz} slices, beam push, renew) "
              f"in {secs:.1f} s; CPU restatement of the reference algorithm (FP32, OpenMP, "
              f"{threads} threads), not the Fortran binary")
    line = {"impl": "reference", "metric": "plasma particle-slices/s", "value": value,
            "unit": "particle-slices/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "timed_3d_steps": 1, "ms_per_step": secs * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded reference loaders)",
            "config": {"workload": workload_desc(cfg, args.config), "plasma_particles": npl,
                       "slices": nz, "iter": cfg["iter"], "tol": cfg.get("tol", 0.0),
                       "passes_per_slice": round(passes / nz, 3),
                       "unconverged_slices": unconv, "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": "particle-slices/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "particle-slices/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--config", default="medium", choices=sorted(CONFIGS))
    ap.add_argument("--prof-slices", type=int, default=32,
                    help="slices of the profiled step whose launches are timed")
    ap.add_argument("--error-samples", type=int, default=24,
                    help="slices of one step checked against the FP64 oracle (and timed on "
                    "the FP32 oracle for the CPU baseline)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--case", default="step",
                    choices=["step", "fft", "amjdp", "push", "scan", "nn_train"],
                    help="step: the 3D step (the benchmark); fft: transform kernels alone; "
                    "amjdp / push: one particle routine alone; scan: the batched "
                    "parameter scan (--scan-n instances); nn_train: training steps of the "
                    "learned B start (the tensor-core kernels alone)")
    ap.add_argument("--scan-n", type=int, default=64)
    ap.add_argument("--graphs", type=int, default=1, choices=[0, 1],
                    help="1: each slice replayed from a captured CUDA graph (use_graphs)")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if args.case == "scan":
        run_scan_case(args)
        return
    if args.case == "fft":
        run_fft_case(args, cfg)
        return
    if args.case in ("amjdp", "push"):
        run_particle_case(args, cfg)
        return
    if args.case == "nn_train":
        run_nn_train_case(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args, cfg)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    r = run_engine(args, cfg, rank, world, local_rank, dist)
    cpu = None
    if rank == 0 and r["cpu"] is not None:
        c = r["cpu"]
        cpu = {"value": c["value"], "unit": "particle-slices/s", "cores": os.cpu_count() or 1,
               "kind": "port", "passes_per_slice": round(c["passes_per_slice"], 3),
               "sample": f"{c['slices']} slices spread evenly over one {args.config} 3D step "
                         f"(head, beam and wake), each run by the oracle from the engine's "
                         f"state before it, {c['seconds']:.1f} s of slice time (CPU restatement "
                         f"of the reference algorithm, FP32, OpenMP; the beam deposit and "
                         f"push are not in this sample, --impl reference times a whole step)"}
    if rank == 0:
        line = {"metric": "plasma particle-slices/s", "value": r["value"],
                "unit": "particle-slices/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["t_ms"] / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded reference loaders)",
                "config": {"workload": workload_desc(cfg, args.config),
                           "plasma_particles": r["npl"], "beam_particles": r["beam_np"],
                           "slices": r["nz"], "iter": cfg["iter"], "tol": cfg.get("tol", 0.0),
                           "passes_per_slice": round(r["passes_per_slice"], 3),
                           "unconverged_slices": r["unconverged"],
                           "l2": "inputs larger than L2: each 3D step writes >4 GB of 3D fields",
                           "slice_graphs": bool(args.graphs),
                           "parallelism": "replicas" if world > 1 else "single"},
                "step_time_ms": r["t_ms"] / args.steps,
                "e2e": r["e2e"], "roofline": r["roofline"], "cpu_baseline": cpu,
                "fp64_error": r["errors"],
                "gpu_launches": r["launches"], "clocks": r["clocks"],
                "regrowths": r["regrow"], "kernels": r["kernels"]}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
