"""Benchmark: Mpts/s of bit-exact 3D Delaunay triangulation on one B200.

Workload (one step = one full triangulation): the 8,000,000-point clustered
cloud (60% uniform in [0,1)^3, 40% from a 64-cluster Gaussian mixture with
sigma 0.01), FP64, PBA grid 1024^3. `--workload` selects the other
configurations (1M mixed at 512^3, 500k degenerate at 512^3, 100k uniform at
256^3, the 4,096-cloud batch).

  value      device throughput of the plain method: points already in HBM,
             tetrahedra left in HBM
  learned_proposal  the same step with the learned star proposal (trained,
             untimed, on another seeded cloud of the same configuration)
  e2e        the public API with pinned host buffers: H2D of the points and D2H
             of all tetrahedra inside every timed step
  roofline   the PBA phase (HBM-bound), CUDA events on the library's stream;
             algorithmic bytes 20*G^3 per triangulation (z pass writes 4 B per
             voxel, y and x passes read and write 4 B per voxel)
  batch      (default line) the 4,096-cloud batch: clouds/s batched, end to
             end, and one call per cloud
  cpu_baseline  the CPU oracle (a C restatement of the same pipeline, OpenMP
             over all host cores) on a random 1/8 subset of the same cloud at
             half the grid width (same voxel density), median of 3 runs

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload NAME]

With N > 1 (torchrun) every rank triangulates its own cloud: replicas, weak
scaling; the time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

import numpy as np  # noqa: E402

METRIC = "Mpts/s to bit-exact 3D DT on 1 B200: learned-proposal vs plain; batched clouds/s"
DEFAULT_WORKLOAD = "clustered8m"
WORKLOADS = {
    "clustered8m": {"workload": "clustered-8M", "points": 8_000_000, "grid": 1024,
                    "distribution": "60% U[0,1)^3 + 40% 64-cluster N(c, 0.01^2), FP64", "seed": 1},
    "mixed1m": {"workload": "mixed-1M", "points": 1_000_000, "grid": 512,
                "distribution": "50% U[0,1)^3 + 50% N(0.5,0.1^2) clipped, FP64", "seed": 1},
    "uniform100k": {"workload": "uniform-100k", "points": 100_000, "grid": 256,
                    "distribution": "U[0,1)^3, FP64", "seed": 1},
    "degenerate500k": {"workload": "degenerate-500k", "points": 500_000, "grid": 512,
                       "distribution": "50% sphere r=0.4, 30% 1/1024 lattice, 20% U[0,1)^3, FP64", "seed": 1},
    "batch4096": {"workload": "batch-4096", "clouds": 4096, "grid": "autotuned per (size bucket, distribution)",
                  "distribution": "sizes log-uniform in [64, 50000]; each uniform, N(0.5, 0.1^2) or 8-cluster "
                                  "N(c, 0.02^2), FP64", "seed": 1},
}
# CPU samples: a random 1/F subset of the workload's cloud at grid G / F^(1/3)
# (the same voxel density). The main line's cpu_baseline uses CPU_SAMPLE (median
# of 3 runs); the reference arm runs K + W steps, so each of its steps is the
# smaller REF_SAMPLE and the whole arm ends within a few minutes.
CPU_SAMPLE = {"clustered8m": 8, "mixed1m": 1, "degenerate500k": 1, "uniform100k": 1}
REF_SAMPLE = {"clustered8m": 64, "mixed1m": 8, "degenerate500k": 8, "uniform100k": 1}

# DRAM traffic of one PBA (z, y and x passes) per voxel for each form of the
# y and x passes, from ncu (dram__bytes_read.sum + dram__bytes_write.sum of the
# three kernels, one launch each) on a 1,000,000-point cloud of the clustered
# configuration at 512^3 (the 8M cloud's voxel density); the capture and its
# command are in profiles/pba_forms_clustered1m_g512.md. Scaled to a grid by
# its voxel count (the passes' traffic is proportional to it).
PBA_TRAFFIC_PER_VOXEL = {0: 4.929e9 / 512 ** 3, 1: 2.532e9 / 512 ** 3}
PBA_TRAFFIC_SOURCE = "profiles/pba_forms_clustered1m_g512.md (ncu at 512^3, scaled by voxel count)"


def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every 5 ms from a thread (the device found by its UUID,
    so CUDA_VISIBLE_DEVICES is honoured), else nvidia-smi at 200 ms. Reads
    only; no setting of the GPU is changed."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm MHz, reason bits)
        self.max_mhz = None
        self.stop_flag = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(self.device).uuid)
        try:
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
        return pynvml, h

    def start(self):
        try:
            self.nvml, self.h = self._nvml_handle()
            self.max_mhz = float(self.nvml.nvmlDeviceGetMaxClockInfo(self.h, self.nvml.NVML_CLOCK_SM))
            self._poll_once()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _poll_once(self):
        n = self.nvml
        mhz = float(n.nvmlDeviceGetClockInfo(self.h, n.NVML_CLOCK_SM))
        get = getattr(n, "nvmlDeviceGetCurrentClocksEventReasons", None) or n.nvmlDeviceGetCurrentClocksThrottleReasons
        self.samples.append((mhz, int(get(self.h))))

    def _poll(self):
        while not self.stop_flag.wait(0.005):
            try:
                self._poll_once()
            except Exception:
                return

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml:
            self.stop_flag.set()
            self.t.join(timeout=5)
            try:
                self._poll_once()
            except Exception:
                pass
            sm = [m for m, _ in self.samples]
            reasons = sorted({k for _, bits in self.samples for k, b in self.BITS.items() if bits & b})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(sm), "source": "nvml, 5 ms"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def cpu_sample(workload, frac, seed):
    """A random 1/frac subset of the workload's cloud and its grid (same voxel
    density); frac is a power of 8."""
    from gstar4d_b200 import workloads
    pts, G = workloads.config_cloud(workload, seed=seed)
    if frac > 1:
        rng = np.random.default_rng(12345)
        keep = np.sort(rng.choice(len(pts), len(pts) // frac, replace=False))
        pts = np.ascontiguousarray(pts[keep])
        G = int(round(G / round(frac ** (1.0 / 3.0))))
    return pts, G


def cpu_run(pts, G, runs, threads):
    """The oracle on a CPU sample; returns (Mpts/s of the median run, seconds)."""
    from oracle import oracle_py
    oracle_py.build() if not os.path.exists(oracle_py.LIB_PATH) else None
    times = []
    for _ in range(runs):
        t0 = time.perf_counter()
        oracle_py.triangulate(pts, G, threads=threads)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return len(pts) / t / 1e6, t


def _sample_text(workload, frac, n, G, runs, what):
    cfg = WORKLOADS[workload]
    part = "random 1/%d subset (%d points) of the %s cloud" % (frac, n, cfg["workload"]) if frac > 1 else \
        "the %s cloud (%d points)" % (cfg["workload"], n)
    return "%s at grid %d^3 (same voxel density as %d^3), %s of %d run%s" % (
        part, G, cfg["grid"], what, runs, "" if runs == 1 else "s")


def reference_arm(args):
    """The reference arm: the oracle (the reference pipeline restated in C,
    OpenMP over all host cores) on the host; rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = args.workload if args.workload in REF_SAMPLE else DEFAULT_WORKLOAD
    threads = os.cpu_count() or 1
    frac = REF_SAMPLE[wl]
    pts, G = cpu_sample(wl, frac, WORKLOADS[wl]["seed"])
    for _ in range(args.warmup):
        cpu_run(pts, G, 1, threads)
    times = []
    for _ in range(max(1, args.steps)):
        _, t = cpu_run(pts, G, 1, threads)
        times.append(t)
    total = sum(times)
    v = len(pts) * len(times) / total / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": "Mpts/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total / len(times) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(WORKLOADS[wl]),
        "cpu_baseline": {"value": round(v, 4), "unit": "Mpts/s", "cores": threads, "kind": "port",
                         "sample": _sample_text(wl, frac, len(pts), G, len(times), "total time")},
        "e2e": {"value": round(v, 4), "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def _timed(fn, ext, flush, steps):
    """Device time of `steps` calls of fn on the library's stream (CUDA events,
    the L2 flushed before each); returns (list of ms, last result)."""
    import torch
    ms, res = [], None
    for _ in range(steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(ext)
        res = fn()
        e.record(ext)
        e.synchronize()
        ms.append(s.elapsed_time(e))
    return ms, res


def run_batch(args, local, rank, steps):
    """4,096 clouds with autotuned grid widths. value: clouds/s of the batched
    call on device-resident points (tetrahedra left on the device); e2e: the
    batched call from pinned host points into a pinned host buffer;
    one_call_per_cloud: the same clouds through one call each (same widths,
    same context)."""
    import torch
    import gstar4d_b200
    from gstar4d_b200 import workloads
    cfg = dict(WORKLOADS["batch4096"])
    clouds, pts, offs = workloads.batch_clouds(cfg["clouds"], seed=cfg["seed"] + rank)
    tri = gstar4d_b200.Triangulator(grid_size=-1, device=local)
    ext = torch.cuda.ExternalStream(tri.stream, device=local)
    d_pts = torch.from_numpy(pts).to(f"cuda:{local}")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=f"cuda:{local}")
    for _ in range(max(1, args.warmup)):  # the first call also tunes the grid widths
        tri.triangulate_batch_device(d_pts.data_ptr(), offs)
    sampler = ClockSampler(local)
    sampler.start()
    ms, res = _timed(lambda: tri.triangulate_batch_device(d_pts.data_ptr(), offs), ext, flush, steps)
    clocks = sampler.stop()
    _, ntet, _, st = res
    value = len(clouds) / (statistics.mean(ms) / 1e3)
    # end to end: pinned host points in, pinned host tetrahedra out (copied
    # pass by pass while later passes compute)
    h_pts = torch.from_numpy(pts).pin_memory()
    h_out = torch.empty((int(ntet * 1.02) + 4096, 8), dtype=torch.int32).pin_memory()
    pts_np, out_np = h_pts.numpy(), h_out.numpy().view(gstar4d_b200.TET_DTYPE).reshape(-1)
    tri.triangulate_batch(pts_np, offs, out=out_np)
    e2e_ms, _ = _timed(lambda: tri.triangulate_batch(pts_np, offs, out=out_np), ext, flush, steps)
    e2e = len(clouds) / (statistics.mean(e2e_ms) / 1e3)
    # one call per cloud through the same context (same tuned widths)
    for c in range(8):
        tri.triangulate_device(d_pts[offs[c]:offs[c + 1]].data_ptr(), int(offs[c + 1] - offs[c]))
        tri.triangulate(clouds[c])

    def singles_device():
        for c in range(len(clouds)):
            tri.triangulate_device(d_pts[offs[c]:offs[c + 1]].data_ptr(), int(offs[c + 1] - offs[c]))

    def singles_host():
        for c in clouds:
            tri.triangulate(c)

    (single_dev_ms,), _ = _timed(singles_device, ext, flush, 1)
    (single_ms,), _ = _timed(singles_host, ext, flush, 1)
    single_dev = len(clouds) / (single_dev_ms / 1e3)
    single = len(clouds) / (single_ms / 1e3)
    tri.close()
    return {
        "metric": "clouds/s, 4096-cloud batch to bit-exact 3D DT on 1 B200", "value": round(value, 1),
        "unit": "clouds/s", "steps": steps, "ms_per_step": round(statistics.mean(ms), 3),
        "config": dict(cfg, points=int(offs[-1]), l2="256 MB buffer written between timed steps; inputs 737 MB"),
        "e2e": {"value": round(e2e, 1), "unit": "clouds/s", "h2d_bytes_per_step": int(offs[-1]) * 24,
                "d2h_bytes_per_step": int(ntet) * 32},
        "one_call_per_cloud": {"value": round(single_dev, 1), "unit": "clouds/s", "ms": round(single_dev_ms, 1),
                               "api": "device-resident points and tetrahedra, one call per cloud"},
        "one_call_per_cloud_e2e": {"value": round(single, 1), "unit": "clouds/s", "ms": round(single_ms, 1),
                                   "api": "host points in, host tetrahedra out, one call per cloud"},
        "batched_over_one_call_per_cloud": round(value / single_dev, 2),
        "batched_over_one_call_per_cloud_e2e": round(e2e / single, 2),
        "splay": {"loops_max": st["loops"], "insertions": st["splay_insertions"], "tets": int(ntet),
                  "large_stars": st["large_stars"]},
        "stages_ms": {k: round(st[k], 3) for k in ("t_init_ms", "t_pba_ms", "t_star_ms", "t_splay_ms",
                                                    "t_out_ms", "t_total_ms")},
        "clocks": clocks, "gpu_launches": int(st["gpu_launches"]) * steps,
    }


def batch_main(args):
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    b = run_batch(args, local, rank, args.steps)
    if rank == 0:
        line = dict(b, n_gpus=1, warmup=args.warmup, higher_is_better=True, scaling="weak", vs_baseline=None,
                    dtype="f64", data="synthetic")
        print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--points", type=int, default=None)
    ap.add_argument("--grid", type=int, default=None)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "batch4096":
        return batch_main(args)

    import torch
    import torch.distributed as dist
    import gstar4d_b200
    from gstar4d_b200 import workloads

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    cfg = dict(WORKLOADS[args.workload])
    base_points = cfg["points"]
    args.points = args.points or cfg["points"]
    args.grid = args.grid or cfg["grid"]
    cfg["points"], cfg["grid"] = args.points, args.grid
    pts, _ = workloads.config_cloud(args.workload, scale=args.points / base_points, seed=cfg["seed"] + rank)
    n = len(pts)
    tri = gstar4d_b200.Triangulator(grid_size=args.grid, device=local)
    ext = torch.cuda.ExternalStream(tri.stream, device=local)
    d_pts = torch.from_numpy(pts).to(f"cuda:{local}")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=f"cuda:{local}")  # 256 MB > L2

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world > 1:
            t = torch.tensor([x], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    # ---- device throughput (value) ----
    for _ in range(args.warmup):
        tri.triangulate_device(d_pts.data_ptr(), n)
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    stats = []

    def step():
        r = tri.triangulate_device(d_pts.data_ptr(), n)
        stats.append(r[2])
        return r

    step_ms, (_, ntets, last) = _timed(step, ext, flush, args.steps)
    barrier()
    clocks = sampler.stop()
    total_ms = max_over_ranks(sum(step_ms))
    value = world * n * args.steps / (total_ms / 1e3) / 1e6
    pba_ms = [s["t_pba_ms"] for s in stats]
    launches = sum(int(s["gpu_launches"]) for s in stats)

    # ---- learned star proposal: trained (untimed) on another seeded cloud of the
    # same configuration with labels from the plain method, then timed like value
    learned = None
    if not args.no_learned:
        # features are in voxel units, so a 1/8-size cloud of the configuration
        # at half the grid width (the same voxel density) trains as well and
        # 8x faster
        small = args.grid >= 256 and args.points >= 800_000
        train_pts, _ = workloads.config_cloud(args.workload, scale=args.points / base_points / (8 if small else 1),
                                              seed=cfg["seed"] + 1000 + rank)
        with gstar4d_b200.Triangulator(grid_size=args.grid // 2 if small else args.grid, device=local) as tt:
            t0 = time.perf_counter()
            loss = tt.train_proposal(train_pts, epochs=4, lr=2e-3)
            train_s = time.perf_counter() - t0
            weights = tt.proposal_weights()
        del train_pts
        tl = gstar4d_b200.Triangulator(grid_size=args.grid, device=local, proposal=1)
        tl.proposal_weights(weights)
        extl = torch.cuda.ExternalStream(tl.stream, device=local)
        for _ in range(args.warmup):
            tl.triangulate_device(d_pts.data_ptr(), n)
        barrier()
        lstats = []

        def lstep():
            r = tl.triangulate_device(d_pts.data_ptr(), n)
            lstats.append(r[2])
            return r

        lms, (_, ntl, stl) = _timed(lstep, extl, flush, args.steps)
        barrier()
        lt = max_over_ranks(sum(lms))
        launches += sum(int(s["gpu_launches"]) for s in lstats)
        lv = world * n * args.steps / (lt / 1e3) / 1e6
        learned = {"value": round(lv, 3), "unit": "Mpts/s", "over_plain": round(lv / value, 3),
                   "ms_per_step": round(lt / args.steps, 3), "tets": ntl, "same_tets_as_plain": ntl == ntets,
                   "star_insertions_per_point": round(stl["star_insertions"] / n, 3),
                   "splay_insertions_per_point": round(stl["splay_insertions"] / n, 3),
                   "proposed_per_point": round(stl["proposed"] / n, 3), "loops": stl["loops"],
                   "stages_ms": {k: round(stl[k], 3) for k in ("t_pba_ms", "t_star_ms", "t_splay_ms", "t_out_ms")},
                   "training": {"cloud": ("1/8-size cloud of the same configuration, seed + 1000, at half the grid "
                                          "width (same voxel density)") if small else
                                         "same configuration, seed + 1000", "epochs": 4,
                                "final_loss": round(loss, 4), "seconds": round(train_s, 2)}}
        tl.close()

    # ---- end to end through the public API with pinned host buffers ----
    h_pts = torch.from_numpy(pts).pin_memory()
    cap = int(ntets * 1.2) + 1024
    h_out = torch.empty((cap, 8), dtype=torch.int32).pin_memory()
    out_np = h_out.numpy().view(gstar4d_b200.TET_DTYPE).reshape(-1)
    pts_np = h_pts.numpy()
    for _ in range(max(1, min(args.warmup, 2))):
        tri.triangulate(pts_np, out=out_np)
    barrier()
    e2e_ms, (tets, _, _) = _timed(lambda: tri.triangulate(pts_np, out=out_np), ext, flush, args.steps)
    e2e_total = max_over_ranks(sum(e2e_ms))
    e2e = world * n * args.steps / (e2e_total / 1e3) / 1e6
    ntet_e2e = len(tets)
    tri.close()
    del d_pts, h_out, out_np, tets
    torch.cuda.empty_cache()

    # ---- the 4,096-cloud batch (extra key of the default line, N = 1) ----
    batch = None
    if world == 1 and not args.no_batch and args.workload == DEFAULT_WORKLOAD:
        batch = run_batch(args, local, rank, min(args.steps, 5))

    if rank == 0:
        peak, peak_kind = _peaks()
        G = args.grid
        alg_bytes = 20.0 * G ** 3
        pba_avg = statistics.mean(pba_ms)
        achieved = alg_bytes / (pba_avg / 1e3) / 1e9
        form = last.get("pba_form", -1)
        traffic = PBA_TRAFFIC_PER_VOXEL[form] * G ** 3 if form in PBA_TRAFFIC_PER_VOXEL else None
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mpts/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(cfg, method="plain PBA stars with voxel-block workset pairs (learned proposal in learned_proposal)",
                           l2="256 MB buffer written between timed steps", parallelism="replicas"),
            "e2e": {"value": round(e2e, 3), "unit": "Mpts/s", "h2d_bytes_per_step": int(n * 24),
                    "d2h_bytes_per_step": int(ntet_e2e * 32)},
            "roofline": {"kernel": "pba (z, y, x passes; %s form)" % ("per-line" if form == 0 else "tile"),
                         "bound": "hbm", "achieved": round(achieved, 1),
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "traffic_source": PBA_TRAFFIC_SOURCE if traffic else None,
                         "algorithmic_bytes": alg_bytes, "avg_ms": round(pba_avg, 4)},
            "stages_ms": {k: round(last[k], 3) for k in ("t_init_ms", "t_pba_ms", "t_star_ms", "t_splay_ms",
                                                          "t_out_ms", "t_total_ms")},
            "splay": {"loops": last["loops"], "star_insertions_per_point": round(last["star_insertions"] / n, 3),
                      "splay_insertions_per_point": round(last["splay_insertions"] / n, 3),
                      "proofs": last["proofs"], "exact_predicates": last["exact_predicates"],
                      "large_stars": last["large_stars"], "tets": ntets},
            "learned_proposal": learned,
            "batch": batch,
            "clocks": clocks,
            "gpu_launches": int(launches),
        }
        if not args.no_cpu and world == 1 and args.workload in CPU_SAMPLE:  # an N=1 figure
            threads = os.cpu_count() or 1
            frac = CPU_SAMPLE[args.workload]
            cp, cG = cpu_sample(args.workload, frac, cfg["seed"])
            v, t = cpu_run(cp, cG, 3, threads)
            line["cpu_baseline"] = {"value": round(v, 4), "unit": "Mpts/s", "cores": threads, "kind": "port",
                                    "sample": _sample_text(args.workload, frac, len(cp), cG, 3, "median")}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
