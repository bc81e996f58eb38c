"""Benchmark: Mpts/s of bit-exact 3D Delaunay triangulation on B200.

Workload (one step = one full triangulation): the 1,000,000-point mixed cloud
(half uniform in [0,1)^3, half N(0.5, 0.1^2) clipped), FP64, PBA grid 512^3.

  value  device throughput: points already in HBM, tetrahedra left in HBM
  e2e    the public API with pinned host buffers: H2D of the points and D2H of
         all tetrahedra inside every timed step
  roofline  the PBA phase (HBM-bound) measured with CUDA events on the
         library's stream: algorithmic bytes 20*G^3 per launch set (z pass
         writes 4 B/voxel, y and x passes read and write 4 B/voxel)
  cpu_baseline  the CPU oracle (a C restatement of the same pipeline, OpenMP over
         all host cores) on a bounded sample of the same distribution

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

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

WORKLOAD = {"workload": "mixed-1M", "points": 1_000_000, "grid": 512,
            "distribution": "50% U[0,1)^3 + 50% N(0.5,0.1^2) clipped, FP64", "seed": 1}
# the other configurations, measured with --workload (parity cases, not the headline line)
WORKLOADS = {
    "mixed1m": WORKLOAD,
    "uniform100k": {"workload": "uniform-100k", "points": 100_000, "grid": 256,
                    "distribution": "U[0,1)^3, FP64", "seed": 1},
    "degenerate500k": {"workload": "degenerate-500k", "points": 500_000, "grid": 512,
                       "distribution": "50% sphere r=0.4, 30% 1/1024 lattice, 20% U[0,1)^3, FP64", "seed": 1},
    "clustered8m": {"workload": "clustered-8M", "points": 8_000_000, "grid": 1024,
                    "distribution": "60% U[0,1)^3 + 40% 64-cluster N(c, 0.01^2), FP64", "seed": 1},
    "batch4096": {"workload": "batch-4096", "clouds": 4096, "grid": "per cloud (134 voxels/point rule)",
                  "distribution": "sizes log-uniform in [64, 50000]; each uniform, N(0.5, 0.1^2) or 8-cluster "
                                  "N(c, 0.02^2), FP64", "seed": 1},
}
METRIC = "Mpts/s to bit-exact 3D DT on 1 B200"
SAMPLE_POINTS, SAMPLE_GRID = 125_000, 256  # same voxel density (134 voxels/point)


def _pba_traffic(G):
    """DRAM bytes of one PBA (z, y, x passes) from the committed ncu summary,
    scaled from its grid to G by the voxel count; None when absent."""
    try:
        with open(os.path.join(REPO, "profiles", "pba_mixed100k_g512.md")) as f:
            for line in f:
                if line.startswith("traffic_per_launch_bytes:"):
                    return float(line.split()[1]) * (G / 512.0) ** 3
    except OSError:
        pass
    return None


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


def cpu_run(steps, threads):
    """The oracle on the bounded sample; returns (Mpts/s, seconds per run)."""
    from oracle import oracle_py
    from gstar4d_b200 import workloads
    oracle_py.build() if not os.path.exists(oracle_py.LIB_PATH) else None
    pts = workloads.mixed(SAMPLE_POINTS, seed=WORKLOAD["seed"])
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        oracle_py.triangulate(pts, SAMPLE_GRID, threads=threads)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return len(pts) / t / 1e6, t, len(pts)


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_run(1, threads)
    v, t, n = cpu_run(max(1, args.steps), threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": "Mpts/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(WORKLOAD),
        "cpu_baseline": {"value": round(v, 4), "unit": "Mpts/s", "cores": threads, "kind": "port",
                         "sample": "%d-point mixed cloud at grid %d^3 (same distribution and voxel density), "
                                   "median of %d runs" % (n, SAMPLE_GRID, max(1, args.steps))},
        "e2e": {"value": round(v, 4), "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def batch_main(args):
    """4,096 clouds with autotuned grid widths. value: clouds/s of the batched
    call on device-resident points (tetrahedra left on the device); e2e: the
    batched call from pinned host points into a pinned host buffer;
    one_call_per_cloud: the same clouds through one host call each (same
    widths, same context)."""
    import torch
    import gstar4d_b200
    from gstar4d_b200 import workloads
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    cfg = dict(WORKLOADS["batch4096"])
    clouds, pts, offs = workloads.batch_clouds(cfg["clouds"], seed=cfg["seed"] + rank)
    tri = gstar4d_b200.Triangulator(grid_size=-1, device=local, log_verbose=int(os.environ.get("G4D_VERBOSE", "0")))
    ext = torch.cuda.ExternalStream(tri.stream, device=local)
    d_pts = torch.from_numpy(pts).to(f"cuda:{local}")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=f"cuda:{local}")
    for _ in range(max(1, args.warmup)):  # the first call also tunes the grid widths
        tri.triangulate_batch_device(d_pts.data_ptr(), offs)
    sampler = ClockSampler(local)
    sampler.start()
    ms = []
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(ext)
        _, ntet, _, st = tri.triangulate_batch_device(d_pts.data_ptr(), offs)
        e.record(ext)
        e.synchronize()
        ms.append(s.elapsed_time(e))
    clocks = sampler.stop()
    value = len(clouds) / (statistics.mean(ms) / 1e3)
    # end to end: pinned host points in, pinned host tetrahedra out (copied
    # pass by pass while later passes compute)
    h_pts = torch.from_numpy(pts).pin_memory()
    h_out = torch.empty((int(ntet * 1.02) + 4096, 8), dtype=torch.int32).pin_memory()
    pts_np, out_np = h_pts.numpy(), h_out.numpy().view(gstar4d_b200.TET_DTYPE).reshape(-1)
    tri.triangulate_batch(pts_np, offs, out=out_np)
    e2e_ms = []
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(ext)
        tets, toffs, _ = tri.triangulate_batch(pts_np, offs, out=out_np)
        e.record(ext)
        e.synchronize()
        e2e_ms.append(s.elapsed_time(e))
    e2e = len(clouds) / (statistics.mean(e2e_ms) / 1e3)
    # one call per cloud through the same context (same tuned widths): device-
    # resident points and tetrahedra, and host points to host tetrahedra
    for c in range(8):
        tri.triangulate_device(d_pts[offs[c]:offs[c + 1]].data_ptr(), int(offs[c + 1] - offs[c]))
        tri.triangulate(clouds[c])
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(ext)
    for c in range(len(clouds)):
        tri.triangulate_device(d_pts[offs[c]:offs[c + 1]].data_ptr(), int(offs[c + 1] - offs[c]))
    e.record(ext)
    e.synchronize()
    single_dev_ms = s.elapsed_time(e)
    single_dev = len(clouds) / (single_dev_ms / 1e3)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(ext)
    for c in clouds:
        tri.triangulate(c)
    e.record(ext)
    e.synchronize()
    single_ms = s.elapsed_time(e)
    single = len(clouds) / (single_ms / 1e3)
    if rank == 0:
        line = {
            "metric": "clouds/s, 4096-cloud batch to bit-exact 3D DT on 1 B200", "value": round(value, 1),
            "unit": "clouds/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(statistics.mean(ms), 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(cfg, points=int(offs[-1]), grid="autotuned per (size bucket, distribution)",
                           l2="256 MB buffer written between timed steps; inputs 737 MB"),
            "e2e": {"value": round(e2e, 1), "unit": "clouds/s", "h2d_bytes_per_step": int(offs[-1]) * 24,
                    "d2h_bytes_per_step": int(ntet) * 32},
            "one_call_per_cloud": {"value": round(single_dev, 1), "unit": "clouds/s",
                                   "ms": round(single_dev_ms, 1),
                                   "api": "device-resident points and tetrahedra, one call per cloud"},
            "one_call_per_cloud_e2e": {"value": round(single, 1), "unit": "clouds/s", "ms": round(single_ms, 1),
                                       "api": "host points in, host tetrahedra out, one call per cloud"},
            "batched_over_one_call_per_cloud": round(value / single_dev, 2),
            "batched_over_one_call_per_cloud_e2e": round(e2e / single, 2),
            "splay": {"loops_max": st["loops"], "insertions": st["splay_insertions"], "tets": int(ntet),
                      "large_stars": st["large_stars"]},
            "stages_ms": {k: round(st[k], 3) for k in ("t_init_ms", "t_pba_ms", "t_star_ms", "t_splay_ms",
                                                        "t_out_ms", "t_total_ms")},
            "clocks": clocks, "gpu_launches": int(st["gpu_launches"]),
        }
        print(json.dumps(line))
    tri.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed1m", choices=sorted(WORKLOADS))
    ap.add_argument("--points", type=int, default=None)
    ap.add_argument("--grid", type=int, default=None)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
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
    args.points = args.points or cfg["points"]
    args.grid = args.grid or cfg["grid"]
    cfg["points"], cfg["grid"] = args.points, args.grid
    pts, _ = workloads.config_cloud(args.workload, scale=args.points / WORKLOADS[args.workload]["points"],
                                    seed=cfg["seed"] + rank)
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

    # ---- device throughput (value) ----
    for _ in range(args.warmup):
        tri.triangulate_device(d_pts.data_ptr(), n)
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    step_ms, pba_ms, launches, ntets = [], [], 0, 0
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(ext)
        _, ntets, st = tri.triangulate_device(d_pts.data_ptr(), n)
        e.record(ext)
        e.synchronize()
        step_ms.append(s.elapsed_time(e))
        pba_ms.append(st["t_pba_ms"])
        launches += st["gpu_launches"]
        last = st
    barrier()
    clocks = sampler.stop()
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * n * args.steps / (total_ms / 1e3) / 1e6

    # ---- learned star proposal: trained (untimed) on another seeded cloud of the
    # same distribution with labels from the plain method, then timed like value
    learned = None
    if not args.no_learned:
        train_pts, _ = workloads.config_cloud(args.workload, scale=args.points / WORKLOADS[args.workload]["points"],
                                              seed=cfg["seed"] + 1000 + rank)
        with gstar4d_b200.Triangulator(grid_size=args.grid, device=local) as tt:
            t0 = time.perf_counter()
            loss = tt.train_proposal(train_pts, epochs=4, lr=2e-3)
            train_s = time.perf_counter() - t0
            weights = tt.proposal_weights()
        tl = gstar4d_b200.Triangulator(grid_size=args.grid, device=local, proposal=1)
        tl.proposal_weights(weights)
        extl = torch.cuda.ExternalStream(tl.stream, device=local)
        for _ in range(args.warmup):
            tl.triangulate_device(d_pts.data_ptr(), n)
        barrier()
        lms = []
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(extl)
            _, ntl, stl = tl.triangulate_device(d_pts.data_ptr(), n)
            e.record(extl)
            e.synchronize()
            lms.append(s.elapsed_time(e))
        barrier()
        lt = sum(lms)
        if world > 1:
            tt_ = torch.tensor([lt], device=f"cuda:{local}")
            dist.all_reduce(tt_, op=dist.ReduceOp.MAX)
            lt = float(tt_.item())
        learned = {"value": round(world * n * args.steps / (lt / 1e3) / 1e6, 3), "unit": "Mpts/s",
                   "ms_per_step": round(lt / args.steps, 3), "tets": ntl,
                   "star_insertions_per_point": round(stl["star_insertions"] / n, 3),
                   "splay_insertions_per_point": round(stl["splay_insertions"] / n, 3),
                   "proposed_per_point": round(stl["proposed"] / n, 3), "loops": stl["loops"],
                   "stages_ms": {k: round(stl[k], 3) for k in ("t_pba_ms", "t_star_ms", "t_splay_ms", "t_out_ms")},
                   "training": {"cloud": "same distribution, seed + 1000", "epochs": 4, "final_loss": round(loss, 4),
                                "seconds": round(train_s, 2)}}
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
    e2e_ms = []
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(ext)
        tets, _, _ = tri.triangulate(pts_np, out=out_np)
        e.record(ext)
        e.synchronize()
        e2e_ms.append(s.elapsed_time(e))
    e2e_total = sum(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e_total], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e = world * n * args.steps / (e2e_total / 1e3) / 1e6

    if rank == 0:
        peak, peak_kind = _peaks()
        G = args.grid
        alg_bytes = 20.0 * G ** 3
        pba_avg = statistics.mean(pba_ms)
        achieved = alg_bytes / (pba_avg / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mpts/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(cfg, l2="256 MB buffer written between timed steps", parallelism="replicas"),
            "e2e": {"value": round(e2e, 3), "unit": "Mpts/s", "h2d_bytes_per_step": int(n * 24),
                    "d2h_bytes_per_step": int(len(tets) * 32)},
            "roofline": {"kernel": "pba (z,y,x passes)", "bound": "hbm", "achieved": round(achieved, 1),
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": _pba_traffic(G), "traffic_source": "profiles/pba_mixed100k_g512.md (ncu)",
                         "algorithmic_bytes": alg_bytes, "avg_ms": round(pba_avg, 4)},
            "stages_ms": {k: round(last[k], 3) for k in ("t_init_ms", "t_pba_ms", "t_star_ms", "t_splay_ms",
                                                          "t_out_ms", "t_total_ms")},
            "splay": {"loops": last["loops"], "star_insertions_per_point": round(last["star_insertions"] / n, 3),
                      "splay_insertions_per_point": round(last["splay_insertions"] / n, 3),
                      "proofs": last["proofs"], "exact_predicates": last["exact_predicates"],
                      "large_stars": last["large_stars"], "tets": ntets},
            "learned_proposal": learned,
            "clocks": clocks,
            "gpu_launches": int(launches),
        }
        if not args.no_cpu and world == 1:  # the CPU baseline is an N=1 figure
            threads = os.cpu_count() or 1
            v, t, ns = cpu_run(1, threads)
            line["cpu_baseline"] = {"value": round(v, 4), "unit": "Mpts/s", "cores": threads, "kind": "port",
                                    "sample": "%d-point mixed cloud at grid %d^3 (same distribution and voxel "
                                              "density), one run" % (ns, SAMPLE_GRID)}
        print(json.dumps(line))
    tri.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
