"""Benchmark of the BVH build-and-trace hot path (one JSON line on rank 0).

Default workload: the 1M-triangle displaced sphere (1024x512 UV sphere, 1,046,528 triangles, radius 1 with
4-octave value-noise displacement 0.05) and 4M rays from a radius-3 sphere into the inward hemisphere;
PLOC r = 16 over 30-bit Morton codes, binary FP32 BVH, closest hit with the reference-exact leaf test.

A step = one build over the resident triangles + one closest-hit trace of the resident rays.
  value          build throughput, Mtri/s (triangles / build time, CUDA events on the build stream)
  trace          closest-hit throughput, Mrays/s (CUDA events around the trace launch)
  e2e            the same step through the public API with HOST inputs: pinned vertex arrays copied in,
                 build, rays copied in, trace, hits copied out; Mtri/s over the whole step
  roofline       build pipeline against HBM (algorithmic bytes per triangle from the byte model in
                 DESIGN.md, over the measured build time), plus the trace kernel's own roofline
  cpu_baseline   the reference's SBvh::Build + SBvh::Intersect (oracle/_ref, compiled from the
                 reference's sources) on the host cores, on a bounded sample of the same workload

--impl reference runs only the reference CPU implementation on the same workload and prints its line.
Multi-GPU (torchrun): replicas only; every rank builds and traces its own copy (weak scaling).
"""
from __future__ import annotations

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

METRIC = "PLOC build Mtri/s + closest-hit Mrays/s on 1 B200; batched vs plain; SAH cost"
HBM_FALLBACK_GBS = 6650.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """Samples SM clocks and clock-event (throttle) reasons through NVML while the timed region runs.

    NVML reads take about a millisecond, so even a timed region of a few tens of milliseconds gets a few
    dozen samples (nvidia-smi itself takes ~100 ms per query). Falls back to nvidia-smi when NVML is absent.
    """

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, index, period_s=0.01):
        self.index = index
        self.period = period_s
        self.samples = []  # (sm_mhz, max_mhz, reason_bits)
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        self._h = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            h = None
            try:
                pr = torch.cuda.get_device_properties(index)
                bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self._nvml, self._h = pynvml, h
        except Exception:
            self._nvml = None

    def _sample(self):
        if self._nvml is not None:
            n = self._nvml
            sm = n.nvmlDeviceGetClockInfo(self._h, n.NVML_CLOCK_SM)
            mx = n.nvmlDeviceGetMaxClockInfo(self._h, n.NVML_CLOCK_SM)
            rs = n.nvmlDeviceGetCurrentClocksEventReasons(self._h)
            return float(sm), float(mx), int(rs)
        out = subprocess.run(["nvidia-smi", "-i", str(self.index),
                              "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active",
                              "--format=csv,noheader,nounits"], capture_output=True, text=True,
                             timeout=5).stdout.strip()
        a = [x.strip() for x in out.split(",")]
        return float(a[0]), float(a[1]), int(a[2], 16)

    def _run(self):
        while True:
            try:
                self.samples.append(self._sample())
            except Exception:
                pass
            if self._stop.wait(self.period):
                break

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [s[0] for s in self.samples]
        reasons = sorted({name for s in self.samples for name, bit in self.REASONS if s[2] & bit})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": reasons, "samples": len(self.samples),
                "source": "nvml" if self._nvml is not None else "nvidia-smi"}


def workload(name, rays_override=None):
    from diplodocus_b200 import scenes as S
    if name == "displaced_sphere":
        tris, rays = S.displaced_sphere(n_rays=rays_override or 4 * 1024 * 1024)
        desc = "1024x512 displaced UV sphere (1,046,528 tris), 4M inward-hemisphere rays from r=3"
    elif name == "small":
        tris, rays = S.small_scene()
        desc = "open box + 64x32 sphere (3,978 tris), 512x512 pinhole primary rays"
    elif name == "soup16m":
        tris = S.soup(16 * 1024 * 1024, seed=3)
        rays = S.random_rays(rays_override or 16 * 1024 * 1024, seed=3)
        desc = "16M log-normal triangle soup, 16M random rays"
    else:
        raise SystemExit(f"unknown workload {name}")
    return tris, rays, desc


# ---------------------------------------------------------------------------------------------------
# Reference arm: the reference's own CPU code (SBvh) on the host cores.
# ---------------------------------------------------------------------------------------------------
def cpu_reference_step_stats(tris, rays, sample_rays, threads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ref = O.RefOracle()
    t0 = time.perf_counter()
    sb = ref.sbvh(tris)
    build_s = time.perf_counter() - t0
    idx = np.linspace(0, len(rays) - 1, sample_rays).astype(np.int64)
    sample = np.ascontiguousarray(rays[idx])
    t0 = time.perf_counter()
    sb.trace(sample, threads=threads)
    trace_s = time.perf_counter() - t0
    sah = sb.sah_cost()[0]
    sb.close()
    return build_s, trace_s, sah


def run_reference(args, rank, world):
    if rank != 0:
        return
    tris, rays, desc = workload(args.workload, args.rays)
    threads = os.cpu_count() or 1
    sample_rays = min(len(rays), args.ref_sample_rays)
    for _ in range(args.warmup if args.warmup <= 1 else 1):
        cpu_reference_step_stats(tris, rays[:4096], 4096, threads)
    builds, traces = [], []
    sah = None
    for _ in range(args.steps):
        b, t, sah = cpu_reference_step_stats(tris, rays, sample_rays, threads)
        builds.append(b)
        traces.append(t)
    n = len(tris)
    value = n / np.mean(builds) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "Mtri/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * (np.mean(builds) + np.mean(traces)), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "description": desc, "triangles": n, "rays": len(rays),
                   "build": "SBvh binned SAH (bin_count 16, leaf < 4, depth 32)"},
        "trace": {"value": round(sample_rays / np.mean(traces) / 1e6, 4), "unit": "Mrays/s",
                  "sample_rays": sample_rays},
        "sah_cost": round(sah, 4),
        "cpu_baseline": {"value": round(value, 4), "unit": "Mtri/s", "cores": 1, "kind": "reference",
                         "sample": f"SBvh::Build of all {n} triangles on 1 thread (it is single-threaded); "
                                   f"SBvh::Intersect of {sample_rays} of {len(rays)} rays on {threads} threads"},
        "e2e": {"value": round(value, 4), "unit": "Mtri/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------------
# GPU arm.
# ---------------------------------------------------------------------------------------------------
# DRAM bytes (read + write) of one build and of one 4M-ray closest-hit trace of the default workload, from ncu
# captures (dram__bytes_read.sum + dram__bytes_write.sum, summed over the build's kernels and over the trace's
# two kernels): profiles/dram_traffic_displaced_sphere_1m.md, profiles/trace_kernel_displaced_sphere_1m.md.
# Other workloads report null.
MEASURED_TRAFFIC = {"displaced_sphere": {"build": 526.72e6, "trace": 348.9e6, "rays": 4194304,
                                         "triangles": 1046528}}


def measured_traffic(workload, kind, n_tri, n_rays):
    m = MEASURED_TRAFFIC.get(workload)
    if not m or m["triangles"] != n_tri or m["rays"] != n_rays:
        return None
    return m[kind]


def max_over_ranks(values, world, device=None):
    """Per-rank device times -> their maximum over all ranks (every rank gets it; identity when world == 1).
    The job's time is its slowest replica's."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def build_bytes_per_tri(code_type, digit_bits=8, node_bytes_per_tri=None):
    """Algorithmic bytes of one build per triangle (byte model, Morton30: 176 B, EMC60: 308 B)."""
    k = 4 if code_type == 0 else 8
    passes = -(-(30 if code_type == 0 else 60) // 8)
    node = 64.0 if node_bytes_per_tri is None else node_bytes_per_tri
    return 36 + (k + 4) + passes * 2 * (k + 4) + node + 4


def run_gpu(args, rank, world, local_rank):
    import ctypes as C

    import torch
    import torch.distributed as dist

    from diplodocus_b200 import _lib as L
    from diplodocus_b200 import accel as A

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = L.load()
    tris, rays_np, desc_txt = workload(args.workload, args.rays)
    n, nr = len(tris), len(rays_np)
    kind = {"morton30": A.AccelerationStructureType.kPloc, "emc60": A.AccelerationStructureType.kPlocEmc}[args.code]
    cfg = A.AccelerationStructureConfig(kind, nn_search_radius=args.radius, leaf_test=args.leaf_test)
    v = A.soa_vertices(tris, dev)
    rays = A.as_device_rays(rays_np, dev)
    hits = torch.empty((nr, 4), dtype=torch.int32, device=dev)
    desc = A.make_desc(*v, cfg)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    lt = A._leaf_test(args.leaf_test)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > L2 (126 MB)

    def step(ev=None):
        h = C.c_void_p(0)
        if ev is not None:
            ev[0].record(stream)
        L.check(lib.dipl_bvh_build(C.byref(desc), C.byref(h), sp), "dipl_bvh_build")
        if ev is not None:
            ev[1].record(stream)
        L.check(lib.dipl_bvh_trace_closest(h, C.c_void_p(rays.data_ptr()), nr, C.c_void_p(hits.data_ptr()), lt, 0,
                                           sp), "dipl_bvh_trace_closest")
        if ev is not None:
            ev[2].record(stream)
        return h

    def destroy(h):
        lib.dipl_bvh_destroy(h)

    for _ in range(args.warmup):
        destroy(step())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    launches0 = lib.dipl_kernel_launch_count()
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        wall0 = time.perf_counter()
        for k in range(args.steps):
            flush.zero_()  # L2 flushed between steps; outside the events
            h = step(evs[k])
            destroy(h)
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
    launches = lib.dipl_kernel_launch_count() - launches0
    build_ms = [e[0].elapsed_time(e[1]) for e in evs]
    trace_ms = [e[1].elapsed_time(e[2]) for e in evs]
    step_ms = [e[0].elapsed_time(e[2]) for e in evs]
    t_step = float(np.sum(step_ms))
    t_build = float(np.sum(build_ms))
    t_trace = float(np.sum(trace_ms))
    t_step, t_build, t_trace = max_over_ranks([t_step, t_build, t_trace], world, dev)

    # SAH cost and info of one build (outside the timed region)
    h = step()
    sah = C.c_double(0)
    lib.dipl_bvh_sah_cost(h, C.byref(sah), sp)
    info = L.BvhInfo()
    lib.dipl_bvh_get_info(h, C.byref(info))
    # counted trace for the trace byte model (same kernel, same rays)
    ctr = torch.zeros(2, dtype=torch.int64, device=dev)
    lib.dipl_bvh_trace_closest_counted(h, C.c_void_p(rays.data_ptr()), nr, C.c_void_p(hits.data_ptr()), lt, 0,
                                       C.c_void_p(ctr.data_ptr()), sp)
    torch.cuda.synchronize()
    visits, tests = [int(x) for x in ctr.cpu().tolist()]
    hit_rate = float((hits[:, 0] >= 0).float().mean().item())
    destroy(h)

    # ---- e2e through the public API with host buffers -------------------------------------------------
    # Every step copies its inputs from pinned host memory and its hits back, as a user tracing frame after
    # frame would: uploads on a copy stream into one of two device input sets (step k+1's uploads overlap
    # step k's build and trace), build and trace on the compute stream, hit downloads on a third stream.
    host_v = [x.cpu().pin_memory() for x in v]
    host_rays = rays.cpu().pin_memory()
    host_hits = [torch.empty((nr, 4), dtype=torch.int32).pin_memory() for _ in range(2)]
    sets = [{"v": [torch.empty_like(x) for x in v], "rays": torch.empty_like(rays), "hits": torch.empty_like(hits)}
            for _ in range(2)]
    edescs = [A.make_desc(*st_["v"], cfg) for st_ in sets]
    copy_s, d2h_s = torch.cuda.Stream(), torch.cuda.Stream()
    ev_v = [torch.cuda.Event() for _ in range(2)]
    ev_r = [torch.cuda.Event() for _ in range(2)]
    ev_done = [torch.cuda.Event() for _ in range(2)]

    def upload(k):
        b = k % 2
        if k >= 2:
            copy_s.wait_event(ev_done[b])  # step k-2 no longer reads this input set
        with torch.cuda.stream(copy_s):
            for d_, h_ in zip(sets[b]["v"], host_v):
                d_.copy_(h_, non_blocking=True)
            ev_v[b].record(copy_s)
            sets[b]["rays"].copy_(host_rays, non_blocking=True)
            ev_r[b].record(copy_s)

    def compute_download(k):
        b = k % 2
        stream.wait_event(ev_v[b])
        hh = C.c_void_p(0)
        L.check(lib.dipl_bvh_build(C.byref(edescs[b]), C.byref(hh), sp), "dipl_bvh_build")
        stream.wait_event(ev_r[b])
        L.check(lib.dipl_bvh_trace_closest(hh, C.c_void_p(sets[b]["rays"].data_ptr()), nr,
                                           C.c_void_p(sets[b]["hits"].data_ptr()), lt, 0, sp),
                "dipl_bvh_trace_closest")
        ev_done[b].record(stream)
        d2h_s.wait_event(ev_done[b])
        with torch.cuda.stream(d2h_s):
            host_hits[b].copy_(sets[b]["hits"], non_blocking=True)
        destroy(hh)

    def e2e_run(steps_):
        upload(0)
        for k in range(steps_):
            if k + 1 < steps_:
                upload(k + 1)
            compute_download(k)

    e2e_run(2)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(copy_s)
    e2e_run(args.steps)
    d2h_s.wait_stream(stream)
    d2h_s.wait_stream(copy_s)
    e1.record(d2h_s)
    torch.cuda.synchronize()
    t_e2e = e0.elapsed_time(e1)
    (t_e2e,) = max_over_ranks([t_e2e], world, dev)
    h2d = sum(x.numel() * 4 for x in v) + rays.numel() * 4
    d2h = hits.numel() * 4

    if rank != 0:
        return
    peak, peak_kind = peaks()
    steps = args.steps
    build_s = t_build / 1e3 / steps
    trace_s = t_trace / 1e3 / steps
    bpt = build_bytes_per_tri(desc.code_type, 8, info.node_bytes / max(n, 1))
    achieved_build = bpt * n / build_s / 1e9
    ray_bytes = 32 + 16 + (visits / nr) * 64 + (tests / nr) * 36
    achieved_trace = ray_bytes * nr / trace_s / 1e9
    value = world * n / build_s / 1e6
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mtri/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": round(t_step / steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "description": desc_txt, "triangles": n, "rays": nr,
                   "code": args.code, "nn_search_radius": args.radius, "leaf_test": args.leaf_test,
                   "layout": "binary", "max_triangles_per_leaf": 4, "l2": "flushed between steps (256 MB write)",
                   "parallelism": f"replicas x{world}"},
        "trace": {"value": round(world * nr / trace_s / 1e6, 3), "unit": "Mrays/s", "hit_rate": round(hit_rate, 4),
                  "node_visits_per_ray": round(visits / nr, 3), "tri_tests_per_ray": round(tests / nr, 3)},
        "build_ms": round(build_s * 1e3, 4), "trace_ms": round(trace_s * 1e3, 4),
        "sah_cost": round(sah.value, 4), "ploc_iterations": int(info.ploc_iterations), "bvh_depth": int(info.depth),
        "roofline": {"bound": "hbm", "achieved": round(achieved_build, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved_build / peak, 4),
                     "traffic": measured_traffic(args.workload, "build", n, nr) if args.code == "morton30" else None,
                     "kernel": "build pipeline (bounds, codes, sort, PLOC, layout)",
                     "traffic_note": "bytes per build from one ncu capture (cold caches per kernel), "
                                     "profiles/dram_traffic_displaced_sphere_1m.md",
                     "bytes_per_unit": round(bpt, 1), "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"},
        "roofline_trace": {"bound": "hbm", "achieved": round(achieved_trace, 1), "peak": peak, "unit": "GB/s",
                           "frac": round(achieved_trace / peak, 4), "bytes_per_ray": round(ray_bytes, 1),
                           "traffic": measured_traffic(args.workload, "trace", n, nr)
                           if args.leaf_test == "ref_mt" and args.code == "morton30" else None},
        "e2e": {"value": round(world * n * steps / (t_e2e / 1e3) / 1e6, 3), "unit": "Mtri/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "note": "whole step per triangle: H2D vertices and rays from pinned memory, build, trace, D2H "
                        "hits; uploads on a copy stream overlap the previous step's build and trace (two device "
                        "input sets), downloads on a third stream"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "wall_s_timed_region": round(wall, 4),
    }
    if not args.no_cpu_baseline and world == 1:
        threads = os.cpu_count() or 1
        sample_rays = min(nr, args.ref_sample_rays)
        try:
            b, t, rsah = cpu_reference_step_stats(tris, rays_np, sample_rays, threads)
            line["cpu_baseline"] = {"value": round(n / b / 1e6, 4), "unit": "Mtri/s", "cores": 1, "kind": "reference",
                                    "sample": f"one SBvh::Build of all {n} triangles (1 thread); SBvh::Intersect of "
                                              f"{sample_rays} rays on {threads} threads: "
                                              f"{sample_rays / t / 1e6:.3f} Mrays/s",
                                    "trace_mrays_per_s": round(sample_rays / t / 1e6, 4),
                                    "trace_threads": threads, "sah_cost": round(rsah, 4)}
        except Exception as e:  # the harness is absent when it was never built here
            line["cpu_baseline"] = {"value": None, "unit": "Mtri/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    print(json.dumps(line), flush=True)




# ---------------------------------------------------------------------------------------------------
# The other configured workloads (one JSON line each; the default line above is the contract's).
# ---------------------------------------------------------------------------------------------------
def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _time(fn, reps, warm=2):
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    a, b = _events()
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def _line(workload, value, unit, extra):
    d = {"metric": METRIC, "workload": workload, "value": round(value, 4), "unit": unit, "n_gpus": 1,
         "higher_is_better": True, "dtype": "f32", "data": "synthetic"}
    d.update(extra)
    print(json.dumps(d), flush=True)


def run_small(args):
    """Small scene as a frame of the renderer path, all on the device: pinhole primary rays, closest hits, one
    cosine bounce per hit, bounce hits (the GPU frontend). Agreement classes of the frame's rays against the
    reference's SBvh and brute force."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from diplodocus_b200 import accel as A
    from diplodocus_b200 import scenes as S
    tris, _ = S.small_scene(width=8, height=8)
    w = h = 512
    cam = dict(S.SMALL_CAMERA)
    ref = O.RefOracle()
    sb = ref.sbvh(tris)
    bvh = A.GpuPlocBvh().Build(A.AccelerationStructureConfig(), A.Stats(), torch.from_numpy(tris))
    prim_rays, hits, bounce, bhits = A.trace_frame(bvh, cam, w, h, seed=11)
    hit = (hits.prim >= 0).cpu().numpy()
    rays = np.concatenate([prim_rays.cpu().numpy(), bounce.cpu().numpy()[hit]])
    gp = np.concatenate([hits.prim.cpu().numpy(), bhits.prim.cpu().numpy()[hit]])
    gt = np.concatenate([hits.t.cpu().numpy(), bhits.t.cpu().numpy()[hit]])
    ms_build = _time(lambda: A.GpuPlocBvh().Build(A.AccelerationStructureConfig(), A.Stats(), torch.from_numpy(tris)), 10)
    ms_frame = _time(lambda: A.trace_frame(bvh, cam, w, h, 11), 20)
    hs = sb.trace(rays)
    hb = ref.brute(tris, rays)
    exact = (gp == hb.prim) & (gt.view(np.uint32) == hb.t.view(np.uint32))
    vs_sbvh_same = gp == hs.prim
    diff = ~vs_sbvh_same
    sb_t = np.where(hs.prim >= 0, hs.t, np.inf)
    s_class = diff & exact & (sb_t >= gt)  # SBvh missed or took a farther/later-tied hit that brute force beats
    _line("small", len(tris) / ms_build / 1e3, "Mtri/s", {
        "config": {"workload": "small", "triangles": len(tris), "rays": len(rays),
                   "rays_detail": "512x512 pinhole primary rays + one cosine bounce per primary hit, generated "
                                  "and traced on the device (one frame)"},
        "build_ms": round(ms_build, 4),
        "frame": {"ms": round(ms_frame, 4), "rays": len(rays), "value": round(len(rays) / ms_frame / 1e3, 2),
                  "unit": "Mrays/s", "steps": "generate primary, trace, generate bounce, trace"},
        "sah_cost": round(bvh.sah_cost(), 4), "sbvh_sah_cost": round(sb.sah_cost()[0], 4),
        "agreement_vs_brute_force": {"E_or_T_bit_exact": int(exact.sum()), "F": int((~exact).sum())},
        "agreement_vs_sbvh": {"same_id": int(vs_sbvh_same.sum()), "S_sbvh_wrong": int(s_class.sum()),
                              "F": int((diff & ~s_class).sum())},
        "sbvh_build_ms": round(sb.build_ms, 3)})


def write_obj_scene(dirpath, name="sphere_room"):
    """A Cornell-style OBJ scene of ~1M triangles as the reference's app would load it: the 1024x512 displaced
    sphere as an indexed mesh (shared vertices), a floor quad, an emissive lamp quad, an MTL file and a .meta
    camera. Coordinates are written with 9 significant digits, so they read back to the same float32."""
    from diplodocus_b200 import scenes as S
    tris, _ = S.displaced_sphere(n_rays=16)
    flat = tris.reshape(-1, 3)
    verts, inv = np.unique(flat, axis=0, return_inverse=True)
    faces = inv.reshape(-1, 3) + 1
    os.makedirs(dirpath, exist_ok=True)
    with open(os.path.join(dirpath, name + ".obj"), "w") as f:
        f.write("mtllib %s.mtl\ng floor\nusemtl floor\n" % name)
        f.write("v -4 -1.2 -4\nv 4 -1.2 -4\nv 4 -1.2 4\nv -4 -1.2 4\nf -4 -3 -2 -1\n")
        f.write("g lamp\nusemtl lamp\nv -0.5 2.5 -0.5\nv 0.5 2.5 -0.5\nv 0.5 2.5 0.5\nv -0.5 2.5 0.5\n"
                "f -1 -2 -3 -4\ng sphere\nusemtl sphere\n")
        np.savetxt(f, verts, fmt="v %.9g %.9g %.9g")
        np.savetxt(f, faces + 8, fmt="f %d %d %d")
    with open(os.path.join(dirpath, name + ".mtl"), "w") as f:
        f.write("newmtl floor\nKd 0.7 0.7 0.7\nnewmtl lamp\nKd 0.8 0.8 0.8\nKe 12 12 11\n"
                "newmtl sphere\nKd 0.6 0.3 0.2\nKs 0.1 0.1 0.1\nNs 20\n")
    with open(os.path.join(dirpath, name + ".meta"), "w") as f:
        f.write("cam_pos 0 0.2 -3.5\ncam_dir 0 -0.05 1\ncam_up 0 1 0\ncam_fov 0.9\ncam_far 100\n"
                "point_light 0 2 -1 1 1 1 50\n")
    return name, len(tris) + 4, os.path.getsize(os.path.join(dirpath, name + ".obj"))


def run_obj_scene(args):
    """OBJ scene path end to end: the reference's scene files (OBJ + MTL + .meta) -> the library's host loader
    -> host-to-device copy -> PLOC build -> one device frame (pinhole + bounce), beside the reference's own
    ObjSceneLoader and SBvh build on the same files."""
    import tempfile

    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from diplodocus_b200 import accel as A
    from diplodocus_b200 import scene_io as SI
    d = tempfile.mkdtemp(prefix="dipl_obj_")
    name, n, size = write_obj_scene(d)
    w = h = 512

    def best(fn, k):
        out = 1e30
        for _ in range(k):
            t0 = time.perf_counter()
            fn()
            out = min(out, time.perf_counter() - t0)
        return out * 1e3

    ms_load = best(lambda: SI.load_obj_scene(d, name), 3)
    sc = SI.load_obj_scene(d, name)
    host = torch.from_numpy(sc.triangles()).pin_memory()
    dev = torch.empty_like(host, device="cuda")
    ms_h2d = _time(lambda: dev.copy_(host, non_blocking=True), 5)
    cfg = A.AccelerationStructureConfig()
    ms_build = _time(lambda: A.GpuPlocBvh().Build(cfg, A.Stats(), dev), 5)
    bvh = A.GpuPlocBvh().Build(cfg, A.Stats(), dev)
    cam = sc.camera.as_dict()
    ms_frame = _time(lambda: A.trace_frame(bvh, cam, w, h, 3), 10)
    stats = A.Stats()
    rays, hits, bounce, bhits = A.trace_frame(bvh, cam, w, h, 3, stats=stats)
    n_rays = w * h + stats.rt_stats.secondary_ray_count

    def e2e():
        s2 = SI.load_obj_scene(d, name)
        t = torch.from_numpy(s2.triangles()).cuda()
        b = A.GpuPlocBvh().Build(cfg, A.Stats(), t)
        A.trace_frame(b, s2.camera.as_dict(), w, h, 3)
        torch.cuda.synchronize()
    ms_e2e = best(e2e, 3)
    ref = O.RefOracle()
    ms_ref_load = best(lambda: ref.obj_scene(d, name), 2)
    sb = ref.sbvh(sc.triangles())
    ms_ref_build = sb.build_ms
    sb.close()
    _line("obj_scene", n / (ms_load + ms_h2d + ms_build) / 1e3, "Mtri/s", {
        "config": {"workload": "obj_scene", "triangles": n, "obj_bytes": size, "frame": f"{w}x{h} pinhole + bounce",
                   "description": "indexed OBJ: 1024x512 displaced sphere + floor + emissive lamp, MTL, .meta"},
        "value_note": "scene file to device BVH: host load + host-to-device copy + PLOC build",
        "load_ms": round(ms_load, 2), "load_mtri_s": round(n / ms_load / 1e3, 2),
        "h2d_ms": round(ms_h2d, 3), "build_ms": round(ms_build, 3),
        "frame": {"ms": round(ms_frame, 4), "rays": n_rays, "value": round(n_rays / ms_frame / 1e3, 2),
                  "unit": "Mrays/s"},
        "e2e": {"ms": round(ms_e2e, 2), "value": round(n / ms_e2e / 1e3, 3), "unit": "Mtri/s",
                "steps": "load file, copy to the device, build, one frame, synchronise"},
        "host_threads": os.cpu_count(),
        "cpu_baseline": {"kind": "reference", "value": round(n / (ms_ref_load + ms_ref_build) / 1e3, 3),
                         "unit": "Mtri/s", "cores": 1,
                         "sample": "ObjSceneLoader::Load of the same files + SBvh::Build (1 thread)",
                         "load_ms": round(ms_ref_load, 2), "sbvh_build_ms": round(ms_ref_build, 2)}})


def run_soup16m(args):
    """16M soup: EMC60+SOBB and the 8-wide quantised form against binary FP32 nodes; t/u/v error vs FP64."""
    import torch
    from diplodocus_b200 import accel as A
    from diplodocus_b200 import scenes as S
    n = args.soup_tris
    tris = S.soup(n, seed=3)
    nr = args.rays or (1 << 24)
    rays = torch.from_numpy(S.random_rays(nr, seed=3)).cuda()
    tt = torch.from_numpy(tris).cuda()  # resident in HBM: the timed builds exclude host->device copies
    v = A.soa_vertices(tt)
    lib = __import__("diplodocus_b200._lib", fromlist=["x"]).load()
    import ctypes as C
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def build_only(desc):
        h = C.c_void_p(0)
        lib.dipl_bvh_build(C.byref(desc), C.byref(h), sp)
        lib.dipl_bvh_destroy(h)

    peak, _ = peaks()
    out = {}
    ref_prim = None
    for name, kind, layout in [("ploc_binary", A.AccelerationStructureType.kPloc, "binary"),
                               ("ploc_emc", A.AccelerationStructureType.kPlocEmc, "binary"),
                               ("ploc_emc_sobb", A.AccelerationStructureType.kPlocEmcSobb, "binary"),
                               ("ploc_wide8_q8", A.AccelerationStructureType.kPloc, "wide8_q8")]:
        cfg = A.AccelerationStructureConfig(kind, layout=layout)
        bvh = A.GpuPlocBvh().Build(cfg, A.Stats(), tt)
        desc = A.make_desc(*v, cfg)
        ms_build = _time(lambda: build_only(desc), 3, warm=1)
        ms_trace = _time(lambda: bvh.Intersect(A.Stats(), rays), 2, warm=1)
        st = A.Stats()
        h = bvh.Intersect(st, rays, count=True)  # same kernel with visit counters, same rays
        visits, tests = st.accel_stats.traversal_count / nr, st.accel_stats.intersection_count / nr
        prim = h.prim.cpu().numpy()
        if ref_prim is None:
            ref_prim = prim
        tuv = A.reintersect_f64(bvh._v, rays, h).cpu().numpy()
        hit = prim >= 0
        t32 = h.t.cpu().numpy()[hit].astype(np.float64)
        u32 = h.u.cpu().numpy()[hit].astype(np.float64)
        rel_t = np.abs(t32 - tuv[hit, 0]) / np.maximum(np.abs(tuv[hit, 0]), 1e-30)
        info = bvh.info()
        node_size = info.node_bytes / max(info.num_inner_nodes, 1)
        ray_bytes = 32 + 16 + visits * node_size + tests * 36
        achieved = ray_bytes * nr / (ms_trace / 1e3) / 1e9
        out[name] = {"build_ms": round(ms_build, 3), "build_mtri_s": round(n / ms_build / 1e3, 1),
                     "trace_mrays_s": round(nr / ms_trace / 1e3, 2), "sah_cost": round(bvh.sah_cost(), 3),
                     "node_visits_per_ray": round(visits, 2), "tri_tests_per_ray": round(tests, 2),
                     "roofline_trace": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                                        "unit": "GB/s", "frac": round(achieved / peak, 4),
                                        "bytes_per_ray": round(ray_bytes, 1), "node_bytes": round(node_size, 1)},
                     "node_bytes": int(info.node_bytes), "same_hits_as_binary": float((prim == ref_prim).mean()),
                     "t_rel_err_vs_fp64": {"median": float(np.median(rel_t)), "p99": float(np.quantile(rel_t, 0.99)),
                                           "max": float(rel_t.max())},
                     "u_abs_err_vs_fp64_max": float(np.abs(u32 - tuv[hit, 1]).max())}
        del bvh
        torch.cuda.empty_cache()
    _line("soup16m", out["ploc_emc_sobb"]["build_mtri_s"], "Mtri/s", {
        "config": {"workload": "soup16m", "triangles": n, "rays": nr,
                   "description": "log-normal soup (mu=-6, sigma=1.5, 20% 1:50 skinny), random rays in the cube"},
        "variants": out})


def run_batched(args):
    """256 noise-displaced spheres (1k..2M triangles): one graph-replayed plan vs 256 sequential builds."""
    import torch
    from diplodocus_b200 import accel as A
    from diplodocus_b200 import scenes as S
    meshes = [torch.from_numpy(m) for m in S.batched_meshes(args.batch_count)]
    total = sum(m.shape[0] for m in meshes)
    cfg = A.AccelerationStructureConfig()
    verts = [A.soa_vertices(m) for m in meshes]
    descs = [A.make_desc(*v, cfg) for v in verts]
    lib = __import__("diplodocus_b200._lib", fromlist=["x"]).load()
    import ctypes as C

    def plain_all():
        for d in descs:
            h = C.c_void_p(0)
            lib.dipl_bvh_build(C.byref(d), C.byref(h), C.c_void_p(torch.cuda.current_stream().cuda_stream))
            lib.dipl_bvh_destroy(h)

    ms_plain = _time(plain_all, 2, warm=1)
    cache = os.path.join("/tmp", "dipl_tune_cache.jsonl")
    t0 = time.perf_counter()
    tuned, from_cache, tverts = A.autotune(cfg, meshes, cache)
    tune_s = time.perf_counter() - t0
    plan = A.BuildPlan(cfg, meshes, tuned_descs=tuned)
    del tverts
    ms_plan = _time(plan.launch, 5, warm=2)
    bvhs = plan.bvhs()
    nr = 65536
    rays = torch.from_numpy(S.sphere_inward_rays(nr, seed=4)).cuda()
    ms_tr = [_time(lambda b=b: b.Intersect(A.Stats(), rays), 2, warm=1) for b in bvhs[:: max(1, len(bvhs) // 16)]]
    # hit agreement between the plan's BVHs and plain builds on a few meshes
    agree = []
    for i in range(0, len(meshes), max(1, len(meshes) // 8)):
        ref = A.GpuPlocBvh().Build(cfg, A.Stats(), meshes[i])
        a = ref.Intersect(A.Stats(), rays).prim.cpu().numpy()
        b = bvhs[i].Intersect(A.Stats(), rays).prim.cpu().numpy()
        agree.append(float((a == b).mean()))
    d0 = tuned[0]
    _line("batched", total / ms_plan / 1e3, "Mtri/s", {
        "config": {"workload": "batched", "meshes": len(meshes), "triangles": int(total),
                   "sizes": "log-uniform 1k..2M per mesh", "rays_per_mesh": nr},
        "plan_graph_ms": round(ms_plan, 3), "sequential_plain_ms": round(ms_plain, 3),
        "speedup_batched_vs_plain": round(ms_plain / ms_plan, 3),
        "plain_mtri_s": round(total / ms_plain / 1e3, 1),
        "autotuned": {"radius": d0.nn_search_radius, "block": d0.ploc_block_size, "digits": d0.sort_digit_bits,
                      "from_cache": from_cache, "tune_s": round(tune_s, 2)},
        "trace_mrays_s_per_mesh_median": round(float(np.median([nr / t / 1e3 for t in ms_tr])), 2),
        "hit_agreement_plan_vs_plain": min(agree)})
    plan.close()


def run_diff(args):
    """Differentiation: 65k-triangle displaced sphere, 1024x1024 primary rays, forward + adjoint."""
    import torch
    from diplodocus_b200 import accel as A
    from diplodocus_b200 import scenes as S
    verts, idx, rays_np = S.diff_scene()
    tris = verts[idx].astype(np.float32)
    bvh = A.GpuPlocBvh().Build(A.AccelerationStructureConfig(), A.Stats(), torch.from_numpy(tris))
    rays = torch.from_numpy(rays_np).cuda()
    h = bvh.Intersect(A.Stats(), rays)
    g = torch.stack([torch.where(h.prim >= 0, 0.06 * h.t, torch.zeros_like(h.t)), torch.zeros_like(h.t),
                     torch.zeros_like(h.t)], 1)
    ms_fwd = _time(lambda: bvh.Intersect(A.Stats(), rays), 10)
    ms_adj = _time(lambda: A.trace_adjoint(bvh._v, rays, h, g), 10)
    nr = rays.shape[0]
    _line("diff", nr / ms_adj / 1e3, "Mrays/s", {
        "config": {"workload": "diff", "triangles": len(tris), "rays": nr},
        "forward_mrays_s": round(nr / ms_fwd / 1e3, 2), "adjoint_ms": round(ms_adj, 4),
        "hit_rate": float((h.prim >= 0).float().mean().item()),
        "check": "tests/test_gpu_forms.py::test_adjoint_matches_fp64_central_differences"})

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="dipl", choices=["dipl", "reference"])
    ap.add_argument("--workload", default="displaced_sphere",
                    choices=["displaced_sphere", "small", "soup16m", "batched", "diff", "obj_scene"])
    ap.add_argument("--soup-tris", type=int, default=16 * 1024 * 1024)
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--code", default="morton30", choices=["morton30", "emc60"])
    ap.add_argument("--radius", type=int, default=16)
    ap.add_argument("--leaf-test", default="ref_mt", choices=["ref_mt", "watertight"])
    ap.add_argument("--rays", type=int, default=None)
    ap.add_argument("--ref-sample-rays", type=int, default=1 << 18)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload in ("small", "soup16m", "batched", "diff", "obj_scene") and world == 1:
        import torch
        torch.cuda.set_device(local_rank)
        {"small": run_small, "soup16m": run_soup16m, "batched": run_batched, "diff": run_diff,
         "obj_scene": run_obj_scene}[args.workload](args)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
