"""Benchmark of the BVH build-and-trace hot path (one JSON line on rank 0).

Default workload: the 16M-triangle log-normal soup (16,777,216 triangles: centroids uniform in the unit cube,
edge lengths exp(N(-6, 1.5)), 20% skinny at 1:50, random orientation) and 16M random rays (origins in the cube,
directions uniform on the sphere, tmax = FLT_MAX); PLOC r = 16 over 60-bit extended Morton codes, binary FP32
BVH, closest hit with the reference-exact leaf test. ``--workload displaced_sphere`` runs the 1M displaced
sphere (1024x512 UV sphere, 4M rays from a radius-3 sphere into the inward hemisphere, 30-bit Morton codes).

A step = one build over the resident triangles + one closest-hit trace of the resident rays.
  value          build throughput, Mtri/s (triangles / build time, CUDA events on the build stream)
  trace          closest-hit throughput, Mrays/s (CUDA events around the trace launch)
  e2e            the same step through the public API with HOST inputs: pinned vertex arrays and rays copied in,
                 build, trace, hits copied out; Mtri/s over the whole step
  roofline       the step's dominant kernel against HBM (algorithmic bytes over its measured time);
                 roofline_build / roofline_trace give both
  variants       (soup) Morton30, EMC60 + SOBB and the 8-wide quantised layout on the same triangles and rays
  errors         (soup) FP32 t/u/v of the reference-exact and the watertight leaf test against an FP64
                 re-intersection of the same triangle, and FP64 re-intersection of the rays whose hits differ
  cpu_baseline   the reference's SBvh::Build (1 thread) and SBvh::Intersect (all host threads), compiled from
                 the reference's sources, on the same workload; with ``parity``, a ray sample checked bit for bit
                 against the reference's brute force (DummyAccelerationStucture::Intersect)

--impl reference runs only the reference CPU implementation (SBvh) on a bounded sample of the same workload.
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
L2_FLUSH_BYTES = 256 * 1024 * 1024  # > the 126 MB L2


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


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


# ---------------------------------------------------------------------------------------------------
# Workloads (seeded synthetic inputs of the configured shapes; no dataset is involved).
# ---------------------------------------------------------------------------------------------------
SOUP_TRIANGLES = 16 * 1024 * 1024
DEFAULT_CODE = {"soup16m": "emc60", "displaced_sphere": "morton30"}
# Pre-splitting of large triangles (percent more clustering leaves at most): the soup's log-normal tail of large
# triangles overlaps everywhere; the sphere's triangles are all alike (nothing would split).
DEFAULT_SPLIT = {"soup16m": 40, "displaced_sphere": 0}
# Ray order of the traces: the pre-split soup's random rays trace faster sorted by origin cell and direction octant
# (DIPL_TRACE_COHERENT_ORDER); the sphere's camera-like rays are faster as given (the sort costs more than it saves).
DEFAULT_ORDER = {"soup16m": "coherent", "displaced_sphere": "given"}


def trace_flags(args):
    order = args.trace_order or DEFAULT_ORDER.get(args.workload, "given")
    return 2 if order == "coherent" else 0  # DIPL_TRACE_COHERENT_ORDER


def workload(name, rays_override=None, soup_tris=SOUP_TRIANGLES):
    from diplodocus_b200 import scenes as S
    if name == "displaced_sphere":
        tris, rays = S.displaced_sphere(n_rays=rays_override or 4 * 1024 * 1024)
        desc = "1024x512 displaced UV sphere (1,046,528 tris), 4M inward-hemisphere rays from r=3"
    elif name == "soup16m":
        tris = S.soup(soup_tris, seed=3)
        rays = S.random_rays(rays_override or 16 * 1024 * 1024, seed=3)
        desc = (f"{soup_tris:,}-triangle log-normal soup (centroids U[0,1]^3, edges exp(N(-6,1.5)), 20% 1:50 "
                f"skinny, random orientation), {len(rays):,} random rays (origins in the cube, directions uniform)")
    else:
        raise SystemExit(f"unknown workload {name}")
    return tris, rays, desc


def ray_sample_index(n_rays, k):
    """Evenly spaced sample of k of the (seeded, random) rays."""
    k = min(int(k), int(n_rays))
    return np.linspace(0, n_rays - 1, k).astype(np.int64)


# ---------------------------------------------------------------------------------------------------
# Reference arm: the reference's own CPU code (SBvh) on the host cores.
# ---------------------------------------------------------------------------------------------------
def _ref_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def cpu_reference_step_stats(tris, rays, sample_rays, threads):
    O = _ref_oracle()
    ref = O.RefOracle()
    t0 = time.perf_counter()
    sb = ref.sbvh(tris)
    build_s = time.perf_counter() - t0
    sample = np.ascontiguousarray(rays[ray_sample_index(len(rays), sample_rays)])
    t0 = time.perf_counter()
    sb.trace(sample, threads=threads)
    trace_s = time.perf_counter() - t0
    sah = sb.sah_cost()[0]
    sb.close()
    return build_s, trace_s, sah


def run_reference(args, rank, world):
    """SBvh::Build on 1 host thread (it is single-threaded) per step, and SBvh::Intersect of a ray sample on every
    host thread. On the 16M soup each step builds over a bounded sample of the soup's triangles (the first
    --ref-sample-tris of the same generator: the same distribution at lower density) so that the whole run ends in
    minutes; the full 16M build is the GPU arm's cpu_baseline."""
    if rank != 0:
        return
    from diplodocus_b200 import scenes as S
    threads = os.cpu_count() or 1
    if args.workload == "soup16m":
        n_sample = min(args.ref_sample_tris, args.soup_tris)
        tris = S.soup(n_sample, seed=3)
        rays = S.random_rays(args.rays or 16 * 1024 * 1024, seed=3)
        desc = workload_desc = (f"{args.soup_tris:,}-triangle log-normal soup, {len(rays):,} random rays")
        sample_txt = (f"SBvh::Build of the first {n_sample:,} of the {args.soup_tris:,} soup triangles (same "
                      f"generator and distribution) on 1 thread per step")
        n_full = args.soup_tris
    else:
        tris, rays, desc = workload(args.workload, args.rays)
        workload_desc = desc
        n_sample = n_full = len(tris)
        sample_txt = f"SBvh::Build of all {n_sample:,} triangles on 1 thread per step"
    sample_rays = min(len(rays), args.ref_sample_rays)
    O = _ref_oracle()
    ref = O.RefOracle()
    for _ in range(args.warmup):
        ref.sbvh(tris[: min(len(tris), 65536)]).close()  # warm-up: code and allocator, not the measurement
    builds = []
    sb = None
    for k in range(args.steps):
        if sb is not None:
            sb.close()
        t0 = time.perf_counter()
        sb = ref.sbvh(tris)
        builds.append(time.perf_counter() - t0)
    sample = np.ascontiguousarray(rays[ray_sample_index(len(rays), sample_rays)])
    t0 = time.perf_counter()
    sb.trace(sample, threads=threads)
    trace_s = time.perf_counter() - t0
    sah = sb.sah_cost()[0]
    sb.close()
    value = n_sample / np.mean(builds) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "Mtri/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * np.mean(builds), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "description": workload_desc, "triangles": n_full, "rays": len(rays),
                   "build": "SBvh binned SAH (bin_count 16, leaf < 4, depth 32)"},
        "trace": {"value": round(sample_rays / trace_s / 1e6, 4), "unit": "Mrays/s", "sample_rays": sample_rays,
                  "threads": threads, "note": "SBvh::Intersect of an evenly spaced ray sample over the last step's "
                                              "BVH"},
        "sah_cost": round(sah, 4),
        "cpu_baseline": {"value": round(value, 4), "unit": "Mtri/s", "cores": 1, "kind": "reference",
                         "sample": sample_txt, "cpu_model": cpu_model(), "host_threads": threads},
        "e2e": {"value": round(value, 4), "unit": "Mtri/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_and_parity(tris, rays_np, gpu_hits_np, args, threads):
    """The GPU arm's cpu_baseline: one SBvh::Build of all triangles (1 thread), SBvh::Intersect of a ray sample on
    every host thread, and the same sample through the reference's brute force, against which the GPU's records
    of those rays are classified (E/T/F; S for SBvh's own misses)."""
    O = _ref_oracle()
    ref = O.RefOracle()
    n = len(tris)
    t0 = time.perf_counter()
    sb = ref.sbvh(tris)
    build_s = time.perf_counter() - t0
    idx = ray_sample_index(len(rays_np), args.parity_rays)
    sample = np.ascontiguousarray(rays_np[idx])
    t0 = time.perf_counter()
    hs = sb.trace(sample, threads=threads)
    trace_s = time.perf_counter() - t0
    rsah = sb.sah_cost()[0]
    sb.close()
    t0 = time.perf_counter()
    hb = ref.brute(tris, sample, threads=threads, chunk=8192 if n > 65536 else None)
    brute_s = time.perf_counter() - t0
    prim, t, u, v = (gpu_hits_np[k][idx] for k in range(4))
    classes = O.classify_hits(prim, t, u, v, hb, hs)
    base = {"value": round(n / build_s / 1e6, 4), "unit": "Mtri/s", "cores": 1, "kind": "reference",
            "sample": f"one SBvh::Build of all {n:,} triangles (1 thread); SBvh::Intersect of an evenly spaced "
                      f"sample of {len(idx)} rays on {threads} threads: {len(idx) / trace_s / 1e6:.5f} Mrays/s",
            "trace_mrays_per_s": round(len(idx) / trace_s / 1e6, 6), "trace_threads": threads,
            "sah_cost": round(rsah, 4), "cpu_model": cpu_model(), "host_threads": threads}
    parity = {"sample_rays": len(idx), "oracle": "reference DummyAccelerationStucture::Intersect (brute force, "
                                                  "lowest-id ties), chunked over the triangles",
              "brute_force_s": round(brute_s, 2), **classes}
    return base, parity


# ---------------------------------------------------------------------------------------------------
# GPU arm.
# ---------------------------------------------------------------------------------------------------
# DRAM bytes (read + write) per unit measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum, one pass) on
# the current kernels, per ray of one closest-hit trace and per triangle of one build, for the configuration each
# was captured with (split budget, ray order, size); other configurations report no traffic. Soup trace: the full
# 16M-triangle, 16M-ray launch, 14.71 GB read + 0.84 GB written (profiles/trace_dram_soup16m.md).
MEASURED_TRAFFIC = {("soup16m", "emc60", "trace"): {"split_budget": 40, "order": "coherent", "triangles": 16777216,
                                                    "per_unit": (14.71e9 + 0.845e9) / 16777216},
                    # the first build of the run, all 34 launches (profiles/dram_traffic_build_soup16m.md)
                    ("soup16m", "emc60", "build"): {"split_budget": 40, "order": "coherent", "triangles": 16777216,
                                                    "per_unit": (22778e6 + 7764e6) / 16777216},
                    ("displaced_sphere", "morton30", "build"): {"split_budget": 0, "order": "given",
                                                                "triangles": 1046528,
                                                                "per_unit": (502e6 + 71e6) / 1046528},
                    ("displaced_sphere", "morton30", "trace"): {"split_budget": 0, "order": "given",
                                                                "triangles": 1046528,
                                                                "per_unit": (284.2e6 + 74.6e6 + 28.5e6 + 0.2e6)
                                                                / 4194304}}


def measured_traffic(workload, code, kind, units, split_budget, order, triangles):
    m = MEASURED_TRAFFIC.get((workload, code, kind))
    if m is None or m["split_budget"] != split_budget or m["order"] != order or m["triangles"] != triangles:
        return None
    return round(m["per_unit"] * units)


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


def build_bytes_per_tri(code_type, digit_bits=8, node_bytes_per_tri=None, leaves_per_tri=1.0):
    """Algorithmic bytes of one build per triangle (byte model, Morton30: 176 B, EMC60: 308 B with 64 B/tri of
    nodes): vertices once, code + index written, the sort's passes at 8-bit digits, the node array, the
    permutation; with pre-splitting the per-leaf terms count once per clustering leaf."""
    k = 4 if code_type == 0 else 8
    passes = -(-(30 if code_type == 0 else 60) // 8)
    node = 64.0 if node_bytes_per_tri is None else node_bytes_per_tri
    return 36 + leaves_per_tri * ((k + 4) + passes * 2 * (k + 4) + 4) + node


def trace_bytes_per_ray(visits, tests, node_bytes):
    """Algorithmic bytes of one closest-hit ray: the ray in, the hit out, every node visited, every triangle
    tested (the counts come from the counting build of the same kernel on the same rays)."""
    return 32 + 16 + visits * node_bytes + tests * 36


def _quantiles(x, qs):
    """Quantiles of a 1-D device tensor by sorting (torch.quantile caps its input at 2^24 elements)."""
    import torch
    if x.numel() == 0:
        return [None for _ in qs]
    s, _ = torch.sort(x)
    n = s.numel()
    return [float(s[min(n - 1, int(round(q * (n - 1))))].item()) for q in qs]


KIND_OF = {("morton30", "aabb"): "kPloc", ("emc60", "aabb"): "kPlocEmc", ("morton30", "sobb"): "kPlocSobb",
           ("emc60", "sobb"): "kPlocEmcSobb"}
# The soup's variants beside the main arm (EMC60, AABB, binary): (code, bounding volume, layout).
SOUP_VARIANTS = {"ploc_emc_no_split": ("emc60", "aabb", "binary", 0),
                 "ploc_morton30": ("morton30", "aabb", "binary", None),
                 "ploc_emc_sobb": ("emc60", "sobb", "binary", None),
                 "ploc_emc_wide8_q8": ("emc60", "aabb", "wide8_q8", None)}


def run_gpu(args, rank, world, local_rank):
    import ctypes as C

    import torch
    import torch.distributed as dist

    from diplodocus_b200 import _lib as L
    from diplodocus_b200 import accel as A

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = L.load()
    code = args.code or DEFAULT_CODE[args.workload]
    tris, rays_np, desc_txt = workload(args.workload, args.rays, args.soup_tris)
    n, nr = len(tris), len(rays_np)
    AT = A.AccelerationStructureType

    split = args.split_budget if args.split_budget is not None else DEFAULT_SPLIT.get(args.workload, 0)
    tflags = trace_flags(args)
    order_name = "coherent" if tflags else "given"

    def config(code_, bv="aabb", layout="binary", split_budget=None):
        return A.AccelerationStructureConfig(getattr(AT, KIND_OF[(code_, bv)]), nn_search_radius=args.radius,
                                             leaf_test=args.leaf_test, layout=layout,
                                             split_budget=split if split_budget is None else split_budget)

    cfg = config(code)
    v = A.soa_vertices(tris, dev)
    rays = A.as_device_rays(rays_np, dev)
    hits = torch.empty((nr, 4), dtype=torch.int32, device=dev)
    desc = A.make_desc(*v, cfg)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    lt = A._leaf_test(args.leaf_test)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def build(d):
        h = C.c_void_p(0)
        L.check(lib.dipl_bvh_build(C.byref(d), C.byref(h), sp), "dipl_bvh_build")
        return h

    def trace(h, out, leaf=lt, counters=None):
        if counters is None:
            L.check(lib.dipl_bvh_trace_closest(h, C.c_void_p(rays.data_ptr()), nr, C.c_void_p(out.data_ptr()), leaf,
                                               tflags, sp), "dipl_bvh_trace_closest")
        else:
            L.check(lib.dipl_bvh_trace_closest_counted(h, C.c_void_p(rays.data_ptr()), nr, C.c_void_p(out.data_ptr()),
                                                       leaf, tflags, C.c_void_p(counters.data_ptr()), sp),
                    "dipl_bvh_trace_closest_counted")
            L.check(lib.dipl_bvh_check_errors(h, sp), "dipl_bvh_check_errors")  # synchronises; not in timed loops

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        h = build(desc)
        if ev is not None:
            ev[1].record(stream)
        trace(h, hits)
        if ev is not None:
            ev[2].record(stream)
        return h

    def destroy(h):
        L.check(lib.dipl_bvh_destroy(h), "dipl_bvh_destroy")

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
            destroy(step(evs[k]))
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
    launches = lib.dipl_kernel_launch_count() - launches0
    build_ms = [e[0].elapsed_time(e[1]) for e in evs]
    trace_ms = [e[1].elapsed_time(e[2]) for e in evs]
    step_ms = [e[0].elapsed_time(e[2]) for e in evs]
    t_step, t_build, t_trace = max_over_ranks([float(np.sum(step_ms)), float(np.sum(build_ms)),
                                               float(np.sum(trace_ms))], world, dev)

    # SAH cost, info and the counted trace (same kernel, same rays) of one build, outside the timed region
    h = build(desc)
    sah = C.c_double(0)
    L.check(lib.dipl_bvh_sah_cost(h, C.byref(sah), sp), "dipl_bvh_sah_cost")
    info = L.BvhInfo()
    L.check(lib.dipl_bvh_get_info(h, C.byref(info)), "dipl_bvh_get_info")
    ctr = torch.zeros(2, dtype=torch.int64, device=dev)
    trace(h, hits, counters=ctr)
    torch.cuda.synchronize()
    visits, tests = [int(x) for x in ctr.cpu().tolist()]
    hit_rate = float((hits[:, 0] >= 0).float().mean().item())
    node_bytes = info.node_bytes / max(info.num_inner_nodes, 1)

    extra = {}
    if args.workload == "soup16m" and not args.no_variants:
        extra = soup_forms(args, lib, L, A, torch, C, v, rays, hits, h, cfg, config, build, trace, destroy, flush,
                           stream, sp, n, nr)
    destroy(h)
    hits_np = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        raw = hits.cpu().numpy()
        f = raw.view(np.float32)
        hits_np = (raw[:, 0].copy(), f[:, 1].copy(), f[:, 2].copy(), f[:, 3].copy())

    t_e2e, h2d, d2h = e2e_run(args, lib, L, A, torch, C, v, rays, hits, cfg, stream, sp, world, dev)

    if rank != 0:
        return
    peak, peak_kind = peaks()
    steps = args.steps
    build_s = t_build / 1e3 / steps
    trace_s = t_trace / 1e3 / steps
    bpt = build_bytes_per_tri(desc.code_type, 8, info.node_bytes / max(n, 1), info.num_leaves / max(n, 1))
    achieved_build = bpt * n / build_s / 1e9
    ray_bytes = trace_bytes_per_ray(visits / nr, tests / nr, node_bytes)
    achieved_trace = ray_bytes * nr / trace_s / 1e9
    value = world * n / build_s / 1e6
    roof_build = {"bound": "hbm", "achieved": round(achieved_build, 1), "peak": peak, "unit": "GB/s",
                  "frac": round(achieved_build / peak, 4), "traffic": measured_traffic(args.workload, code, "build", n, split, order_name, n),
                  "kernel": "build pipeline (bounds, codes, sort, PLOC, layout)", "ms": round(build_s * 1e3, 4),
                  "bytes_per_unit": round(bpt, 1), "unit_of_bytes": "triangle",
                  "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"}
    roof_trace = {"bound": "hbm", "achieved": round(achieved_trace, 1), "peak": peak, "unit": "GB/s",
                  "frac": round(achieved_trace / peak, 4),
                  "traffic": (measured_traffic(args.workload, code, "trace", nr, split, order_name, n)
                              if args.leaf_test == "ref_mt" else None),
                  "kernel": "closest-hit trace (trace_kernel + tail_kernel)", "ms": round(trace_s * 1e3, 4),
                  "bytes_per_unit": round(ray_bytes, 1), "unit_of_bytes": "ray", "node_bytes": round(node_bytes, 1),
                  "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"}
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mtri/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": round(t_step / steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "description": desc_txt, "triangles": n, "rays": nr,
                   "code": code, "bounding_volume": "aabb", "split_budget": split,
                   "ray_order": "coherent (sorted on the device)" if tflags else "given",
                   "clustering_leaves": int(info.num_leaves), "nn_search_radius": args.radius,
                   "leaf_test": args.leaf_test, "layout": "binary", "max_triangles_per_leaf": 4,
                   "l2": "inputs larger than L2, and L2 flushed between steps (256 MB write)",
                   "parallelism": f"replicas x{world}"},
        "trace": {"value": round(world * nr / trace_s / 1e6, 3), "unit": "Mrays/s", "hit_rate": round(hit_rate, 4),
                  "node_visits_per_ray": round(visits / nr, 3), "tri_tests_per_ray": round(tests / nr, 3)},
        "build_ms": round(build_s * 1e3, 4), "trace_ms": round(trace_s * 1e3, 4),
        "build_ms_min_max": [round(min(build_ms), 4), round(max(build_ms), 4)],
        "sah_cost": round(sah.value, 4), "ploc_iterations": int(info.ploc_iterations), "bvh_depth": int(info.depth),
        "roofline": roof_trace if trace_s > build_s else roof_build,
        "roofline_build": roof_build, "roofline_trace": roof_trace,
        "e2e": {"value": round(world * n * steps / (t_e2e / 1e3) / 1e6, 3), "unit": "Mtri/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "ms_per_step": round(t_e2e / steps, 4),
                "note": "whole step per triangle through the C ABI: H2D vertices and rays from pinned memory, build, "
                        "trace, D2H hits; uploads on a copy stream overlap the previous step's build and trace (two "
                        "device input sets), downloads on a third stream"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "wall_s_timed_region": round(wall, 4),
    }
    line.update(extra)
    if hits_np is not None:
        threads = os.cpu_count() or 1
        try:
            line["cpu_baseline"], line["parity"] = cpu_baseline_and_parity(tris, rays_np, hits_np, args, threads)
        except FileNotFoundError as e:  # the reference harness is built where the reference tree exists
            line["cpu_baseline"] = {"value": None, "unit": "Mtri/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    print(json.dumps(line), flush=True)


def e2e_run(args, lib, L, A, torch, C, v, rays, hits, cfg, stream, sp, world, dev):
    """The step through the public API from HOST memory. Every step copies its inputs from pinned host memory and
    its hits back, as a user tracing frame after frame would: uploads on a copy stream into one of two device input
    sets (step k+1's uploads overlap step k's build and trace), build and trace on the compute stream, hit downloads
    on a third stream. Returns (device ms over all steps, H2D bytes per step, D2H bytes per step)."""
    nr = rays.shape[0]
    lt = A._leaf_test(args.leaf_test)
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
                                           C.c_void_p(sets[b]["hits"].data_ptr()), lt, trace_flags(args), sp),
                "dipl_bvh_trace_closest")
        ev_done[b].record(stream)
        d2h_s.wait_event(ev_done[b])
        with torch.cuda.stream(d2h_s):
            host_hits[b].copy_(sets[b]["hits"], non_blocking=True)
        L.check(lib.dipl_bvh_destroy(hh), "dipl_bvh_destroy")

    def run(steps_):
        upload(0)
        for k in range(steps_):
            if k + 1 < steps_:
                upload(k + 1)
            compute_download(k)

    run(2)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(copy_s)
    run(args.steps)
    d2h_s.wait_stream(stream)
    d2h_s.wait_stream(copy_s)
    e1.record(d2h_s)
    torch.cuda.synchronize()
    (t_e2e,) = max_over_ranks([e0.elapsed_time(e1)], world, dev)
    h2d = sum(x.numel() * 4 for x in v) + rays.numel() * 4
    d2h = hits.numel() * 4
    del sets, host_v, host_rays, host_hits
    torch.cuda.empty_cache()
    return t_e2e, h2d, d2h


def soup_forms(args, lib, L, A, torch, C, v, rays, hits, h_main, cfg, config, build, trace, destroy, flush, stream,
               sp, n, nr):
    """The soup's forms beside the main arm, all on the same resident triangles and rays:

    * variants: Morton30, EMC60 + SOBB and the 8-wide quantised layout; build and trace times (CUDA events, L2
      flushed before each), SAH, node visits, the trace roofline, and hit agreement with the main arm;
    * errors: FP32 t/u/v of the reference-exact (main) and watertight leaf tests against the FP64 re-intersection of
      the same triangle, per scene;
    * disagreements: rays whose hit differs between two forms, re-intersected in FP64 against both triangles to
      tell which form found the nearer one."""
    peak, _ = peaks()
    main_prim = hits[:, 0].clone()
    f32 = hits.view(torch.float32)

    def ev():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps):
        out = []
        for _ in range(reps):
            flush.zero_()
            # the flush finishes before the timed build is enqueued: builds enqueued behind it measured 1.5-4x
            # their time now and then (unsplit soup 24-65 ms against 16.1 ms; SOBB 67 against 33.5 ms), the same
            # builds after a synchronise 16.1 +- 0.03 ms and 33.5 +- 0.05 ms in five runs
            torch.cuda.synchronize()
            a, b = ev()
            a.record(stream)
            r = fn()
            b.record(stream)
            torch.cuda.synchronize()
            out.append(a.elapsed_time(b))
            if r is not None:
                destroy(r)
        return out

    def reintersect(hts):
        out = torch.empty((nr, 3), dtype=torch.float64, device=rays.device)
        L.check(lib.dipl_reintersect_f64(C.c_void_p(v[0].data_ptr()), C.c_void_p(v[1].data_ptr()),
                                         C.c_void_p(v[2].data_ptr()), C.c_void_p(rays.data_ptr()),
                                         C.c_void_p(hts.data_ptr()), nr, C.c_void_p(out.data_ptr()), sp),
                "dipl_reintersect_f64")
        return out

    def error_stats(hts):
        f = hts.view(torch.float32)
        hit = hts[:, 0] >= 0
        ref = reintersect(hts)
        t64, u64, v64 = ref[hit, 0], ref[hit, 1], ref[hit, 2]
        rel_t = (f[hit, 1].double() - t64).abs() / t64.abs().clamp_min(1e-300)
        du = (f[hit, 2].double() - u64).abs()
        dv = (f[hit, 3].double() - v64).abs()
        q = (0.5, 0.99, 0.9999, 1.0)
        return {"hits": int(hit.sum().item()),
                "t_rel": dict(zip(("median", "p99", "p9999", "max"), _quantiles(rel_t, q))),
                "u_abs": dict(zip(("median", "p99", "p9999", "max"), _quantiles(du, q))),
                "v_abs": dict(zip(("median", "p99", "p9999", "max"), _quantiles(dv, q)))}

    def disagreement(h_a, h_b):
        """Rays whose ids differ between two forms: FP64 t of both forms' triangles along the ray."""
        diff = h_a[:, 0] != h_b[:, 0]
        nd = int(diff.sum().item())
        if nd == 0:
            return {"rays": 0}
        ta = reintersect(h_a)[diff, 0]
        tb = reintersect(h_b)[diff, 0]
        return {"rays": nd, "first_nearer_fp64": int((ta < tb).sum().item()),
                "second_nearer_fp64": int((tb < ta).sum().item()), "equal_fp64": int((ta == tb).sum().item()),
                "first_missed": int((h_a[diff, 0] < 0).sum().item()),
                "second_missed": int((h_b[diff, 0] < 0).sum().item())}

    out = {"errors_vs_fp64": {}, "disagreements": {}, "variants": {}}
    out["errors_vs_fp64"][args.leaf_test] = error_stats(hits)
    # the watertight leaf test on the main BVH
    other = "watertight" if args.leaf_test == "ref_mt" else "ref_mt"
    h_wt = torch.empty_like(hits)
    trace(h_main, h_wt, leaf=A._leaf_test(other))
    out["errors_vs_fp64"][other] = error_stats(h_wt)
    out["disagreements"][f"{args.leaf_test}_vs_{other}"] = disagreement(hits, h_wt)
    del h_wt
    vh = torch.empty_like(hits)
    for name, (code_, bv, layout, split_) in SOUP_VARIANTS.items():
        c = config(code_, bv, layout, split_)
        d = A.make_desc(*v, c)
        timed(lambda: build(d), 1)  # warm-up: the first build of a form sizes its buffers in the memory pool
        b_ms = timed(lambda: build(d), args.variant_builds)
        hv = build(d)
        t_ms = timed(lambda: trace(hv, vh), args.variant_traces)
        ctr = torch.zeros(2, dtype=torch.int64, device=rays.device)
        trace(hv, vh, counters=ctr)
        visits, tests = [x / nr for x in ctr.cpu().tolist()]
        info = L.BvhInfo()
        L.check(lib.dipl_bvh_get_info(hv, C.byref(info)), "dipl_bvh_get_info")
        sah = C.c_double(0)
        L.check(lib.dipl_bvh_sah_cost(hv, C.byref(sah), sp), "dipl_bvh_sah_cost")
        nb = info.node_bytes / max(info.num_inner_nodes, 1)
        rb = trace_bytes_per_ray(visits, tests, nb)
        tm = float(np.median(t_ms))
        ach = rb * nr / (tm / 1e3) / 1e9
        same = float((vh[:, 0] == main_prim).float().mean().item())
        bm = float(np.median(b_ms))
        out["variants"][name] = {
            "code": code_, "bounding_volume": bv, "layout": layout, "split_budget": c.split_budget,
            "build_ms": round(bm, 3), "build_ms_all": [round(x, 3) for x in b_ms],
            "build_mtri_s": round(n / bm / 1e3, 1), "trace_ms": round(tm, 3),
            "trace_mrays_s": round(nr / tm / 1e3, 2), "sah_cost": round(sah.value, 4),
            "node_visits_per_ray": round(visits, 2), "tri_tests_per_ray": round(tests, 2),
            "node_bytes": int(info.node_bytes),
            "roofline_trace": {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                               "frac": round(ach / peak, 4), "bytes_per_ray": round(rb, 1), "node_bytes": round(nb, 1)},
            "same_hits_as_main": same}
        if same < 1.0:
            out["disagreements"][f"main_vs_{name}"] = disagreement(hits, vh)
        destroy(hv)
        torch.cuda.empty_cache()
    del vh
    return out


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


def run_batched(args):
    """256 noise-displaced spheres (1k..2M triangles): one graph-replayed plan vs 256 sequential builds."""
    import ctypes as C

    import torch
    from diplodocus_b200 import _lib as L
    from diplodocus_b200 import accel as A
    from diplodocus_b200 import scenes as S
    meshes_np = S.batched_meshes(args.batch_count)
    meshes = [torch.from_numpy(m) for m in meshes_np]
    total = sum(m.shape[0] for m in meshes)
    cfg = A.AccelerationStructureConfig()
    verts = [A.soa_vertices(m) for m in meshes]
    descs = [A.make_desc(*v, cfg) for v in verts]
    lib = L.load()

    def plain_all():
        sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        for d in descs:
            h = C.c_void_p(0)
            L.check(lib.dipl_bvh_build(C.byref(d), C.byref(h), sp), "dipl_bvh_build")
            L.check(lib.dipl_bvh_destroy(h), "dipl_bvh_destroy")

    ms_plain = _time(plain_all, 2, warm=1)
    cache = os.path.join("/tmp", "dipl_tune_cache.jsonl")
    t0 = time.perf_counter()
    tuned, from_cache, tverts = A.autotune(cfg, meshes, cache)
    tune_s = time.perf_counter() - t0
    plan = A.BuildPlan(cfg, meshes, tuned_descs=tuned)
    del tverts
    launches0 = lib.dipl_kernel_launch_count()
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms_plan = _time(plan.launch, 5, warm=2)
    launches = (lib.dipl_kernel_launch_count() - launches0) // 7
    bvhs = plan.bvhs()
    nr = 65536
    rays_np = S.sphere_inward_rays(nr, seed=4)
    rays = torch.from_numpy(rays_np).cuda()
    ms_tr = [_time(lambda b=b: b.Intersect(A.Stats(), rays), 2, warm=1) for b in bvhs[:: max(1, len(bvhs) // 16)]]
    # hit agreement between the plan's BVHs and plain builds on a few meshes
    agree = []
    for i in range(0, len(meshes), max(1, len(meshes) // 8)):
        ref = A.GpuPlocBvh().Build(cfg, A.Stats(), meshes[i])
        a = ref.Intersect(A.Stats(), rays).prim.cpu().numpy()
        b = bvhs[i].Intersect(A.Stats(), rays).prim.cpu().numpy()
        agree.append(float((a == b).mean()))
    d0 = tuned[0]
    line = {
        "config": {"workload": "batched", "meshes": len(meshes), "triangles": int(total),
                   "sizes": "log-uniform 1k..2M per mesh", "rays_per_mesh": nr},
        "plan_graph_ms": round(ms_plan, 3), "sequential_plain_ms": round(ms_plain, 3),
        "speedup_batched_vs_plain": round(ms_plain / ms_plan, 3),
        "plain_mtri_s": round(total / ms_plain / 1e3, 1),
        "autotuned": {"clustering": "ploc" if d0.clustering == L.CLUSTER_PLOC else "hploc",
                      "radius": d0.nn_search_radius, "block": d0.ploc_block_size, "digits": d0.sort_digit_bits,
                      "from_cache": from_cache, "tune_s": round(tune_s, 2)},
        "trace_mrays_s_per_mesh_median": round(float(np.median([nr / t / 1e3 for t in ms_tr])), 2),
        "hit_agreement_plan_vs_plain": min(agree), "gpu_launches_per_plan": int(launches),
        "clocks": clk.summary()}
    if not args.no_cpu_baseline:
        # SBvh::Build of every 8th mesh on 1 thread (the whole batch would take about a minute), and SBvh::Intersect
        # of the rays over one mid-sized mesh on every host thread; plus the plan's hits on that mesh against brute
        # force
        try:
            O = _ref_oracle()
            ref = O.RefOracle()
            sub = list(range(0, len(meshes_np), 8))
            n_sub = sum(len(meshes_np[i]) for i in sub)
            t0 = time.perf_counter()
            for i in sub:
                ref.sbvh(meshes_np[i]).close()
            build_s = time.perf_counter() - t0
            mid = int(np.argsort([len(m) for m in meshes_np])[len(meshes_np) // 2])
            sb = ref.sbvh(meshes_np[mid])
            threads = os.cpu_count() or 1
            t0 = time.perf_counter()
            sb.trace(rays_np, threads=threads)
            trace_s = time.perf_counter() - t0
            sb.close()
            idx = ray_sample_index(nr, 4096)
            hb = ref.brute(meshes_np[mid], rays_np[idx], threads=threads)
            hg = bvhs[mid].Intersect(A.Stats(), rays)
            g = [x.cpu().numpy()[idx] for x in (hg.prim, hg.t, hg.u, hg.v)]
            line["cpu_baseline"] = {"value": round(n_sub / build_s / 1e6, 4), "unit": "Mtri/s", "cores": 1,
                                    "kind": "reference",
                                    "sample": f"SBvh::Build of every 8th mesh ({len(sub)} meshes, {n_sub:,} triangles) "
                                              f"on 1 thread; SBvh::Intersect of {nr} rays over mesh {mid} "
                                              f"({len(meshes_np[mid]):,} triangles) on {threads} threads",
                                    "trace_mrays_per_s": round(nr / trace_s / 1e6, 4), "cpu_model": cpu_model()}
            line["parity"] = {"mesh": mid, **O.classify_hits(*g, hb)}
        except FileNotFoundError as e:
            line["cpu_baseline"] = {"value": None, "unit": "Mtri/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    _line("batched", total / ms_plan / 1e3, "Mtri/s", line)
    plan.close()


def run_diff(args):
    """Differentiation: 65k-triangle displaced sphere, 1024x1024 primary rays, forward + adjoint."""
    import torch
    from diplodocus_b200 import _lib as L
    from diplodocus_b200 import accel as A
    from diplodocus_b200 import scenes as S
    verts, idx, rays_np = S.diff_scene()
    tris = verts[idx].astype(np.float32)
    bvh = A.GpuPlocBvh().Build(A.AccelerationStructureConfig(), A.Stats(), torch.from_numpy(tris))
    rays = torch.from_numpy(rays_np).cuda()
    h = bvh.Intersect(A.Stats(), rays)
    hit = h.prim >= 0
    zero = torch.zeros_like(h.t)
    g = torch.stack([torch.where(hit, 0.06 * h.t, zero), torch.where(hit, 0.5 * h.u, zero),
                     torch.where(hit, -0.25 * h.v, zero)], 1)
    lib = L.load()
    launches0 = lib.dipl_kernel_launch_count()
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms_fwd = _time(lambda: bvh.Intersect(A.Stats(), rays), 10)
        ms_adj = _time(lambda: A.trace_adjoint(bvh._v, rays, h, g), 10)
    launches = lib.dipl_kernel_launch_count() - launches0
    nr = rays.shape[0]
    line = {"config": {"workload": "diff", "triangles": len(tris), "rays": nr,
                       "upstream": "dL/dt, dL/du, dL/dv all non-zero on hits"},
            "forward_mrays_s": round(nr / ms_fwd / 1e3, 2), "adjoint_ms": round(ms_adj, 4),
            "hit_rate": float(hit.float().mean().item()), "gpu_launches": int(launches), "clocks": clk.summary(),
            "check": "FP64 central differences of t, u and v in the differentiation tests"}
    if not args.no_cpu_baseline:
        # The reference has no adjoint; its nearest CPU counterpart is the forward closest hit (SBvh::Intersect of
        # the same 1M primary rays on every host thread).
        try:
            O = _ref_oracle()
            sb = O.RefOracle().sbvh(tris)
            threads = os.cpu_count() or 1
            t0 = time.perf_counter()
            sb.trace(rays_np, threads=threads)
            trace_s = time.perf_counter() - t0
            sb.close()
            line["cpu_baseline"] = {"value": round(nr / trace_s / 1e6, 4), "unit": "Mrays/s", "cores": threads,
                                    "kind": "reference",
                                    "sample": f"SBvh::Intersect of all {nr} primary rays on {threads} threads (the "
                                              "forward pass; the reference has no adjoint)", "cpu_model": cpu_model()}
        except FileNotFoundError as e:
            line["cpu_baseline"] = {"value": None, "unit": "Mrays/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    _line("diff", nr / ms_adj / 1e3, "Mrays/s", line)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="dipl", choices=["dipl", "reference"])
    ap.add_argument("--workload", default="soup16m",
                    choices=["soup16m", "displaced_sphere", "small", "batched", "diff", "obj_scene"])
    ap.add_argument("--soup-tris", type=int, default=SOUP_TRIANGLES)
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--code", default=None, choices=["morton30", "emc60"],
                    help="code of the main arm (default: emc60 on the soup, morton30 on the sphere)")
    ap.add_argument("--radius", type=int, default=16)
    ap.add_argument("--split-budget", type=int, default=None,
                    help="pre-splitting of large triangles, percent (default: 40 on the soup, 0 on the sphere)")
    ap.add_argument("--leaf-test", default="ref_mt", choices=["ref_mt", "watertight"])
    ap.add_argument("--trace-order", default=None, choices=["given", "coherent"],
                    help="ray order of the traces (default per workload: coherent for the soup, given otherwise)")
    ap.add_argument("--rays", type=int, default=None)
    ap.add_argument("--ref-sample-rays", type=int, default=1 << 12)
    ap.add_argument("--ref-sample-tris", type=int, default=1 << 21,
                    help="reference arm on the soup: triangles per SBvh::Build step")
    ap.add_argument("--parity-rays", type=int, default=4096)
    ap.add_argument("--variant-builds", type=int, default=5)
    ap.add_argument("--variant-traces", type=int, default=2)
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 0 or args.steps < 1:
        raise SystemExit("--steps must be >= 1 and --warmup >= 0")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload in ("small", "batched", "diff", "obj_scene") and world == 1:
        import torch
        torch.cuda.set_device(local_rank)
        {"small": run_small, "batched": run_batched, "diff": run_diff, "obj_scene": run_obj_scene}[args.workload](args)
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
