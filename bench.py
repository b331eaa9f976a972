"""Closest-hit microbenchmark of the B200 path tracer (one JSON line on rank 0).

Workload: 2,097,152 random triangles (centroids uniform in the unit cube,
lognormal edge lengths around 0.005, random orientation) and 4,194,304
incoherent rays (origins uniform in the cube, directions uniform on the
sphere, tmax = 1e30), all seeded. A step traces every ray once through the
scene's GPU-built BVH and writes (prim, t, u, v) per ray.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

For N > 1 (torchrun) every rank holds a full scene replica and traces its
own seeded ray set (weak scaling); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_TRIS = 2097152
N_RAYS = 4194304
METRIC = "closest-hit Mrays/s (2M random tris, 4M incoherent rays, bit-exact vs Ref)"
UNIT = "Mrays/s"
WORKLOAD = "closest-hit BVH microbench: 2,097,152 random triangles, 4,194,304 incoherent rays"


PARITY_CHUNK = 1024
PARITY_FIXTURE = os.path.join(ROOT, "tests", "golden", "headline_ref.npz")


def chunk_digests(records: np.ndarray, chunk: int = PARITY_CHUNK) -> np.ndarray:
    """8-byte BLAKE2b digest of each run of `chunk` hit records ((n, 4)
    uint32: prim, t, u, v bits), as uint64."""
    rec = np.ascontiguousarray(records, np.uint32).reshape(-1, 4)
    import hashlib

    n = (len(rec) + chunk - 1) // chunk
    out = np.zeros(n, np.uint64)
    for k in range(n):
        out[k] = int.from_bytes(hashlib.blake2b(rec[k * chunk:(k + 1) * chunk].tobytes(), digest_size=8).digest(), "little")
    return out


def inputs_sha256(tris: np.ndarray, rays: np.ndarray) -> str:
    import hashlib

    h = hashlib.sha256(np.ascontiguousarray(tris, np.float32).tobytes())
    h.update(np.ascontiguousarray(rays, np.float32).tobytes())
    return h.hexdigest()


def parity_vs_reference(name: str, tris: np.ndarray, rays: np.ndarray, records: np.ndarray, fixture: str = PARITY_FIXTURE) -> dict:
    """Compares this tracer's hits on the full microbench (`records`, (n, 4)
    uint32) with the compiled reference's Ref traversal, stored as per-chunk
    digests in `fixture` (tests/golden/make_headline_fixture.py). Rays where
    the fixture records that the reference deviates from the closest hit with
    ties to the lower triangle index (an exact-t tie kept in traversal order,
    or a box the reference culled) are mapped to the reference's answer when
    this tracer gives the closest hit there; every other difference shows as a
    mismatching chunk."""
    if not os.path.exists(fixture):
        return {"rays": int(len(rays)), "mismatch": None, "fixture": "absent"}
    import hashlib

    fx = np.load(fixture)
    if inputs_sha256(tris, rays) != fx[f"{name}_inputs_sha256"].item().decode():
        return {"rays": int(len(rays)), "mismatch": None, "fixture": "inputs differ from the fixture's"}
    rec = np.array(records, np.uint32, copy=True).reshape(-1, 4)
    idx = fx[f"{name}_dev_idx"]
    ours_ok = np.all(rec[idx] == fx[f"{name}_dev_ours"], axis=1) if len(idx) else np.zeros(0, bool)
    rec[idx[ours_ok]] = fx[f"{name}_dev_ref"][ours_ok]
    dig = chunk_digests(rec, int(fx["chunk"]))
    bad = np.nonzero(dig != fx[f"{name}_digests"])[0]
    kinds = fx[f"{name}_dev_kind"]
    return {"rays": int(len(rays)), "mismatch_chunks": int(len(bad)), "mismatch": int(len(bad)) if len(bad) else 0,
            "bad_chunks": [int(b) for b in bad[:16]], "chunk": int(fx["chunk"]),
            "explained": {"exact_t_ties": int(np.sum(kinds[ours_ok] == 0)), "ref_box_false_negatives": int(np.sum(kinds[ours_ok] == 1))},
            "unexplained_deviation_rays": int(np.sum(~ours_ok)),
            "hits": int(np.sum(rec[:, 0].view(np.int32) >= 0)), "ref_hits": int(fx[f"{name}_hits"]),
            "fixture": hashlib.sha256(open(fixture, "rb").read()).hexdigest()[:16]}


def profiled(name: str = "trace_closest_microbench.txt") -> dict:
    """Machine-readable figures of a committed ncu summary (lines 'key: value'
    at the start of a line): DRAM bytes per launch, L2 throughput and issue
    activity of the traversal kernel on this workload."""
    p = os.path.join(ROOT, "profiles", name)
    out = {}
    if not os.path.exists(p):
        return out
    for line in open(p):
        k, sep, v = line.strip().partition(":")
        if sep and k in ("dram_bytes_per_launch", "l2_throughput_pct", "issue_active_pct", "profiled_launch_ms", "lanes_active"):
            try:
                out[k] = float(v.split()[0])
            except (ValueError, IndexError):
                pass
    return out


def peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def tuned_tuple(info) -> dict:
    """The frame tuner's choice as the renderer reports it after a frame."""
    return {"kernel": {1: "wavefront", 2: "path"}.get(info.kernel, "?"), "sort_mask": f"0x{info.sort_mask:03x}",
            "trace_variant": int(info.trace_variant), "refill": int(info.trace_refill), "block": int(info.trace_block),
            "smem_stack": int(info.trace_stack), "one_triangle_per_step": int(info.trace_one_tri)}


def make_workload(rank: int, n_tris: int = N_TRIS, n_rays: int = N_RAYS):
    """Rank `rank`'s share of an N-GPU run: the same scene on every rank (a
    replica) and the rank's own seeded rays (weak scaling: rays per rank fixed)."""
    from raydemo_b200 import scenes

    tris = scenes.random_triangles(n_tris, seed=0)
    rays = scenes.incoherent_rays(n_rays, seed=1 + rank)
    return tris, rays


def max_over_ranks(ms: float, world: int, device) -> float:
    """The slowest rank's time (the job ends with its last rank): an all-reduce
    MAX over the process group; the value itself with one rank."""
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_reference(tris, rays, sample: int, steps: int, warmup: int):
    """Times the reference's AVX2 closest-hit traversal (oracle/_ref) on all
    host threads. Returns (Mrays/s per step list, threads, build seconds)."""
    from oracle.oracle import RefLib, RefScene
    from raydemo_b200 import scenes

    ref = RefLib()
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    t0 = time.perf_counter()
    sc = RefScene(ref, True)
    attrs, idx = scenes.triangle_soup_mesh(tris)
    m = sc.add_material(0)
    sc.add_instance(sc.add_mesh(attrs, idx, [(m, 0xFFFFFFFF, 0, len(idx))]))
    build_s = time.perf_counter() - t0
    rng = np.random.default_rng(123)
    vals = []
    for s in range(warmup + steps):
        sub = rays[rng.integers(0, len(rays), sample)]
        t0 = time.perf_counter()
        sc.trace_closest(sub, nthreads=threads, backend=1)
        dt = time.perf_counter() - t0
        if s >= warmup:
            vals.append(sample / dt / 1e6)
    return vals, threads, build_s


RENDER_WORKLOAD = "Cornell box (seed 0): 1,316 tris, 256x256, 1 sample per frame, 4 bounces, ray sorting off"


def build_scene(api, r, spec: dict):
    """A scene spec (raydemo_b200.scenes) through the public API, committed."""
    sc = r.CreateScene()
    if "env" in spec:
        sc.SetEnvironment(**spec["env"])
    for rgba, srgb, mips in spec.get("textures", []):
        sc.AddTexture(rgba, is_srgb=srgb, generate_mipmaps=mips)
    for m in spec.get("materials", []):
        sc.AddMaterial(**m)
    for attrs, idx, shapes, layout in spec.get("meshes", []):
        sc.AddMesh(attrs, idx, shapes, layout=layout)
    for mesh, xf in spec.get("instances", []):
        sc.AddMeshInstance(mesh, xf)
    for l in spec.get("lights", []):
        sc.AddLight(**l)
    sc.set_current_cam(sc.AddCamera(api.CameraDesc(**spec["camera"])))
    sc.Commit()
    return sc


def render_frames(args, dev, stream, rank: int, world: int) -> dict:
    """The render loop on the small render configuration: frames of the
    Cornell box through RenderScene, timed with CUDA events on the renderer's
    stream; rays per frame from the renderer's counters; the image compared
    with the reference's Ref renderer on the same sample sequence."""
    import torch
    import torch.distributed as dist

    from raydemo_b200 import api, scenes

    spec = scenes.cornell_box(0)
    w, h = spec["size"]
    r = api.Renderer(w, h, device=dev.index)
    r.set_stream(stream.cuda_stream)
    sc = build_scene(api, r, spec)
    # first frame: the image compared with the reference
    r.Clear()
    reg = api.RegionContext()
    r.RenderScene(sc, reg)
    first = r.get_pixels_ref()
    info = r.frame_info()
    if info.error_flags:
        raise RuntimeError(f"render reported error flags {info.error_flags}")
    rays_per_frame = info.rays + info.shadow_rays
    frames = max(10, args.steps * 10)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(kernel: int) -> float:
        """ms per frame with the given kernel choice (0: the renderer's own choice by timing)."""
        r.set_kernel(kernel)
        for _ in range(max(24, args.warmup)):  # covers the tuner's timed frames (2 per variant, up to 8 variants)
            r.RenderScene(sc, reg)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        ev0.record(stream)
        for _ in range(frames):
            r.RenderScene(sc, reg)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        return max_over_ranks(ev0.elapsed_time(ev1) / frames, world, dev)

    by_kernel = {"wavefront": round(timed(1), 4), "path": round(timed(2), 4)}
    ms_frame = timed(0)
    chosen_info = r.frame_info()
    chosen = {1: "wavefront", 2: "path"}.get(chosen_info.kernel, "?")
    # end to end through the public API: RenderScene, then the pixels read back to the host
    e_frames = max(5, min(frames, 50))
    ev0.record(stream)
    for _ in range(e_frames):
        r.RenderScene(sc, reg)
        r.get_pixels_ref()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e = ev0.elapsed_time(ev1) / e_frames
    out = {"workload": RENDER_WORKLOAD, "ms_per_frame": round(ms_frame, 4), "frames": frames,
           "mrays_per_s": round(world * rays_per_frame / (ms_frame * 1e-3) / 1e6, 2), "rays_per_frame": int(rays_per_frame),
           "closest_hit_rays_per_frame": int(info.rays), "shadow_rays_per_frame": int(info.shadow_rays),
           "e2e_ms_per_frame": round(ms_e2e, 4), "e2e_d2h_bytes_per_frame": w * h * 16, "kernel": chosen,
           "tuned": tuned_tuple(chosen_info),
           "ms_per_frame_by_kernel": by_kernel}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle.oracle import RefLib, RefRenderer
            from tests.render_scenes import build_ref

            ref = RefLib()
            rsc = build_ref(ref, spec)
            rr = RefRenderer(ref, w, h, RefRenderer.REF, True)
            t0 = time.perf_counter()
            rr.render(rsc, 1, reset=True, nthreads=1)
            ref_ms = (time.perf_counter() - t0) * 1e3
            img = rr.pixels()
            d = img.astype(np.float64) - first.astype(np.float64)
            out["rmse_vs_ref"] = float(np.sqrt(np.mean(d[..., :3] ** 2)))
            out["identical_px_vs_ref"] = float(np.mean(np.all(img == first, axis=-1)))
            threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
            ra = RefRenderer(ref, w, h, RefRenderer.AVX2, True)
            ra.render(rsc, 1, reset=True, nthreads=threads)  # warm-up
            t0 = time.perf_counter()
            n_cpu = 5
            ra.render(rsc, n_cpu, reset=False, nthreads=threads)
            avx_ms = (time.perf_counter() - t0) * 1e3 / n_cpu
            out["cpu_baseline"] = {"ms_per_frame": round(avx_ms, 3), "cores": threads, "kind": "reference",
                                   "sample": f"{n_cpu} frames, AVX2 renderer, 64-px buckets on {threads} threads",
                                   "ref_1core_ms_per_frame": round(ref_ms, 2)}
        except FileNotFoundError as e:
            out["cpu_baseline"] = {"ms_per_frame": None, "kind": "reference", "sample": f"unavailable: {e}"}
    r.set_stream(0)
    return out


BATCH_WORKLOAD = ("batched form: 64 scenes (ground plane + displaced icospheres, 962..491,522 tris, log-uniform target "
                  "[1e3, 5e5]), resolutions from {64..1024}^2 (19.9 Mpixel), 4 samples, max 6 bounces, sun + sky")


def batch_frames(args, dev, stream, n_scenes: int = 64, samples: int = 4) -> dict:
    """The batched configuration: `samples` samples of every scene as ONE
    ray_render_batch call, against the plain loop of RenderScene per scene
    and sample (each renderer with its own kernel choice), on one stream.
    Both loops render the same images (compared bit for bit)."""
    import torch

    from raydemo_b200 import api, scenes

    specs = [scenes.batch_scene(i) for i in range(n_scenes)]
    rs, scs = [], []
    for sp in specs:
        w, h = sp["size"]
        r = api.Renderer(w, h, device=dev.index)
        r.set_stream(stream.cuda_stream)
        sc = build_scene(api, r, sp)
        rs.append(r)
        scs.append(sc)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def plain_pass() -> list:
        regs = [api.RegionContext() for _ in rs]
        for r, sc, g in zip(rs, scs, regs):
            r.Clear()
            for _ in range(samples):
                r.RenderScene(sc, g)
        return regs

    def batch_pass() -> list:
        regs = [api.RegionContext() for _ in rs]
        for r in rs:
            r.Clear()
        api.render_batch(rs, scs, regs, samples)
        return regs

    plain_ms, plain_imgs, kernels = None, None, []
    if not args.batch_no_plain:
        # warm-up: the plain loop twice (each renderer times both kernels on its first frames)
        for _ in range(6):  # 24 frames per renderer: past its tuner's timed frames (2 per variant)
            plain_pass()
        plain_ms = float("inf")
        for _ in range(3):  # the best of three, as for the batch
            torch.cuda.synchronize(dev)
            ev0.record(stream)
            plain_pass()
            ev1.record(stream)
            torch.cuda.synchronize(dev)
            plain_ms = min(plain_ms, ev0.elapsed_time(ev1))
        plain_imgs = [r.get_pixels_ref() for r in rs]
        kernels = [r.frame_info().kernel for r in rs]
    if args.batch_no_plain:  # profiling: the batch alone, wavefront
        rs[0].set_kernel(1)
        batch_pass()
        batch_pass()
        torch.cuda.synchronize(dev)
        return {"workload": BATCH_WORKLOAD, "profiling_run": True}

    def timed_batch(kernel: int, warm: int, sort: int = -1, reps: int = 3) -> float:
        """The best of `reps` timed calls after `warm` untimed ones."""
        rs[0].set_kernel(kernel)  # the batch follows the first renderer's settings
        rs[0].set_ray_sort(sort)
        for _ in range(warm):
            batch_pass()
        best = float("inf")
        for _ in range(reps):
            torch.cuda.synchronize(dev)
            ev0.record(stream)
            batch_pass()
            ev1.record(stream)
            torch.cuda.synchronize(dev)
            best = min(best, ev0.elapsed_time(ev1))
        return best

    by_kernel = {"wavefront": round(timed_batch(1, 1, 0), 3), "wavefront_sorted": round(timed_batch(1, 1, 0x3FF), 3),
                 "path": round(timed_batch(2, 1, 0, reps=1), 3)}
    batch_ms = timed_batch(0, 20)  # the default: kernel, sort and trace settings chosen by timing the first calls (2 per variant)
    info = rs[0].frame_info()
    if info.error_flags:
        raise RuntimeError(f"batch reported error flags {info.error_flags}")
    identical, worst = 0, 0.0
    for r, a in zip(rs, plain_imgs):
        b = r.get_pixels_ref()
        identical += int(np.array_equal(a.view(np.uint32), b.view(np.uint32)))
        worst = max(worst, float(np.sqrt(np.mean((a[..., :3].astype(np.float64) - b[..., :3]) ** 2))))
    rays = info.rays + info.shadow_rays
    return {"workload": BATCH_WORKLOAD, "scenes": n_scenes, "samples": samples, "tris_total": int(sum(s["tris"] for s in specs)),
            "pixels_per_sample": int(sum(s["size"][0] * s["size"][1] for s in specs)), "batch_ms": round(batch_ms, 3),
            "plain_loop_ms": round(plain_ms, 3), "speedup_vs_plain": round(plain_ms / batch_ms, 3),
            "batch_mrays_per_s": round(rays / (batch_ms * 1e-3) / 1e6, 1), "rays": int(rays),
            "plain_kernels": {"wavefront": kernels.count(1), "path": kernels.count(2)},
            "batch_kernel": {1: "wavefront", 2: "path"}.get(info.kernel, "?"), "tuned": tuned_tuple(info),
            "batch_ms_by_kernel": by_kernel,
            "images_identical_to_plain": f"{identical}/{n_scenes}", "max_rmse_vs_plain": worst}


ATRIUM_WORKLOAD = ("metallic-roughness atrium (seed 0): 20x4x60 room (12 tris) + 16 displaced icospheres of subdivision 5 "
                   "(327,680 tris), GGX roughness U[0.05,1], metallic Bernoulli(0.3), 1024^2 value-noise albedo, sun 5 + 4 quad "
                   "lights; 1280x720, 16 samples per frame, max 8 bounces")


def atrium_frames(args, dev, stream, rank: int, world: int) -> dict:
    """The metallic-roughness configuration: 16-sample frames of the atrium
    through RenderScene (16 calls), timed with CUDA events per variant (the
    wavefront without ray sorting, sorting before every bounce, the mask the
    timing chooses; the path kernel) and with the renderer's own choice; the
    image compared with the oracle's CPU restatement on the same sample
    sequence, whose time is the CPU baseline."""
    import torch
    import torch.distributed as dist

    from raydemo_b200 import api, scenes

    spp = 16
    spec = scenes.atrium(0)
    w, h = spec["size"]
    r = api.Renderer(w, h, device=dev.index)
    r.set_stream(stream.cuda_stream)
    sc = build_scene(api, r, spec)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def frame(reg):
        for _ in range(spp):
            r.RenderScene(sc, reg)

    # the 16-sample image (wavefront, no sorting) and its ray counts
    r.set_kernel(1)
    r.set_ray_sort(0)
    r.Clear()
    reg = api.RegionContext()
    rays = shadow = 0
    for _ in range(spp):
        r.RenderScene(sc, reg)
        info = r.frame_info()
        if info.error_flags:
            raise RuntimeError(f"render reported error flags {info.error_flags}")
        rays += info.rays
        shadow += info.shadow_rays
    image = r.get_pixels_ref()
    frames = max(2, min(args.steps // 10, 5))

    phase_us = {}  # per variant: the stats' phase times per frame (us)

    def timed(kernel: int, sort: int) -> float:
        r.set_kernel(kernel)
        r.set_ray_sort(sort)
        g = api.RegionContext()
        for _ in range(max(2, args.warmup // 3)):  # 16 RenderScene calls each: covers the tuner's timed frames
            frame(g)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        r.ResetStats()
        ev0.record(stream)
        for _ in range(frames):
            frame(g)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        phase_us[(kernel, sort)] = {k: int(v) // frames for k, v in r.GetStats().items()}
        return max_over_ranks(ev0.elapsed_time(ev1) / frames, world, dev)

    variants = {"wavefront_sort_off": timed(1, 0), "wavefront_sort_all": timed(1, 0x3FF), "wavefront_sort_auto": timed(1, -1)}
    auto_mask = r.frame_info().sort_mask
    variants["path"] = timed(2, 0)
    r.ResetStats()
    ms_frame = timed(0, -1)
    chosen = r.frame_info()
    stats = r.GetStats()
    # end to end: the 16 RenderScene calls and the pixels read back to the host
    g = api.RegionContext()
    ev0.record(stream)
    frame(g)
    img_h = r.get_pixels_ref()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e = ev0.elapsed_time(ev1)
    all_rays = rays + shadow
    out = {"workload": ATRIUM_WORKLOAD, "tris": int(spec["tris"]), "samples_per_frame": spp, "ms_per_frame": round(ms_frame, 3),
           "frames": frames, "mrays_per_s": round(world * all_rays / (ms_frame * 1e-3) / 1e6, 1), "rays_per_frame": int(all_rays),
           "closest_hit_rays_per_frame": int(rays), "shadow_rays_per_frame": int(shadow),
           "ms_per_frame_by_variant": {k: round(v, 3) for k, v in variants.items()},
           "auto_sort_mask": f"0x{auto_mask:03x}", "tuned": tuned_tuple(chosen),
           "phase_us_per_frame": {"wavefront_sort_off": phase_us.get((1, 0)), "wavefront_sort_all": phase_us.get((1, 0x3FF))},
           "chosen": {"kernel": {1: "wavefront", 2: "path"}.get(chosen.kernel, "?"),
                                                              "sort_mask": f"0x{chosen.sort_mask:03x}"},
           "e2e_ms_per_frame": round(ms_e2e, 3), "e2e_d2h_bytes_per_frame": w * h * 16, "data": "synthetic (seeded procedural scene)",
           "stats_us": {k: int(v) for k, v in stats.items()}}
    # ray sorting before every bounce against none: its cost in the sort phase and what it changes in the
    # secondary traces (the phase events of the two variants' timed frames)
    po, pa = phase_us.get((1, 0)) or {}, phase_us.get((1, 0x3FF)) or {}
    if po and pa:
        sort_ms = pa.get("time_secondary_sort_us", 0) / 1e3 - po.get("time_secondary_sort_us", 0) / 1e3
        tr_off, tr_all = po.get("time_secondary_trace_us", 0) / 1e3, pa.get("time_secondary_trace_us", 0) / 1e3
        out["ray_sorting"] = {"sort_ms_per_frame": round(sort_ms, 2), "secondary_trace_ms_unsorted": round(tr_off, 2),
                              "secondary_trace_ms_sorted": round(tr_all, 2),
                              "reading": ("sorting every bounce costs more than the sorted order saves in the secondary traces"
                                          if sort_ms > tr_off - tr_all else "the sorted order saves more than the sort costs")}
    del img_h
    if rank == 0 and world == 1 and args.atrium_oracle_spp > 0:
        from oracle.oracle import Oracle

        threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
        n = min(spp, args.atrium_oracle_spp)
        orc = Oracle()
        ps = orc.principled_scene(spec)
        t0 = time.perf_counter()
        ref = orc.render_principled(spec, n, nthreads=threads, scene=ps)
        cpu_s = time.perf_counter() - t0
        if n == spp:
            d = ref[..., :3].astype(np.float64) - image[..., :3]
            out["rmse_vs_oracle"] = float(np.sqrt(np.mean(d ** 2)))
            out["identical_px_vs_oracle"] = float(np.mean(np.all(ref == image, axis=-1)))
            out["max_abs_vs_oracle"] = float(np.max(np.abs(d)))
        out["cpu_baseline"] = {"ms_per_frame": round(cpu_s * 1e3 * spp / n, 1), "mrays_per_s": round(all_rays * n / spp / cpu_s / 1e6, 2),
                               "cores": threads, "kind": "port",
                               "sample": f"{n} of the frame's {spp} samples by the oracle's CPU restatement (single-ray BVH "
                                         f"traversal, {threads} threads); rays counted by the GPU renderer on the same paths"}
    r.set_stream(0)
    return out


DIFF_WORKLOAD = ("differentiable form: the atrium (16 displaced icospheres of subdivision 5, 8 materials) at 256x256, 8 samples, max 4 "
                 "bounces; parameters: 512x512 RGB albedo, 8 roughness slots; L2 image loss; path-replay adjoint")


def sort_frames(args, dev, stream) -> dict:
    """The ray sort (ray_sort_rays: get_ray_hash, then the stable one-sweep
    radix sort of the 32-bit keys, SortRays_CPU's order) on 921,600 rays (one
    1280x720 wavefront) and 4,194,304 rays, with and without the gather of
    the ray records; device buffers, CUDA events on the stream."""
    import ctypes as C

    import torch

    from raydemo_b200 import api, capi, scenes

    r = api.Renderer(16, 16, device=dev.index)
    L = capi.lib()
    rm = (C.c_float * 3)(0.0, 0.0, 0.0)
    cs = (C.c_float * 3)(1 / 255, 1 / 255, 1 / 255)
    out = {"workload": "ray hash + stable radix sort (+ gather of the 32-byte ray records), rays uniform in the unit cube"}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(5, min(args.steps, 50))
    for n in (921600, 4194304):
        rays = torch.from_numpy(scenes.incoherent_rays(n, seed=5)).to(dev)
        perm = torch.empty(n, dtype=torch.int32, device=dev)
        rout = torch.empty((n, 8), dtype=torch.float32, device=dev)
        for gather in (False, True):
            def call():
                capi.check(L.ray_sort_rays(r.handle, rays.data_ptr(), n, rm, cs, None, perm.data_ptr(),
                                           rout.data_ptr() if gather else None, stream.cuda_stream))
            for _ in range(3):
                call()
            torch.cuda.synchronize(dev)
            e0.record(stream)
            for _ in range(reps):
                call()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            out[f"us_{n}{'_gather' if gather else ''}"] = round(e0.elapsed_time(e1) / reps * 1e3, 1)
    return out


def diff_frames(args, dev, stream, rank: int, world: int) -> dict:
    """The differentiable configuration: forward (ray_render_diff) and adjoint
    (ray_render_adjoint) times through the torch harness, the adjoint's
    gradients against central differences (h = 1e-3) of this renderer and of
    the oracle, and Adam steps of inverse rendering from albedo 0.5 and
    roughness 0.5 towards a 1,024-sample image of the hidden parameters."""
    import torch

    from raydemo_b200 import api, diff, scenes

    spp, h_fd = 8, 1e-3
    spec = scenes.diff_atrium(0)
    w, h = spec["size"]
    r = api.Renderer(w, h, device=dev.index)
    sc = build_scene(api, r, spec)
    slots = spec["material_slot"]
    tgt_a = torch.tensor(spec["albedo_target"], device=dev)
    tgt_r = torch.tensor(spec["rough_target"], device=dev)

    def render(a, g, frozen=None):
        return diff.render(a, g, r, sc, slots, 1, spp, frozen)

    with torch.no_grad():
        target = render(tgt_a, tgt_r).clone()
    albedo = torch.full_like(tgt_a, 0.5).requires_grad_(True)
    rough = torch.full_like(tgt_r, 0.5).requires_grad_(True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    n_t = max(5, min(args.steps, 20))
    # forward alone, then forward + loss + adjoint (the gradient step); both warmed up first
    for _ in range(3):
        with torch.no_grad():
            render(albedo, rough)
        albedo.grad = rough.grad = None
        ((render(albedo, rough) - target) ** 2).sum().backward()
    torch.cuda.synchronize(dev)
    ev[0].record()
    for _ in range(n_t):
        with torch.no_grad():
            render(albedo, rough)
    ev[1].record()
    for _ in range(n_t):
        albedo.grad = rough.grad = None
        loss = ((render(albedo, rough) - target) ** 2).sum()
        loss.backward()
    ev[2].record()
    torch.cuda.synchronize(dev)
    fwd_ms = ev[0].elapsed_time(ev[1]) / n_t
    step_ms = ev[1].elapsed_time(ev[2]) / n_t
    ga = albedo.grad.detach().cpu().numpy().reshape(-1)
    gr = rough.grad.detach().cpu().numpy()

    def loss_of(a, g, frozen=None):
        with torch.no_grad():
            return float(((render(a, g, frozen).double() - target.double()) ** 2).sum())

    # gradient checks: 64 texels drawn at random from those the view sees well (the top fifth by gradient
    # magnitude: elsewhere the differences of a float32 image drown in its rounding), every roughness slot
    rng = np.random.default_rng(0)
    seen = np.flatnonzero(ga != 0.0)
    well = seen[np.argsort(-np.abs(ga[seen]))][: max(64, len(seen) // 5)]
    texels = rng.choice(well, size=min(64, len(well)), replace=False)
    a0, r0 = albedo.detach(), rough.detach()
    errs_a = []
    for i in texels:
        ap, am = a0.clone(), a0.clone()
        ap.view(-1)[int(i)] += h_fd
        am.view(-1)[int(i)] -= h_fd
        fd = (loss_of(ap, r0) - loss_of(am, r0)) / (2 * h_fd)
        errs_a.append(abs(ga[i] - fd) / max(abs(fd), 1e-12))
    errs_r, fd_r, fd_r_attached = [], [], []
    for k in range(len(gr)):
        gp, gm = r0.clone(), r0.clone()
        gp[k] += h_fd
        gm[k] -= h_fd
        fd = (loss_of(a0, gp, r0) - loss_of(a0, gm, r0)) / (2 * h_fd)
        fd_r.append(fd)
        errs_r.append(abs(gr[k] - fd) / max(abs(fd), 1e-12))
        fd_r_attached.append((loss_of(a0, gp) - loss_of(a0, gm)) / (2 * h_fd))
    out = {"workload": DIFF_WORKLOAD, "samples": spp, "forward_ms": round(fwd_ms, 3), "grad_step_ms": round(step_ms, 3),
           "adjoint_ms": round(step_ms - fwd_ms, 3), "grad_step_over_forward": round(step_ms / fwd_ms, 3),
           "fd_h": h_fd, "albedo_texels_checked": len(texels), "albedo_max_rel_err_vs_fd": round(float(max(errs_a)), 5),
           "albedo_within_2pct": f"{sum(e <= 0.02 for e in errs_a)}/{len(errs_a)}",
           "roughness_grad": [round(float(x), 4) for x in gr], "roughness_fd_frozen_sampling": [round(float(x), 4) for x in fd_r],
           "roughness_max_rel_err_vs_fd": round(float(max(errs_r)), 5),
           "roughness_within_2pct": f"{sum(e <= 0.02 for e in errs_r)}/{len(errs_r)}",
           "roughness_fd_same_samples_unfrozen": [round(float(x), 2) for x in fd_r_attached]}
    if rank == 0 and world == 1 and args.diff_oracle_fd:
        from oracle.oracle import Oracle

        orc = Oracle()
        threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
        tnp = target.cpu().numpy().astype(np.float64)
        a_np, r_np = a0.cpu().numpy(), r0.cpu().numpy()

        def oloss(a, g):
            ps = orc.principled_scene(spec, a, g, slots, roughness_sampling=r_np)
            img = orc.render_principled(spec, spp, nthreads=threads, scene=ps, plain_mean=True)[..., :3].astype(np.float64)
            return float(((img - tnp) ** 2).sum())

        t0 = time.perf_counter()
        oerr_r = []
        for k in range(len(gr)):
            gp, gm = r_np.copy(), r_np.copy()
            gp[k] += h_fd
            gm[k] -= h_fd
            fd = (oloss(a_np, gp) - oloss(a_np, gm)) / (2 * h_fd)
            oerr_r.append(abs(gr[k] - fd) / max(abs(fd), 1e-12))
        oerr_a = []
        for i in texels[:8]:
            ap, am = a_np.copy().reshape(-1), a_np.copy().reshape(-1)
            ap[i] += h_fd
            am[i] -= h_fd
            fd = (oloss(ap.reshape(a_np.shape), r_np) - oloss(am.reshape(a_np.shape), r_np)) / (2 * h_fd)
            oerr_a.append(abs(ga[i] - fd) / max(abs(fd), 1e-12))
        out["oracle_fd"] = {"roughness_max_rel_err": round(float(max(oerr_r)), 5), "albedo_texels": len(oerr_a),
                            "albedo_max_rel_err": round(float(max(oerr_a)), 5), "seconds": round(time.perf_counter() - t0, 1),
                            "threads": threads}
    # inverse rendering: Adam steps (cosine-decayed learning rates) towards a 1,024-sample target, whose noise
    # floor sits far below the per-step loss. Each step takes the residual from one render and the adjoint from
    # an independent one (other samples): with the same samples for both, the gradient would also follow the
    # estimator's variance, which pulls the parameters away from the truth. A call's samples stay inside one
    # block of 256 iterations of the sample tables, so the target is 16 calls of 64 samples over four blocks, the
    # optimisation draws from a fifth and the 64-sample loss checks from a sixth.
    ispp = args.diff_inverse_spp
    with torch.no_grad():
        firsts = [1, 65, 129] + [256 * b + 64 * k for b in (1, 2, 3) for k in range(4)] + [1024]
        acc = torch.zeros_like(target)
        for f in firsts:
            acc += diff.render(tgt_a, tgt_r, r, sc, slots, f, 64)
        target = acc / len(firsts)
    albedo = torch.full_like(tgt_a, 0.5).requires_grad_(True)
    rough = torch.full_like(tgt_r, 0.5).requires_grad_(True)
    opt = torch.optim.Adam([{"params": [albedo], "lr": args.diff_lr_albedo}, {"params": [rough], "lr": args.diff_lr_rough}])
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, max(1, args.diff_steps))

    def loss64():  # the image loss at 64 samples (its noise floor far below the per-step loss's)
        with torch.no_grad():
            return float(((diff.render(albedo, rough, r, sc, slots, 1600, 64) - target) ** 2).sum())

    with torch.no_grad():  # the floor: another 64-sample render at the hidden parameters
        loss64_truth = float(((diff.render(tgt_a, tgt_r, r, sc, slots, 1600, 64) - target) ** 2).sum())
    loss64_start = loss64()
    losses = []
    t0 = time.perf_counter()
    for step in range(args.diff_steps):
        opt.zero_grad()
        first = 1280 + (2 * ispp * step) % (256 - 2 * ispp)
        with torch.no_grad():
            resid = diff.render(albedo, rough, r, sc, slots, first, ispp) - target
        img = diff.render(albedo, rough, r, sc, slots, first + ispp, ispp)
        (2.0 * resid * img).sum().backward()  # gradient 2 (I_a - T) dI_b
        opt.step()
        sched.step()
        with torch.no_grad():
            albedo.clamp_(0.0, 1.0)
            rough.clamp_(0.05, 1.0)
        losses.append(float((resid ** 2).sum()))
    torch.cuda.synchronize(dev)

    def rmse(values, idx):
        mask = torch.zeros(tgt_a.numel(), dtype=torch.bool, device=dev)
        mask[torch.as_tensor(idx, device=dev)] = True
        return float(((values.reshape(-1) - tgt_a.reshape(-1))[mask] ** 2).mean().sqrt())

    half = torch.full_like(tgt_a, 0.5)
    secs = time.perf_counter() - t0
    loss64_end = loss64()
    out["inverse"] = {"steps": args.diff_steps, "seconds": round(secs, 2), "samples_per_render": ispp,
                      "lr": [args.diff_lr_albedo, args.diff_lr_rough], "lr_schedule": "cosine", "target_samples": 64 * len(firsts),
                      "loss_first": round(losses[0], 3), "loss_last": round(losses[-1], 3),
                      "loss64_start": round(loss64_start, 3), "loss64_end": round(loss64_end, 3),
                      "loss64_ratio": round(loss64_end / loss64_start, 5), "loss64_at_hidden_parameters": round(loss64_truth, 3),
                      "roughness_mae_start": round(float((0.5 - tgt_r).abs().mean()), 4),
                      "roughness_mae_end": round(float((rough.detach() - tgt_r).abs().mean()), 4),
                      "albedo_rmse_seen_start": round(rmse(half, seen), 4), "albedo_rmse_seen_end": round(rmse(albedo.detach(), seen), 4),
                      "albedo_texels_well_seen": int(len(well)),
                      "albedo_rmse_well_seen_start": round(rmse(half, well), 4),
                      "albedo_rmse_well_seen_end": round(rmse(albedo.detach(), well), 4)}
    r.set_stream(0)
    return out


def run_reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    tris, rays = make_workload(0)
    sample = args.cpu_sample
    vals, threads, build_s = cpu_reference(tris, rays, sample, max(1, args.steps), max(0, args.warmup))
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(sample / (v * 1e6) * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene and rays)",
            "config": {"workload": WORKLOAD, "rays_per_step": sample, "tris": N_TRIS, "bvh_build_s": round(build_s, 2)},
            "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{sample} rays drawn from the 4,194,304-ray set per step; Ref SAH wide BVH; AVX2 8-ray packets"},
            "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_gpu_arm(args) -> None:
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    from raydemo_b200.api import Renderer
    from raydemo_b200 import scenes

    if args.render_only or args.batch_only or args.atrium_only or args.diff_only or args.sort_only:  # one part alone (for profiling)
        stream = torch.cuda.Stream(dev)
        torch.cuda.set_stream(stream)
        args.no_cpu_baseline = True
        if args.sort_only:
            out = {"sort": sort_frames(args, dev, stream)}
        elif args.render_only:
            out = {"render": render_frames(args, dev, stream, rank, world)}
        elif args.batch_only:
            out = {"batch": batch_frames(args, dev, stream, n_scenes=args.batch_scenes)}
        elif args.atrium_only:
            out = {"atrium": atrium_frames(args, dev, stream, rank, world)}
        else:
            out = {"diff": diff_frames(args, dev, stream, rank, world)}
        if rank == 0:
            print(json.dumps(out), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    tris, rays = make_workload(rank)
    r = Renderer(64, 64, device=local)
    sc = r.CreateScene()
    attrs, idx = scenes.triangle_soup_mesh(tris)
    mat = sc.AddMaterial()
    sc.AddMeshInstance(sc.AddMesh(attrs, idx, [(mat, 0, len(idx))]))
    t0 = time.perf_counter()
    sc.Commit()
    build_s = time.perf_counter() - t0
    info = sc.mesh_bvh_info(0)

    rays_d = torch.from_numpy(rays).to(dev)
    hits_d = torch.empty((N_RAYS, 4), dtype=torch.float32, device=dev)
    # an explicit stream: the kernels and the timing events share it (a null
    # handle would mean the scene's own stream to the C ABI)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream

    def step():
        sc.trace_closest_device(rays_d.data_ptr(), N_RAYS, hits_d.data_ptr(), 0, sptr)

    # the library's trace tuner (ray_scene_tune_trace) on this scene and these
    # rays: kernel, L2 residency, cache hint, refill threshold, block size with
    # stack depth and trace order, one at a time, each the best of two timed
    # traces; the timed steps use its choice (--trace-tuning default: the
    # library's defaults instead)
    tune_report = {}
    if args.trace_tuning == "auto":
        chosen, rep = sc.tune_trace_device(rays_d.data_ptr(), N_RAYS, hits_d.data_ptr(), sptr, force=True)
        for item in rep.split(";"):
            k, sep, v = item.partition("=")
            if sep:
                tune_report[k] = v if k == "chosen" else round(float(v), 4)
    tuning = sc.get_trace_tuning()
    names = ("kernel", "refill_min", "deep_stack", "reorder", "reorder_bits", "block", "smem_stack", "stream_hint", "l2_persist")
    # kernels per step: the trace; with a trace order also the key kernel, the
    # sort's histogram and digit passes (and its copy when they are odd)
    passes = (tuning[4] + 7) // 8
    launches_per_step = 1 + ((2 + passes + (passes & 1)) if tuning[3] else 0)

    # counting pass: node visits and triangle tests of this BVH (algorithmic bytes)
    sc.set_counting(True)
    step()
    cnt = sc.last_trace_info()
    sc.set_counting(False)
    if cnt.error_flags:
        raise RuntimeError(f"trace reported error flags {cnt.error_flags}")
    node_visits, tri_tests = cnt.node_visits, cnt.tri_tests

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    if sc.last_trace_info().error_flags:
        raise RuntimeError("trace reported an error during the timed steps")
    ms_max = max_over_ranks(ms, world, dev)
    ms_step = ms_max / args.steps
    value = world * N_RAYS / (ms_step * 1e-3) / 1e6

    # end to end through the C ABI with pinned host buffers (H2D + kernel + D2H)
    rays_h = torch.from_numpy(rays).pin_memory()
    hits_h = torch.empty((N_RAYS, 4), dtype=torch.float32).pin_memory()
    from raydemo_b200 import capi

    def e2e_step():
        capi.check(capi.lib().ray_scene_trace_closest(sc.handle, rays_h.data_ptr(), N_RAYS, hits_h.data_ptr(), None,
                                                      capi.RAY_MEM_HOST, sptr))

    for _ in range(2):
        e2e_step()
    e_steps = max(3, min(args.steps, 20))
    if world > 1:
        dist.barrier()
    ev0.record(stream)
    for _ in range(e_steps):
        e2e_step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    te_max = max_over_ranks(ev0.elapsed_time(ev1) / e_steps, world, dev)
    e2e_value = world * N_RAYS / (te_max * 1e-3) / 1e6
    hits_dev = hits_d.cpu().numpy().view(np.uint32)
    ok = np.array_equal(hits_h.numpy().view(np.uint32), hits_dev)
    # every hit of the timed workload against the compiled reference (digests of its Ref traversal)
    parity = parity_vs_reference("inc", tris, rays, hits_dev) if world == 1 or rank == 0 else None

    # the same scene and kernel on 4,194,304 coherent rays (a pinhole camera at 2048x2048 outside the cube)
    coh_rays = scenes.coherent_rays(2048, 2048)
    coh = torch.from_numpy(coh_rays).to(dev)
    for _ in range(3):
        sc.trace_closest_device(coh.data_ptr(), N_RAYS, hits_d.data_ptr(), 0, sptr)
    torch.cuda.synchronize(dev)
    ev0.record(stream)
    c_steps = max(3, min(args.steps, 20))
    for _ in range(c_steps):
        sc.trace_closest_device(coh.data_ptr(), N_RAYS, hits_d.data_ptr(), 0, sptr)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    coh_ms = ev0.elapsed_time(ev1) / c_steps
    coh_hits = hits_d[:, 0].view(torch.int32)
    coherent = {"rays": N_RAYS, "ms_per_step": round(coh_ms, 4), "mrays_per_s": round(N_RAYS / (coh_ms * 1e-3) / 1e6, 1),
                "hit_rate": round(float((coh_hits >= 0).float().mean()), 4),
                "camera": "pinhole at (0.5, 0.5, -1.5), fov 45 deg, one ray per pixel centre of 2048x2048",
                "parity": parity_vs_reference("coh", tris, coh_rays, hits_d.cpu().numpy().view(np.uint32)) if rank == 0 else None}
    del coh

    # roofline of the traversal kernel (the only kernel in the timed region).
    # achieved = the algorithmic byte stream (rays, hits, nodes visited,
    # triangles tested) per launch over the launch time: a request stream
    # served mostly by L1/L2, stated against the HBM copy peak as the
    # contract's frac. The kernel is bound by instruction issue (divergent
    # traversal), not by DRAM: dram_frac (ncu DRAM bytes of one launch over
    # the same launch time) and the profile's issue and L2 figures say so.
    p = peaks()
    bytes_per_launch = N_RAYS * 44 + node_visits * 80 + tri_tests * 48
    launch_s = ms / args.steps * 1e-3
    achieved = bytes_per_launch / launch_s / 1e9
    prof = profiled()
    traffic = args.traffic_bytes if args.traffic_bytes is not None else prof.get("dram_bytes_per_launch")
    roofline = {"bound": "issue", "achieved": round(achieved, 1), "peak": p["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / p["hbm_gbs"], 4), "traffic": traffic, "peak_source": p["source"],
                "achieved_is": "algorithmic request stream (44 B per ray + 80 B per node visit + 48 B per triangle test), served by L1/L2",
                "dram_frac": round(traffic / launch_s / 1e9 / p["hbm_gbs"], 4) if traffic else None,
                "l2_frac": round(prof["l2_throughput_pct"] / 100, 4) if "l2_throughput_pct" in prof else None,
                "issue_active_frac": round(prof["issue_active_pct"] / 100, 4) if "issue_active_pct" in prof else None,
                "lanes_active_of_32": prof.get("lanes_active"),
                "profile": "profiles/trace_closest_microbench.txt",
                "alg_bytes_per_launch": int(bytes_per_launch), "node_visits_per_ray": round(node_visits / N_RAYS, 3),
                "tri_tests_per_ray": round(tri_tests / N_RAYS, 3)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            vals, threads, bs = cpu_reference(tris, rays, args.cpu_sample, 3, 1)
            cpu = {"value": round(statistics.median(vals), 4), "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"{args.cpu_sample} rays x 3 steps from the same 4,194,304-ray set; Ref SAH wide BVH "
                             f"(build {bs:.1f} s, excluded); AVX2 8-ray packets"}
        except FileNotFoundError as e:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}

    sort = sort_frames(args, dev, stream) if rank == 0 and not args.no_sort else None
    render = None if args.no_render else render_frames(args, dev, stream, rank, world)
    batch = None if args.no_batch else batch_frames(args, dev, stream)
    atrium = None if args.no_atrium else atrium_frames(args, dev, stream, rank, world)
    diffr = None if args.no_diff else diff_frames(args, dev, stream, rank, world)

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded procedural scene and rays)",
                "config": {"workload": WORKLOAD, "rays_per_step_per_gpu": N_RAYS, "tris": N_TRIS,
                           "l2": "inputs larger than L2 (rays 128 MiB per step, hits 64 MiB)", "bvh_build_s": round(build_s, 3),
                           "bvh_nodes": info.nodes, "bvh_depth": info.depth, "parallelism": f"replicas x{world}",
                           "trace_tuning": {"chosen": dict(zip(names, tuning)), "tuner": args.trace_tuning,
                                            "ms_per_trace_by_candidate": tune_report}},
                "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": N_RAYS * 32, "d2h_bytes_per_step": N_RAYS * 16,
                        "matches_device_path": bool(ok)},
                "parity": parity, "gpu_launches": args.steps * launches_per_step, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(), "coherent": coherent,
                "sort": sort, "render": render, "batch": batch,
                "atrium": atrium, "diff": diffr}
        print(json.dumps(line), flush=True)
    del sc, r
    if world > 1:
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=262144)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-render", action="store_true", help="skip the render-loop frames")
    ap.add_argument("--render-only", action="store_true", help="only the render-loop frames (no microbench, no CPU baseline)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-form measurement")
    ap.add_argument("--batch-only", action="store_true", help="only the batched-form measurement")
    ap.add_argument("--batch-no-plain", action="store_true", help="with --batch-only: two wavefront batches, nothing timed (profiling)")
    ap.add_argument("--batch-scenes", type=int, default=64, help="with --batch-only: the first N scenes of the batch")
    ap.add_argument("--no-atrium", action="store_true", help="skip the metallic-roughness atrium frames")
    ap.add_argument("--atrium-only", action="store_true", help="only the atrium frames")
    ap.add_argument("--atrium-oracle-spp", type=int, default=16,
                    help="samples the oracle renders for the atrium's image check and CPU time (16: the whole frame; 0: none)")
    ap.add_argument("--no-diff", action="store_true", help="skip the differentiable form")
    ap.add_argument("--diff-only", action="store_true", help="only the differentiable form")
    ap.add_argument("--sort-only", action="store_true", help="only the ray sort")
    ap.add_argument("--no-sort", action="store_true", help="skip the ray sort measurement")
    ap.add_argument("--diff-steps", type=int, default=200, help="Adam steps of the inverse-rendering run")
    ap.add_argument("--diff-inverse-spp", type=int, default=32, help="samples per render in an inverse-rendering step")
    ap.add_argument("--diff-lr-albedo", type=float, default=2e-3)
    ap.add_argument("--diff-lr-rough", type=float, default=2e-3)
    ap.add_argument("--no-diff-oracle-fd", dest="diff_oracle_fd", action="store_false",
                    help="skip the oracle's finite differences in the differentiable form")
    ap.add_argument("--trace-tuning", default="auto", choices=["auto", "default"],
                    help="auto: the library's trace tuner picks the settings of the timed steps; default: its defaults")
    ap.add_argument("--traffic-bytes", type=float, default=None,
                    help="DRAM bytes per launch of the traversal kernel from an ncu capture (reported as roofline.traffic)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
