#!/usr/bin/env python
"""Benchmark of the B200 path tracer on the plain-method scenes.

One "step" is one complete render of the workload: every pixel traced until
it reaches its sample budget or converges (pt_render with no wave limit),
starting from a reset accumulator with the scene resident in HBM.  The
default workload is plain-large (972k-triangle stochastic tree, 1024x1024,
adaptive 16-1024 spp, depth 12); --config plain-small selects the 20k-triangle
2D tree at 256x256, 64 spp; --config batch the 64-scene batching workload
(scenes built on the device, all rendered by one pt_render; the line also
carries the time of the same scenes rendered one per pt_render); --config
adjoint the differentiation workload (path-replay gradient, Adam steps);
--config forest the instanced forest (263M instanced triangles, sun + sky, 4
views of 1920x1080 per launch; a step takes about a minute, so run it with
--steps 1).

  value  Msamples/s of the device-timed steps (CUDA events on the stream the
         library launches on), summed over ranks, time = max over ranks.
  e2e    the same metric through the public API with HOST buffers: per step
         the mesh is uploaded from pinned host memory (and the BVH rebuilt),
         camera and params set, the image rendered and read back to pinned
         host memory.
  roofline  for the closest-hit traversal kernel (the dominant kernel):
         algorithmic bytes per ray (80 B per compressed node + 48 B per
         triangle visited, + 32 B ray in + 16 B hit out) x rays per launch /
         launch time.
  cpu_baseline  the reference's own render code compiled for the host
         (oracle/_ref, OpenMP over pixels) on a bounded pixel sample.

Multi-GPU: for the plain, adjoint and forest workloads every rank renders its
own copy of the workload (pixels and scenes are independent; no data-path
collective) -> weak scaling.  The batch workload is split by whole scenes over
the ranks by estimated cost (lsystemeditor_b200/partition.py), each rank
renders its scenes in one batch and every image is gathered once to rank 0
inside the timed step -> strong scaling.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import signal
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Msamples/s"
L2_FLUSH_BYTES = 256 << 20


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--config", choices=["plain-small", "plain-large", "batch", "adjoint", "forest"],
                    default="plain-large")
    ap.add_argument("--opt-steps", type=int, default=200, help="Adam steps of the adjoint workload's optimisation")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the leg that times the reference's own CUDA kernels on this GPU")
    ap.add_argument("--no-autotune", action="store_true", help="batch workload: keep the default scheduling knobs")
    ap.add_argument("--estimator", choices=["mis", "reference"], default="mis",
                    help="batch workload: the emitter MIS estimator (short emissive shadow rays) or the "
                         "reference's estimator (emitters found by BSDF sampling only)")
    ap.add_argument("--rel-err", type=float, default=0.02,
                    help="batch workload: per-pixel relative standard error at which a pixel stops")
    ap.add_argument("--spp-cap", type=int, default=512,
                    help="batch workload: samples per pixel at which a pixel stops at the latest (the workload "
                         "definition's 512; pixels lit through the foliage stay above the relative-MSE target "
                         "at 4096 too)")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="batch workload: skip the FP64-oracle check of the batch's relative MSE")
    ap.add_argument("--spectral", default="auto", choices=["auto", "0", "4", "8"],
                    help="hero wavelengths per path: auto = the workload's own (plain-small 4, plain-large 8, "
                         "batch and adjoint RGB), 0 = RGB like the reference's integrator")
    return ap.parse_args()


def make_workload(name: str):
    from lsystemeditor_b200.scene import SceneSpec, batch_scenes, config0_scene, config1_scene
    if name == "plain-small":
        return config0_scene()
    if name == "plain-large":
        return config1_scene()
    if name == "adjoint":
        from lsystemeditor_b200.scene import config3_scene
        return config3_scene()
    if name == "batch":
        # host-side stand-in for the CPU arms: the scene of the batch with the
        # median triangle count, lofted on the host, with the batch's params
        tubes, cams, sizes, params = batch_scenes()
        order = np.argsort([t.triangle_count for t in tubes], kind="stable")
        k = int(order[len(order) // 2])
        mesh = tubes[k].host_mesh()
        w, h = sizes[k]
        return SceneSpec(f"batch scene {k} of 64 ({mesh.triangle_count} triangles, {w}x{h}, adaptive 16-512 spp "
                         "to relative std-error 0.03, depth 12)", mesh, cams[k], params, w, h, 512)
    raise ValueError(name)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
REASON_BITS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}


class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 4:
                    continue
                try:
                    sm.append(float(parts[0]))
                    smax.append(float(parts[1]))
                    bits = int(parts[3], 16)
                except ValueError:
                    continue
                for b, name in REASON_BITS.items():
                    if bits & b and name != "gpu_idle":
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's render code on the host cores
# ---------------------------------------------------------------------------
CONFIG0_GRAMMAR = "F(0.1,0.02)\nF(h,r) -> F(h,r)[Yaw(25.7)F(h,r)]F(h,r)[Yaw(0-25.7)F(h,r)]F(h,r)"


def host_stage_times(chk, spec) -> dict:
    """The reference's host stages: its L-system evaluator, turtle, spline frames
    and loft on the plain-small grammar (the reference's syntax, 4 iterations,
    8 sides; oracle/_ref/libptref_gen.so), and its BVH + emissive-CDF build
    (MeshAccelScene::build, meshAccelBuildBvh) of the workload's mesh."""
    out = {}
    try:
        from oracle.bindings import ReferenceGenerator, reference_generator_available
        if reference_generator_available():
            g = ReferenceGenerator().build(CONFIG0_GRAMMAR, 4, rotation_deg=(0.0, 90.0, 0.0), sides=8)
            out["plain_small_generator"] = {k: round(float(v), 3) for k, v in g["ms"].items()}
            out["plain_small_generator"]["triangles"] = int(g["positions"].shape[0])
    except Exception as e:  # reported, never fatal
        out["plain_small_generator"] = f"unavailable: {e}"
    t0 = time.perf_counter()
    sc = chk.scene(spec.mesh)
    out["bvh_and_scene_build"] = {"ms": round((time.perf_counter() - t0) * 1e3, 1),
                                  "triangles": int(spec.mesh.triangle_count), "nodes": sc.bvh_node_count()}
    return out


def cpu_render_rate(spec, min_seconds: float = 10.0, max_pixels: int | None = None, seed: int = 0):
    """Times the host render (reference build when present, else the oracle port) on a pixel sample."""
    from oracle.bindings import Checker, reference_available
    kind = "reference" if reference_available() else "port"
    chk = Checker("ref" if kind == "reference" else "oracle")
    stages = host_stage_times(chk, spec)
    sc = chk.scene(spec.mesh)
    threads = chk.max_threads()
    P = spec.width * spec.height
    rng = np.random.default_rng(seed)
    # calibrate on a small sample, then size the sample for ~min_seconds
    n = min(P, 256)
    pix = np.sort(rng.choice(P, n, replace=False)).astype(np.int32)
    t0 = time.perf_counter()
    st = sc.render(spec.camera, spec.params, spec.width, spec.height, spec.waves, pixels=pix, threads=threads)
    dt = max(time.perf_counter() - t0, 1e-3)
    per_pixel = dt / n
    n = int(min(P, max(256, min_seconds / per_pixel)))
    if max_pixels:
        n = min(n, max_pixels)
    pix = np.sort(rng.choice(P, n, replace=False)).astype(np.int32)
    # whole frames when the image is small: repeat (fresh accumulation, new seeds) until min_seconds
    samples, reps = 0, 0
    t0 = time.perf_counter()
    while True:
        st = sc.render(spec.camera, spec.params, spec.width, spec.height, spec.waves, pixels=pix, threads=threads,
                       seed_base=1 + reps * spec.waves)
        samples += int(st["counts"][pix].sum())
        reps += 1
        dt = time.perf_counter() - t0
        if dt >= min_seconds or reps >= 1000:
            break
    return {"value": samples / dt / 1e6, "unit": METRIC, "cores": int(threads), "kind": kind,
            "sample": f"{n} of {P} pixels x up to {spec.waves} samples, {reps} frame(s) ({samples} path samples, "
                      f"{dt:.1f} s), same scene/camera/params, PCG32 random numbers",
            "host_stages_ms": stages}


def reference_gpu_leg(spec, pt, stream, max_waves: int = 0):
    """The reference's own megakernel (PathTracer.cu compiled unchanged for sm_100a,
    oracle/_ref/libptref_gpu.so) on this GPU, driven by its render loop's wave
    sequence, on the workload's scene, camera, resolution and sample budget with
    the reference's estimator (RGB, relative std-dev stop test); beside it the
    B200 path on exactly those parameters.  A baseline leg: reported, not the
    headline value."""
    import torch

    from oracle.bindings import ReferenceGpu, reference_gpu_available
    if not reference_gpu_available():
        return {"unavailable": "oracle/_ref/libptref_gpu.so not built (no reference tree where build() ran)"}
    params = np.array(spec.params, copy=True)
    params["spectral_wavelengths"] = 0
    params["adaptive_criterion"] = 0
    rg = ReferenceGpu()
    sc = rg.scene(spec.mesh)
    sc.render(spec.camera, params, spec.width, spec.height, max_waves=4)  # warm-up: module load, first launches
    torch.cuda.synchronize()
    r = sc.render(spec.camera, params, spec.width, spec.height, max_waves=max_waves)
    ref_value = r["samples"] / (r["device_ms"] / 1e3) / 1e6
    # the B200 path on the same parameters (RGB, the reference's stop test)
    saved = pt.params()
    pt.set_params(params)
    pt.reset_accumulation()
    pt.render(max_waves)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pt.reset_accumulation()
    a.record(stream)
    pt.render(max_waves)
    b.record(stream)
    torch.cuda.synchronize()
    ours_ms = a.elapsed_time(b)
    ours_samples = float(pt.stats()["samples"])
    _, counts, _ = pt.readback()
    pt.set_params(saved)
    same_counts = float(np.mean(counts.reshape(-1) == r["counts"]))
    return {
        "value": ref_value, "unit": METRIC, "kind": "reference megakernel (PathTracer.cu sampleAdaptiveKernel, "
        "unchanged, nvcc for sm_100a) driven by its render loop's wave sequence, per-wave host wait",
        "estimator": "RGB, relative std-dev < %g, %d-%d spp" % (float(params["relative_error_threshold"]),
                                                               int(params["min_samples"]),
                                                               int(params["max_samples_per_pixel"])),
        "frame_ms": r["device_ms"], "waves": r["waves"], "samples": r["samples"],
        "host_bvh_build_ms": sc.build_ms, "bvh_nodes": sc.bvh_node_count(),
        "b200_same_params": {"value": ours_samples / (ours_ms / 1e3) / 1e6, "unit": METRIC, "frame_ms": ours_ms,
                             "samples": ours_samples, "pixels_with_equal_counts": same_counts},
    }


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    spec = make_workload(args.config)
    try:
        from oracle.bindings import reference_available
        kind = "reference" if reference_available() else "port"
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"host checker cannot be built: {e}"}))
        return 0
    # bounded sample per step: ~5 s of CPU work
    for _ in range(args.warmup):
        cpu_render_rate(spec, min_seconds=1.0)
    rates, descr = [], None
    t0 = time.perf_counter()
    for k in range(args.steps):
        r = cpu_render_rate(spec, min_seconds=5.0, seed=k + 1)
        rates.append(r["value"])
        descr = r
    wall = time.perf_counter() - t0
    value = float(np.mean(rates))
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {**workload_config(spec, args.config), "colour": colour_note(0) + "; the B200 arm renders "
                   + colour_note(wavelengths(args))},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": descr["cores"], "kind": kind,
                         "sample": descr["sample"]},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


WORKLOAD_WAVELENGTHS = {"plain-small": 4, "plain-large": 8, "batch": 0, "adjoint": 0, "forest": 8}


def wavelengths(args) -> int:
    return WORKLOAD_WAVELENGTHS[args.config] if args.spectral == "auto" else int(args.spectral)


def colour_note(nw: int) -> str:
    if nw == 0:
        return "RGB (the reference's integrator)"
    return (f"hero-wavelength spectral, {nw} wavelengths per path over 380-780 nm, CIE 1931 x D65 -> linear sRGB "
            "per sample")


def workload_config(spec, name):
    m = spec.mesh
    return {"workload": spec.name, "width": spec.width, "height": spec.height,
            "spp": int(spec.params["max_samples_per_pixel"]), "min_spp": int(spec.params["min_samples"]),
            "adaptive": ("relative std-error" if int(spec.params["adaptive_criterion"]) == 1 else "relative std-dev")
            + f" < {float(spec.params['relative_error_threshold']):g}",
            "max_depth": int(spec.params["max_path_depth"]), "triangles": int(m.triangle_count),
            "materials": int(len(m.materials)), "seed": "reference per-(pixel, sample) seed",
            "l2": "flushed between timed steps (256 MiB write, untimed)"}


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def run_b200(args):
    import torch

    from lsystemeditor_b200.pathtracer import PROFILE_COUNT_VISITS, PROFILE_STAGE_TIMES, PathTracer
    from lsystemeditor_b200.replicas import Replicas

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    # one replica of the workload per GPU; ranks meet only for the timing (NCCL)
    reps = Replicas(backend="nccl", device="cuda", timeout_s=300.0)
    world, rank = reps.world, reps.rank
    barrier, max_over_ranks, sum_over_ranks = reps.barrier, reps.max, reps.sum

    spec = make_workload(args.config)
    nw = wavelengths(args)
    spec.params["spectral_wavelengths"] = nw
    stream = torch.cuda.current_stream()
    pt = PathTracer(local)
    pt.set_stream(stream.cuda_stream)
    pt.configure(spec.width, spec.height, spec.mesh)
    pt.set_camera(spec.camera)
    pt.set_params(spec.params)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def step():
        pt.reset_accumulation()
        pt.render(0)

    # warm-up (also allocates path state and sample buffers)
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    # ---- timed region: K device-timed renders ----------------------------
    launches0 = pt.stats()["launches"]
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    samples = 0
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    for k in range(args.steps):
        flush.zero_()
        evs[k][0].record(stream)
        step()
        evs[k][1].record(stream)
        samples += pt.stats()["samples"]
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = pt.stats()["launches"] - launches0
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(float(sum(step_ms)))
    total_samples = sum_over_ranks(float(samples))
    value = total_samples / (total_ms / 1e3) / 1e6

    # ---- the same K renders again with CUDA events around every stage launch
    # (on the launch stream) for the kernel durations of the roofline ---------
    pt.set_profiling(PROFILE_STAGE_TIMES)
    stages = {}
    ext_ms, ext_launches, ext_rays = 0.0, 0, 0
    for k in range(args.steps):
        flush.zero_()
        step()
        prof = pt.profile()
        for key, v in prof.items():
            if key.startswith("ms_"):
                stages[key[3:]] = stages.get(key[3:], 0.0) + v / args.steps
        ext_ms += prof["ms_extend"]
        ext_launches += prof["launches_extend"]
        ext_rays += prof["rays_extend"]
    pt.set_profiling(0)

    # ---- traversal statistics for the roofline (untimed counting pass) ----
    pt.set_profiling(PROFILE_COUNT_VISITS | PROFILE_STAGE_TIMES)
    step()
    cp = pt.profile()
    pt.set_profiling(0)
    nodes_per_ray = cp["nodes_extend"] / max(cp["rays_extend"], 1)
    tris_per_ray = cp["tris_extend"] / max(cp["rays_extend"], 1)
    bytes_per_ray = 80.0 * nodes_per_ray + 48.0 * tris_per_ray + 32.0 + 16.0
    rays_per_launch = ext_rays / max(ext_launches, 1)
    launch_ms = ext_ms / max(ext_launches, 1)
    achieved = bytes_per_ray * rays_per_launch / (launch_ms / 1e3) / 1e9 if launch_ms > 0 else None
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    # the traversal's working set (nodes + leaf triangles) fits in L2 for the
    # plain scenes: its own roof is the L2-resident read bandwidth, measured here
    l2_peak = pt.measure_l2(32 << 20, 64)
    working_set = 80.0 * pt.stats()["bvh_nodes"] + 48.0 * spec.mesh.triangle_count
    # DRAM bytes per k_extend ray from an ncu capture (profiles/), scaled to a launch
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_extend.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            t = json.load(f).get(args.config, {})
        if t.get("bytes_per_ray"):
            traffic = t["bytes_per_ray"] * rays_per_launch

    # ---- end to end through the public API with host buffers ---------------
    m = spec.mesh.contiguous()

    def pinned(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        v = t.numpy().view(a.dtype).reshape(a.shape)
        v[...] = a
        return t, v

    keep = []
    pm = type(m)(*[None] * 6)
    for field in ("positions", "normals", "uvs", "material_ids", "materials", "textures"):
        t, v = pinned(getattr(m, field))
        keep.append(t)
        setattr(pm, field, v)
    # the step's result is read back into pinned host memory
    rgba_t = torch.empty((spec.height, spec.width, 4), dtype=torch.float32, pin_memory=True)
    counts_t = torch.empty((spec.height, spec.width), dtype=torch.int32, pin_memory=True)
    conv_t = torch.empty((spec.height, spec.width), dtype=torch.uint8, pin_memory=True)
    out_bufs = (rgba_t.numpy(), counts_t.numpy().view(np.uint32), conv_t.numpy())
    h2d = sum(getattr(m, f).nbytes for f in ("positions", "normals", "uvs", "material_ids", "materials",
                                                "textures")) + 80 + 64
    d2h = spec.width * spec.height * (16 + 4 + 1)

    def e2e_step():
        pt.set_mesh(pm)
        pt.set_camera(spec.camera)
        pt.set_params(spec.params)
        pt.render(0)
        pt.readback(out_bufs)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    e_evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    e_samples = 0
    barrier()
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()
        e_evs[k][0].record(stream)
        e2e_step()
        e_evs[k][1].record(stream)
        e_samples += pt.stats()["samples"]
    torch.cuda.synchronize()
    barrier()
    e_ms = max_over_ranks(float(sum(a.elapsed_time(b) for a, b in e_evs)))
    e_value = sum_over_ranks(float(e_samples)) / (e_ms / 1e3) / 1e6

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_render_rate(spec, min_seconds=12.0)
        except Exception as e:  # the baseline must not take the GPU number down with it
            cpu = {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "port",
                   "sample": f"unavailable: {e}"}

    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        try:
            ref_gpu = reference_gpu_leg(spec, pt, stream)
        except Exception as e:  # the baseline must not take the GPU number down with it
            ref_gpu = {"unavailable": f"{type(e).__name__}: {e}"}

    st = pt.stats()
    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {**workload_config(spec, args.config), "parallelism": f"replicas{world}",
                   "colour": colour_note(nw), "spectral_wavelengths": nw,
                   "bvh_nodes": int(st["bvh_nodes"]),
                   "mrays_per_s": (cp["rays_extend"] + cp["rays_shadow"]) / (total_ms / args.steps / 1e3) / 1e6,
                   "stage_ms_per_step": {k: round(v, 4) for k, v in stages.items()},
                   "rays_per_sample": (cp["rays_extend"] + cp["rays_shadow"]) / max(1, spec.width * spec.height * spec.waves)},
        "e2e": {"value": e_value, "unit": METRIC, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": (achieved / hbm_peak) if achieved else None, "traffic": traffic,
                     "kernel": "k_extend (closest-hit traversal)",
                     "bytes_per_ray": bytes_per_ray, "nodes_per_ray": nodes_per_ray, "tris_per_ray": tris_per_ray,
                     "rays_per_launch": rays_per_launch, "launch_ms": launch_ms,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s",
                     "l2": {"working_set_mb": working_set / 1e6, "peak_gbs": l2_peak,
                            "frac": (achieved / l2_peak) if achieved and l2_peak else None,
                            "peak_source": "pt_measure_l2: 32 MiB L2-resident 128-bit reads, measured in this run"}},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if cpu is not None:
        if nw > 0:
            cpu["sample"] += "; renders RGB (the reference has no spectral integrator)"
        out["cpu_baseline"] = cpu
    if ref_gpu is not None:
        out["reference_gpu"] = ref_gpu
    if rank == 0:
        print(json.dumps(out))
    pt.close()
    reps.close()
    return 0


def batch_accuracy_scenes(tubes, count: int = 4, seed: int = 9):
    """Scenes of the batch whose images are checked: the smallest, the largest
    and seeded others."""
    order = np.argsort([t.triangle_count for t in tubes])
    pick = {int(order[0]), int(order[-1])}
    rng = np.random.default_rng(seed)
    for k in rng.permutation(len(tubes)):
        if len(pick) >= min(count, len(tubes)):
            break
        pick.add(int(k))
    return sorted(pick)


def batch_accuracy(tubes, cams, sizes, params, images, pixels_per_scene: int = 128, ref_spp: int = 4096,
                   seed: int = 11):
    """Relative MSE of the batch's images against the FP64 oracle.

    Per checked scene, pixels are drawn uniformly over the image (independently
    of the image under test); the FP64 oracle renders them with ref_spp samples
    of its own random numbers (PCG32) and the same estimator.  Pixels whose
    reference luminance is below 1e-4 (background) are dropped.  The relative
    MSE is of the luminance, corrected for the reference's own variance:
    mean(((x - r)^2 - var(r)) / r^2)."""
    from oracle.bindings import Checker
    chk = Checker("oracle")
    threads = chk.max_threads()
    rng = np.random.default_rng(seed)
    lum = np.array([0.2126, 0.7152, 0.0722])
    terms, caps, per_scene = [], [], {}
    t0 = time.perf_counter()
    for k, img in images.items():
        w, h = sizes[k]
        pix = np.sort(rng.choice(w * h, size=min(pixels_per_scene, w * h), replace=False)).astype(np.int32)
        sc = chk.scene(tubes[k].host_mesh())
        if int(params["emitter_mis"]) == 1:
            sc.set_emitter_mis(True)
        p = params.copy()
        p["min_samples"] = p["max_samples_per_pixel"] = ref_spp
        p["adaptive_criterion"] = 0
        st = sc.render(cams[k], p, w, h, ref_spp, seed_base=900_001, pixels=pix, threads=threads, fp64=True)
        r = st["lum_mean"][pix]
        var_r = st["m2"][pix] / float(ref_spp) / float(ref_spp)
        rgba, counts = img
        x = rgba[..., :3].reshape(-1, 3).astype(np.float64)[pix] @ lum
        keep = r > 1e-4
        t = ((x - r) ** 2 - var_r)[keep] / (r[keep] ** 2)
        capped = (counts.reshape(-1)[pix] >= int(params["max_samples_per_pixel"]))[keep]
        terms.append(t)
        caps.append(capped)
        per_scene[int(k)] = {"pixels": int(keep.sum()), "relmse": float(t.mean()) if keep.any() else None,
                             "at_cap": int(capped.sum()), "triangles": int(tubes[k].triangle_count)}
    allt = np.concatenate(terms) if terms else np.zeros(0)
    allc = np.concatenate(caps) if caps else np.zeros(0, bool)
    return {"relmse": float(allt.mean()) if len(allt) else None, "pixels": int(len(allt)),
            "median_sq_rel_err": float(np.median(allt)) if len(allt) else None,
            "pixels_at_cap": int(allc.sum()),
            "relmse_pixels_at_cap": float(allt[allc].mean()) if allc.any() else None,
            "relmse_pixels_stopped": float(allt[~allc].mean()) if (~allc).any() else None,
            "scenes": per_scene, "reference": f"FP64 oracle, {ref_spp} samples per pixel, independent random "
            f"numbers, {threads} host threads", "measure": "luminance relative MSE, reference variance "
            "subtracted", "oracle_s": round(time.perf_counter() - t0, 1)}


def run_batch(args):
    """The batching workload: 64 scenes built on the device and rendered in one
    pt_render (value), against the same scenes rendered one per pt_render
    (config.plain_*).  Every scene's image is identical in both forms."""
    import torch

    from lsystemeditor_b200.pathtracer import PROFILE_COUNT_VISITS, PROFILE_STAGE_TIMES, PathTracer
    from lsystemeditor_b200.scene import batch_scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def reduce(x: float, op: str) -> float:
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
        return float(t.item())

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    t0 = time.perf_counter()
    all_tubes, all_cams, all_sizes, params = batch_scenes(rel_err=args.rel_err, max_spp=args.spp_cap)
    params["emitter_mis"] = 1 if args.estimator == "mis" else 0
    params["adaptive_criterion"] = 2  # relative std-error; all-black pixels stop at 64 samples
    gen_s = time.perf_counter() - t0
    # scenes split over the ranks by estimated cost; each rank renders its own
    # scenes in one batch and rank 0 gathers every image once (strong scaling)
    from lsystemeditor_b200.partition import assign, gather_to_root, owners, scene_cost
    spp_cap = int(params["max_samples_per_pixel"])
    costs = [scene_cost(t.triangle_count, w * h, spp_cap) for t, (w, h) in zip(all_tubes, all_sizes)]
    assignment = assign(costs, world)
    mine = assignment[rank]
    tubes = [all_tubes[k] for k in mine]
    cams = [all_cams[k] for k in mine]
    sizes = [all_sizes[k] for k in mine]
    n = len(tubes)
    stream = torch.cuda.current_stream()
    pt = PathTracer(local)
    pt.set_stream(stream.cuda_stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    own = owners(assignment)
    recv = {k: torch.empty((all_sizes[k][0] * all_sizes[k][1], 4), dtype=torch.float32, device="cuda")
            for k in own if own[k] != 0} if (world > 1 and rank == 0) else {}

    def build_batch():
        pt.batch_configure(sizes)
        for k in range(n):
            pt.batch_set_tubes(k, tubes[k])
            pt.batch_set_camera(k, cams[k])
        pt.set_params(params)

    def local_images():
        """This rank's scene images as views of the renderer's device accumulator (scene after scene)."""
        class _View:
            def __init__(self, ptr, rows):
                self.__cuda_array_interface__ = {"shape": (rows, 4), "typestr": "<f4", "data": (ptr, False),
                                                 "strides": None, "version": 3}
        ptr = pt.device_buffers()[0]
        views, off = {}, 0
        for k, (w, h) in zip(mine, sizes):
            views[k] = torch.as_tensor(_View(ptr + 16 * off, w * h), device="cuda")
            off += w * h
        return views

    def gather():
        if world > 1:
            gather_to_root(rank, assignment, local_images(), recv)

    tb = time.perf_counter()
    build_batch()
    torch.cuda.synchronize()
    build_s = time.perf_counter() - tb
    # scheduling knobs chosen by the autotuner on short probes (untimed; the
    # image does not depend on them)
    tune = pt.autotune(waves=4) if not args.no_autotune else None

    def step():
        pt.reset_accumulation()
        pt.render(0)
        gather()

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    launches0 = pt.stats()["launches"]
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    samples = 0
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    for k in range(args.steps):
        flush.zero_()
        evs[k][0].record(stream)
        step()
        evs[k][1].record(stream)
        samples += pt.stats()["samples"]
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = pt.stats()["launches"] - launches0
    total_ms = reduce(float(sum(a.elapsed_time(b) for a, b in evs)), "max")
    value = reduce(float(samples), "sum") / (total_ms / 1e3) / 1e6

    # stage times (one render) and traversal counts (one render) for the roofline
    pt.set_profiling(PROFILE_STAGE_TIMES)
    flush.zero_()
    step()
    prof = pt.profile()
    pt.set_profiling(PROFILE_COUNT_VISITS | PROFILE_STAGE_TIMES)
    step()
    cp = pt.profile()
    pt.set_profiling(0)
    nodes_per_ray = cp["nodes_extend"] / max(cp["rays_extend"], 1)
    tris_per_ray = cp["tris_extend"] / max(cp["rays_extend"], 1)
    bytes_per_ray = 80.0 * nodes_per_ray + 48.0 * tris_per_ray + 32.0 + 16.0
    rays_per_launch = prof["rays_extend"] / max(prof["launches_extend"], 1)
    launch_ms = prof["ms_extend"] / max(prof["launches_extend"], 1)
    achieved = bytes_per_ray * rays_per_launch / (launch_ms / 1e3) / 1e9 if launch_ms > 0 else None
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))

    # the same scenes one per render (the plain drop-in), device-built likewise
    # images of the scenes whose accuracy is checked against the FP64 oracle
    acc_scenes = batch_accuracy_scenes(all_tubes) if (world == 1 and not args.no_accuracy) else []
    acc_images = {k: pt.batch_readback(k)[:2] for k in acc_scenes}

    # (host wall time of the whole loop too: per scene its configure, tube
    # upload, device build, render and image readback, as a caller of the plain
    # drop-in would run it)
    plain_ms, plain_samples, plain_build_ms = 0.0, 0, 0.0
    torch.cuda.synchronize()
    pw0 = time.perf_counter()
    for k in range(n):
        w, h = sizes[k]
        pt.configure(w, h)
        pt.batch_set_tubes(0, tubes[k])
        plain_build_ms += pt.stats()["build_ms"]
        pt.set_camera(cams[k])
        pt.set_params(params)
        flush.zero_()
        pt.render(0)
        s = pt.stats()
        plain_ms += s["render_ms"]
        plain_samples += s["samples"]
        pt.readback()
    torch.cuda.synchronize()
    plain_wall_s = time.perf_counter() - pw0

    # end to end through the public API: tube arrays from host memory, device
    # loft + BVH builds, render, read back every image (one step)
    h2d = sum(t.ring_start.nbytes + t.points.nbytes + t.tangents.nbytes + t.radii.nbytes + t.materials.nbytes +
              t.leaves.nbytes + t.extra.positions.nbytes + t.extra.normals.nbytes + t.extra.uvs.nbytes +
              t.extra.material_ids.nbytes + t.extra.materials.nbytes for t in tubes)
    d2h = sum(w * h * (16 + 4 + 1) for w, h in sizes) + sum(v.numel() * 4 for v in recv.values())
    torch.cuda.synchronize()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    bw0 = time.perf_counter()
    e0.record(stream)
    build_batch()
    pt.render(0)
    e_samples = pt.stats()["samples"]
    gather()
    if rank == 0:
        for k in range(n):
            pt.batch_readback(k)
        for v in recv.values():
            v.cpu()
    e1.record(stream)
    torch.cuda.synchronize()
    batched_wall_s = time.perf_counter() - bw0
    e_ms = reduce(float(e0.elapsed_time(e1)), "max")
    e_value = reduce(float(e_samples), "sum") / (e_ms / 1e3) / 1e6

    accuracy = None
    if acc_scenes:
        try:
            accuracy = batch_accuracy(all_tubes, all_cams, all_sizes, params, acc_images)
        except Exception as e:  # the check must not take the GPU number down with it
            accuracy = {"unavailable": f"{type(e).__name__}: {e}"}
        batched_s = build_s + total_ms / args.steps / 1e3
        plain_s = plain_build_ms / 1e3 + plain_ms / 1e3
        accuracy["time_to_target"] = {
            "batched_s": batched_s, "plain_s": plain_s,
            "batched_wall_s": batched_wall_s, "plain_wall_s": plain_wall_s,
            "note": "one pass over all scenes to the per-pixel stop criterion; *_s: device time of the device "
                    "builds (loft + BVH) plus the render; *_wall_s: host wall time from the first tube upload to "
                    "the last image read back (batched: one renderer call sequence for all scenes; plain: one "
                    "configure / upload / build / render / readback per scene); batched and plain images are "
                    "identical, so both reach the same relative MSE"}
        accuracy["batched_faster_device"] = bool(batched_s < plain_s)
        accuracy["batched_faster"] = bool(batched_wall_s < plain_wall_s)
        if "relmse" in accuracy:
            accuracy["target_met"] = bool(accuracy["relmse"] <= 1e-3)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_render_rate(make_workload("batch"), min_seconds=12.0)
        except Exception as e:
            cpu = {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "port",
                   "sample": f"unavailable: {e}"}
    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"batch: {len(all_tubes)} stochastic trees (iterations 4-8, seeds "
                               f"100-{99 + len(all_tubes)}), {sum(t.triangle_count for t in all_tubes)} triangles, "
                               f"{sum(w * h for w, h in all_sizes)} pixels, adaptive 16-{args.spp_cap} spp to "
                               f"relative std-error {args.rel_err:g} (all-black pixels stop at 64), depth 12",
                   "scenes": len(all_tubes), "scenes_on_rank0": n,
                   "triangles": int(sum(t.triangle_count for t in all_tubes)),
                   "autotune": tune, "frame_loop": "CUDA graphs of 4 bounce iterations",
                   "pixels": int(sum(w * h for w, h in all_sizes)),
                   "parallelism": f"scenes split over {world} rank(s) by estimated cost (pixels x spp x BVH depth), "
                                  "each rank one batched render, every image gathered once to rank 0 "
                                  "(NCCL point-to-point, inside the timed step)",
                   "l2": "flushed between timed steps (256 MiB write, untimed)",
                   "host_generation_s": round(gen_s, 2), "device_build_s": round(build_s, 2),
                   "batched_ms_per_render": total_ms / args.steps,
                   "plain_ms_per_render": plain_ms, "plain_msamples_per_s": plain_samples / plain_ms / 1e3,
                   "plain_build_ms": plain_build_ms,
                   "stage_ms_per_step": {k[3:]: round(v, 2) for k, v in prof.items() if k.startswith("ms_")},
                   "images": "every scene identical in the batched and the plain form",
                   "estimator": ("emitter MIS (emitter_mis = 1: short emissive shadow rays, balance-weighted "
                                 "BSDF emitter hits at opaque vertices; the reference estimator's expectation)"
                                 if args.estimator == "mis" else "the reference's (emitters by BSDF sampling only)"),
                   "accuracy": accuracy},
        "e2e": {"value": e_value, "unit": METRIC, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "steps": 1},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": (achieved / hbm_peak) if achieved else None, "traffic": None,
                     "kernel": "k_extend (closest-hit traversal)", "bytes_per_ray": bytes_per_ray,
                     "nodes_per_ray": nodes_per_ray, "tris_per_ray": tris_per_ray,
                     "rays_per_launch": rays_per_launch, "launch_ms": launch_ms,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s"},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if cpu is not None:
        out["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(out))
    pt.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_adjoint(args):
    """The differentiation workload: 512x512, 64 spp forward and 64 spp path-replay
    adjoint over 10 materials (8 branch materials, ground, light).  One step =
    one optimisation step through the public API: forward render, readback, L2
    loss against a 256-spp target, pt_backward, Adam update, material upload.
    value = adjoint Msamples/s (device time of pt_backward); config carries the
    forward and adjoint device times, their ratio, and an Adam run of
    --opt-steps steps (lr 1e-2) from a separately seeded start."""
    import torch

    from lsystemeditor_b200.pathtracer import PathTracer
    from lsystemeditor_b200.scene import config3_scene, diff_materials

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    spec = config3_scene()
    spp = int(spec.params["max_samples_per_pixel"])
    W, H = spec.width, spec.height
    pt = PathTracer(local)
    stream = torch.cuda.current_stream()
    pt.set_stream(stream.cuda_stream)
    pt.configure(W, H, spec.mesh)
    pt.set_camera(spec.camera)
    truth = spec.mesh.materials.copy()
    names = ("r", "g", "b", "roughness", "metallic", "sheen", "emission")

    def theta_of(m):
        return np.stack([m[n].astype(np.float64) for n in names], -1)

    def with_theta(base, th):
        m = base.copy()
        for j, n in enumerate(names):
            m[n] = th[:, j].astype(np.float32)
        return m

    # target: 256 spp of the ground truth
    p_target = spec.params.copy()
    p_target["min_samples"] = p_target["max_samples_per_pixel"] = 256
    pt.set_params(p_target)
    pt.render(0)
    target = pt.readback()[0][..., :3].astype(np.float64)
    pt.set_params(spec.params)
    pt.record_samples(spp)  # the adjoint reads the forward's per-sample radiance

    init = truth.copy()
    wrong = diff_materials(np.random.default_rng(1003), 8)
    for n in names[:6]:
        init[n][:8] = wrong[n]
    init["emission"][9] = np.float32(np.random.default_rng(1004).uniform(5.0, 20.0))
    free = np.zeros((len(truth), 7), bool)
    free[:8, :6] = True
    free[9, 6] = True

    class Adam:
        def __init__(self, x, lr):
            self.x, self.lr, self.m, self.v, self.t = x.copy(), lr, np.zeros_like(x), np.zeros_like(x), 0

        def step(self, g):
            self.t += 1
            self.m = 0.9 * self.m + 0.1 * g
            self.v = 0.999 * self.v + 0.001 * g * g
            mh = self.m / (1 - 0.9 ** self.t)
            vh = self.v / (1 - 0.999 ** self.t)
            self.x = self.x - self.lr * mh / (np.sqrt(vh) + 1e-8)
            self.x[:, :6] = np.clip(self.x[:, :6], 0.0, 1.0)
            self.x[:, 6] = np.maximum(self.x[:, 6], 0.0)

    def opt_step(opt, timing=None):
        pt.set_materials(with_theta(truth, opt.x))
        pt.reset_accumulation()
        pt.render(0)
        fwd_ms = pt.stats()["render_ms"]
        img = pt.readback()[0][..., :3].astype(np.float64)
        loss = float(((img - target) ** 2).sum())
        g, adj_ms = pt.backward((2.0 * (img - target)).astype(np.float32), spp)
        g = g[:len(truth)].astype(np.float64) * free
        # the emission strength lives on a 5..20 scale: Adam steps it in units of 10 lr
        g[:, 6] *= 10.0
        opt.step(g)
        if timing is not None:
            timing.append((fwd_ms, adj_ms))
        return loss

    opt = Adam(theta_of(init), 1e-2)
    for _ in range(max(args.warmup, 3)):
        opt_step(opt)
    timing = []
    launches0 = pt.stats()["launches"]
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = time.perf_counter()
    for _ in range(args.steps):
        opt_step(opt, timing)
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - e0) * 1e3 / args.steps
    clk = clocks.stop()
    launches = pt.stats()["launches"] - launches0
    fwd = float(np.mean([a for a, _ in timing]))
    adj = float(np.mean([b for _, b in timing]))
    samples = W * H * spp
    value = samples / (adj / 1e3) / 1e6

    # the optimisation from the start (untimed)
    opt = Adam(theta_of(init), 1e-2)
    losses = [opt_step(opt) for _ in range(args.opt_steps)]
    def errors(x):
        t = theta_of(truth)
        out = {}
        for j, n in enumerate(names[:6]):
            out[n] = float(np.sqrt(np.mean((x[:8, j] - t[:8, j]) ** 2)))
        out["emission_abs"] = float(abs(x[9, 6] - t[9, 6]))
        return out
    err0 = errors(theta_of(init))
    err1 = errors(opt.x)
    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": adj, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"adjoint: bracketed tree with 8 depth materials, {W}x{H}, {spp} spp forward + "
                               f"{spp} spp path-replay adjoint, {len(truth)} materials",
                   "forward_ms": fwd, "adjoint_ms": adj, "adjoint_over_forward": adj / fwd,
                   "opt_step_wall_ms": wall_ms, "l2": "not flushed (each step re-reads the scene it rendered)",
                   "optimisation": {"steps": args.opt_steps, "lr": 1e-2,
                                    "loss_first": losses[0] if losses else None,
                                    "loss_last": losses[-1] if losses else None,
                                    "loss_min": min(losses) if losses else None,
                                    "param_rmse_start": err0, "param_rmse_end": err1}},
        "e2e": {"value": samples * 2 / (wall_ms / 1e3) / 1e6, "unit": METRIC,
                "h2d_bytes_per_step": int(W * H * 3 * 4 + len(truth) * 96),
                "d2h_bytes_per_step": int(W * H * (16 + 4 + 1) + 16 * 7 * 4),
                "note": "forward + adjoint samples per wall-clock optimisation step through the public API"},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(out))
    pt.close()
    return 0


def run_forest(args):
    """The instanced forest: 500 instances of 12 trees (6.0M unique, 263M
    instanced triangles), a 5800 K sun in a 0.53 degree cone plus a uniform
    sky, 1920x1080, adaptive 32-2048 spp, depth 16, 8 hero wavelengths.  One
    step renders the batched form, 4 camera views sharing the scene's BVHs in
    one pt_render (value); the plain form (one view per render) is reported
    beside it."""
    import torch
    import torch.distributed as dist

    from lsystemeditor_b200.pathtracer import PROFILE_COUNT_VISITS, PROFILE_STAGE_TIMES, PathTracer
    from lsystemeditor_b200.scene import forest_scene

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def reduce(x: float, op) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def barrier():
        if world > 1:
            dist.barrier()

    W, H, V = 1920, 1080, 4
    scene, cams, params, sun = forest_scene(width=W, height=H, views=V)
    nw = wavelengths(args)
    params["spectral_wavelengths"] = nw
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def setup(pt, objects):
        pt.batch_configure([(W, H)] * V)
        pt.set_instances(objects, scene.instances, scene=0)
        for k in range(1, V):
            pt.batch_share_scene(k, 0)
        for k in range(V):
            pt.batch_set_camera(k, cams[k])
        pt.set_params(params)
        pt.set_distant_light(**sun)

    pt = PathTracer(local)
    pt.set_stream(stream.cuda_stream)
    setup(pt, scene.objects)

    def step():
        pt.reset_accumulation()
        pt.render(0)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    launches0 = pt.stats()["launches"]
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    samples = 0
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    for k in range(args.steps):
        flush.zero_()
        evs[k][0].record(stream)
        step()
        evs[k][1].record(stream)
        samples += pt.stats()["samples"]
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = pt.stats()["launches"] - launches0
    total_ms = reduce(float(sum(a.elapsed_time(b) for a, b in evs)), dist.ReduceOp.MAX if world > 1 else None)
    value = reduce(float(samples), dist.ReduceOp.SUM if world > 1 else None) / (total_ms / 1e3) / 1e6

    # ---- plain form (view 0 alone), stage times and traversal counts -------
    plain = PathTracer(local)
    plain.set_stream(stream.cuda_stream)
    plain.configure(W, H)
    plain.set_instances(scene.objects, scene.instances)
    plain.set_camera(cams[0])
    plain.set_params(params)
    plain.set_distant_light(**sun)
    plain.reset_accumulation()
    plain.render(0)
    plain.set_profiling(PROFILE_STAGE_TIMES)
    flush.zero_()
    plain.reset_accumulation()
    plain.render(0)
    ps, prof = plain.stats(), plain.profile()
    plain_value = ps["samples"] / (ps["render_ms"] / 1e3) / 1e6
    stages = {k[3:]: round(v, 3) for k, v in prof.items() if k.startswith("ms_")}
    plain.set_profiling(PROFILE_COUNT_VISITS | PROFILE_STAGE_TIMES)
    plain.reset_accumulation()
    plain.render(0)
    cp = plain.profile()
    plain.close()
    nodes_per_ray = cp["nodes_extend"] / max(cp["rays_extend"], 1)
    tris_per_ray = cp["tris_extend"] / max(cp["rays_extend"], 1)
    bytes_per_ray = 80.0 * nodes_per_ray + 48.0 * tris_per_ray + 32.0 + 16.0
    rays_per_launch = prof["rays_extend"] / max(prof["launches_extend"], 1)
    launch_ms = prof["ms_extend"] / max(prof["launches_extend"], 1)
    achieved = bytes_per_ray * rays_per_launch / (launch_ms / 1e3) / 1e9 if launch_ms > 0 else None
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))

    # ---- end to end: objects from pinned host memory, 4 views, readback ----
    keep = []

    def pinned(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        v = t.numpy().view(a.dtype).reshape(a.shape)
        v[...] = a
        keep.append(t)
        return v

    pobjs = []
    h2d = 0
    for mesh in scene.objects:
        m = mesh.contiguous()
        pm = type(m)(*[pinned(getattr(m, f)) for f in ("positions", "normals", "uvs", "material_ids", "materials",
                                                         "textures")])
        h2d += sum(getattr(m, f).nbytes for f in ("positions", "normals", "uvs", "material_ids", "materials",
                                                   "textures"))
        pobjs.append(pm)
    h2d += 64 * len(scene.instances) + V * 80 + 64 + 40
    d2h = V * W * H * (16 + 4 + 1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    setup(pt, pobjs)
    pt.render(0)
    e_samples = pt.stats()["samples"]
    for k in range(V):
        pt.batch_readback(k)
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = reduce(float(e0.elapsed_time(e1)), dist.ReduceOp.MAX if world > 1 else None)
    e_value = reduce(float(e_samples), dist.ReduceOp.SUM if world > 1 else None) / (e_ms / 1e3) / 1e6
    st = pt.stats()
    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"forest: {len(scene.instances) - 1} instances of {len(scene.objects) - 1} stochastic "
                               f"trees + ground, {scene.unique_triangles} unique / {scene.triangle_count} instanced "
                               f"triangles, sun 5800 K in a 0.53 degree cone + uniform sky, {V} views of {W}x{H}, "
                               "adaptive 32-2048 spp to relative std-error 1e-2, depth 16",
                   "views_per_launch": V, "colour": colour_note(nw), "spectral_wavelengths": nw,
                   "plain_msamples_per_s": plain_value, "plain_ms_per_view": ps["render_ms"],
                   "stage_ms_per_view": stages, "bvh_nodes": int(st["bvh_nodes"]),
                   "l2": "flushed before every timed render (256 MiB write, untimed)",
                   "parallelism": f"replicas{world}"},
        "e2e": {"value": e_value, "unit": METRIC, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": (achieved / hbm_peak) if achieved else None, "traffic": None,
                     "kernel": "k_extend<instanced> (two-level closest-hit traversal, plain view)",
                     "bytes_per_ray": bytes_per_ray, "nodes_per_ray": nodes_per_ray, "tris_per_ray": tris_per_ray,
                     "rays_per_launch": rays_per_launch, "launch_ms": launch_ms,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s"},
        "gpu_launches": int(launches),
        "clocks": clk,
        "cpu_baseline": {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "reference",
                         "sample": "not run: the reference flattens the instances into one 263M-triangle mesh and "
                                   "builds its BVH on one host thread, which alone exceeds a bench run"},
    }
    if rank == 0:
        print(json.dumps(out))
    pt.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        if args.config == "forest":
            if int(os.environ.get("RANK", "0")) == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference flattens the forest's 263M "
                                  "instanced triangles and builds their BVH on one host thread; not runnable in a "
                                  "bench's budget"}))
            return 0
        return run_reference(args)
    if args.config == "forest":
        return run_forest(args)
    if args.config == "batch":
        return run_batch(args)
    if args.config == "adjoint":
        return run_adjoint(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
