"""Command-line renderer for the named workloads (plain methods and one view of the instanced forest).

  python -m lsystemeditor_b200.render --workload plain-large --width 512 --height 512 --spp 8 --frames 3

Renders the workload ``--frames`` times from a fresh accumulation (each frame
runs every pixel to its sample budget or to convergence) and prints one line
of statistics per frame; ``--save`` writes the last frame's linear RGBA as a
``.npy`` array.  The reduced forms (smaller image, fixed spp, fewer path
slots) keep the scene and the kernels of the full workload, which makes them
the bounded cases used for kernel profiles.
"""
from __future__ import annotations

import argparse
import sys
import time

import numpy as np


def make_spec(workload: str, width: int = 0, height: int = 0):
    from .scene import config0_scene, config1_scene
    if workload == "plain-small":
        return config0_scene(**({"width": width, "height": height} if width else {}))
    if workload == "plain-large":
        return config1_scene(**({"width": width, "height": height} if width else {}))
    raise ValueError(f"unknown workload {workload!r}")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", choices=["plain-small", "plain-large", "forest"], default="plain-small")
    ap.add_argument("--width", type=int, default=0, help="image width (0 = the workload's)")
    ap.add_argument("--height", type=int, default=0, help="image height (0 = the workload's)")
    ap.add_argument("--spp", type=int, default=0, help="fixed samples per pixel (0 = the workload's min/max)")
    ap.add_argument("--frames", type=int, default=1)
    ap.add_argument("--capacity", type=int, default=0, help="path slots in flight (0 = library default)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--spectral", default="auto", choices=["auto", "0", "4", "8"],
                    help="hero wavelengths per path (auto: plain-small 4, plain-large 8; 0 = RGB)")
    ap.add_argument("--emitter-mis", action="store_true",
                    help="emitter MIS estimator (short emissive shadow rays; not the reference's estimator)")
    ap.add_argument("--save", default="")
    ap.add_argument("--stage-times", action="store_true",
                    help="time every stage launch with CUDA events and print the per-stage totals and ray counts")
    a = ap.parse_args(argv)
    if (a.width > 0) != (a.height > 0):
        ap.error("--width and --height go together")

    from .pathtracer import PROFILE_STAGE_TIMES, PathTracer
    forest = None
    if a.workload == "forest":
        # one view of the instanced forest (objects, instances, sun + sky)
        from .scene import forest_scene
        fw, fh = (a.width, a.height) if a.width else (1920, 1080)
        scene, cams, fparams, sun = forest_scene(width=fw, height=fh, views=1)
        forest = (scene, cams[0], sun)

        class _Spec:
            name = "forest: one view"
            width, height, params, camera, mesh = fw, fh, fparams, cams[0], None
        spec = _Spec()
    else:
        spec = make_spec(a.workload, a.width, a.height)
    params = spec.params.copy()
    params["spectral_wavelengths"] = {"plain-small": 4, "plain-large": 8, "forest": 8}[a.workload] \
        if a.spectral == "auto" else int(a.spectral)
    if a.spp > 0:
        params["min_samples"] = a.spp
        params["max_samples_per_pixel"] = a.spp
    if a.emitter_mis:
        params["emitter_mis"] = 1
    t0 = time.perf_counter()
    with PathTracer(a.device) as pt:
        if a.capacity:
            pt.set_tuning(a.capacity, 0)
        if forest is None:
            pt.configure(spec.width, spec.height, spec.mesh)
            triangles = spec.mesh.triangle_count
        else:
            pt.configure(spec.width, spec.height)
            pt.set_instances(forest[0].objects, forest[0].instances)
            pt.set_distant_light(**forest[2])
            triangles = sum(o.triangle_count for o in forest[0].objects)
        pt.set_camera(spec.camera)
        pt.set_params(params)
        if a.stage_times:
            pt.set_profiling(PROFILE_STAGE_TIMES)
        nw = int(params["spectral_wavelengths"])
        colour = f"{nw} wavelengths" if nw else "RGB"
        print(f"{spec.name}: {triangles} triangles, {spec.width}x{spec.height}, "
              f"{colour}, "
              f"scene ready in {time.perf_counter() - t0:.2f} s", flush=True)
        launched = pt.stats()["launches"]
        for f in range(a.frames):
            pt.reset_accumulation()
            pt.render(0)
            s = pt.stats()
            print(f"frame {f}: {s['render_ms']:.2f} ms, {s['samples']} samples, "
                  f"{s['samples'] / max(s['render_ms'], 1e-9) / 1e3:.1f} Msamples/s, launches {s['launches'] - launched}",
                  flush=True)
            launched = s["launches"]
            if a.stage_times:
                p = pt.profile()
                print("  stages ms: " + ", ".join(f"{k[3:]} {v:.3f}" for k, v in p.items() if k.startswith("ms_")) +
                      f"; extend launches {p['launches_extend']} rays {p['rays_extend']}; "
                      f"shadow launches {p['launches_shadow']} rays {p['rays_shadow']}", flush=True)
        if a.save:
            rgba, counts, converged = pt.readback()
            np.save(a.save, rgba)
    return 0


if __name__ == "__main__":
    sys.exit(main())
