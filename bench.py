#!/usr/bin/env python
"""Benchmark of the spectral path-tracing hot path on B200.

Workload: the mixed-material mesh scene (seeded displaced icosphere, subdivision 8, 64
spheres of 2048 triangles and a ground plane: 1,441,794 triangles; 40% diffuse / 40% GGX
conductor / 20% dielectric; 2 point + 2 spot lights and a constant environment) at
1920x1080, 16 spp, depth 16, four hero wavelengths per sample, Sobol/Owen sampler, seed 1.

One step renders all 16 spp of the 1080p film (33,177,600 samples) into the device FP64
film.  ``value`` is Msamples/s with the scene resident; ``e2e`` is the same metric through the
public API (build the scene from host arrays, render into a host film, read it back).

``--impl reference`` times the reference's CPU path (the oracle restatement, all host
threads) on bounded samples of the same workload.

Multi-GPU (torchrun): every rank renders its own sample range of the same film (independent
units, no data-path collective); ``value`` is all ranks' samples over the slowest rank's time.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "spectral path Msamples/s"
UNIT = "Msamples/s"
WORKLOAD = "mixed_material_1080p_16spp_depth16"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--width", type=int, default=1920)
    p.add_argument("--height", type=int, default=1080)
    p.add_argument("--spp", type=int, default=16)
    p.add_argument("--depth", type=int, default=16)
    p.add_argument("--subdivisions", type=int, default=8)
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-secondary", action="store_true",
                   help="skip the fog, batched-views and adjoint workloads (run at N=1 only)")
    p.add_argument("--adam-steps", type=int, default=200)
    return p.parse_args()


def config(args, n):
    return {"workload": WORKLOAD, "width": args.width, "height": args.height, "spp": args.spp,
            "max_depth": args.depth, "triangles": None, "sampler": "sobol-owen", "seed": 1,
            "hero_wavelengths": 4, "film": "fp64 device film, box filter",
            "l2": "inputs larger than L2 (path-state pool and BVH exceed 126 MB) and a 256 MB L2 flush between steps",
            "parallelism": f"replicas{n}" if n > 1 else "single"}


class Clocks:
    """nvidia-smi clock/throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.stop_flag = threading.Event()
        self.thread = threading.Thread(target=self.run, daemon=True)

    def run(self):
        while not self.stop_flag.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self.stop_flag.wait(0.2)

    def __enter__(self):
        self.thread.start()
        return self

    def __exit__(self, *a):
        self.stop_flag.set()
        self.thread.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        peaks = json.load(open(path))
        return float(peaks["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def trace_profile():
    """The closest-hit kernel's ncu figures, per ray, from the small-case capture recorded in
    rypath_b200/data/k_trace_ncu.json (DRAM and L2 bytes per ray, issue activity, SIMD
    efficiency); {} if the file is absent."""
    path = os.path.join(ROOT, "rypath_b200", "data", "k_trace_ncu.json")
    return json.load(open(path)) if os.path.exists(path) else {}


def l2_copy_gbs(torch):
    """This GPU's L2 bandwidth, measured here: device-to-device copies between two buffers that
    both stay resident in the 126 MB L2 (16, 24 and 32 MB each), repeated 200 times; the best
    rate of bytes read plus written per second."""
    best = 0.0
    for mb in (16, 24, 32):
        src = torch.empty(mb << 20, dtype=torch.uint8, device="cuda")
        dst = torch.empty_like(src)
        for _ in range(20):
            dst.copy_(src)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        for _ in range(200):
            dst.copy_(src)
        stop.record()
        torch.cuda.synchronize()
        best = max(best, 2 * src.numel() * 200 / (start.elapsed_time(stop) / 1e3) / 1e9)
    return best


BAND = 8  # rows per contiguous block of the CPU sample


def strided_rows(w, h, lanes, max_spp):
    """A bounded sample of the whole film, independent of how it is timed: blocks of BAND
    consecutive rows spread evenly over the film (one block every `stride` rows, the smallest
    multiple of BAND that keeps the blocks' pixels within `lanes`), at as many absolute samples
    (0, 1, ...) as then fit, at most max_spp.  Returns the blocks' first rows and row counts,
    and the samples."""
    fit = max(1, lanes // (BAND * w))   # blocks within the budget
    total = -(-h // BAND)                # blocks of the whole film
    stride = BAND * -(-total // fit)
    blocks = [(r, min(BAND, h - r)) for r in range(((stride - BAND) // 2) // BAND * BAND, h, stride)]
    pixels = sum(n for _, n in blocks) * w
    spp = max(1, min(max_spp, lanes // max(1, pixels)))
    return blocks, spp


def cpu_baseline(orc, args, seconds, threads=0):
    """The oracle (the reference's CPU path restated) on a bounded sample of the workload: blocks
    of whole rows spread over the film (strided_rows), sized from a short probe to about
    `seconds`; one oracle call per block, so every host thread has work."""
    from tests.oracle_lib import request

    w, h = args.width, args.height

    def render(blocks, spp):
        t0 = time.perf_counter()
        outs = [orc.sample(request(w, h, spp, pixel_begin=r * w, pixel_count=n * w), threads=threads)
                for r, n in blocks]
        return np.concatenate(outs), time.perf_counter() - t0

    probe, _ = strided_rows(w, h, 4 * BAND * w, 1)
    out, dt = render(probe, 1)
    rate = out.size / max(dt, 1e-6)
    blocks, spp = strided_rows(w, h, int(max(BAND * w, rate * seconds)), args.spp)
    out, dt = render(blocks, spp)
    ok = int((out["status"] == 0).sum())
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    stride = blocks[1][0] - blocks[0][0] if len(blocks) > 1 else h
    return {"value": out.size / dt / 1e6, "unit": UNIT, "cores": cores, "kind": "port", "seconds": dt,
            "sample": f"{out.size} lanes: {len(blocks)} blocks of {BAND} whole rows of the {w}x{h} film, one every "
                      f"{stride} rows from row {blocks[0][0]}, absolute samples 0..{spp - 1}, depth {args.depth}; "
                      f"{dt:.2f} s, {ok} succeeded"}


def run_reference(args, rank):
    if rank != 0:
        return
    from rypath_b200 import scenes

    from tests.oracle_lib import OracleScene

    scene = scenes.mixed_scene(args.width, args.height, args.spp, args.depth, subdivisions=args.subdivisions)
    orc = OracleScene(scene)
    for _ in range(args.warmup):
        cpu_baseline(orc, args, 1.0)
    values = [cpu_baseline(orc, args, args.cpu_seconds / max(args.steps, 1)) for _ in range(args.steps)]
    value = statistics.median(v["value"] for v in values)
    cfg = config(args, 1)
    cfg["triangles"] = scene.triangle_count
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.median(v["seconds"] * 1e3 for v in values),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": cfg, "cpu_baseline": dict(values[-1], value=value),
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def bench_fog(torch, cpu_seconds):
    """Scalar volpath: the Cornell-style box filled with a homogeneous medium (sigma_s mean 0.5,
    albedo 0.9, HG g = 0.7), 1024x1024, 64 spp, depth 32, one wavelength per sample."""
    from rypath_b200 import abi, renderer, scenes

    from tests.oracle_lib import OracleScene, request

    w, spp = 1024, 64
    scene = scenes.cornell_fog(w, w, spp, 32)
    rs = renderer.build_renderer(scene).scene
    film = torch.zeros(w * w * abi.FILM_PIXEL_BYTES // 8, dtype=torch.float64, device="cuda")
    probe = renderer.RenderSettings(w, w, samples=8, batch_size=8, seed=1)
    rs.render_film_device(probe, film.data_ptr())
    rs.set_counting(True)
    film.zero_()
    rs.render_film_device(probe, film.data_ptr())
    counts = rs.timing()
    rs.set_counting(False)
    film.zero_()
    rs.render_film_device(renderer.RenderSettings(w, w, samples=spp, batch_size=spp, seed=1), film.data_ptr(),
                          sample_begin=8)
    t = rs.timing()
    rays_per_sample = (counts.closest_rays + counts.shadow_rays) / counts.samples
    value = t.samples / t.total_ms / 1e3
    rs.close()
    orc = OracleScene(scene)
    n = 16384
    t0 = time.perf_counter()
    orc.sample_scalar(request(w, w, 1, pixel_begin=(w * w - n) // 2, pixel_count=n))
    rate = n / (time.perf_counter() - t0)
    n = int(min(w * w, max(n, rate * cpu_seconds)))
    t0 = time.perf_counter()
    out = orc.sample_scalar(request(w, w, 1, pixel_begin=(w * w - n) // 2, pixel_count=n))
    dt = time.perf_counter() - t0
    return {"workload": "cornell_fog_1024x1024_64spp_depth32 (scalar volpath, homogeneous medium)",
            "metric": "scalar path Msamples/s", "value": value, "unit": UNIT, "ms_per_step": t.total_ms,
            "kernel": "k_scalar_walk + k_scalar_step (wavefront over 262,144 resident path slots)",
            "rays_per_sample": rays_per_sample, "mrays_per_s": value * rays_per_sample,
            "cpu_baseline": {"value": out.size / dt / 1e6, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": f"{out.size} lanes (1 spp of pixels around the film centre), {dt:.2f} s"}}


def bench_views(torch):
    """Batched form: 64 seeded views of the mixed scene (resolutions U[256x256, 1280x720],
    spp from {4, 8, 16, 32, 64}) in one wavefront with graph replay and tuned shapes, against
    one plain wavefront per view; both films are compared bit for bit."""
    from rypath_b200 import abi, renderer, scenes

    scene = scenes.mixed_scene(64, 64, 1, 16)
    views = scenes.view_batch(scene, count=64, seed=1)
    total = renderer.pack_views(views)
    lanes = sum(v.width * v.height * v.sample_count for v in views)
    rs = renderer.build_renderer(scene).scene
    film = torch.zeros(total * abi.FILM_PIXEL_BYTES, dtype=torch.uint8, device="cuda")
    t0 = time.perf_counter()
    chosen = rs.tune_views(views, renderer.BatchRequest())
    tune_s = time.perf_counter() - t0
    req = renderer.BatchRequest(wave_lanes=chosen.wave_lanes, trace_block=chosen.trace_block,
                                shade_block=chosen.shade_block, blocks_per_sm=chosen.blocks_per_sm, use_graph=1)
    batched_ms = []
    for _ in range(2):
        film.zero_()
        rs.render_views_device(views, req, film.data_ptr())
        batched_ms.append(rs.timing().total_ms)
    batched = film.clone()
    rs.close()
    # the plain form: one scene per view (the reference renders one camera per job), each view
    # rendered through rp_cuda_render_film_device into its part of the film
    import copy

    film.zero_()
    plain_ms = 0.0
    for v in views:
        one = copy.copy(scene)
        one.camera, one.width, one.height, one._keep = v.camera, v.width, v.height, []
        plain = renderer.build_renderer(one).scene
        sub = film[v.film_offset * abi.FILM_PIXEL_BYTES:(v.film_offset + v.width * v.height) * abi.FILM_PIXEL_BYTES]
        plain.render_film_device(renderer.RenderSettings(v.width, v.height, samples=v.sample_count,
                                                         batch_size=v.sample_count, seed=1),
                                 sub.data_ptr(), sample_begin=v.sample_begin)
        plain_ms += plain.timing().total_ms
        plain.close()
    identical = bool(torch.equal(batched, film))
    ms = min(batched_ms)
    return {"workload": "64 views of the mixed scene, resolutions U[256x256, 1280x720], spp {4..64}",
            "metric": "batched Msamples/s (all views)", "value": lanes / ms / 1e3, "unit": UNIT,
            "plain_per_view_value": lanes / plain_ms / 1e3, "speedup_vs_plain": plain_ms / ms,
            "films_identical_to_plain": identical, "lanes": lanes, "batched_ms": ms, "plain_ms": plain_ms,
            "plain_form": "one scene per view, rp_cuda_render_film_device per view (render time only)",
            "tuned": {"wave_lanes": chosen.wave_lanes, "trace_block": chosen.trace_block,
                      "shade_block": chosen.shade_block, "blocks_per_sm": chosen.blocks_per_sm,
                      "probe_ms_per_mlane": chosen.probe_ms_per_mlane, "tuning_s": tune_s},
            "equal_rmse": "identical films: the batched form renders exactly the plain lanes"}


def bench_images(torch, plain_value):
    """Row f3 workloads: the benchmark scene with its constant environment replaced by a
    256x256 equal-area sky image (importance-sampled light, image radiance on escape), at the
    headline configuration, against the plain scene's value; and the textured Cornell box
    (sRGB trilinear, float EWA and half point image reflectance, RGB reflectance) at 1024x1024,
    64 spp, depth 8, against the untextured box."""
    from rypath_b200 import abi, renderer, scenes

    def render(scene, w, h, spp):
        built = renderer.build_renderer(scene)
        assert built.status == abi.RP_SUCCESS, built.diagnostic
        rs = built.scene
        film = torch.zeros(w * h * abi.FILM_PIXEL_BYTES // 8, dtype=torch.float64, device="cuda")
        warm = renderer.RenderSettings(w, h, samples=4, batch_size=4, seed=1)
        rs.render_film_device(warm, film.data_ptr(), fresh=True)
        best = None
        for _ in range(2):
            rs.render_film_device(renderer.RenderSettings(w, h, samples=spp, batch_size=spp, seed=1),
                                  film.data_ptr(), fresh=True)
            t = rs.timing()
            best = t if best is None or t.total_ms < best.total_ms else best
        rs.close()
        return best.samples / best.total_ms / 1e3, best.total_ms

    env_value, env_ms = render(scenes.with_environment_image(scenes.mixed_scene()), 1920, 1080, 16)
    tex_value, tex_ms = render(scenes.cornell_features("texture", 1024, 1024, 64), 1024, 1024, 64)
    box_value, box_ms = render(scenes.cornell_box(1024, 1024, 64, 8), 1024, 1024, 64)
    return {"environment_image": {"workload": "mixed_scene_1920x1080_16spp_depth16 with a 256x256 float sky image "
                                              "(compensated importance tables) for the constant environment",
                                  "value": env_value, "unit": UNIT, "ms_per_step": env_ms,
                                  "vs_constant_environment": env_value / plain_value if plain_value else None},
            "textured_cornell": {"workload": "cornell_texture_1024x1024_64spp_depth8 (trilinear sRGB, EWA float, "
                                             "point half image reflectance; RGB reflectance)",
                                 "value": tex_value, "unit": UNIT, "ms_per_step": tex_ms,
                                 "untextured_value": box_value, "vs_untextured": tex_value / box_value}}


def bench_demo(torch, cpu_seconds):
    """`--render-demo` at its own defaults: rypath's demo scene (make_demo_scene) at 256x192,
    128 spp, depth 5, the independent (Philox) sampler, scalar transport, into a device film;
    the oracle's scalar demo lanes on the host cores beside it."""
    from rypath_b200 import abi, renderer, scenes

    from tests.oracle_lib import OracleScene, request

    w, h, spp = 256, 192, 128
    scene = scenes.demo_scene(w, h, spp)
    rs = renderer.build_renderer(scene).scene
    film = torch.zeros(w * h * abi.FILM_PIXEL_BYTES // 8, dtype=torch.float64, device="cuda")
    settings = renderer.RenderSettings(w, h, samples=spp, batch_size=spp, seed=1, sampler=abi.SAMPLER_INDEPENDENT)
    rs.render_film_device(renderer.RenderSettings(w, h, samples=8, batch_size=8, seed=1,
                                                  sampler=abi.SAMPLER_INDEPENDENT), film.data_ptr(), fresh=True)
    best = None
    for _ in range(3):
        rs.render_film_device(settings, film.data_ptr(), fresh=True)
        t = rs.timing()
        best = t if best is None or t.total_ms < best.total_ms else best
    rs.close()
    value = best.samples / best.total_ms / 1e3
    orc = OracleScene(scene)
    t0 = time.perf_counter()
    out = orc.sample_scalar(request(w, h, 64, sampler=abi.SAMPLER_INDEPENDENT))
    dt = time.perf_counter() - t0
    return {"workload": "demo_v1_256x192_128spp_depth5 (rypath --render-demo defaults, scalar transport, "
                        "independent sampler)",
            "value": value, "unit": UNIT, "ms_per_step": best.total_ms,
            "cpu_baseline": {"value": out.size / dt / 1e6, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": f"{out.size} lanes (64 spp of every pixel), {dt:.2f} s"}}


def bench_adjoint(torch, adam_steps):
    """Differentiation: 16 reflectance groups x 32 knots of the Cornell geometry, 512x512,
    32 spp, depth 8, L2 loss on film-mean XYZ against a 128-spp render of seeded true
    spectra.  The path-replay adjoint gradient against central differences (h = 1e-3, common
    random numbers) of the same renders; errors against a 32x-spp adjoint gradient on another
    seed, and the adjoint's sample count at which its error matches the differences'."""
    from rypath_b200 import abi, renderer, scenes

    w, spp, params = 512, 32, 512
    scene, truth = scenes.cornell_groups(w, w, spp, 8)
    mats = list(range(16))
    rs = renderer.build_renderer(scene).scene
    rt = renderer.build_renderer(truth).scene

    def mean(r, n, seed):
        doubles = abi.FILM_PIXEL_BYTES // 8
        film = torch.zeros(w * w * doubles, dtype=torch.float64, device="cuda")
        r.render_film_device(renderer.RenderSettings(w, w, samples=n, batch_size=n, seed=seed), film.data_ptr())
        torch.cuda.synchronize()
        f = film.reshape(w * w, doubles)
        return (f[:, 0:3] + f[:, 3:6]) / (f[:, 6:7] + f[:, 7:8]), r.timing().total_ms

    def adjoint(r, n, seed, g):
        grad = torch.zeros(params, dtype=torch.float32, device="cuda")
        r.adjoint_device(renderer.RenderSettings(w, w, samples=n, batch_size=n, seed=seed), mats,
                         g.contiguous().data_ptr(), grad.data_ptr())
        torch.cuda.synchronize()
        return grad.cpu().numpy().astype(np.float64), r.timing().total_ms

    target, _ = mean(rt, 128, 11)
    rt.close()
    theta0 = np.concatenate([scene.knots[32 * g:32 * g + 32, 1] for g in range(16)]).astype(np.float32)
    for _ in range(2):
        m, f_ms = mean(rs, spp, 1)
        grad, b_ms = adjoint(rs, spp, 1, 2 * (m - target))
    # the reference gradient: the adjoint at 32x the samples, on another seed
    mref, _ = mean(rs, 32 * spp, 7)
    gref, _ = adjoint(rs, 32 * spp, 7, 2 * (mref - target))
    sub = list(range(3, params, 32))
    fd, fd_ms = [], 0.0
    h = 1e-3
    for j in sub:
        th = theta0.copy()
        th[j] += h
        rs.set_knot_values(0, th)
        mp, a = mean(rs, spp, 1)
        th[j] -= 2 * h
        rs.set_knot_values(0, th)
        mm, b = mean(rs, spp, 1)
        fd_ms += a + b
        fd.append((float(((mp - target) ** 2).sum()) - float(((mm - target) ** 2).sum())) / (2 * h))
    rs.set_knot_values(0, theta0)
    fd = np.array(fd)
    rel = lambda x, y: float(np.linalg.norm(x - y) / np.linalg.norm(y))
    fd_error = rel(fd, gref[sub])
    fd_full_ms = fd_ms / len(sub) * params
    # equal gradient error: the adjoint at growing sample counts until its error on the same
    # parameters is at most the finite differences' error; that adjoint's time against theirs
    ladder = []
    matched = None
    for n in (spp, 2 * spp, 4 * spp, 8 * spp, 16 * spp):
        for _ in range(2):
            m, a = mean(rs, n, 1)
            g, b = adjoint(rs, n, 1, 2 * (m - target))
        err = rel(g[sub], gref[sub])
        ladder.append({"spp": n, "ms": a + b, "relative_error_subset": err, "relative_error_all": rel(g, gref)})
        if err <= fd_error:
            matched = ladder[-1]
            break
    th, mom, vel, losses, dev_ms = theta0.copy(), np.zeros(params), np.zeros(params), [], 0.0
    t0 = time.perf_counter()
    for k in range(1, adam_steps + 1):
        rs.set_knot_values(0, th)
        m, a = mean(rs, spp, k)
        gr, b = adjoint(rs, spp, k, 2 * (m - target))
        dev_ms += a + b
        losses.append(float(((m - target) ** 2).sum()))
        mom = 0.9 * mom + 0.1 * gr
        vel = 0.999 * vel + 0.001 * gr * gr
        step = 0.02 * (mom / (1 - 0.9 ** k)) / (np.sqrt(vel / (1 - 0.999 ** k)) + 1e-8)
        th = np.clip(th - step, 0.01, 1.0).astype(np.float32)
    adam_s = time.perf_counter() - t0
    rs.close()
    adjoint_ms = f_ms + b_ms
    return {"workload": "cornell_groups 512x512, 32 spp, depth 8, 16 groups x 32 knots, L2 on XYZ",
            "metric": "gradient ms (forward + backward)", "value": adjoint_ms, "unit": "ms", "higher_is_better": False,
            "forward_ms": f_ms, "backward_ms": b_ms,
            "finite_difference_ms": fd_full_ms, "speedup_vs_finite_difference": fd_full_ms / adjoint_ms,
            "finite_difference": f"central, h = {h}, common random numbers, {len(sub)} of {params} parameters "
                                 f"timed ({fd_ms:.0f} ms), whole-gradient time scaled by parameter count",
            "relative_error_vs_32x_adjoint": {"adjoint_all": rel(grad, gref), "adjoint_subset": rel(grad[sub], gref[sub]),
                                              "finite_difference_subset": fd_error},
            "equal_error": {"adjoint_ladder": ladder, "matched": matched,
                            "speedup_vs_finite_difference": (fd_full_ms / matched["ms"]) if matched else None,
                            "rule": "smallest adjoint spp (32 x 2^k) whose error on the finite-difference parameters "
                                    "is at most the finite differences' error at 32 spp; both against the "
                                    "1024-spp adjoint on another seed"},
            "adam": {"steps": adam_steps, "lr": 0.02, "loss_first": losses[0] if losses else None,
                     "loss_last": losses[-1] if losses else None, "device_ms_per_step": dev_ms / max(1, adam_steps),
                     "wall_s": adam_s}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from rypath_b200 import abi, renderer, scenes, shard

    scene = scenes.mixed_scene(args.width, args.height, args.spp, args.depth, subdivisions=args.subdivisions)
    pixels = args.width * args.height
    settings = renderer.RenderSettings(args.width, args.height, samples=args.spp, batch_size=args.spp)
    built = renderer.build_renderer(scene, device=local)
    if built.status != abi.RP_SUCCESS:
        raise SystemExit(f"build_renderer failed: {built.diagnostic}")
    rs = built.scene
    film = torch.zeros(pixels * abi.FILM_PIXEL_BYTES // 8, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    # each rank's disjoint block of absolute samples: the counting render, warm-up and timed steps
    per_rank = args.spp * (args.warmup + args.steps + 1)
    sample_base, _ = shard.sample_range(per_rank * world, rank, world)

    # exact traversal counts for the roofline (an untimed counting render of the same workload)
    rs.set_counting(True)
    film.zero_()
    rs.render_film_device(settings, film.data_ptr(), sample_begin=sample_base)
    counts = rs.timing()
    rs.set_counting(False)

    for i in range(args.warmup):
        film.zero_()
        rs.render_film_device(settings, film.data_ptr(), sample_begin=sample_base + (i + 1) * args.spp)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    steps = []
    with Clocks(local) as clocks:
        for i in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            film.zero_()
            rs.render_film_device(settings, film.data_ptr(),
                                  sample_begin=sample_base + (args.warmup + 1 + i) * args.spp)
            steps.append(rs.timing())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    total_ms = sum(t.total_ms for t in steps)
    samples = sum(t.samples for t in steps)
    if dist:
        v = torch.tensor([total_ms, float(samples)], dtype=torch.float64, device="cuda")
        mx = v.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(v, op=dist.ReduceOp.SUM)
        job_ms, job_samples = float(mx[0]), float(v[1])
    else:
        job_ms, job_samples = total_ms, float(samples)
    value = job_samples / (job_ms / 1e3) / 1e6

    # roofline of the dominant kernel: closest-hit traversal
    trace_ms = sum(t.trace_ms for t in steps)
    trace_launches = sum(t.trace_launches for t in steps)
    rays = counts.closest_rays
    node_bytes, tri_bytes = 80, 48  # compressed 8-wide node, one triangle (3 float4)
    state_bytes = 4 + 16 + 32 + 16  # queue entry, flags, ray read, hit write
    algo_per_ray = (counts.nodes_visited * node_bytes + counts.triangles_tested * tri_bytes) / max(
        1, counts.closest_rays) + state_bytes
    trace_bytes_per_step = algo_per_ray * rays
    achieved = trace_bytes_per_step * len(steps) / (trace_ms / 1e3) / 1e9 if trace_ms > 0 else None
    peak, peak_kind = measured_peaks()
    ncu = trace_profile()
    tpr = ncu.get("dram_bytes_per_ray")
    l2_peak = l2_copy_gbs(torch)
    avg_launch_s = trace_ms / max(1, trace_launches) / 1e3
    rays_per_launch = rays / max(1, counts.trace_launches)
    # launch time per kernel group over the summed launch time of all groups (the shadow walks of
    # one event overlap the next event's closest-hit walk on a second stream, so the groups'
    # launch times add up to more than the step time)
    group_ms = {k: sum(getattr(t, k + "_ms") for t in steps) for k in ("trace", "shadow", "shade", "other")}
    shares = {k: v / max(sum(group_ms.values()), 1e-9) for k, v in group_ms.items()}

    line = None
    if rank == 0:
        cfg = config(args, world)
        cfg["triangles"] = scene.triangle_count
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": job_ms / len(steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": cfg,
            "roofline": {"bound": "hbm", "kernel": "k_trace (closest-hit traversal)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": (tpr * rays_per_launch) if tpr else None,
                         "algorithmic_bytes_per_launch": trace_bytes_per_step / max(1, counts.trace_launches),
                         "algorithmic_bytes_per_ray": algo_per_ray, "peak_kind": peak_kind,
                         "avg_launch_ms": trace_ms / max(1, trace_launches),
                         # what limits the walk: most of its bytes come from L2, and it is
                         # issue-bound at low SIMD efficiency (ncu, rypath_b200/data/k_trace_ncu.json)
                         "limiter": "issue (SIMD efficiency of uneven ray lengths), not HBM",
                         "l2": {"peak_gbs": l2_peak, "peak_kind": "measured here (L2-resident device copy)",
                                "achieved_gbs": (ncu["l2_bytes_per_ray"] * rays_per_launch / avg_launch_s / 1e9)
                                if ncu.get("l2_bytes_per_ray") and trace_ms > 0 else None,
                                "algorithmic_frac": (achieved / l2_peak) if achieved else None,
                                "bytes_per_ray": ncu.get("l2_bytes_per_ray")},
                         "issue": {"issue_active": ncu.get("issue_active"), "simd_efficiency": ncu.get("simd_efficiency"),
                                   "useful_lane_fraction": (ncu["issue_active"] * ncu["simd_efficiency"])
                                   if ncu.get("issue_active") else None},
                         "ncu_source": ncu.get("capture")},
            "traversal_per_ray": {
                "closest": {"nodes": counts.nodes_visited / max(1, counts.closest_rays),
                            "triangles": counts.triangles_tested / max(1, counts.closest_rays),
                            "ns_per_ray": trace_ms / len(steps) * 1e6 / max(1, counts.closest_rays)},
                "shadow": {"nodes": counts.shadow_nodes_visited / max(1, counts.shadow_rays),
                           "triangles": counts.shadow_triangles_tested / max(1, counts.shadow_rays),
                           "ns_per_ray": group_ms["shadow"] / len(steps) * 1e6 / max(1, counts.shadow_rays)}},
            "shade_family_ms_per_step": dict(zip(("diffuse", "conductor", "dielectric", "escape"),
                                                 list(counts.shade_family_ms))),
            "kernel_share": shares,
            "kernel_group_ms_per_step": {k: v / len(steps) for k, v in group_ms.items()},
            "rays_per_step": {"closest": counts.closest_rays, "shadow": counts.shadow_rays},
            "mrays_per_s": (counts.closest_rays + counts.shadow_rays) * len(steps) / (total_ms / 1e3) / 1e6,
            "gpu_launches": int(sum(t.kernel_launches for t in steps)),
            "scene_build_ms": {"total": counts.build_ms, "host": counts.build_host_ms, "lbvh": counts.build_bvh_ms},
            "clocks": clocks.summary(),
        }
    # end to end through the public API: build the scene from pinned host arrays, render into a
    # pinned host film, read it back.  The resident scene is released first so its device
    # memory returns to the pool the next scene draws from.
    rs.close()
    if not args.no_e2e:
        def pinned(a):
            t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
            out = t.numpy().view(a.dtype).reshape(a.shape)
            out[...] = a
            return out, t

        scene.positions, keep_p = pinned(np.ascontiguousarray(scene.positions, np.float32))
        scene.triangles, keep_t = pinned(np.ascontiguousarray(scene.triangles, np.uint32))
        film_host, keep_f = pinned(np.zeros(pixels, abi.film_dtype()))
        desc_bytes = (scene.positions.nbytes + scene.triangles.nbytes + scene.knots.nbytes +
                      len(scene.emissions) * 1888 + len(scene.positional) * 1948 + 234208 + 471 * 4)
        film_bytes = pixels * abi.FILM_PIXEL_BYTES

        def e2e_step(i):
            # a new render each step: the film starts empty on the device and is read back
            st, diag, _ = renderer.render_progressive(
                scene, renderer.RenderSettings(args.width, args.height, samples=args.spp, batch_size=args.spp,
                                               seed=1), device=local, film=film_host, fresh=True)
            if st != abi.RP_SUCCESS:
                raise SystemExit(f"e2e render failed: {diag}")

        for i in range(args.warmup):
            e2e_step(i)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        times = []
        for i in range(args.steps):
            t0 = time.perf_counter()
            e2e_step(i)
            times.append(time.perf_counter() - t0)
        e2e_s = sum(times) / len(times)
        # one more, untimed step through the same calls, split into its parts
        t0 = time.perf_counter()
        built = renderer.build_renderer(scene, device=local)
        t1 = time.perf_counter()
        st, diag, _ = built.scene.render_film(
            renderer.RenderSettings(args.width, args.height, samples=args.spp, batch_size=args.spp, seed=1),
            film_host, fresh=True)
        t2 = time.perf_counter()
        device_ms = built.scene.timing().total_ms
        built.scene.close()
        t3 = time.perf_counter()
        breakdown = {"build_ms": (t1 - t0) * 1e3, "render_call_ms": (t2 - t1) * 1e3,
                     "render_device_ms": device_ms, "close_ms": (t3 - t2) * 1e3}
        if dist:
            v = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
            dist.all_reduce(v, op=dist.ReduceOp.MAX)
            e2e_s = float(v[0])
        if line is not None:
            line["e2e"] = {"value": pixels * args.spp * world / e2e_s / 1e6, "unit": UNIT,
                           "h2d_bytes_per_step": desc_bytes, "d2h_bytes_per_step": film_bytes,
                           "seconds_per_step": e2e_s, "steps": args.steps, "warmup": args.warmup,
                           "breakdown_of_one_step": breakdown,
                           "includes": "scene upload from pinned host arrays, light tables, LBVH and wide-tree build, "
                                       "render into a fresh device film, readback into a pinned host film"}
    if line is not None and not args.no_cpu_baseline:
        from tests.oracle_lib import OracleScene

        line["cpu_baseline"] = cpu_baseline(OracleScene(scene), args, args.cpu_seconds)
    if line is not None and world == 1 and not args.no_secondary:
        line["secondary"] = {"volpath": bench_fog(torch, 4.0), "batched_views": bench_views(torch),
                             "adjoint": bench_adjoint(torch, args.adam_steps),
                             "images": bench_images(torch, line["value"]), "demo": bench_demo(torch, 4.0)}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
