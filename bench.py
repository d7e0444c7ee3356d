#!/usr/bin/env python
"""Benchmark: Mrays/s of the geodesic spectral ray tracer on B200.

A "step" is one render of the workload (default: the Kerr a=0.9 thin-disk scene
at 1024^2, 64 spectral bins, tolerance 1e-8) on each GPU. Multi-GPU runs are
weak-scaled: every rank renders its own frame (rays are independent; there is
no data-path collective), and the value is all ranks' rays / max-over-ranks
device time.

`--impl reference` times the reference's CPU algorithm instead: the FP64 C++
restatement of the reference's CPU integrator (the reference is Julia, which
is not installed), on the host's cores, on a bounded pixel sample.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s Kerr 1024² at ≤1e-3 rel err: FP32-mixed vs FP64 on 1 B200; adjoint grad/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="kerr_thin_disk")
    ap.add_argument("--x-pix", type=int, default=1024)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-fp64-leg", action="store_true", help="skip the FP64 comparison leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=8192, help="rays in the CPU baseline sample")
    ap.add_argument("--no-batched", action="store_true", help="skip the 96-frame batched leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the synchrotron-torus adjoint leg")
    ap.add_argument("--no-scenes", action="store_true", help="skip the per-bin scene leg (Powehi, Synchro_Test, wormhole, Cartesian sphere)")
    ap.add_argument("--no-plain-leg", action="store_true", help="skip the plain FP64 GPU path leg")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the cfg1-cfg3 legs (Minkowski sphere 256^2, Schwarzschild 1024^2, Kerr thick 2048^2)")
    ap.add_argument("--adjoint-x-pix", type=int, default=512)
    ap.add_argument("--torus-forward-only", action="store_true",
                    help="time only the synchrotron torus's forward render (FP32-mixed, FSAL) at --adjoint-x-pix "
                         "(one warm-up, --steps timed) and print one JSON line")
    ap.add_argument("--strong", action="store_true",
                    help="N>1: report the strong-scaling leg (one frame over N GPUs in interleaved tiles) as the "
                         "headline value")
    ap.add_argument("--block-warps", type=int, default=0)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_init(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def all_max(v, world):
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([c.strip() for c in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# the CPU legs (oracle restatement of the reference's CPU integrator)
# ---------------------------------------------------------------------------
def steps_hist(steps):
    """Step attempts per ray: quantiles and a log2-binned histogram."""
    st = np.asarray(steps, dtype=np.int64)
    q = {f"p{k}": int(np.quantile(st, k / 100)) for k in (1, 10, 50, 90, 99)}
    q["max"] = int(st.max())
    q["mean"] = float(st.mean())
    edges = [0] + [2 ** k for k in range(4, 15)]
    h, _ = np.histogram(st, bins=edges + [1 << 62])
    q["hist_log2"] = {f"<{e2}" if e2 < (1 << 62) else f">={e1}": int(c)
                      for e1, e2, c in zip(edges, edges[1:] + [1 << 62], h)}
    return q


def cpu_sample_ids(P, n):
    n = min(n, P)
    return np.unique(np.linspace(0, P - 1, n).round().astype(np.int64))


def rel_err_y(g_xyz, ref_xyz):
    """Relative error of linear Y against the oracle, denominator
    max(|ref|, 1e-6 max|ref|)."""
    y_r = np.asarray(ref_xyz)[:, 1]
    y_g = np.asarray(g_xyz)[:, 1].astype(np.float64)
    den = np.maximum(np.abs(y_r), 1e-6 * np.abs(y_r).max() + 1e-300)
    return np.abs(y_g - y_r) / den


def parity_block(g_cls, g_xyz, ref, sel=None):
    """Class match and intensity error of GPU pixels against the FP64 oracle on
    the same pixels (sel: a boolean subset of them)."""
    same = np.asarray(g_cls) == ref["class"]
    err = rel_err_y(g_xyz, ref["xyz"])
    if sel is None:
        sel = np.ones(same.size, bool)
    if not sel.any():
        return {"px": 0}
    ok = sel & same
    out = {"px": int(sel.sum()), "class_match": float(np.mean(same[sel]))}
    if ok.any():
        e = err[ok]
        out.update({"within_1e-3": float(np.mean(e <= 1e-3)), "p99_rel_err": float(np.quantile(e, 0.99)),
                    "max_rel_err": float(e.max())})
    return out


def _short(block, with_px=True):
    """A parity block rounded for the summary line."""
    if not block:
        return {}
    keys = (("px", "px"), ("class_match", "class"), ("within_1e-3", "in_1e-3"), ("p99_rel_err", "p99"))
    out = {}
    for k, o in keys:
        if k in block and (with_px or k != "px"):
            v = block[k]
            out[o] = v if isinstance(v, int) else float(f"{v:.4g}")
    return out


def shadow_annulus(cls_img, x_pix, y_pix, width=3):
    """Pixels within `width` of the shadow edge: horizon-class pixels with a
    non-horizon 4-neighbour, dilated by width pixels. This band holds the
    critical curve and the photon-ring images around it."""
    hz = np.asarray(cls_img).reshape(y_pix, x_pix) == 2  # RTW_CLASS_HORIZON
    pad = np.pad(hz, 1, mode="edge")
    inner = pad[:-2, 1:-1] & pad[2:, 1:-1] & pad[1:-1, :-2] & pad[1:-1, 2:]
    band = hz & ~inner
    for _ in range(width):
        pb = np.pad(band, 1)
        band = band | pb[:-2, 1:-1] | pb[2:, 1:-1] | pb[1:-1, :-2] | pb[1:-1, 2:]
    return np.flatnonzero(band.ravel())


def cpu_time(scene, cam, colors, n, threads=0, keep=False, skybox=(None, None), gaunt_lut=None):
    from oracle import oracle as O
    O.build()
    P = cam.x_pix * cam.y_pix
    ids = cpu_sample_ids(P, n)
    t = time.perf_counter()
    want = ("xyz", "class", "steps", "state") + (("spectrum",) if gaunt_lut is not None else ())
    res = O.render(scene, cam, colors, pixel_ids=ids, threads=threads, want=want, skybox=skybox, gaunt_lut=gaunt_lut)
    dt = time.perf_counter() - t
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    if keep:
        return ids.size / dt / 1e6, ids.size, dt, cores, res
    return ids.size / dt / 1e6, ids.size, dt, cores


def run_reference(args):
    """--impl reference: the reference's CPU algorithm (oracle port), rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from rtwca_b200 import configs
    scene, cam, colors = configs.workload(args.workload, x_pix=args.x_pix)
    for _ in range(args.warmup):
        cpu_time(scene, cam, colors, max(64, args.cpu_sample // 8))
    vals = []
    t_all = 0.0
    for _ in range(args.steps):
        v, n, dt, cores = cpu_time(scene, cam, colors, args.cpu_sample)
        vals.append(v)
        t_all += dt
    value = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_all / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.workload} {args.x_pix}x{cam.y_pix}, 64 bins, tol {cam.tolerance:g}",
                   "sample_rays_per_step": n},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": cores, "kind": "port",
                         "sample": f"{n} evenly spaced pixels of the {args.x_pix}^2 frame per step, "
                                   "C++ FP64 restatement of the reference's CPU integrator, OpenMP"},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# the B200 arm
# ---------------------------------------------------------------------------
def op_model(renderer, scene_kind, stats, n_bins):
    """Algorithmic FP operations of one render from the library's own operation
    counts (rtw_op_counts) and the render's counters."""
    oc = renderer.op_counts(scene_kind)
    att = stats["step_attempts"]
    emit_att = stats["emitting_steps"]
    spec = stats["spectral_steps"]
    # 6 right-hand sides per attempt (k1 is carried); emitting attempts are
    # counted as emitting in all 6 stages (an upper bound of that share)
    flops = (att * (6 * oc["rhs_vacuum"] + oc["step_overhead"]) + emit_att * 6 * (oc["rhs_emit"] - oc["rhs_vacuum"])
             + spec * n_bins * oc["bin_step"])
    mufu = (att * (6 * oc["rhs_vacuum_mufu"] + oc["step_overhead_mufu"])
            + emit_att * 6 * (oc["rhs_emit_mufu"] - oc["rhs_vacuum_mufu"]) + spec * n_bins * oc["bin_step_mufu"])
    return flops, mufu, oc


# DRAM bytes per step attempt of the FP32-mixed Kerr trace kernel, from one ncu
# capture at 512^2: the main launch's dram__bytes_read+write (22.1 + 1.1 MB; the
# outputs, 17 B per ray, are still in L2 when the launch ends) over the render's
# step attempts (the tail launch, 10 % of that render's time, returned no counters)
TRAFFIC_B_PER_ATTEMPT = 23.20e6 / 357227232


def batched_leg(r, world, rank, stream, barrier_fn):
    """96 Kerr frames (r ~ U[5, 40] M, inclination ~ U[10, 85] deg, numpy
    default_rng(0); 32 frames each at 256^2, 512^2, 1024^2; tolerance 1e-6 /
    1e-8 alternating) in ONE persistent, graph-captured, autotuned FP32-mixed
    launch per GPU (frames sharded over ranks by estimated cost). Per-frame
    latency from the kernel's global-timer stamps. Against it, FP64 with one
    frame per launch, on the 24 frames k % 8 in {0, 1} (every size and both
    tolerances), also run batched-mixed for a like-for-like ratio."""
    import torch
    from rtwca_b200 import abi, configs, shard

    scene, cams, colors, meta = configs.batched_frames(96, seed=0)
    mine = shard.frames_of_rank(cams, world, rank)
    dev = torch.device("cuda", torch.cuda.current_device())

    def outputs(cs):
        P = sum(c.x_pix * abi.y_pixels(c.x_pix, c.fov_hor, c.fov_vert) for c in cs)
        xyz = torch.empty((P, 3), dtype=torch.float32, device=dev)
        cl = torch.empty(P, dtype=torch.uint8, device=dev)
        o = abi.Outputs()
        o.xyz, o.term_class, o.on_device = xyz.data_ptr(), cl.data_ptr(), 1
        return P, o, (xyz, cl)

    def run(cs, precision, graph, autotune):
        prm = r.params(colors, precision=precision, stream=stream.cuda_stream, graph=graph, autotune=autotune)
        P, o, keep = outputs(cs)
        # warm-up on the same frame list shrunk to 16 px wide (allocations, tuning)
        small = [abi.make_camera(list(c.position), list(c.direction), c.speed, list(c.pointing), 16, c.fov_hor,
                                 c.fov_vert, c.tolerance, c.max_steps) for c in cs]
        r.render_raw(scene, small, prm, outputs(small)[1])
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r.render_raw(scene, cs, prm, o)
        e1.record(stream)
        e1.synchronize()
        return P, e0.elapsed_time(e1), r.stats()

    barrier_fn()
    cs = [cams[i] for i in mine]
    P, ms, st = run(cs, abi.PREC_MIXED, True, True)
    ft = r.frame_times(len(cs))
    # like-for-like subset: batched mixed vs one frame per launch in FP64
    sub = [k for k in mine if k % 8 in (0, 1)]
    sc = [cams[i] for i in sub]
    Ps, ms_sub, _ = run(sc, abi.PREC_MIXED, True, True) if sc else (0, 0.0, None)
    ms64, lat64 = 0.0, []
    prm64 = r.params(colors, precision=abi.PREC_FP64, stream=stream.cuda_stream)
    if sc:  # warm-up of the FP64 kernel
        r.render_raw(scene, [sc[0]], prm64, outputs([sc[0]])[1])
    for c in sc:
        Pc, o, keep = outputs([c])
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r.render_raw(scene, [c], prm64, o)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1)
        ms64 += t
        lat64.append(ms64)
    barrier_fn()
    ms_all = all_max(ms, world)
    rays_all = sum(cams[i].x_pix * abi.y_pixels(cams[i].x_pix, cams[i].fov_hor, cams[i].fov_vert) for i in range(96))
    if world > 1:
        import torch.distributed as dist
        gathered = [None] * world
        dist.all_gather_object(gathered, (list(ft["done"]), ms_sub, Ps, ms64, lat64))
    else:
        gathered = [(list(ft["done"]), ms_sub, Ps, ms64, lat64)]
    done = np.concatenate([np.asarray(g[0]) for g in gathered])
    sub_ms = max(g[1] for g in gathered)
    sub_rays = sum(g[2] for g in gathered)
    f64_ms = max(g[3] for g in gathered)
    f64_lat = np.concatenate([np.asarray(g[4]) for g in gathered]) if sub_rays else np.zeros(1)
    return {
        "workload": "kerr_thin_disk, 96 frames (32 x 256^2, 32 x 512^2, 32 x 1024^2), r ~ U[5,40] M, "
                    "inclination ~ U[10,85] deg, numpy default_rng(0), tol 1e-6/1e-8 alternating",
        "rays": rays_all, "ms": ms_all, "value": rays_all / (ms_all * 1e-3) / 1e6, "unit": "Mrays/s",
        "launches_per_gpu": 1, "graph_replayed": st["graph_replayed"],
        "autotuned": {"block_warps": st["block_warps"], "refill_min": st["refill_min"]},
        "frame_done_ms": {"p50": float(np.quantile(done, 0.5)), "p99": float(np.quantile(done, 0.99))},
        "subset_24_frames": {
            "rays": sub_rays,
            "batched_mixed": {"ms": sub_ms, "value": sub_rays / (sub_ms * 1e-3) / 1e6},
            "one_frame_per_launch_fp64": {"ms": f64_ms, "value": sub_rays / (f64_ms * 1e-3) / 1e6,
                                          "frame_done_ms": {"p50": float(np.quantile(f64_lat, 0.5)),
                                                            "p99": float(np.quantile(f64_lat, 0.99))}},
        },
    }


def scenes_leg(r, rank, cpu=True):
    """Four of the reference's per-bin scenes through the per-bin kernels,
    each at 1024 px wide with the reference's default field
    of view and colours (400/550/700 nm), tolerance 1e-6: Powehi ("m87": Kerr
    a = 0.9, disk + jet) and Synchro_Test ("synch": flat Cartesian space,
    camera inside the cylinder), the Dneg wormhole ("wormhole", two
    synthetic 64-texel cube maps from numpy default_rng(0) standing in for the
    reference's missing skybox PNGs) and the Cartesian blackbody sphere
    ("minkowski_t,x,y,z_sphere", the first of those maps as its skybox), and the
    bremsstrahlung torus (the Gaunt-factor lookup of emission_functions.jl:54-78
    on a smooth stand-in table on the van Hoof grid; 512^2, 230 GHz +- 20 %,
    8 bins, the torus camera; its parity on the spectra). FP32-mixed and FP64,
    the reference's step.
    Device time of the kernel (1 warm-up + 3 timed renders, mean); on rank 0
    the FP64 oracle on 4096 evenly spaced pixels on all host cores gives the
    CPU rate and a parity sample (linear Y within 1e-3)."""
    from rtwca_b200 import abi, configs

    def rel_err(g, ref):
        den = np.maximum(np.abs(ref), 1e-6 * np.abs(ref).max() + 1e-300)
        return np.abs(np.asarray(g, np.float64) - ref) / den

    col = np.array([400.0, 550.0, 700.0])
    out = {}
    rng = np.random.default_rng(0)
    sky = tuple(rng.uniform(0, 1, (3 * 64, 4 * 64, 3)).astype(np.float32) for _ in range(2))
    for name, sc, camf, kw in (("m87_powehi", configs.powehi_scene(), configs.powehi_camera, {}),
                               ("synch_synchro_test", configs.synchro_scene(), configs.synchro_camera, {}),
                               ("wormhole", configs.wormhole_scene(), configs.wormhole_camera, {"skybox": sky}),
                               ("minkowski_cart_sphere", configs.cart_sphere_scene(), configs.cart_sphere_camera,
                                {"skybox": (sky[0], None)}),
                               ("brems_torus", configs.brems_scene(), configs.torus_camera,
                                {"gaunt_lut": configs.smooth_gaunt_table()})):
        cam = camf(1024 if name != "brems_torus" else 512, tol=1e-6)
        P = cam.x_pix * cam.y_pix
        colv = configs.torus_colors(8) if name == "brems_torus" else col
        leg = {"workload": f"{name} {cam.x_pix}x{cam.y_pix}, {colv.size} bins, tol 1e-6, reference step"}
        for pname, prec in (("mixed", abi.PREC_MIXED), ("fp64", abi.PREC_FP64)):
            wv = ("spectrum",) if name == "brems_torus" else ("xyz",)
            r.render(sc, [cam], colv, want=wv, precision=prec, integrator=abi.DP45_REF_COMPAT, **kw)
            ms = []
            for _ in range(3):
                g = r.render(sc, [cam], colv, want=wv, precision=prec, integrator=abi.DP45_REF_COMPAT, **kw)
                ms.append(r.stats()["kernel_ms"])
            t = float(np.mean(ms))
            leg[pname] = {"Mrays_s": P / t / 1e3, "ms": t, "step_attempts": r.stats()["step_attempts"]}
            if pname == "mixed":
                gx = g["spectrum"] if name == "brems_torus" else g["xyz"]
        if cpu and rank == 0:
            v, n, dt, cores, ref = cpu_time(sc, cam, colv, 4096, keep=True, skybox=kw.get("skybox", (None, None)),
                                            gaunt_lut=kw.get("gaunt_lut"))
            ids = cpu_sample_ids(P, 4096)
            if name == "brems_torus":  # mm-wave bins: the spectra (the CIE weights vanish there)
                e = rel_err(gx[ids].ravel(), ref["spectrum"].ravel())
            else:
                e = rel_err(gx[ids, 1], ref["xyz"][:, 1])
            leg["cpu_oracle"] = {"Mrays_s": v, "pixels": n, "s": dt, "cores": cores}
            leg["mixed_over_cpu"] = leg["mixed"]["Mrays_s"] / v
            leg["parity_sample_within_1e-3"] = float(np.mean(e <= 1e-3))
        out[name] = leg
    return out


def render_timed(r, scene, cam, colors, prec, reps, integrator=None, want=("xyz", "class")):
    """One warm-up and `reps` timed renders (device time of the kernel); the
    last render's host outputs and counters."""
    from rtwca_b200 import abi
    integ = abi.DP45_REF_COMPAT if integrator is None else integrator
    r.render(scene, [cam], colors, want=("class",), precision=prec, integrator=integ)
    ms = []
    g = None
    for _ in range(reps):
        g = r.render(scene, [cam], colors, want=want, precision=prec, integrator=integ)
        ms.append(r.stats()["kernel_ms"])
    return g, float(np.mean(ms)), r.stats()


def config_legs(r, rank, cpu=True, sample=2048):
    """The workload configs besides the headline, each at its stated size,
    FP32-mixed and FP64 (device time of the kernel), each precision's error
    stated against the FP64 oracle:
      cfg1 minkowski_sphere 256^2 (64 bins, tol 1e-8): the whole frame;
      cfg2 schwarzschild_disk 1024^2 (64 bins, tol 1e-8): `sample` evenly
           spaced pixels;
      cfg3 kerr_thick_disk 2048^2 (64 bins, tol 1e-7, orbiting camera at
           r = 5 M): `sample` evenly spaced pixels."""
    from rtwca_b200 import abi, configs
    out = {}
    for key, name, reps in (("cfg1_minkowski_sphere_256", "minkowski_sphere", 3),
                            ("cfg2_schwarzschild_1024", "schwarzschild_disk", 2),
                            ("cfg3_kerr_thick_2048", "kerr_thick_disk", 1)):
        scene, cam, colors = configs.workload(name)
        P = cam.x_pix * cam.y_pix
        leg = {"workload": f"{name} {cam.x_pix}x{cam.y_pix}, 64 bins, tol {cam.tolerance:g}"}
        gs = {}
        for pname, prec in (("mixed", abi.PREC_MIXED), ("fp64", abi.PREC_FP64)):
            g, ms, st = render_timed(r, scene, cam, colors, prec, reps)
            gs[pname] = g
            leg[pname] = {"Mrays_s": P / ms / 1e3, "ms": ms, "step_attempts": st["step_attempts"],
                          "promoted_steps": st["promoted_steps"]}
        leg["mixed_over_fp64"] = leg["mixed"]["Mrays_s"] / leg["fp64"]["Mrays_s"]
        if cpu and rank == 0:
            ids = np.arange(P) if name == "minkowski_sphere" else cpu_sample_ids(P, sample)
            v, n, dt, cores, ref = cpu_time(scene, cam, colors, ids.size, keep=True)
            leg["oracle"] = {"Mrays_s": v, "pixels": n, "s": dt, "cores": cores}
            for pname in ("mixed", "fp64"):
                leg[pname]["parity"] = parity_block(gs[pname]["class"][ids], gs[pname]["xyz"][ids], ref)
        out[key] = leg
    return out


def photon_ring_leg(scene, cam, colors, g_cls, g_xyz, n_max=4096):
    """The headline frame's shadow-edge annulus (3 px either side of the
    shadow boundary of the GPU render, at most n_max evenly spaced pixels)
    against the FP64 oracle. Photon-ring pixels are those whose oracle ray
    wound more than once around the hole (|phi_end - phi_camera| > 2 pi) or
    crossed the equatorial plane at least twice; they are reported apart from
    the rest of the band."""
    from oracle import oracle as O
    ids = shadow_annulus(g_cls, cam.x_pix, cam.y_pix)
    if ids.size > n_max:
        ids = ids[np.unique(np.linspace(0, ids.size - 1, n_max).round().astype(np.int64))]
    t = time.perf_counter()
    ref = O.render(scene, cam, colors, pixel_ids=ids, want=("xyz", "class", "state", "crossings"))
    dt = time.perf_counter() - t
    ring = (np.abs(ref["state"][:, 3] - cam.position[3]) > 2 * np.pi) | (ref["crossings"] >= 2)
    return {"band_px": int(ids.size), "oracle_s": dt,
            "criterion": "oracle |dphi| > 2 pi or >= 2 equatorial crossings",
            "ring": parity_block(g_cls[ids], g_xyz[ids], ref, ring),
            "rest_of_band": parity_block(g_cls[ids], g_xyz[ids], ref, ~ring)}


def strong_leg(r, world, rank, scene, cam, colors, barrier_fn, reps=2):
    """One frame over `world` GPUs (strong scaling): interleaved 16 x 16 pixel
    tiles (tile t -> rank t mod world), each rank's tiles in one batched
    launch, one gather of the tiles to rank 0, which assembles the image.
    Device time (CUDA events around the whole call, gather included), max
    over ranks."""
    import torch
    from rtwca_b200 import abi, shard
    P = cam.x_pix * cam.y_pix
    shard.render_frame_tiles(r, scene, cam, colors, world, rank, precision=abi.PREC_MIXED)  # warm-up
    ms = []
    for _ in range(reps):
        barrier_fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        img = shard.render_frame_tiles(r, scene, cam, colors, world, rank, precision=abi.PREC_MIXED)
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = all_max(float(np.mean(ms)), world)
    out = {"value": P / (t * 1e-3) / 1e6, "unit": "Mrays/s", "ms": t, "tile": 16,
           "tiles_per_rank": -(-len(shard.tile_windows(cam.x_pix, cam.y_pix)) // world),
           "exchange": "one gather of the tiles to rank 0"}
    if rank == 0 and img is not None:
        out["pixels_assembled"] = int(img["class"].size)
    return out


def adjoint_leg(r, x_pix, world=1, rank=0):
    """Differentiable synchrotron torus: Kerr a = 0.94, inclination 17 deg,
    x_pix^2 rays, 32 bins over 230 GHz +- 20 %, FP32-mixed, tolerance 1e-6.
    Loss = sum (I - target)^2 against the image at parameters perturbed by
    5 % normal deviates from numpy default_rng(1). One rtw_adjoint call =
    forward render + record pass + reverse sweep (checkpoints every 16
    accepted steps). Rays that take a polar escape are left out of the
    gradient (counted in escape_rays). Times are device times of the call.
    On N GPUs every rank takes the interleaved pixels rank, rank + N, ...
    (strong scaling) and one all-reduce sums the loss and the gradient; the
    time is the max over ranks."""
    from rtwca_b200 import abi, configs

    tp = configs.torus_target_params(1)
    scT, camT, col = configs.torus_problem(x_pix=x_pix, tol=1e-6, params=tp)
    target = r.render(scT, [camT], col, want=("spectrum",), precision=abi.PREC_MIXED,
                      integrator=abi.DP45_FSAL)["spectrum"]
    sc, cam, col = configs.torus_problem(x_pix=x_pix, tol=1e-6)
    # forward alone, for the ratio (warm-up first)
    r.render(sc, [cam], col, want=("spectrum",), precision=abi.PREC_MIXED, integrator=abi.DP45_FSAL)
    r.render(sc, [cam], col, want=("spectrum",), precision=abi.PREC_MIXED, integrator=abi.DP45_FSAL)
    fwd = r.stats()
    a = r.adjoint(sc, cam, col, target, precision=abi.PREC_MIXED, exclude_escape_rays=True, rays=(rank, 0, world))
    P = cam.x_pix * cam.y_pix
    if world > 1:
        import torch
        import torch.distributed as dist
        v = torch.tensor([a["loss"]] + list(a["grad"]) + [float(a["escape_rays"]), float(a["events"])],
                         dtype=torch.float64, device="cuda")
        dist.all_reduce(v)
        t = torch.tensor([a["total_ms"], a["forward_ms"], a["record_ms"], a["reverse_ms"]], dtype=torch.float64,
                         device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        v, t = v.cpu().tolist(), t.cpu().tolist()
        a["loss"], a["grad"], a["escape_rays"], a["events"] = v[0], v[1:6], int(v[6]), int(v[7])
        a["total_ms"], a["forward_ms"], a["record_ms"], a["reverse_ms"] = t
    return {
        "workload": f"synchrotron torus {cam.x_pix}x{cam.y_pix}, 32 bins 230 GHz +-20%, a=0.94, i=17 deg, tol 1e-6, "
                    "FP32-mixed, FSAL",
        "metric": "adjoint grad/s", "value": 1000.0 / a["total_ms"], "unit": "gradients/s",
        "adjoint_ms": a["total_ms"], "forward_render_ms": fwd["kernel_ms"],
        "adjoint_over_forward": a["total_ms"] / fwd["kernel_ms"],
        "parts_ms": {"forward": a["forward_ms"], "record": a["record_ms"], "reverse": a["reverse_ms"]},
        "forward_Mrays_s": P / fwd["kernel_ms"] / 1e3, "step_attempts": fwd["step_attempts"],
        "loss": a["loss"], "grad": dict(zip(abi.ADJOINT_PARAMS, [float(v) for v in a["grad"]])),
        "events": a["events"], "checkpoints": a["checkpoints"], "scratch_GB": a["scratch_bytes"] / 1e9,
        "escape_rays": a["escape_rays"], "escape_rays_policy": "left out of the gradient",
        "target_params": tp, "n_gpus": world,
        "sharding": "interleaved pixels, one all-reduce of loss + gradient" if world > 1 else "one GPU",
    }


def run_b200(args):
    import torch
    from rtwca_b200 import Renderer, abi, configs

    rank, world, local = dist_init(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scene, cam, colors = configs.workload(args.workload, x_pix=args.x_pix)
    P = cam.x_pix * cam.y_pix
    N = len(colors)
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    r = Renderer(local)
    stream = torch.cuda.current_stream(dev)
    # device outputs (inputs are the camera descriptors, uploaded by every render)
    xyz = torch.empty((P, 3), dtype=torch.float32, device=dev)
    cls = torch.empty(P, dtype=torch.uint8, device=dev)
    steps = torch.empty(P, dtype=torch.int32, device=dev)
    out = abi.Outputs()
    out.xyz, out.term_class, out.steps, out.on_device = xyz.data_ptr(), cls.data_ptr(), steps.data_ptr(), 1
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    def params(p, integ=abi.DP45_REF_COMPAT):
        return r.params(colors, precision=p, integrator=integ, stream=stream.cuda_stream,
                        block_warps=args.block_warps, ctas_per_sm=args.ctas_per_sm)

    def timed_renders(p, k, w, integ=abi.DP45_REF_COMPAT):
        prm = params(p, integ)
        for _ in range(w):
            r.render_raw(scene, [cam], prm, out)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        total = 0.0
        kernel = 0.0
        launches = 0
        st = None
        for _ in range(k):
            flush.fill_(1.0)  # evict L2 between timed renders
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r.render_raw(scene, [cam], prm, out)
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
            st = r.stats()
            kernel += st["kernel_ms"]
            launches += st["launches"]
        torch.cuda.synchronize()
        barrier(world)
        st = dict(st, launches_total=launches)
        return total, kernel, st

    peaks = r.measure_peaks() if rank == 0 else None
    with ClockSampler(local) as clk:
        total_ms, kernel_ms, st = timed_renders(prec, args.steps, args.warmup)
    total_ms = all_max(total_ms, world)
    value = world * P * args.steps / (total_ms * 1e-3) / 1e6
    ms_per_step = total_ms / args.steps

    # FP64 comparison leg (same workload, same timing rules)
    fp64 = None
    if not args.no_fp64_leg and prec == abi.PREC_MIXED:
        t64, _, st64 = timed_renders(abi.PREC_FP64, max(1, args.steps // 2), 1)
        t64 = all_max(t64, world)
        fp64 = {"value": world * P * max(1, args.steps // 2) / (t64 * 1e-3) / 1e6,
                "ms_per_step": t64 / max(1, args.steps // 2)}

    # textbook FSAL Dormand-Prince (k1 = f(y)) instead of the reference's
    # carried average slope: same workload, same timing rules
    fsal = None
    if not args.no_fp64_leg:
        tf, _, _ = timed_renders(prec, max(1, args.steps // 2), 1, abi.DP45_FSAL)
        tf = all_max(tf, world)
        fsal = {"value": world * P * max(1, args.steps // 2) / (tf * 1e-3) / 1e6,
                "ms_per_step": tf / max(1, args.steps // 2)}

    # the plain FP64 GPU path (one thread per pixel, the reference's full state
    # and right-hand side): one timed render of the same frame after a warm-up
    # on a 128^2 frame; single-GPU runs only (it takes tens of seconds)
    plain = None
    if not args.no_plain_leg and not args.no_fp64_leg and world == 1:
        pp = params(abi.PREC_FP64_PLAIN)
        _, camw, _ = configs.workload(args.workload, x_pix=128)
        r.render_raw(scene, [camw], pp, out)
        torch.cuda.synchronize()
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r.render_raw(scene, [cam], pp, out)
        e1.record(stream)
        e1.synchronize()
        tp = e0.elapsed_time(e1)
        plain = {"value": P / (tp * 1e-3) / 1e6, "ms_per_step": tp, "mixed_over_plain": value / (P / (tp * 1e-3) / 1e6),
                 "what": "one FP64 thread per pixel over a grid, the reference's 8 + 2N state and per-bin right-hand "
                         "side, no warp cooperation (RTW_PREC_FP64_PLAIN)"}

    strong = None
    if world > 1 or args.strong:
        strong = strong_leg(r, world, rank, scene, cam, colors, lambda: barrier(world))
        if args.strong:
            value = strong["value"]
            ms_per_step = strong["ms"]

    batched = None
    if not args.no_batched:
        batched = batched_leg(r, world, rank, stream, lambda: barrier(world))
    adjoint = None
    if not args.no_adjoint:
        barrier(world)
        adjoint = adjoint_leg(r, args.adjoint_x_pix, world, rank)
    scenes = None
    if not args.no_scenes:
        # no collectives in this leg: a failure in it is reported in the line
        # instead of ending the run before the headline's end-to-end leg
        try:
            scenes = scenes_leg(r, rank, cpu=not args.no_cpu_baseline)
        except Exception as exc:
            scenes = {"error": f"{type(exc).__name__}: {exc}"[:400]}

    configs_leg = None
    if not args.no_configs and world == 1:
        configs_leg = config_legs(r, rank, cpu=not args.no_cpu_baseline)

    # end to end through the public API: the synchronous rtw_render call with
    # pinned host outputs, timed by the host clock around the call (frame
    # set-up, table uploads, kernel, device-to-host copies of XYZ, class and
    # step counts)
    hx = torch.empty((P, 3), dtype=torch.float32, pin_memory=True)
    hc = torch.empty(P, dtype=torch.uint8, pin_memory=True)
    hs = torch.empty(P, dtype=torch.int32, pin_memory=True)
    hout = abi.Outputs()
    hout.xyz, hout.term_class, hout.steps, hout.on_device = hx.data_ptr(), hc.data_ptr(), hs.data_ptr(), 0
    prm = r.params(colors, precision=prec, block_warps=args.block_warps, ctas_per_sm=args.ctas_per_sm)
    r.render_raw(scene, [cam], prm, hout)
    barrier(world)
    e2e_s = 0.0
    ke = max(1, args.steps // 2)
    for _ in range(ke):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r.render_raw(scene, [cam], prm, hout)   # synchronous: returns with the outputs on the host
        e2e_s += time.perf_counter() - t0
    e2e_ms = all_max(e2e_s * 1e3, world)
    e2e_val = world * P * ke / (e2e_ms * 1e-3) / 1e6
    h2d = 8 * 4 * 128 + 256  # bins table + one frame descriptor
    d2h = P * (12 + 1 + 4)

    if rank == 0:
        flops, mufu, oc = op_model(r, scene.kind, st, N)
        kms = kernel_ms / args.steps
        achieved = flops / (kms * 1e-3) / 1e12
        peak = peaks["fp32_flops"] / 1e12 if prec == abi.PREC_MIXED else peaks["fp64_flops"] / 1e12
        cpu = None
        parity = None
        ring = None
        ref_form = None
        g_cls, g_xyz = hc.numpy(), hx.numpy()
        if not args.no_cpu_baseline:
            v, n, dt, cores, ref = cpu_time(scene, cam, colors, args.cpu_sample, keep=True)
            cpu = {"value": v, "unit": "Mrays/s", "cores": cores, "kind": "port",
                   "sample": f"{n} evenly spaced pixels of the {args.x_pix}^2 frame ({dt:.1f} s), C++ FP64 "
                             "restatement of the reference's CPU integrator, OpenMP"}
            # the same pixels of the (end-to-end) render against the FP64 oracle
            ids = cpu_sample_ids(P, args.cpu_sample)
            parity = parity_block(g_cls[ids], g_xyz[ids], ref)
            parity["of"] = "evenly spaced pixels vs the FP64 oracle, reference step; error on linear Y"
            if args.workload in ("kerr_thin_disk", "schwarzschild_disk"):
                ring = photon_ring_leg(scene, cam, colors, g_cls, g_xyz)
            # the work of the reference's form: the oracle's own integration of
            # the same pixels over a counting scalar (its own step counts),
            # scaled to the frame
            from oracle import oracle as O
            wk = O.work(scene, cam, colors, pixel_ids=ids)
            fw = wk["flops"] * P / ids.size
            ref_form = {"achieved": round(fw / (kms * 1e-3) / 1e12, 3),
                        "frac": round(fw / (kms * 1e-3) / 1e12 / peak, 4),
                        "flops_per_attempt": round(wk["flops"] / wk["attempts"]),
                        "kernel_flops_per_attempt": round(flops / st["step_attempts"]),
                        "source": "oracle counting-scalar run of the cpu sample, scaled to the frame"}
        fp64_v = fp64["value"] if fp64 else None
        summary = {
            "mixed_Mrays_s": value if prec == abi.PREC_MIXED else None,
            "fp64_Mrays_s": fp64_v,
            "mixed_over_fp64": value / fp64_v if fp64_v else None,
            "plain_fp64_Mrays_s": plain["value"] if plain else None,
            "mixed_over_plain_fp64": plain["mixed_over_plain"] if plain else None,
            "fsal_Mrays_s": fsal["value"] if fsal else None,
            "batched_Mrays_s": batched["value"] if batched else None,
            "strong_Mrays_s": strong["value"] if strong else None,
            "batched_frame_done_ms_p50_p99": ([round(batched["frame_done_ms"]["p50"]), round(batched["frame_done_ms"]["p99"])]
                                              if batched else None),
            "adjoint_grad_per_s": adjoint["value"] if adjoint else None,
            "adjoint_over_forward": adjoint["adjoint_over_forward"] if adjoint else None,
            "parity": _short(parity),
            "photon_ring": ({"band_px": ring["band_px"], "ring": _short(ring["ring"]),
                             "rest": _short(ring["rest_of_band"])} if ring else None),
        }
        if configs_leg:
            for k, leg in configs_leg.items():
                summary[k] = {pn: {"Mrays_s": round(leg[pn]["Mrays_s"], 4), **_short(leg[pn].get("parity"), False)}
                              for pn in ("mixed", "fp64")}
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong" if args.strong else "weak",
            "vs_baseline": None, "dtype": "f32+f64" if prec == abi.PREC_MIXED else "f64", "data": "synthetic",
            "gpu_launches": st["launches_total"],
            "config": {"workload": f"{args.workload} {cam.x_pix}x{cam.y_pix}, 64 bins, tol {cam.tolerance:g}, "
                                   f"{'FP32-mixed' if prec == abi.PREC_MIXED else 'FP64'}, reference step",
                       "rays_per_gpu": P // world if args.strong else P,
                       "parallelism": (f"strong x{world} (one frame in interleaved 16x16 tiles)" if args.strong
                                       else f"weak x{world} (one frame per GPU)"),
                       "l2": "flushed (256 MB write) between timed renders"},
            "summary": summary,
            "roofline": {"bound": "fp32" if prec == abi.PREC_MIXED else "fp64", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": (st["step_attempts"] * TRAFFIC_B_PER_ATTEMPT
                                     if prec == abi.PREC_MIXED and args.workload == "kerr_thin_disk" else None),
                         "peak_source": "measured in-run FMA probe (rtw_measure_peaks)",
                         "mufu_gops": mufu / (kms * 1e-3) / 1e9, "mufu_peak_gops": peaks["mufu_ops"] / 1e9,
                         "reference_form": ref_form},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": "Mrays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "timer": "host clock around the synchronous rtw_render call"},
            "clocks": clk.summary(),
        }
        details = {
            "fp64": fp64, "fsal": fsal, "plain_fp64": plain, "batched": batched, "adjoint": adjoint, "strong": strong,
            "scenes": scenes, "configs": configs_leg, "photon_ring": ring, "parity_sample": parity,
            "integrator": "reference step (k1 = previous sum b_i k_i)",
            "traffic_source": "ncu dram__bytes_read+write of one capture of this kernel at 512^2, scaled by step "
                              "attempts",
            "op_counts": oc, "steps_per_ray": steps_hist(hs.numpy()),
            "counters": {k: st[k] for k in ("step_attempts", "rejected_steps", "promoted_steps", "spectral_steps",
                                            "emitting_steps", "escape_substeps", "nan_rays", "tail_rays")},
        }
        # every leg in full on stderr (one JSON line), the summary on stdout
        sys.stderr.write("BENCH_DETAILS " + json.dumps(details) + "\n")
        sys.stderr.flush()
        print(json.dumps(line), flush=True)
    r.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def torus_forward_only(args):
    """The per-bin forward kernel alone on the synchrotron torus (the forward
    render of the adjoint leg, without the adjoint's record pool)."""
    from rtwca_b200 import Renderer, abi, configs
    sc, cam, col = configs.torus_problem(x_pix=args.adjoint_x_pix, tol=1e-6)
    r = Renderer(0)
    r.render(sc, [cam], col, want=("spectrum",), precision=abi.PREC_MIXED, integrator=abi.DP45_FSAL)
    ms = []
    for _ in range(max(1, args.steps)):
        r.render(sc, [cam], col, want=("spectrum",), precision=abi.PREC_MIXED, integrator=abi.DP45_FSAL)
        ms.append(r.stats()["kernel_ms"])
    P = cam.x_pix * cam.y_pix
    st = r.stats()
    print(json.dumps({"metric": "torus forward Mrays/s", "value": P / float(np.mean(ms)) / 1e3, "unit": "Mrays/s",
                      "ms": ms, "step_attempts": st["step_attempts"],
                      "workload": f"synchrotron torus {cam.x_pix}x{cam.y_pix}, 32 bins, tol 1e-6, FP32-mixed, FSAL"}))
    r.close()


def main():
    args = parse()
    if args.torus_forward_only:
        torus_forward_only(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
