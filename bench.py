#!/usr/bin/env python
"""Benchmark of the distance-estimation raymarcher on B200.

Metric: DE evaluations per second (CalculateDistance calls, counted on the
device) of the FP32 batched (persistent wavefront) kernel, next to the plain
FP64 kernel on the same frame, at stated error against the FP64 frame.
Workload (default): Mandelbox s=-1.5, 1920x1080, camera A (0,-6,0) FOV 53,
N=50, bailout 100, 5 binary steps, Lambert + hard shadow, 16 AO rays per hit.

One step = one full frame rendered by one kernel launch.  Under torchrun each
rank renders its own frame (own jitter stream): weak scaling, no collective on
the data path; timing is max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DE evals/s & Mpix/s: FP32-batched vs plain FP64 kernel, 1 B200, fixed error"
UNIT = "DE evals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--engine", default=None,
                    help="default per workload: wavefront_fp32 (wide views, GI), wavefront_auto (deep zoom, batch)")
    ap.add_argument("--baseline-engine", default="plain_fp64")
    ap.add_argument("--workload", default="mandelbox_1080p_A", choices=WORKLOADS)
    ap.add_argument("--fract", default=None,
                    help="render the scene of a mandelbulber2 settings file (.fract) instead of a named workload")
    ap.add_argument("--spp", type=int, default=16, help="GI samples per pixel (hybrid_gi_2160p)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-baseline", action="store_true")
    a = ap.parse_args()
    if a.fract:
        a.workload = "fract:" + a.fract
    return a


WORKLOADS = ("mandelbox_1080p_A", "mandelbox_1080p_B", "mandelbulb_512", "hybrid_gi_2160p", "batch_2048")


def workload(name: str, spp: int = 16):
    """Scene, camera, parameters and description of a frame workload."""
    from mandelbulber2_b200 import configs

    if name == "mandelbox_1080p_A":
        sc, cam, p = configs.mandelbox_1080p("A")
        desc = {"workload": "mandelbox s=-1.5 1920x1080 camera A (0,-6,0) fov 53, N=50, bailout 100, "
                            "5 binary steps, lambert + hard shadow, 16 AO rays", "width": 1920, "height": 1080,
                "formula": "mandelbox", "maxiter": 50, "ao_rays": 16}
    elif name == "mandelbox_1080p_B":
        sc, cam, p = configs.mandelbox_1080p("A")  # camera B is placed from view A's centre hit in main()
        desc = {"workload": "mandelbox s=-1.5 1920x1080 camera B: 1e-5 in front of view A's centre hit, fov 0.5, "
                            "16 AO rays (deep zoom)", "width": 1920, "height": 1080, "formula": "mandelbox",
                "maxiter": 50, "ao_rays": 16}
    elif name == "mandelbulb_512":
        sc, cam, p = configs.mandelbulb_512()
        desc = {"workload": "mandelbulb p=8 512x512 camera (0,-3,0) fov 53, N=250, bailout 10, 5 binary steps, "
                            "lambert + hard shadow", "width": 512, "height": 512, "formula": "mandelbulb",
                "maxiter": 250}
    elif name == "hybrid_gi_2160p":
        sc, cam, p = configs.hybrid_gi_2160p(spp=spp)
        desc = {"workload": f"hybrid mandelbulb(1-3)+menger(4-12) 3840x2160 monte carlo GI {spp} spp, 4 bounces, "
                            "thin lens aperture 0.02 focus 3", "width": 3840, "height": 2160, "formula": "hybrid",
                "spp": spp}
    elif name.startswith("fract:"):
        # a scene read from a settings file through mbr_fract_parse
        from mandelbulber2_b200 import settings

        path = name[len("fract:"):]
        s = settings.load_from_file(path)
        if not s.ok:
            raise SystemExit(f"{path}: {s.report}")
        sc, cam, p = s.scene, s.camera, s.params
        used = range(sc.n_fractals) if sc.hybrid_fractal_enable else range(1)
        names = {2: "mandelbulb", 7: "menger", 8: "mandelbox"}
        forms = "+".join(names[sc.fractal[i].formula] for i in used if sc.fractal[i].formula in names)
        desc = {"workload": f"settings file {os.path.basename(path)}: {forms} {cam.width}x{cam.height}, "
                            f"N={sc.formula_maxiter}, {p.ao_rays} AO rays", "width": cam.width,
                "height": cam.height, "formula": forms, "maxiter": sc.formula_maxiter, "ao_rays": p.ao_rays}
    else:
        raise SystemExit(f"unknown workload {name}")
    return sc, cam, p, desc


DEFAULT_ENGINE = {"mandelbox_1080p_A": "wavefront_fp32", "mandelbox_1080p_B": "wavefront_auto",
                  "mandelbulb_512": "wavefront_fp32", "hybrid_gi_2160p": "wavefront_fp32",
                  "batch_2048": "wavefront_auto"}


def kernels_per_frame(engine: str, p) -> int:
    """Kernel launches of one frame: the plain engines launch one kernel; the
    wavefront pipeline launches stage P, N (normals wanted), D and S (shadow or
    AO), the finish kernel and the pixel counter; a GI frame launches the
    primary paths, per bounce level (bounces + 1 of them) the normal and vertex
    stages, the per-pixel sum and the pixel counter; the auto engine launches
    the policy kernel and both pipelines, whose kernels of the precision not
    chosen return at once."""
    if "wavefront" not in engine:
        return 1
    if p.gi_samples > 0:
        n = 1 + 2 * (p.gi_bounces + 1) + 2
        return 1 + 2 * n if engine == "wavefront_auto" else n
    n = 4  # primary, normals (the bench asks for normals), finish, pixel count
    if p.ao_rays > 0 or (p.shading_enable and p.shadow_enable):
        n += 2  # directions, shadow/AO marches
    if engine == "wavefront_auto":
        return 1 + 2 * n
    return n


# ---- clocks ---------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons sampled every 2 ms during the timed
    region through NVML (read-only queries; nvidia-smi's 100 ms period misses
    timed regions of a few tens of milliseconds), with an nvidia-smi fallback."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int, pci_bus_id: str | None = None):
        self.index = index
        self.pci = pci_bus_id
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []
        self.stop_flag = threading.Event()

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        h = None
        if self.pci:
            try:
                h = pynvml.nvmlDeviceGetHandleByPciBusId(self.pci)
            except pynvml.NVMLError:
                h = None
        if h is None:
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        return pynvml, h

    def start(self):
        try:
            self.nvml, self.handle = self._nvml_handle()
            self.smax = float(self.nvml.nvmlDeviceGetMaxClockInfo(self.handle, self.nvml.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _poll(self):
        nv, h = self.nvml, self.handle
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        while not self.stop_flag.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((sm, [n for n, b in bits.items() if rs & b]))
            except Exception:
                pass
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.nvml is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            sm = [x[0] for x in self.samples]
            reasons = sorted({r for x in self.samples for r in x[1]})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax, "reasons": reasons,
                    "samples": len(sm), "source": "NVML, 2 ms period"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(self.NAMES, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 100 ms period"}


def pci_bus_id(torch, local: int) -> str | None:
    try:
        pr = torch.cuda.get_device_properties(local)
        return f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
    except Exception:
        return None


# ---- helpers ----------------------------------------------------------------------
def l2_flush_buffer(torch, device):
    return torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)


def time_engine(r, torch, cam, p, bufs, engine, steps, warmup, flush, dist, world):
    """Renders warmup + steps frames; returns (device seconds max over ranks, stats of the timed steps, per-step ms)."""
    from mandelbulber2_b200.render import STATS_FIELDS, stats_dict

    dev = r.device
    stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        r.render_into(cam, p, bufs, stats, engine)
    r.sync()
    stats.zero_()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    for k in range(steps):
        flush.fill_(float(k))  # L2 flush: a 256 MiB write between timed frames (outside the events)
        evs[k][0].record(stream)
        r.render_into(cam, p, bufs, stats, engine)
        evs[k][1].record(stream)
    torch.cuda.synchronize(dev)
    r.sync()
    if dist is not None:
        dist.barrier()
    ms = [a.elapsed_time(b) for a, b in evs]
    t = sum(ms) / 1e3
    if dist is not None:
        tt = torch.tensor([t], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    return t, stats_dict(stats), ms


def compare_frames(fast: dict, ref: dict) -> dict:
    import numpy as np

    hf, hr = fast["hit"].astype(bool), ref["hit"].astype(bool)
    both = hf & hr
    out = {"hit_mismatch": float((hf != hr).mean())}
    if both.any():
        rel = np.abs(fast["depth"][both] - ref["depth"][both]) / np.abs(ref["depth"][both])
        out.update(depth_rel_median=float(np.median(rel)), depth_rel_p99=float(np.quantile(rel, 0.99)),
                   depth_rel_max=float(rel.max()), frac_depth_rel_le_1e4=float((rel <= 1e-4).mean()))
        nf, nr = fast["normal"][both].astype(np.float64), ref["normal"][both].astype(np.float64)
        if np.abs(nr).sum() > 0:  # GI frames carry no normal output
            cos = np.clip((nf * nr).sum(1), -1, 1)
            ang = np.degrees(np.arccos(cos))
            out.update(normal_deg_median=float(np.median(ang)), normal_deg_p99=float(np.quantile(ang, 0.99)))
        if "rgb8" in fast and "rgb8" in ref:
            mse = float(np.mean((fast["rgb8"].astype(np.float64) - ref["rgb8"].astype(np.float64)) ** 2))
            out["psnr_rgb8"] = float("inf") if mse == 0 else 10.0 * np.log10(255.0 ** 2 / mse)
    return out


def load_json(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def cpu_baseline(sc, cam, p, seconds: float) -> dict:
    """The oracle as the reference ships it (-O3 -ffast-math, OpenMP over rows,
    all host threads) on a centred band of rows sized to about `seconds`."""
    from oracle.oracle import Oracle

    o = Oracle("fast")
    threads = o.threads()
    h = cam.height
    rows = max(2, min(8, h))
    while True:
        r0 = h // 2 - rows // 2
        t0 = time.perf_counter()
        _, st = o.render(sc, cam, p, rows=(r0, r0 + rows), threads=threads, outputs=("depth",))
        dt = time.perf_counter() - t0
        if dt >= seconds * 0.5 or rows >= h:
            break
        rows = min(h, max(rows * 2, int(rows * seconds / max(dt, 1e-3))))
    return {"value": st["de_evals"] / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"rows {r0}..{r0 + rows - 1} of the {cam.width}x{h} frame ({rows * cam.width} pixels), "
                      f"{dt:.2f} s", "mpix_per_s": rows * cam.width / dt / 1e6,
            "formula_iterations_per_s": st["formula_iterations"] / dt, "seconds": dt}


def product_library_mapped() -> bool:
    """True when libmbr.so is mapped into this process (Linux)."""
    try:
        with open("/proc/self/maps") as f:
            return any(line.rstrip().endswith("/libmbr.so") for line in f)
    except OSError:
        return False


def reference_centre_depth(o, sc, cam, p) -> float:
    """Depth of view A's centre pixel rendered by the CPU restatement (camera B
    of the deep-zoom workload is placed from it without a GPU)."""
    import numpy as np

    y = cam.height // 2
    out, _ = o.render(sc, cam, p, rows=(y, y + 1), threads=o.threads(), outputs=("depth",))
    return float(np.asarray(out["depth"])[cam.width // 2])


def run_reference(a) -> None:
    """The reference's CPU path (the oracle built as the reference ships it,
    OpenMP over rows on every host thread) on the GPU arm's workload: the
    same scene, camera and parameters, filled from the oracle's restatement
    of the reference's defaults so that the product library is never loaded.
    A step is one full frame when the run fits in about three minutes, else a
    centred band of rows (named in `sample`)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from mandelbulber2_b200 import abi
    from oracle.oracle import Oracle

    o = Oracle("fast")
    abi.use_defaults_from(o.lib, "oracle_")
    if a.workload == "batch_2048":
        print(json.dumps({"impl": "reference", "unavailable": "the batch workload has no CPU arm in this bench"}))
        return
    sc, cam, p, desc = workload(a.workload, a.spp)
    if a.workload == "mandelbox_1080p_B":
        from mandelbulber2_b200 import configs

        cdepth = reference_centre_depth(o, sc, cam, p)
        sc, cam, p = configs.mandelbox_1080p("B", centre_depth=cdepth, camera_rotation=o.camera_rotation)
        desc["centre_depth"] = cdepth
    threads = o.threads()
    # probe: a band of rows, to size the step
    rows = 8
    r0 = cam.height // 2 - rows // 2
    t0 = time.perf_counter()
    o.render(sc, cam, p, rows=(r0, r0 + rows), threads=threads, outputs=("depth",))
    probe = time.perf_counter() - t0
    full = probe * cam.height / rows
    budget = 180.0
    if full * a.steps + probe * a.warmup <= budget:
        r0, rows = 0, cam.height
    else:
        per_step = budget / max(1, a.steps)
        rows = int(max(8, min(cam.height, rows * per_step / max(probe, 1e-3))))
        r0 = cam.height // 2 - rows // 2
    for _ in range(a.warmup):  # warm-up: a small band (caches, thread pool)
        o.render(sc, cam, p, rows=(cam.height // 2 - 4, cam.height // 2 + 4), threads=threads, outputs=("depth",))
    tot_de, tot_t = 0, 0.0
    for _ in range(a.steps):
        t0 = time.perf_counter()
        _, st = o.render(sc, cam, p, rows=(r0, r0 + rows), threads=threads,
                         outputs=("depth", "iters", "hit", "normal", "rgb8"))
        tot_t += time.perf_counter() - t0
        tot_de += st["de_evals"]
    v = tot_de / tot_t
    if rows == cam.height:
        sample = f"the whole {cam.width}x{cam.height} frame per step"
    else:
        sample = f"rows {r0}..{r0 + rows - 1} of {cam.width}x{cam.height} per step ({rows * cam.width} pixels)"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": tot_t / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (procedural fractal scene, no dataset)",
            "config": bench_config(desc, a.gpus),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                             "build": "oracle/mbr_oracle.cpp -O3 -ffast-math -fopenmp (as the reference ships)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "mpix_per_s": rows * cam.width * a.steps / tot_t / 1e6,
            "product_library_loaded": product_library_mapped()}
    print(json.dumps(line), flush=True)


def bench_config(desc: dict, gpus: int) -> dict:
    """The workload block of the JSON line, the same in both arms."""
    return dict(desc, parallelism=f"replicas x{gpus} (one frame per GPU)",
                l2="GPU arm: a 256 MiB buffer is written between timed frames")


def run_batch(a, torch, dist, world, rank, local) -> None:
    """2048 render jobs of uneven size in one graph-captured wavefront launch,
    against the plain FP64 kernel rendering the same jobs one by one."""
    import numpy as np

    from mandelbulber2_b200 import abi, configs
    from mandelbulber2_b200.render import Renderer, STATS_FIELDS, alloc_outputs, outputs_struct, stats_dict
    scenes, cams, offsets, total = configs.batch_jobs(2048, seed=7)
    # jobs of this rank (weak scaling: every rank renders a full set of 2048 jobs)
    p = configs.base_params(5, 20.0)
    p.shading_enable = 0
    p.shadow_enable = 0
    p.ao_rays = 0
    r = Renderer(local)
    jobs = (abi.Job * len(cams))()
    for i, c in enumerate(cams):
        jobs[i].camera = c
        jobs[i].scene_index = i
        jobs[i].pixel_offset = offsets[i]
    sc_arr = (abi.Scene * len(scenes))(*scenes)
    names = ("depth", "normal")
    bufs = alloc_outputs(total, r.device, names)
    stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=r.device)
    o = outputs_struct(bufs, stats)
    b = C.c_void_p()
    lib = abi.load()
    engines = {v: k for k, v in abi.ENGINE_NAMES.items()}
    st = lib.mbr_batch_create(r.ctx, sc_arr, len(scenes), jobs, len(cams), C.byref(p), C.byref(o),
                              engines[a.engine], None, C.byref(b))
    if st != abi.MBR_OK:
        raise SystemExit(lib.mbr_last_error_string(r.ctx).decode())
    wide_jobs = C.c_int32(0)
    n_groups = lib.mbr_batch_groups(b, C.byref(wide_jobs))
    s = torch.cuda.current_stream()
    for _ in range(a.warmup):
        lib.mbr_batch_launch(b, C.c_void_p(s.cuda_stream))
    r.sync()
    stats.zero_()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local, pci_bus_id(torch, local))
    clocks.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(a.steps):
        lib.mbr_batch_launch(b, C.c_void_p(s.cuda_stream))
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    r.sync()
    t = e0.elapsed_time(e1) / 1e3
    sd = stats_dict(stats)
    fast = {k: v.cpu().numpy() for k, v in bufs.items()}
    lib.mbr_batch_destroy(b)
    # plain FP64, job by job (one launch per job)
    base = None
    if not a.no_baseline:
        bstats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=r.device)
        torch.cuda.synchronize()
        e0.record()
        for i, (sc, cam) in enumerate(zip(scenes, cams)):
            r.set_scene(sc)
            n = cam.width * cam.height
            view = {k: v[offsets[i]: offsets[i] + n] for k, v in bufs.items()}
            r.render_into(cam, p, view, bstats, abi.ENGINE_PLAIN_FP64)
        e1.record()
        torch.cuda.synchronize()
        bt = e0.elapsed_time(e1) / 1e3
        bsd = stats_dict(bstats)
        ref = {k: v.cpu().numpy() for k, v in bufs.items()}
        hf, hr = fast["depth"] < 1e19, ref["depth"] < 1e19
        both = hf & hr
        rel = np.abs(fast["depth"][both] - ref["depth"][both]) / ref["depth"][both]
        # jobs whose camera sits inside the solid: every pixel hits at a depth
        # near 0, where a relative depth error compares rounding noise
        inside = np.zeros(total, dtype=bool)
        for i, cam in enumerate(cams):
            n = cam.width * cam.height
            d = ref["depth"][offsets[i]: offsets[i] + n]
            h = d < 1e19
            if h.any() and np.median(d[h]) < 1e-6:
                inside[offsets[i]: offsets[i] + n] = True
        out_both = both & ~inside
        rel_out = np.abs(fast["depth"][out_both] - ref["depth"][out_both]) / ref["depth"][out_both]
        base = {"engine": "plain_fp64 (one launch per job)", "value": bsd["de_evals"] / bt, "unit": UNIT,
                "seconds": bt, "mpix_per_s": bsd["pixels"] / bt / 1e6,
                "hit_mismatch": float((hf != hr).mean()), "depth_rel_median": float(np.median(rel)),
                "depth_rel_p99": float(np.quantile(rel, 0.99)),
                "frac_depth_rel_le_1e4": float((rel <= 1e-4).mean()),
                "camera_outside_solid": {"pixels": int((~inside).sum()),
                                         "hit_mismatch": float((hf != hr)[~inside].mean()),
                                         "depth_rel_median": float(np.median(rel_out)),
                                         "depth_rel_p99": float(np.quantile(rel_out, 0.99)),
                                         "frac_depth_rel_le_1e4": float((rel_out <= 1e-4).mean())},
                "camera_inside_solid": {"jobs": int(sum(1 for i, c in enumerate(cams)
                                                        if inside[offsets[i]])),
                                        "pixels": int(inside.sum())}}
    value = sd["de_evals"] / t
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": t / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (procedural fractal scenes, no dataset)",
                "config": {"workload": "2048 jobs, resolutions {64..1024}^2, cameras on a sphere r U[2.5,4], "
                                       "mandelbulb (p U[2,12], N=100) / mandelbox (scale U[-2.5,-1.5] or U[1.5,3], "
                                       "minR2 U[0.1,0.5], N=40), seed 7; outputs depth + normals",
                           "pixels": total, "engine": f"{a.engine} batch (one graph launch)",
                           "pipelines": n_groups, "fp64_jobs": wide_jobs.value,
                           "l2": "outputs (11 GB) larger than L2"},
                "mpix_per_s": sd["pixels"] / t / 1e6, "stats_per_step": {k: v / a.steps for k, v in sd.items()},
                "fp64_baseline": base, "speedup_vs_fp64": value / base["value"] if base else None,
                "wall_speedup_vs_fp64": (base["seconds"] / (t / a.steps)) if base else None,
                "gpu_launches": a.steps * n_groups * 4, "clocks": clk}
        print(json.dumps(line), flush=True)
    r.close()


def main() -> None:
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    import numpy as np
    import torch

    from mandelbulber2_b200 import abi
    from mandelbulber2_b200.render import Renderer, alloc_outputs, STATS_FIELDS

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
        dist = tdist
    torch.cuda.set_device(local)
    engines = {v: k for k, v in abi.ENGINE_NAMES.items()}
    if a.engine is None:
        a.engine = DEFAULT_ENGINE.get(a.workload, "wavefront_auto")
    if a.workload == "batch_2048":
        run_batch(a, torch, dist, world, rank, local)
        return
    engine = engines[a.engine]
    base_engine = engines[a.baseline_engine]

    sc, cam, p, desc = workload(a.workload, a.spp)
    p.seed = rank  # each rank: its own frame (jitter stream)
    r = Renderer(local)
    r.set_scene(sc)
    if a.workload == "mandelbox_1080p_B":
        # camera B: 1e-5 in front of the surface point hit by view A's centre ray
        from mandelbulber2_b200 import configs

        fa = r.render(cam, p, abi.ENGINE_PLAIN_FP64, outputs=("depth", "hit"))
        cdepth = float(fa["depth"].cpu().numpy()[(cam.height // 2) * cam.width + cam.width // 2])
        sc, cam, p = configs.mandelbox_1080p("B", centre_depth=cdepth)
        p.seed = rank
        desc["centre_depth"] = cdepth
    tuning = None
    if "wavefront" in a.engine:
        t_ = r.autotune(cam, p, engine)  # the library's own autotuner picks the launch shape
        tuning = {"block_size": t_.block_size, "ctas_per_sm": t_.ctas_per_sm, "refill_k": t_.refill_k,
                  "queue_layout": t_.queue_layout}
    n = cam.width * cam.height
    names = ("depth", "iters", "hit", "normal", "rgb8")
    bufs = alloc_outputs(n, r.device, names)
    flush = l2_flush_buffer(torch, r.device)

    clocks = ClockSampler(local, pci_bus_id(torch, local))
    clocks.start()
    t, st, ms = time_engine(r, torch, cam, p, bufs, engine, a.steps, a.warmup, flush, dist, world)
    clk = clocks.stop()
    de_total = torch.tensor([st["de_evals"], st["pixels"], st["formula_iterations"]], dtype=torch.float64,
                            device=r.device)
    if dist is not None:
        dist.all_reduce(de_total)
    de_all, pix_all, it_all = (float(x) for x in de_total.tolist())
    value = de_all / t
    fast_frame = {k: v.cpu().numpy() for k, v in bufs.items()}

    # plain FP64 kernel on the same frame, and the error of the fast frame against it
    base = None
    err = None
    if not a.no_baseline:
        bbufs = alloc_outputs(n, r.device, names)
        bsteps = max(1, min(a.steps, 3))
        bt, bst, bms = time_engine(r, torch, cam, p, bbufs, base_engine, bsteps, 1, flush, dist, world)
        btot = torch.tensor([bst["de_evals"]], dtype=torch.float64, device=r.device)
        if dist is not None:
            dist.all_reduce(btot)
        base = {"engine": a.baseline_engine, "value": float(btot.item()) / bt, "unit": UNIT,
                "ms_per_step": bt / bsteps * 1e3,
                "mpix_per_s": n * world * bsteps / bt / 1e6}
        err = compare_frames(fast_frame, {k: v.cpu().numpy() for k, v in bbufs.items()})
        del bbufs

    # end to end through the public API with host buffers: every step copies
    # its inputs (the scene, camera and parameter structs, pinned) to the device
    # and reads all outputs back to pinned host memory
    hbufs = {k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True) for k, v in bufs.items()}
    in_bytes = C.sizeof(abi.Scene) + C.sizeof(abi.Camera) + C.sizeof(abi.RenderParams)
    host_in = torch.empty(in_bytes, dtype=torch.uint8, pin_memory=True)
    C.memmove(host_in.data_ptr(), C.addressof(sc), C.sizeof(abi.Scene))
    C.memmove(host_in.data_ptr() + C.sizeof(abi.Scene), C.addressof(cam), C.sizeof(abi.Camera))
    C.memmove(host_in.data_ptr() + C.sizeof(abi.Scene) + C.sizeof(abi.Camera), C.addressof(p),
              C.sizeof(abi.RenderParams))
    dev_in = torch.empty(in_bytes, dtype=torch.uint8, device=r.device)
    stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=r.device)
    e_steps = a.steps
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e_steps):
        dev_in.copy_(host_in, non_blocking=True)
        r.set_scene(sc)
        r.render_into(cam, p, bufs, stats, engine)
        for k in bufs:
            hbufs[k].copy_(bufs[k], non_blocking=True)
        r.sync()
    torch.cuda.synchronize()
    te = time.perf_counter() - t0
    if dist is not None:
        tt = torch.tensor([te], dtype=torch.float64, device=r.device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        te = float(tt.item())
    d2h = sum(v.numel() * v.element_size() for v in bufs.values())
    e2e = {"value": de_all / a.steps * e_steps / te, "unit": UNIT, "h2d_bytes_per_step": in_bytes,
           "d2h_bytes_per_step": d2h, "ms_per_step": te / e_steps * 1e3,
           "api": "mbr_scene_set + mbr_render + D2H of depth/iters/hit/normal/rgb8 + mbr_sync"}

    # roofline: algorithmic flops of the formula iterations (per-iteration
    # counts from the op-counting oracle, profiles/opcount.json) per launch
    # over the measured launch time, against the measured FP32 FMA peak
    peak = C.c_double()
    fp64_peak = C.c_double()
    abi.load().mbr_fma_peak(0, 4096, None, C.byref(peak))
    abi.load().mbr_fma_peak(1, 1024, None, C.byref(fp64_peak))
    ops = load_json(os.path.join(ROOT, "profiles", "opcount.json")) or {}
    per_iter = ops.get(desc["formula"], {}).get("flops_per_iteration")
    launch_s = t / a.steps
    roofline = None
    # the precision the formula iteration ran in: FP64 engines, and the auto
    # engine when its policy picked FP64 for this view
    iter_fp64 = a.engine in ("plain_fp64", "plain_fp64_strict", "wavefront_fp64") or (
        a.engine == "wavefront_auto" and r.choose_precision(cam, p) == 1)
    if per_iter:
        achieved = st["formula_iterations"] / a.steps * per_iter / launch_s / 1e12
        pk = (fp64_peak if iter_fp64 else peak).value / 1e12
        traffic = load_json(os.path.join(ROOT, "profiles", "traffic.json")) or {}
        tr = traffic.get(a.engine, {}).get(a.workload)
        probe = "DFMA probe (mbr_fma_peak), FP64" if iter_fp64 else "FFMA probe (mbr_fma_peak), FP32 non-tensor"
        roofline = {"bound": "fma", "achieved": achieved, "peak": pk, "unit": "TFLOP/s", "frac": achieved / pk,
                    "traffic": tr, "peak_source": f"measured live: {probe}; MEASURED_PEAKS.json has no FMA "
                                                  "figure for non-tensor arithmetic",
                    "iteration_precision": "f64" if iter_fp64 else "f32",
                    "flops_per_iteration": per_iter, "fp32_peak": peak.value / 1e12,
                    "fp64_peak": fp64_peak.value / 1e12}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        try:
            cpu = cpu_baseline(sc, cam, p, a.cpu_seconds)
        except Exception as e:  # the baseline must not hide the GPU line
            cpu = {"error": str(e)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": t / a.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if iter_fp64 else "f32",
            "data": "synthetic (procedural fractal scene, no dataset)",
            "config": bench_config(desc, world), "engine": a.engine, "tuning": tuning,
            "mpix_per_s": pix_all / t / 1e6, "formula_iterations_per_s": it_all / t,
            "de_evals_per_frame": st["de_evals"] / a.steps, "stats_per_frame": {k: v / a.steps for k, v in st.items()},
            "fp64_baseline": base, "speedup_vs_fp64": (value / base["value"]) if base else None,
            "error_vs_fp64": err, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": a.steps * kernels_per_frame(a.engine, p), "clocks": clk, "per_step_ms": ms,
        }
        print(json.dumps(line), flush=True)
    r.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
