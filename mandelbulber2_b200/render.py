"""Python host API over the C-ABI, mirroring the reference's render interface.

``Renderer`` plays the part of cRenderer/cRenderWorker for one GPU: a scene
(the fractal/hybrid node with its sFractal parameters, cf. mbr_scene) is set
once, then frames are rendered for a camera and render parameters.  Device
buffers are torch tensors (torch is the allocator and stream provider here,
nothing more); every pixel is computed by the CUDA kernels in libmbr.so.
There is no CPU path: without CUDA or without the library, construction
fails.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import abi

OUTPUT_SPECS = {
    # name: (dtype, channels)
    "depth": (torch.float64, 1),
    "iters": (torch.int32, 1),
    "hit": (torch.uint8, 1),
    "normal": (torch.float32, 3),
    "shade": (torch.float32, 1),
    "ao": (torch.float32, 1),
    "rgb": (torch.float32, 3),
    "rgb8": (torch.uint8, 3),
}
STATS_FIELDS = [f for f, _ in abi.Stats._fields_]


class MbrError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def check(lib, ctx, status: int) -> None:
    if status != abi.MBR_OK:
        msg = lib.mbr_last_error_string(ctx).decode() if ctx else ""
        raise MbrError(status, msg)


@dataclass
class Frame:
    """Device outputs of one render plus the launch counters."""

    buffers: dict
    stats: dict
    width: int
    height: int

    def __getitem__(self, k):
        return self.buffers[k]


def alloc_outputs(n_pixels: int, device, names) -> dict:
    out = {}
    for n in names:
        dt, ch = OUTPUT_SPECS[n]
        shape = (n_pixels,) if ch == 1 else (n_pixels, ch)
        out[n] = torch.empty(shape, dtype=dt, device=device)
    return out


def outputs_struct(bufs: dict, stats_tensor) -> abi.Outputs:
    o = abi.Outputs()
    for n in OUTPUT_SPECS:
        setattr(o, n, bufs[n].data_ptr() if n in bufs and bufs[n] is not None else None)
    o.stats = stats_tensor.data_ptr() if stats_tensor is not None else None
    return o


def stats_dict(t: torch.Tensor) -> dict:
    v = t.cpu().tolist()
    return {k: int(x) & 0xFFFFFFFFFFFFFFFF for k, x in zip(STATS_FIELDS, v)}


class Renderer:
    """One rendering context on one GPU (mbr_ctx)."""

    def __init__(self, device: int = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA is not available: the renderer has no CPU path")
        self.lib = abi.load()
        self.device = torch.device("cuda", device)
        ctx = C.c_void_p()
        st = self.lib.mbr_create(C.byref(ctx), device)
        if st != abi.MBR_OK:
            raise MbrError(st, "mbr_create failed")
        self.ctx = ctx
        self.scene = None

    def close(self) -> None:
        if self.ctx:
            self.lib.mbr_destroy(self.ctx)
            self.ctx = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        check(self.lib, self.ctx, st)

    def set_scene(self, scene: abi.Scene) -> None:
        self._check(self.lib.mbr_scene_set(self.ctx, C.byref(scene)))
        self.scene = scene

    def render_into(self, camera: abi.Camera, params: abi.RenderParams, bufs: dict, stats: torch.Tensor | None,
                    engine: int, stream: torch.cuda.Stream | None = None) -> None:
        """Queues one frame into caller-provided device buffers (asynchronous)."""
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        o = outputs_struct(bufs, stats)
        self._check(self.lib.mbr_render(self.ctx, C.byref(camera), C.byref(params), C.byref(o), engine,
                                        C.c_void_p(s.cuda_stream)))

    def render(self, camera: abi.Camera, params: abi.RenderParams, engine: int = abi.ENGINE_PLAIN_FP64,
               outputs=("depth", "iters", "hit", "normal", "shade", "ao", "rgb", "rgb8")) -> Frame:
        n = camera.width * camera.height
        bufs = alloc_outputs(n, self.device, outputs)
        stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=self.device)
        self.render_into(camera, params, bufs, stats, engine)
        self.sync()
        return Frame(bufs, stats_dict(stats), camera.width, camera.height)

    def sync(self, stream: torch.cuda.Stream | None = None) -> None:
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        self._check(self.lib.mbr_sync(self.ctx, C.c_void_p(s.cuda_stream)))

    def distance(self, points: torch.Tensor, detail: float, normal_mode: bool = False,
                 engine: int = abi.ENGINE_PLAIN_FP64):
        """CalculateDistance at points (N x 3 float64 CUDA tensor)."""
        pts = points.to(device=self.device, dtype=torch.float64).contiguous()
        n = pts.shape[0]
        dist = torch.empty(n, dtype=torch.float64, device=self.device)
        iters = torch.empty(n, dtype=torch.int32, device=self.device)
        s = torch.cuda.current_stream(self.device)
        self._check(self.lib.mbr_distance(self.ctx, C.c_void_p(pts.data_ptr()), n, detail, int(normal_mode),
                                          C.c_void_p(dist.data_ptr()), C.c_void_p(iters.data_ptr()), engine,
                                          C.c_void_p(s.cuda_stream)))
        self.sync()
        return dist, iters

    def choose_precision(self, camera: abi.Camera, params: abi.RenderParams) -> int:
        """1 when MBR_ENGINE_WAVEFRONT_AUTO iterates this view in FP64, else 0."""
        flag = C.c_int32(0)
        self._check(self.lib.mbr_choose_precision(self.ctx, C.byref(camera), C.byref(params), C.byref(flag)))
        return int(flag.value)

    def set_tuning(self, block_size: int, ctas_per_sm: int, refill_k: int, queue_layout: int) -> None:
        t = abi.Tuning(block_size, ctas_per_sm, refill_k, queue_layout)
        self._check(self.lib.mbr_set_tuning(self.ctx, C.byref(t)))

    def get_tuning(self) -> abi.Tuning:
        t = abi.Tuning()
        self._check(self.lib.mbr_get_tuning(self.ctx, C.byref(t)))
        return t

    def autotune(self, camera: abi.Camera, params: abi.RenderParams, engine: int = abi.ENGINE_WAVEFRONT_FP32):
        n = camera.width * camera.height
        bufs = alloc_outputs(n, self.device, ("depth", "iters", "hit", "normal", "rgb"))
        stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=self.device)
        o = outputs_struct(bufs, stats)
        t = abi.Tuning()
        s = torch.cuda.current_stream(self.device)
        self._check(self.lib.mbr_autotune(self.ctx, C.byref(camera), C.byref(params), C.byref(o), engine,
                                          C.c_void_p(s.cuda_stream), C.byref(t)))
        return t

    def adjoint(self, camera: abi.Camera, params: abi.RenderParams, depth: torch.Tensor, hit: torch.Tensor,
                dl_ddepth: torch.Tensor | None, dl_dshade: torch.Tensor | None,
                engine: int = abi.ENGINE_PLAIN_FP64) -> torch.Tensor:
        grad = torch.zeros(abi.GRAD_COUNT, dtype=torch.float64, device=self.device)
        s = torch.cuda.current_stream(self.device)
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
        self._check(self.lib.mbr_adjoint(self.ctx, C.byref(camera), C.byref(params), ptr(depth), ptr(hit),
                                         ptr(dl_ddepth), ptr(dl_dshade), ptr(grad), engine,
                                         C.c_void_p(s.cuda_stream)))
        self.sync()
        return grad


def camera_rotation(camera: abi.Camera):
    """(mRot row-major 3x3 as a list of 9, [yaw, pitch, roll]) from the library's host set-up."""
    m = (C.c_double * 9)()
    a = (C.c_double * 3)()
    st = abi.load().mbr_camera_rotation(C.byref(camera), m, a)
    if st != abi.MBR_OK:
        raise MbrError(st, "mbr_camera_rotation")
    return list(m), list(a)


def scene_sequence(scene: abi.Scene):
    """(sequence table, length, DE function, per-slot bailout) from the library's host builder."""
    seq = (C.c_int32 * abi.MBR_SEQUENCE_LENGTH)()
    length, fn = C.c_int32(), C.c_int32()
    bail = (C.c_double * abi.MBR_MAX_FRACTALS)()
    st = abi.load().mbr_scene_sequence(C.byref(scene), seq, C.byref(length), C.byref(fn), bail)
    if st != abi.MBR_OK:
        raise MbrError(st, "mbr_scene_sequence")
    return list(seq)[: length.value], length.value, fn.value, list(bail)
