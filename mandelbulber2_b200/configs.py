"""Named workloads: scene, camera and render parameters of the benchmark and
parity configurations, in the reference's parameter vocabulary.

  mandelbulb_512   Mandelbulb p=8, 512x512, Lambert + hard shadow
  mandelbox_1080p  Mandelbox s=-1.5, 1920x1080, camera A (wide) or B (deep zoom), 16 AO rays
  batch_jobs       render jobs of uneven size (multi-job persistent launch)
  adjoint_256      256x256 Mandelbulb / Mandelbox depth + Lambert renders for the adjoint
  hybrid_gi_2160p  Mandelbulb(1-3) + Menger(4-12) hybrid, 3840x2160 Monte Carlo GI
"""
from __future__ import annotations

import math

import numpy as np

from . import abi

SUN = (1.0, -1.0, 1.0)


def mandelbulb_scene(power: float = 8.0, maxiter: int = 250) -> abi.Scene:
    s = abi.scene_defaults(abi.FORMULA_MANDELBULB)
    s.formula_maxiter = maxiter
    s.fractal[0].bulb_power = power
    return s


def mandelbox_scene(scale: float = -1.5, min_radius: float = 0.5, maxiter: int = 50) -> abi.Scene:
    s = abi.scene_defaults(abi.FORMULA_MANDELBOX)
    s.formula_maxiter = maxiter
    f = s.fractal[0]
    f.mandelbox_scale = scale
    f.mandelbox_folding_limit = 1.0
    f.mandelbox_folding_value = 2.0
    f.mandelbox_folding_min_radius = min_radius
    f.mandelbox_folding_fixed_radius = 1.0
    return s


def menger_scene(maxiter: int = 12) -> abi.Scene:
    s = abi.scene_defaults(abi.FORMULA_MENGER_SPONGE)
    s.formula_maxiter = maxiter
    return s


def hybrid_scene() -> abi.Scene:
    """Hybrid node: Mandelbulb p=8 for 3 iterations, then Menger sponge (scale 3) for 9; 12 iterations."""
    s = abi.scene_defaults(abi.FORMULA_MANDELBULB)
    s.hybrid_fractal_enable = 1
    s.n_fractals = 2
    s.formula_maxiter = 12
    s.fractal[0].bulb_power = 8.0
    s.fractal[0].formula_iterations = 3
    abi.fractal_defaults(s.fractal[1], abi.FORMULA_MENGER_SPONGE)
    s.fractal[1].formula_iterations = 9
    s.fractal[1].transf_scale3 = 3.0
    return s


def camera(pos, target=(0.0, 0.0, 0.0), fov=53.0, width=512, height=512, top=(0.0, 0.0, 1.0)) -> abi.Camera:
    c = abi.camera_defaults()
    c.camera[:] = list(pos)
    c.target[:] = list(target)
    c.top[:] = list(top)
    c.fov_deg = fov
    c.width = width
    c.height = height
    c.use_angles = 0
    return c


def base_params(binary_steps: int = 5, view_distance_max: float = 20.0) -> abi.RenderParams:
    p = abi.params_defaults()
    p.detail_level = 1.0
    p.de_factor = 1.0
    p.max_raymarching_steps = 10000
    p.binary_steps = binary_steps
    p.view_distance_max = view_distance_max
    p.smoothness = 1.0
    p.jitter = 1
    p.seed = 0
    p.shading_enable = 1
    p.shadow_enable = 1
    # the benchmark configurations use a hard, non-penetrating shadow
    # (the library's defaults are the reference's: a 1 degree soft cone, penetrating)
    p.soft_shadow_cone = 0.0
    p.penetrating = 0
    p.light_direction[:] = list(SUN)
    p.light_intensity = 1.0
    p.material_shading = 1.0
    p.albedo = 1.0
    p.ambient_intensity = 0.0
    p.ao_rays = 0
    return p


def mandelbulb_512(width: int = 512, height: int = 512, binary_steps: int = 5):
    """Plain FP64 Mandelbulb: p=8, N=250, bailout 10, camera (0,-3,0) -> 0, FOV 53,
    detail 1, <=10000 steps, 5 binary steps, miss at t>20, Lambert + hard shadow."""
    return (mandelbulb_scene(8.0, 250), camera((0.0, -3.0, 0.0), width=width, height=height),
            base_params(binary_steps, 20.0))


def mandelbox_1080p(view: str = "A", width: int = 1920, height: int = 1080, ao_rays: int = 16,
                    centre_depth: float | None = None, camera_rotation=None):
    """Mandelbox s=-1.5, limit 1, min r 0.5 (mR2 0.25), fixed r 1, N=50, bailout 100, r/|dr|.

    View A: camera (0,-6,0) aimed at the origin, FOV 53.  View B: camera 1e-5 in
    front of the surface point that view A's centre ray hits (`centre_depth`
    along that ray), same direction, FOV 0.5.  AO: 16 cosine rays from PCG32
    (state 1234, stream = pixel).  `camera_rotation(camera) -> (mRot, angles)`
    places the centre ray (default: the library's mbr_camera_rotation).
    """
    sc = mandelbox_scene(-1.5, 0.5, 50)
    p = base_params(5, 20.0)
    p.ao_rays = ao_rays
    p.ao_seed = 1234
    p.light_intensity = 0.6
    p.ambient_intensity = 0.4
    cam_a = camera((0.0, -6.0, 0.0), fov=53.0, width=width, height=height)
    if view == "A":
        return sc, cam_a, p
    if centre_depth is None:
        raise ValueError("view B needs the depth of view A's centre ray")
    d = centre_ray(cam_a, camera_rotation)
    hit = np.array(cam_a.camera[:]) + d * centre_depth
    pos = hit - d * 1e-5
    cam_b = camera(tuple(pos), target=tuple(hit + d), fov=0.5, width=width, height=height)
    return sc, cam_b, p


def centre_ray(cam: abi.Camera, camera_rotation=None) -> np.ndarray:
    """Unit direction of the ray through the image centre (pixel W/2, H/2)."""
    if camera_rotation is None:
        from .render import camera_rotation

    m, _ = camera_rotation(cam)
    fov = 2.0 * math.tan(cam.fov_deg / 360.0 * math.pi)
    ix = ((1.0 / cam.width) * (cam.width // 2) - 0.5) * (cam.width / cam.height)
    iy = (-1.0 / cam.height) * (cam.height // 2) + 0.5
    v = np.array([ix * fov, 1.0, iy * fov])
    v = v / np.linalg.norm(v)
    M = np.array(m).reshape(3, 3)
    d = M @ v
    return d / np.linalg.norm(d)


def hybrid_gi_2160p(width: int = 3840, height: int = 2160, spp: int = 16):
    """Hybrid Mandelbulb(1-3)/Menger(4-12); GI 16 spp, 4 bounces, albedo 0.7, sky 0.3,
    sun 3 along normalize(1,-1,1), thin lens aperture 0.02 focus 3."""
    sc = hybrid_scene()
    cam = camera((0.0, -3.0, 0.0), fov=53.0, width=width, height=height)
    p = base_params(5, 20.0)
    p.jitter = 0
    p.gi_samples = spp
    p.gi_bounces = 4
    p.albedo = 0.7
    p.gi_sky = 0.3
    p.gi_sun = 3.0
    p.dof_aperture = 0.02
    p.dof_focus = 3.0
    p.gi_seed = 0
    return sc, cam, p


def batch_jobs(n_jobs: int = 2048, seed: int = 7, sizes=(64, 128, 256, 512, 1024)):
    """Uneven render jobs: resolution from `sizes`^2, camera on a sphere of radius
    U[2.5, 4] aimed at the origin, Mandelbulb (p U[2,12], N=100) or Mandelbox
    (scale U[-2.5,-1.5] or U[1.5,3], min r^2 U[0.1,0.5], N=40), 50/50.

    Returns (scenes, cameras, pixel_offsets, total_pixels)."""
    rng = np.random.default_rng(seed)
    scenes, cams, offsets = [], [], []
    off = 0
    for _ in range(n_jobs):
        res = int(rng.choice(sizes))
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        radius = rng.uniform(2.5, 4.0)
        pos = u * radius
        top = (0.0, 0.0, 1.0) if abs(u[2]) < 0.95 else (0.0, 1.0, 0.0)
        if rng.uniform() < 0.5:
            sc = mandelbulb_scene(float(rng.uniform(2.0, 12.0)), 100)
        else:
            scale = float(rng.uniform(-2.5, -1.5)) if rng.uniform() < 0.5 else float(rng.uniform(1.5, 3.0))
            mr2 = float(rng.uniform(0.1, 0.5))
            sc = mandelbox_scene(scale, math.sqrt(mr2), 40)
        scenes.append(sc)
        cams.append(camera(tuple(pos), fov=53.0, width=res, height=res, top=top))
        offsets.append(off)
        off += res * res
    return scenes, cams, offsets, off


def adjoint_256(kind: str = "mandelbulb", width: int = 256, height: int = 256):
    """Depth + Lambert render for the adjoint: camera given by position and
    yaw/pitch/roll, refine = root so that depth is smooth in the parameters."""
    if kind == "mandelbulb":
        sc = mandelbulb_scene(8.0, 250)
        pos = (0.0, -3.0, 0.0)
    else:
        sc = mandelbox_scene(-1.5, 0.5, 50)
        pos = (0.0, -6.0, 0.0)
    cam = camera(pos, fov=53.0, width=width, height=height)
    cam.use_angles = 1
    cam.angles[:] = [0.0, 0.0, 0.0]
    p = base_params(60, 20.0)
    p.refine = abi.REFINE_ROOT
    p.jitter = 0
    p.shadow_enable = 0
    return sc, cam, p
