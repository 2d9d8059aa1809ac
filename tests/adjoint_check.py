"""Loss, finite-difference and dual-number references for the adjoint tests.

The loss of a depth + Lambert render against a target rendered with every
differentiated parameter perturbed by 1 %:
    L(θ) = Σ_M (t(θ) - t*)² + (s(θ) - s*)²
over a fixed pixel mask M (pixels hit in every render of the check, with
smooth depth and shade in every parameter - no jump of the distance estimate
between θ-h and θ+h - and away from the Lambert kink).  t comes from the FP64 oracle
render with root refinement, s = max(N·L, 0) from the oracle's FP64
central-difference normal at that depth.
"""
import math

import numpy as np

from mandelbulber2_b200 import abi

PARAMS = {
    "mandelbulb": [abi.GRAD_BULB_POWER, abi.GRAD_CAMERA_X, abi.GRAD_CAMERA_Y, abi.GRAD_CAMERA_Z, abi.GRAD_YAW],
    "mandelbox": [abi.GRAD_MANDELBOX_SCALE, abi.GRAD_MANDELBOX_MIN_R2, abi.GRAD_CAMERA_X, abi.GRAD_CAMERA_Y,
                  abi.GRAD_CAMERA_Z, abi.GRAD_YAW],
}


def get(sc, cam, k):
    if k == abi.GRAD_BULB_POWER:
        return sc.fractal[0].bulb_power
    if k == abi.GRAD_MANDELBOX_SCALE:
        return sc.fractal[0].mandelbox_scale
    if k == abi.GRAD_MANDELBOX_MIN_R2:
        return sc.fractal[0].mandelbox_folding_min_radius ** 2
    if k in (abi.GRAD_CAMERA_X, abi.GRAD_CAMERA_Y, abi.GRAD_CAMERA_Z):
        return cam.camera[k - abi.GRAD_CAMERA_X]
    return cam.angles[0]


def put(sc, cam, k, v):
    if k == abi.GRAD_BULB_POWER:
        sc.fractal[0].bulb_power = v
    elif k == abi.GRAD_MANDELBOX_SCALE:
        sc.fractal[0].mandelbox_scale = v
    elif k == abi.GRAD_MANDELBOX_MIN_R2:
        sc.fractal[0].mandelbox_folding_min_radius = math.sqrt(v)
    elif k in (abi.GRAD_CAMERA_X, abi.GRAD_CAMERA_Y, abi.GRAD_CAMERA_Z):
        cam.camera[k - abi.GRAD_CAMERA_X] = v
    else:
        cam.angles[0] = v


def copy(sc, cam):
    s2, c2 = abi.Scene(), abi.Camera()
    import ctypes as C

    C.memmove(C.addressof(s2), C.addressof(sc), C.sizeof(sc))
    C.memmove(C.addressof(c2), C.addressof(cam), C.sizeof(cam))
    return s2, c2


def depth_shade(oracle, sc, cam, p):
    """FP64 depth (root refinement) and FP64 Lambert term per pixel."""
    b, _ = oracle.render(sc, cam, p, outputs=("depth", "hit"))
    _, _, s = oracle.pixel_gradients(sc, cam, p, b["depth"], b["hit"])
    return b["depth"], b["hit"].astype(bool), s


def perturbed(sc, cam, kind, rel=0.01):
    s2, c2 = copy(sc, cam)
    for k in PARAMS[kind]:
        v = get(s2, c2, k)
        put(s2, c2, k, v * (1.0 + rel) if v != 0.0 else rel)
    return s2, c2


def root_ok(oracle, sc, cam, p, t0, hit0, tol=1e-6):
    """|dist(p(t)) - thr(t)| <= tol * thr at the stored depth of each hit pixel."""
    W, H = cam.width, cam.height
    ok = np.zeros(W * H, dtype=bool)
    idx = np.nonzero(hit0)[0]
    if len(idx) == 0:
        return ok
    dirs = np.array([oracle.view(cam, int(i % W), int(i // W)) for i in idx])
    pts = np.array(cam.camera[:])[None, :] + dirs * t0[idx, None]
    fov = 2.0 * math.tan(cam.fov_deg / 360.0 * math.pi)
    thr = np.linalg.norm(pts - np.array(cam.camera[:])[None, :], axis=1) * (1.0 / H) * fov / p.detail_level
    d = np.array([oracle.distance(sc, pts[j:j + 1], thr[j])[0][0] for j in range(len(idx))])
    ok[idx] = np.abs(d - thr) <= tol * thr
    return ok


def fd_check(oracle, sc, cam, p, kind, h=1e-5):
    """Returns (mask, weights dL/dt, dL/ds at θ, depth at θ, hit at θ, fd gradient dict)."""
    ts, tc = perturbed(sc, cam, kind)
    tt, thit, tsh = depth_shade(oracle, ts, tc, p)
    t0, hit0, s0 = depth_shade(oracle, sc, cam, p)
    mask = hit0 & thit & (s0 > 1e-3) & (tsh > 0.0)
    plus, minus = {}, {}
    for k in PARAMS[kind]:
        v = get(sc, cam, k)
        for sign, store in ((1.0, plus), (-1.0, minus)):
            s2, c2 = copy(sc, cam)
            put(s2, c2, k, v + sign * h)
            store[k] = depth_shade(oracle, s2, c2, p)
            mask &= store[k][1] & (store[k][2] > 0.0)
        # a smooth pixel has a second difference of O(h^2); a jump of the
        # distance estimate (an orbit's bailout iteration changing between
        # θ-h and θ+h, which makes r/|dr| discontinuous) does not
        d2t = np.abs(plus[k][0] - 2.0 * t0 + minus[k][0])
        d2s = np.abs(plus[k][2] - 2.0 * s0 + minus[k][2])
        mask &= (d2t <= 1e-9 * np.maximum(t0, 1.0)) & (d2s <= 1e-7)
    # pixels whose depth is a root of F = dist - thr (not a jump of the estimate)
    mask &= root_ok(oracle, sc, cam, p, t0, hit0)
    wt = np.where(mask, 2.0 * (t0 - tt), 0.0)
    ws = np.where(mask, 2.0 * (s0 - tsh), 0.0)

    def loss(t, s):
        return float(np.sum(np.where(mask, (t - tt) ** 2 + (s - tsh) ** 2, 0.0)))

    fd = {k: (loss(plus[k][0], plus[k][2]) - loss(minus[k][0], minus[k][2])) / (2 * h) for k in PARAMS[kind]}
    return mask, wt, ws, t0, hit0, fd
