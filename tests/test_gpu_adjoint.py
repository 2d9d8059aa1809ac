"""The adjoint kernel (through the C-ABI) against FP64 central differences of
the oracle's loss and against the oracle's forward-mode dual-number gradient.

Bar: gradients within 1e-3 relative of the FP64 finite differences; the FP64
adjoint equal to the dual-number reference within 1e-6 relative (same
mathematics, same FP64 precision).  The forward render for the adjoint is the
FP32 march with FP64 root refinement (MBR_ENGINE_PLAIN_MIXED, refine = root),
whose depth agrees with the FP64 oracle's to 1e-9 relative.
"""
import numpy as np
import pytest
import torch

from mandelbulber2_b200 import abi, configs

from .adjoint_check import PARAMS, fd_check

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["mandelbulb", "mandelbox"])
def test_adjoint_matches_finite_differences_and_dual_numbers(renderer, oracle, kind):
    sc, cam, p = configs.adjoint_256(kind, 64, 64)
    mask, wt, ws, t0, hit0, fd = fd_check(oracle, sc, cam, p, kind)
    assert mask.sum() > 200
    renderer.set_scene(sc)
    # FP32-march forward with FP64 root refinement: depth close to the FP64 oracle's
    fr = renderer.render(cam, p, abi.ENGINE_PLAIN_MIXED, outputs=("depth", "hit"))
    gdepth, ghit = fr["depth"].cpu().numpy(), fr["hit"].cpu().numpy().astype(bool)
    both = ghit & hit0
    rel = np.abs(gdepth[both] - t0[both]) / t0[both]
    assert np.quantile(rel, 0.99) <= 1e-9, np.quantile(rel, 0.99)
    dev = renderer.device
    depth = torch.from_numpy(t0).to(dev)
    hit = torch.from_numpy(hit0.astype(np.uint8)).to(dev)
    dlt = torch.from_numpy(wt.astype(np.float32)).to(dev)
    dls = torch.from_numpy(ws.astype(np.float32)).to(dev)
    g64 = renderer.adjoint(cam, p, depth, hit, dlt, dls, abi.ENGINE_PLAIN_FP64).cpu().numpy()
    g32 = renderer.adjoint(cam, p, depth, hit, dlt, dls, abi.ENGINE_PLAIN_MIXED).cpu().numpy()
    # dual-number reference with the same (float32-rounded) weights
    dt, ds, _ = oracle.pixel_gradients(sc, cam, p, t0, hit0.astype(np.uint8))
    gref = (wt.astype(np.float32).astype(np.float64)[:, None] * dt).sum(0) + \
           (ws.astype(np.float32).astype(np.float64)[:, None] * ds).sum(0)
    ks = PARAMS[kind]
    scale = max(abs(fd[k]) for k in ks)
    for k in ks:
        print(kind, k, "fd", fd[k], "adjoint64", g64[k], "adjoint32", g32[k], "dual", gref[k])
        assert abs(g64[k] - gref[k]) <= 1e-6 * max(abs(gref[k]), 1e-3 * scale), k
        assert abs(g64[k] - fd[k]) <= 1e-3 * max(abs(fd[k]), 1e-2 * scale), k
        assert abs(g32[k] - g64[k]) <= 2e-2 * max(abs(g64[k]), 1e-2 * scale), k


def test_adjoint_rejects_unsupported(renderer):
    from mandelbulber2_b200.render import MbrError

    sc, cam, p = configs.adjoint_256("mandelbulb", 16, 16)
    renderer.set_scene(sc)
    z = torch.zeros(256, dtype=torch.float64, device=renderer.device)
    h = torch.zeros(256, dtype=torch.uint8, device=renderer.device)
    cam.use_angles = 0
    with pytest.raises(MbrError):
        renderer.adjoint(cam, p, z, h, None, None)
    cam.use_angles = 1
    renderer.set_scene(configs.menger_scene())
    with pytest.raises(MbrError):
        renderer.adjoint(cam, p, z, h, None, None)
