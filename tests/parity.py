"""Comparison metrics between a GPU frame and the oracle frame."""
import numpy as np


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    mse = float(np.mean((a - b) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(255.0 ** 2 / mse)


def compare(gpu: dict, ora: dict) -> dict:
    """Hit/iteration agreement, depth relative error on common hits, 8-bit PSNR, normal angle."""
    hg, ho = gpu["hit"].astype(bool), ora["hit"].astype(bool)
    n = hg.size
    both = hg & ho
    out = {"pixels": n, "hit_frac": float(ho.mean()), "hit_mismatch": float((hg != ho).mean())}
    if "iters" in gpu and "iters" in ora:
        out["iters_match"] = float((gpu["iters"] == ora["iters"]).mean())
        out["hit_iters_match"] = float(((gpu["iters"] == ora["iters"]) & (hg == ho)).mean())
    if both.any():
        dg, do = gpu["depth"][both], ora["depth"][both]
        rel = np.abs(dg - do) / np.abs(do)
        out["depth_rel_max"] = float(rel.max())
        out["depth_rel_median"] = float(np.median(rel))
        out["depth_rel_p99"] = float(np.quantile(rel, 0.99))
        out["depth_rel_le_1e-9"] = float((rel <= 1e-9).mean())
        out["depth_rel_le_1e-4"] = float((rel <= 1e-4).mean())
        if "normal" in gpu and "normal" in ora and np.abs(ora["normal"][both]).sum() > 0:
            ng, no = gpu["normal"][both].astype(np.float64), ora["normal"][both].astype(np.float64)
            cos = np.clip((ng * no).sum(1) / np.maximum(np.linalg.norm(ng, axis=1) * np.linalg.norm(no, axis=1), 1e-30),
                          -1, 1)
            ang = np.degrees(np.arccos(cos))
            out["normal_deg_median"] = float(np.median(ang))
            out["normal_deg_p99"] = float(np.quantile(ang, 0.99))
    if "rgb8" in gpu and "rgb8" in ora:
        out["psnr"] = psnr(gpu["rgb8"], ora["rgb8"])
    return out
