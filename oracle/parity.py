"""Comparison of one movie's alignment with the FP64 oracle's.

TEST INFRASTRUCTURE ONLY (imported by tests/ and by bench.py's CPU-checker
leg, never by the product).  The bars are the path's correctness contract:

  * pair list identical (OD_SetEquation_All order, mfunc.h:64-84);
  * integer box peaks identical, except near-ties: the oracle's own CC
    values at the two positions agree within 1e-5 relative (FP32 transforms
    cannot order them); that pair's shift then within 2/32 px;
  * pair shifts on the same 1/32-px grid point, except near-ties: the
    oracle's own upsampled map (FindShift, cufunc.cu:428-481) differs by
    <= 1e-5 relative between the two neighbouring grid points;
  * per-frame shifts within 0.01 px of the oracle;
  * summed image within 1e-5 relative L2 of the oracle.
"""
from __future__ import annotations

import numpy as np

from . import mc_oracle as O

SHIFT_TOL = 0.01
IMAGE_RTOL = 1e-5
TIE_RTOL = 1e-5


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def grid_near_tie(box_map: np.ndarray, nps: int, so, sg) -> bool:
    """The two pair shifts are neighbouring 1/32 grid points at which the
    oracle's upsampled sub-box is flat to TIE_RTOL."""
    if max(abs(so[0] - sg[0]), abs(so[1] - sg[1])) > 1.5 / 32:
        return False
    box = box_map.shape[0]
    ix, iy = O.integer_peak(box_map, nps)
    offx = min(max(ix - 8, 0), box - 16)
    offy = min(max(iy - 8, 0), box - 16)
    f = O.upsampled_subbox(box_map, offx, offy)

    def val(sx, sy):
        X = int(round((sx + box // 2 - offx) * 32))
        Y = int(round((sy + box // 2 - offy) * 32))
        return f[Y % 512, X % 512]
    a, b = val(*so), val(*sg)
    return abs(a - b) <= TIE_RTOL * abs(a)


def compare_alignment(g: dict, ref, nps: int = 0) -> dict:
    """Metrics of a GPU run ``g`` (keys pairs, peak, shift, frame_shifts and
    optionally kept, image) against oracle Result ``ref`` (run with
    keep_boxes=True for the near-tie rules).  ``violations`` lists every
    departure from the bars above that no near-tie explains."""
    out = {"pairs": len(ref.pairs), "violations": []}
    v = out["violations"]
    pl = np.array(ref.pairs, dtype=np.int64).reshape(-1, 2)
    out["pair_list_equal"] = bool(np.array_equal(np.asarray(g["pairs"], dtype=np.int64).reshape(-1, 2), pl))
    if not out["pair_list_equal"]:
        v.append("pair list differs")
    so = np.stack([ref.pair_shift.real, ref.pair_shift.imag], 1)
    sg = np.asarray(g["shift"], dtype=np.float64)
    pk = np.asarray(g["peak"])
    peak_flip = np.nonzero(np.any(pk != ref.pair_peak, axis=1))[0]
    out["peak_flips"] = int(len(peak_flip))
    for r in peak_flip:
        if ref.boxes is None:
            v.append(f"pair {r}: peak {pk[r]} vs {ref.pair_peak[r]} (no oracle windows to check a tie)")
            continue
        (gx, gy), (ox, oy) = pk[r], ref.pair_peak[r]
        vo, vg = ref.boxes[r][oy, ox], ref.boxes[r][gy, gx]
        if abs(vo - vg) > TIE_RTOL * abs(vo):
            v.append(f"pair {r}: peak {pk[r].tolist()} vs {ref.pair_peak[r].tolist()}, CC {vg:.6g} vs {vo:.6g}")
        elif np.max(np.abs(so[r] - sg[r])) > 2.0 / 32 + 1e-9:
            v.append(f"pair {r}: tie peak but shift {sg[r].tolist()} vs {so[r].tolist()}")
    grid = [r for r in np.nonzero(np.any(so != sg, axis=1))[0] if r not in set(peak_flip)]
    out["grid_flips"] = int(len(grid))
    for r in grid:
        if ref.boxes is None or not grid_near_tie(ref.boxes[r], nps, so[r], sg[r]):
            v.append(f"pair {r}: shift {sg[r].tolist()} vs {so[r].tolist()}")
    out["max_pair_shift_diff_px"] = float(np.max(np.abs(so - sg))) if len(so) else 0.0
    if "kept" in g and g["kept"] is not None:
        out["kept_equal"] = [int(x) for x in g["kept"]] == [int(x) for x in ref.goodlist]
    fo = np.stack([ref.frame_shift.real, ref.frame_shift.imag], 1)
    fg = np.asarray(g["frame_shifts"], dtype=np.float64)
    d = fg - fo
    out["shift_max_diff_px"] = float(np.max(np.abs(d)))
    out["shift_rmse_vs_oracle_px"] = float(np.sqrt(np.mean(np.sum(d * d, axis=1))))
    if out["shift_max_diff_px"] > SHIFT_TOL:
        v.append(f"frame shifts differ by {out['shift_max_diff_px']:.4g} px")
    if g.get("image") is not None and ref.image is not None:
        out["sum_rel_l2_vs_oracle"] = rel_l2(g["image"], ref.image)
        if out["sum_rel_l2_vs_oracle"] > IMAGE_RTOL:
            v.append(f"sum relative L2 {out['sum_rel_l2_vs_oracle']:.3g}")
    return out
