"""The tile image of the mixed ion kernel, restated in numpy (CPU).

Per (warp, source tile) the kernel classifies every source against the
bounding box of the warp's 32 targets (centre c, half-width h per axis) and
takes the image the centre gives it, k = rint((x_j - c) / L).  When all
reachable sources share one k and 2 (r_c + h) < L - 2 fm on every axis, the
kernel folds that k into the targets' coordinates and gives no pair its own
image (near_groups_img, disp_tile_x2).  The claim: then every pair inside
r_c gets the reference's conditional minimum image (int_ion_pure.f:147-152),
and every pair outside r_c stays outside.  Checked on random boxes, warps and
tiles, including tiles that straddle the periodic boundary.
"""
import numpy as np


def _min_image(d, L):
    d = np.where(d > L / 2, d - L, d)
    return np.where(d < -L / 2, d + L, d)


def _case(rng, L, rc, hw, tile_w):
    # 32 targets in a box of half-width <= hw somewhere in [0, L)
    c0 = rng.uniform(0, L, 3)
    tgt = np.mod(c0 + rng.uniform(-hw, hw, (32, 3)), L)
    # a tile of 128 sources: a compact region that does not wrap (as a run
    # of a space-filling curve in [0, L)^3)
    s0 = rng.uniform(0, L - tile_w, 3)
    src = s0 + rng.uniform(0, tile_w, (128, 3))
    lo, hi = tgt.min(0), tgt.max(0)
    c = 0.5 * (lo + hi)
    h = 0.5 * (hi - lo)
    # reachable: distance from the source's centre image to the box <= rc
    dm = src - c
    k = np.rint(dm / L)
    dm = dm - k * L
    gap = np.maximum(np.abs(dm) - h, 0.0)
    reach = (gap * gap).sum(1) <= rc * rc
    tile_img = np.all(2 * (rc + h) < L - 2.0)
    return tgt, src, k, reach, tile_img


def test_tile_image_is_the_minimum_image_inside_rc():
    rng = np.random.default_rng(7)
    used = 0
    for trial in range(400):
        L = np.array([rng.uniform(300, 3000)] * 3)
        rc = rng.uniform(0.1, 0.45) * L[0]
        hw = rng.uniform(5, 0.1 * L[0])
        tile_w = rng.uniform(10, 0.4 * L[0])
        tgt, src, k, reach, tile_img = _case(rng, L, rc, hw, tile_w)
        if not (tile_img and reach.any()):
            continue
        ks = k[reach]
        if not np.all(ks == ks[0]):
            continue                  # the kernel takes each pair's own image then
        used += 1
        kt = ks[0]
        raw = src[None, :, :] - tgt[:, None, :]                 # x_j - x_i, all 32 x 128 pairs
        d_ref = _min_image(raw, L)
        r_ref = np.sqrt((d_ref ** 2).sum(2))
        d_tile = raw - kt * L
        r_tile = np.sqrt((d_tile ** 2).sum(2))
        inside = r_ref <= rc
        assert np.array_equal(d_tile[inside], d_ref[inside]), trial
        assert np.all(r_tile[~inside] > rc), trial
        # a source the box test calls unreachable has no pair inside r_c
        assert not np.any(inside & ~reach[None, :]), trial
    assert used > 100
