"""Geometry of the interstitial windows, without a device.

The interstitial passes visit a box of candidate sites around each interstitial (the
window of misa-md-hip_b200/csrc/mb_device.cuh: make_window / window_site) and keep those
whose ideal site lies closer than the reach R = cutoff + skin.  Two facts the kernels and
the host-buffer step rely on are checked here by enumerating the same window with numpy:
the in-reach sites of an interstitial in box layer Z lie in layers Z - ceil(R / a0) ..
Z + ceil(R / a0) (so z-slabs of ceil(R / a0) + 1 layers keep every item's reads within
the neighbouring slabs), and their number fits the per-warp list of 256 entries at the
benchmark reach but not at 9 A (the wide-reach GPU test walks every candidate).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

A0 = 2.855
WIN_LIST = 256  # per-warp list of in-reach window sites (MB_WIN_LIST)


def window_sites(q, a0, reach):
    """Ideal positions and z layers of the in-reach candidates of make_window / window_site
    (half-lattice x index gx; odd gx are the body-centre sites, half a cell up in y and z)."""
    qx, qy, qz = q
    gx = np.arange(math.floor((qx - reach) / (0.5 * a0)), math.ceil((qx + reach) / (0.5 * a0)) + 1)
    gy = np.arange(math.floor((qy - reach) / a0) - 1, math.ceil((qy + reach) / a0) + 1)
    gz = np.arange(math.floor((qz - reach) / a0) - 1, math.ceil((qz + reach) / a0) + 1)
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    h = 0.5 * (X & 1)
    px, py, pz = 0.5 * a0 * X, a0 * (Y + h), a0 * (Z + h)
    keep = (px - qx) ** 2 + (py - qy) ** 2 + (pz - qz) ** 2 < reach * reach
    return np.stack([px[keep], py[keep], pz[keep]], axis=1), Z[keep], int(X.size)


@pytest.mark.parametrize("reach", [5.6 + 0.7, 5.6 + 1.3])
def test_in_reach_sites_stay_within_ceil_reach_layers(reach):
    rng = np.random.default_rng(5)
    span = math.ceil(reach / A0)
    lo, hi = 0, 0
    for _ in range(400):
        layer = 7
        q = rng.uniform(0.0, 10 * A0, size=3)
        q[2] = (layer + rng.uniform(0.0, 1.0)) * A0  # anywhere inside box layer 7
        _, z, _ = window_sites(q, A0, reach)
        lo, hi = min(lo, int(z.min()) - layer), max(hi, int(z.max()) - layer)
    assert -span <= lo and hi <= span  # a slab of span + 1 layers has a layer to spare
    assert hi == span  # the bound is reached (sites a little over two cells up)


@pytest.mark.parametrize("reach,fits", [(5.6 + 0.7, True), (5.6 + 1.3, True), (5.6 + 3.4, False)])
def test_in_reach_site_count_against_the_per_warp_list(reach, fits):
    rng = np.random.default_rng(9)
    counts = [window_sites(rng.uniform(0.0, 20 * A0, size=3), A0, reach)[0].shape[0] for _ in range(200)]
    sphere = 4.0 / 3.0 * math.pi * reach ** 3 * 2.0 / A0 ** 3  # two sites per cubic cell
    assert abs(np.mean(counts) - sphere) < 0.05 * sphere
    assert (max(counts) <= WIN_LIST) == fits


def test_candidates_outnumber_sites_in_reach():
    # the listed walk loads ~1 candidate in 8: the reason for listing first
    pts, _, ncand = window_sites((10.3, 11.7, 12.9), A0, 6.3)
    assert 6 < ncand / pts.shape[0] < 12
