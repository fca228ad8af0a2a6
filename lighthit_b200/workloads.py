"""Seeded synthetic inputs with the shapes of the LightHit workloads.

No public dataset is involved: the workloads are the reference's synthetic
Baikal-like array (``examples/synthetic.py:12-54``) with sources drawn from
stated distributions. These generators restate those draws so that the same
inputs exist on a machine without the reference.
"""
from __future__ import annotations

import numpy as np

__all__ = ["baikal_like_positions", "flash_positions", "flash_batch_sizes"]


def baikal_like_positions(clusters=1, strings=8, modules=6, cluster_pitch_m=180.0,
                          string_radius_m=25.0, vertical_spacing_m=15.0):
    """OM centres of the synthetic array (``examples/synthetic.py:20-35``).

    Clusters along +x every ``cluster_pitch_m``; strings on a circle of
    ``string_radius_m``; modules spaced ``vertical_spacing_m`` about z = 0.
    OMs look down (orientation -z).
    """
    centres = np.zeros((clusters, 3))
    centres[:, 0] = np.arange(clusters) * cluster_pitch_m
    azimuth = np.arange(strings) * 2 * np.pi / strings
    ring = np.column_stack((string_radius_m * np.cos(azimuth),
                            string_radius_m * np.sin(azimuth), np.zeros(strings)))
    heights = (np.arange(modules) - (modules - 1) / 2) * vertical_spacing_m
    column = np.column_stack((np.zeros(modules), np.zeros(modules), heights))
    positions = (centres[:, None, None, :] + ring[None, :, None, :]
                 + column[None, None, :, :]).reshape(-1, 3)
    orientations = np.tile([0.0, 0.0, -1.0], (len(positions), 1))
    return positions, orientations


def flash_positions(count, centre, *, seed=11, radius_m=60.0, height_m=300.0,
                    om_positions=None, min_distance_m=2.0):
    """Flash positions uniform in a vertical cylinder around ``centre``.

    Draw order from one ``default_rng(seed)``: ``r = radius*sqrt(U)`` for all
    flashes, then ``phi = U(0, 2 pi)``, then ``z = U(-h/2, h/2)``. When
    ``om_positions`` is given, flashes closer than ``min_distance_m`` to any OM
    (inside the table's inner radius, where the reference raises) are drawn
    again from the same stream.
    """
    rng = np.random.default_rng(seed)
    centre = np.asarray(centre, float)

    def draw(n):
        r = radius_m * np.sqrt(rng.uniform(size=n))
        phi = rng.uniform(0.0, 2 * np.pi, n)
        z = rng.uniform(-height_m / 2, height_m / 2, n)
        return centre + np.column_stack((r * np.cos(phi), r * np.sin(phi), z))

    out = draw(int(count))
    if om_positions is not None:
        oms = np.asarray(om_positions, float)
        for _ in range(100):
            d = np.linalg.norm(out[:, None, :] - oms[None, :, :], axis=2).min(axis=1)
            bad = np.flatnonzero(d < min_distance_m)
            if not len(bad):
                break
            out[bad] = draw(len(bad))
    return out


def flash_batch_sizes(total, *, seed=12, low=1, high=256):
    """Uneven served batch sizes in ``[low, high]`` that add up to ``total``."""
    rng = np.random.default_rng(seed)
    sizes = []
    left = int(total)
    while left > 0:
        size = int(min(left, rng.integers(low, high + 1)))
        sizes.append(size)
        left -= size
    return sizes
