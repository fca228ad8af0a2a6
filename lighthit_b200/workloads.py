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


FINE_STRUCTURE = 7.2973525693e-3
C_M_PER_NS = 0.299792458


def _rotation_between(source, target):
    """Proper rotation taking unit ``source`` to unit ``target`` (``sources.py:39-57``)."""
    source = np.asarray(source, float) / np.linalg.norm(source)
    target = np.asarray(target, float) / np.linalg.norm(target)
    cosine = float(np.clip(source @ target, -1.0, 1.0))
    if np.isclose(cosine, 1.0, atol=1e-14):
        return np.eye(3)
    if np.isclose(cosine, -1.0, atol=1e-14):
        helper = np.array([1.0, 0.0, 0.0])
        if abs(float(source @ helper)) > 0.9:
            helper = np.array([0.0, 1.0, 0.0])
        axis = np.cross(source, helper)
        axis /= np.linalg.norm(axis)
        return 2 * np.outer(axis, axis) - np.eye(3)
    cross = np.cross(source, target)
    skew = np.array([[0.0, -cross[2], cross[1]], [cross[2], 0.0, -cross[0]],
                     [-cross[1], cross[0], 0.0]])
    return np.eye(3) + skew + skew @ skew * ((1.0 - cosine) / float(cross @ cross))


def gaussian_shower(position_m, direction, *, charged_track_length_m=100.0,
                    longitudinal_sigma_m=1.2, transverse_sigma_m=0.08, elements=64, beta=0.999,
                    seed=0, time_ns=0.0):
    """Spectral elements of ``SyntheticShower.gaussian`` placed at a pose.

    Restates ``sources.py:403-441`` (draws from one ``default_rng(seed)``:
    transverse offsets, then angular offsets) and the pose placement
    ``placed`` (``sources.py:231-262``: the C0-weighted centroid and principal
    axis of the midpoints moved onto the pose). Returns a dict with the
    reference's ``SpectralLightElements`` field names (spectral cones).
    """
    rng = np.random.default_rng(seed)
    z = np.linspace(-3 * longitudinal_sigma_m, 3 * longitudinal_sigma_m, int(elements))
    share = np.exp(-0.5 * (z / longitudinal_sigma_m) ** 2)
    share /= share.sum()
    transverse = rng.normal(scale=transverse_sigma_m, size=(len(z), 2))
    angular = rng.normal(scale=0.025, size=(len(z), 2))
    start = np.column_stack((transverse, z))
    unit = np.column_stack((angular, np.ones(len(z))))
    unit /= np.linalg.norm(unit, axis=1)[:, None]
    unit = unit / np.linalg.norm(unit, axis=1)[:, None]  # SpectralLightElements normalises again
    segment_length = max(0.01, 6 * longitudinal_sigma_m / len(z))
    length = np.full(len(z), segment_length)
    common = 2 * np.pi * FINE_STRUCTURE * 1e9 * charged_track_length_m * share
    t0 = (z - z.min()) / (beta * C_M_PER_NS)
    t1 = t0 + length / (beta * C_M_PER_NS)
    # principal axis of the C0-weighted midpoints (sources.py:22-36)
    points = start + 0.5 * length[:, None] * unit
    weight = common / common.sum()
    centre = np.sum(weight[:, None] * points, axis=0)
    offset = points - centre
    covariance = np.einsum("i,ij,ik->jk", weight, offset, offset)
    values, vectors = np.linalg.eigh(covariance)
    if float(np.max(np.abs(values))) <= 1e-24:
        axis = np.sum(weight[:, None] * unit, axis=0)
    else:
        axis = vectors[:, int(np.argmax(values))]
    if float(np.sum(weight * (unit @ axis))) < 0:
        axis = -axis
    axis = axis / np.linalg.norm(axis)
    rotation = _rotation_between(axis, direction)
    translation = np.asarray(position_m, float) - rotation @ centre
    delay = float(time_ns - np.min(t0))
    return dict(start_m=start @ rotation.T + translation, direction=unit @ rotation.T,
                length_m=length, coefficient0=common, coefficient2=-common / beta ** 2,
                beta=np.full(len(z), float(beta)), start_ns=t0 + delay, end_ns=t1 + delay)


def shower_stream(count, centroid_m, *, seed=21, low_elements=500, high_elements=50000,
                  metres_per_element=0.15, radius_m=200.0, height_m=600.0):
    """Pose and size of each shower of the served stream (seeded).

    One ``default_rng(seed)`` draws, per shower in order: the element count
    ``round(exp(U(ln low, ln high)))``, the vertex ``r = radius sqrt(U)``,
    ``phi = U(0, 2 pi)``, ``z = U(-h/2, h/2)`` around ``centroid_m``, and an
    isotropic direction (``cos theta = U(-1, 1)``, azimuth ``U(0, 2 pi)``).
    The charged track length is ``metres_per_element`` per element. Returns
    dicts with ``position_m``, ``direction``, ``elements``,
    ``charged_track_length_m`` and ``seed`` (the shower's own generator seed).
    """
    rng = np.random.default_rng(seed)
    centroid = np.asarray(centroid_m, float)
    out = []
    for k in range(int(count)):
        n = int(round(float(np.exp(rng.uniform(np.log(low_elements), np.log(high_elements))))))
        r = radius_m * np.sqrt(rng.uniform())
        phi = rng.uniform(0.0, 2 * np.pi)
        z = rng.uniform(-height_m / 2, height_m / 2)
        cos_t = rng.uniform(-1.0, 1.0)
        az = rng.uniform(0.0, 2 * np.pi)
        sin_t = np.sqrt(max(0.0, 1.0 - cos_t * cos_t))
        out.append(dict(position_m=centroid + np.array([r * np.cos(phi), r * np.sin(phi), z]),
                        direction=np.array([sin_t * np.cos(az), sin_t * np.sin(az), cos_t]),
                        elements=n, charged_track_length_m=metres_per_element * n,
                        seed=int(seed) * 1_000_003 + k))
    return out
