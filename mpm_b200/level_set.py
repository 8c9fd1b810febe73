"""Level-set collision objects.

``LevelSetCollisionObject3D`` follows the reference's struct of the same name
(include/collision_object3d.h:9-12: a level set, declared but never applied
there): the signed distance of an obstacle sampled at the scene's grid nodes,
negative inside.  The solver applies it in every grid collision (and particle
collision, when enabled) after the grid boundary, with the friction law of
applyBoundaryCollision (src/collision_object3d.cu:38-51) on the velocity
relative to the object's surface velocity.

The builders return exact signed distances on the node lattice
``origin + stride * (x, y, z)`` as float32 arrays of shape
``(res_z, res_y, res_x)`` (C order = node index x + X (y + Y z)).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence

import numpy as np


@dataclass
class LevelSetCollisionObject3D:
    level_set: np.ndarray            # signed distance per grid node, (res_z, res_y, res_x) or flat
    friction: float = 0.0
    velocity: Sequence[float] = (0.0, 0.0, 0.0)   # surface velocity of the object

    def arrays(self, resolution) -> tuple:
        nodes = int(resolution[0]) * int(resolution[1]) * int(resolution[2])
        phi = np.ascontiguousarray(self.level_set, np.float32).reshape(-1)
        if phi.size != nodes:
            raise ValueError(f"level set has {phi.size} values, the grid has {nodes} nodes")
        vel = np.ascontiguousarray(self.velocity, np.float32).reshape(3)
        return phi, vel


def node_coordinates(origin, resolution, stride):
    """World coordinates of the grid nodes, each of shape (res_z, res_y, res_x)."""
    axes = [np.float64(origin[a]) + np.float64(stride) * np.arange(int(resolution[a]), dtype=np.float64)
            for a in range(3)]
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return x, y, z


def sphere(origin, resolution, stride, center, radius) -> np.ndarray:
    x, y, z = node_coordinates(origin, resolution, stride)
    d = np.sqrt((x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2) - radius
    return d.astype(np.float32)


def box(origin, resolution, stride, lo, hi) -> np.ndarray:
    """Axis-aligned box [lo, hi]."""
    x, y, z = node_coordinates(origin, resolution, stride)
    q = [np.abs(c - 0.5 * (lo[a] + hi[a])) - 0.5 * (hi[a] - lo[a]) for a, c in enumerate((x, y, z))]
    outside = np.sqrt(sum(np.maximum(qa, 0.0) ** 2 for qa in q))
    inside = np.minimum(np.maximum(np.maximum(q[0], q[1]), q[2]), 0.0)
    return (outside + inside).astype(np.float32)


def half_space(origin, resolution, stride, point, normal) -> np.ndarray:
    """Solid on the side opposite to `normal` of the plane through `point`."""
    n = np.asarray(normal, np.float64)
    n = n / np.linalg.norm(n)
    x, y, z = node_coordinates(origin, resolution, stride)
    return ((x - point[0]) * n[0] + (y - point[1]) * n[1] + (z - point[2]) * n[2]).astype(np.float32)


def union(*phis) -> np.ndarray:
    return np.minimum.reduce([np.asarray(p, np.float32) for p in phis])
