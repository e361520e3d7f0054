"""The two trimesh calls the reference's transform() makes on point clouds
(SPH/main.py:133-143): a Trimesh holding float64 vertices, translated in place, and
the rotation about an axis through a point. TEST INFRASTRUCTURE for
tests/golden/make_reference_run.py."""
import types

import numpy as np


class Trimesh:
    def __init__(self, vertices=None, faces=None, **kw):
        self.vertices = np.array(vertices, dtype=np.float64)
        self.faces = faces

    @property
    def center_mass(self):
        # trimesh integrates the mass properties over the faces; a mesh without faces
        # has zero volume, for which trimesh returns a zero center of mass
        if self.faces is None or len(self.faces) == 0:
            return np.zeros(3)
        raise NotImplementedError("center_mass of a mesh with faces")

    def apply_translation(self, t):
        self.vertices = self.vertices + np.asarray(t, np.float64)

    def apply_transform(self, m):
        m = np.asarray(m, np.float64)
        self.vertices = self.vertices @ m[:3, :3].T + m[:3, 3]


def _rotation_matrix(angle, direction, point=None):
    d = np.asarray(direction, np.float64)
    d = d / np.linalg.norm(d)
    c, s = np.cos(angle), np.sin(angle)
    K = np.array([[0, -d[2], d[1]], [d[2], 0, -d[0]], [-d[1], d[0], 0]])
    R = np.eye(3) * c + s * K + (1 - c) * np.outer(d, d)
    M = np.eye(4)
    M[:3, :3] = R
    if point is not None:
        p = np.asarray(point, np.float64)
        M[:3, 3] = p - R @ p
    return M


transformations = types.SimpleNamespace(rotation_matrix=_rotation_matrix)
