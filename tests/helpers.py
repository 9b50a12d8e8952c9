"""Test helpers shared by several test modules."""
from __future__ import annotations


def mesh_by_name(name):
    from walk_on_spheres_b200 import meshes
    return {
        "annulus": meshes.annulus(),
        "circle256": meshes.circle(segments=256),
        "circle1024": meshes.circle(segments=1024),
        "sphere": meshes.uv_sphere(lon=32, lat=16),
        "sphere_full": meshes.uv_sphere(),
    }[name]
