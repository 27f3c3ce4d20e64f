"""Mesh generation (mirrors the reference's ``stream.mesh`` for the 3D alpha shape)."""
from .ashape3d import AlphaShape3D  # noqa: F401
