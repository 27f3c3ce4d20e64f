"""Mesh generation (mirrors the reference's ``stream.mesh``: the 3D and 2D alpha
shapes and the 2D Delaunay mesher)."""
from .ashape2d import AlphaShape2D  # noqa: F401
from .ashape3d import AlphaShape3D  # noqa: F401
from .mesh2d import Mesh2D  # noqa: F401
