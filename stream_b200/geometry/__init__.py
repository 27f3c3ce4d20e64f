"""Spatial trees: the Karras LBVH over 3D spheres."""
from .lbvh import Sphere3DLBVH, Sphere3DTRBVH  # noqa: F401
