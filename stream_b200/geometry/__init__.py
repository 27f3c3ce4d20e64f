"""Spatial trees over 3D spheres: the Karras LBVH, the TRBVH and the LBVHa
(Apetrei's agglomerative build)."""
from .lbvh import Sphere3DLBVH, Sphere3DLBVHa, Sphere3DTRBVH  # noqa: F401
