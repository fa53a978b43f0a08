"""B200 randomized pseudoskeleton (CUR) compression of far-field MoM/EFIE impedance blocks.

Host-side Python over the C ABI of libpskel_b200.so (include/pskel.h):

* :mod:`pskel.mesh` - meshes and RWG topology in the reference's array layout;
* :mod:`pskel.api` - the reference's Julia driver functions (fill wrappers, CUR round,
  adaptive CUR, compressed-matvec error) with the same names, arguments and behaviour;
* :mod:`pskel.octree` - octree grouping and the far-field block list;
* :mod:`pskel.engine` - the handle API: resident mesh, batched far-block compression.
"""
from . import mesh  # noqa: F401

__all__ = ["mesh"]
