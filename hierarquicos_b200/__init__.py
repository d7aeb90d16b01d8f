"""hierarquicos_b200: a B200 (sm_100a) Barnes-Hut force engine.

The force path -- 63-bit Morton keys, stable LSD radix sort, octree from the
sorted keys, FP64 multipole upward pass (monopole / quadrupole / octupole),
warp-cooperative FP32 Kahan-compensated group walk -- is CUDA C++ behind the C
ABI of include/hierarquicos_bh.h.  Python modules:

* ``api3d``        -- drop-in for the reference's f2py module api_mod;
* ``system``       -- device-resident systems (BHSystem, MortonTree, Octree);
* ``initial_values`` -- seeded Plummer / Hernquist / homogeneous / uniform ICs;
* ``metrics``      -- force-error statistics;
* ``build``        -- compiles the library in-tree.
"""
from ._lib import BHError, BHParams, default_params, lib  # noqa: F401

__version__ = "0.1.0"
