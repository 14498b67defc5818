"""skirt7_b200 -- SKIRT7's photon-packet life cycle on NVIDIA B200 (sm_100a).

The compute path is the CUDA library libskirt_b200.so (C ABI: include/skirt_b200.h); this
package is its host side: simulation items named after the reference's classes
(skirt7_b200.scene), a device context and the MonteCarloSimulation phase driver
(skirt7_b200.runtime), and the workload definitions used by the tests and the benchmark
(skirt7_b200.models).  There is no CPU fallback: without the library every call raises.
"""
from . import _abi
from ._abi import SkirtError
from .runtime import Context, MonteCarloSimulation, build_tree, chunk_params, device_count, tree_from_splits
from .scene import (KPC, LSUN, MICRON, MPC, PC, DEG, CartesianDustGrid, ClumpyGeometryDecorator, DustComp,
                    DustMix, ExpDiskGeometry, FaceOnDustCompNormalization, FrameInstrument, FullInstrument,
                    LogWavelengthGrid, OligoWavelengthGrid, PointGeometry, SceneModel, SEDInstrument,
                    SersicGeometry, SimpleInstrument, StellarComp, TreeDustGrid, VoronoiDustGrid)

__all__ = [n for n in dir() if not n.startswith("_")]
