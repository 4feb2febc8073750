"""B200-native pressure projection for NEREUS (RaphaelLaroca/NEREUS_CFD).

The compute lives in ``libnereus_b200.so`` (CUDA for sm_100a behind the C ABI of ``include/nereus_b200.h``);
``pressure.PressureSolver`` mirrors the reference's PressureSolver2D/3D interface over it, ``workloads`` builds the
synthetic cases, ``build`` compiles the library in-tree.
"""

__all__ = ["capi", "pressure", "workloads", "build"]
