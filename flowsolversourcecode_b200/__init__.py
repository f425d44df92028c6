"""B200 (sm_100a) SIMPLE inner loop of the FlowSolverSourceCode finite-volume solver.

The compute runs in libfsb200.so (hand-written CUDA kernels behind the C ABI
of include/fsb200.h); this package holds its ctypes binding (`_lib`), the host
mirror of the reference subroutines (`solver.Solver`), case descriptions
(`case`), meshes and polyMesh I/O (`mesh`) and the build (`build`).
"""
__version__ = "0.1.0"
