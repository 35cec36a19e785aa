"""B200-native Full Binary Pursuit.

Drop-in replacement for the hot path of spikesorting_fullpursuit:
``spikesorting_fullpursuit.parallel.binary_pursuit_parallel.binary_pursuit``.
The pursuit runs in hand-written sm_100a CUDA kernels (libfbp_b200.so, built
in-tree by ``spikesorting_fullpursuit_b200.build``) behind a C ABI
(include/fbp_b200.h); PyTorch only owns device buffers and streams.
"""
__version__ = "0.1.0"

from .parallel.binary_pursuit_parallel import binary_pursuit  # noqa: F401
