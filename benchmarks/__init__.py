"""Measurement programs for the configurations beyond bench.py's headline
(single kernels, batched sub-volumes, gradients, storage precision, shift
measurement). They drive the library through its public Python binding and
are not part of the library."""
