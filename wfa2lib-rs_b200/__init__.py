"""wfa2lib-rs_b200: a B200-native wavefront-alignment hot path behind the
wfa2lib-rs aligner API (src/aligner.rs of the reference crate).

The compute path is the C-ABI shared library built from csrc/ (CUDA kernels
for sm_100a plus the C++ host side); this package is its Python mirror.
"""
