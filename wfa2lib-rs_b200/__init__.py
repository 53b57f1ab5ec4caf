"""wfa2lib-rs_b200: a B200-native wavefront-alignment hot path behind the
wfa2lib-rs aligner API (src/aligner.rs of the reference crate).

The compute path is the C-ABI shared library built from csrc/ (CUDA kernels
for sm_100a plus the C++ host side, lib/libwfa_b200.so); this package is its
Python mirror.  Import it by path (the directory name is not an identifier),
e.g. with importlib; see tests/_pkg.py.
"""
from .aligner import (COMPLETED, EDIT, GAP_AFFINE, GAP_AFFINE_2P, GAP_LINEAR, INDEL,  # noqa: F401
                      RESULT_DTYPE, Cigar, Server, Stream, WavefrontAligner, cigar_rle, lib)
