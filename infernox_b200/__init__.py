"""B200-native covariance-model scan path (QDB CYK / Inside window scanners).

Product code: libcmscan_gpu.so (csrc/, built in-tree by ``build``) behind the
C ABI in include/cmscan_gpu.h, with this package's ctypes mirror of the
reference's scanner entry points (scan.py), model preparation (model.py) and
seeded synthetic inputs (synth.py).
"""
__version__ = "0.1.0"
