"""B200-native radar range-Doppler chain (front end, pulse compression, Doppler, CA-CFAR).

All computation runs in the in-tree CUDA library ``libzkx_rd.so`` (C ABI declared in
``include/zkx_rd.h``); this package is the Python mirror of the reference's operator
interface on top of it.
"""
from ._lib import ZkxError, ZkxValueError, lib
from .radartools import (ambgfun, ca_cfar, cfar_alpha, fft, pulse_compression, pulse_doppler,
                         replica_spectrum)
from .filtering import firfilter, firfilter2, hilbert, resample_poly, resample_poly_taps, upfirdn
from .chain import ChainConfig, RangeDopplerChain, WorkList
from .serving import RdServer, ServerConfig

__all__ = ["ZkxError", "ZkxValueError", "lib", "ambgfun", "ca_cfar", "cfar_alpha", "fft", "pulse_compression",
           "pulse_doppler", "replica_spectrum", "firfilter", "firfilter2", "hilbert", "resample_poly",
           "resample_poly_taps", "upfirdn", "ChainConfig", "RangeDopplerChain", "WorkList", "RdServer", "ServerConfig"]
