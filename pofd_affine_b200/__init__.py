"""B200-native P(D) likelihood hot path of aconley/pofd_affine.

FP64 sm_100a kernels behind a C ABI (include/pofd_b200.h, built into
pofd_affine_b200/_lib/libpofd_b200.so), with Python classes that mirror the
reference's interfaces (beam, PDFactory, calcLike; doublebeam,
calcLikeDouble).
"""
from ._lib import PofdError  # noqa: F401
from .api1d import PD, Context, PDFactory, beam, calcLike  # noqa: F401
from .api2d import PDFactoryDouble, calcLikeDouble, doublebeam  # noqa: F401

__version__ = "0.1.0"
