"""B200-native LDDMM landmark/surface registration with varifold matching.

The compute path is the sm_100a shared library ``liblddmm_b200.so`` (C ABI in
``include/lddmm_b200.h``); ``lddmm_b200.api`` wraps it.  ``problem`` and ``shapes``
are host-side data helpers that import without the library.

Attributes of ``api`` (``Context``, ``LDDMM``, ``objgrd``, ...) are re-exported
lazily, so that importing the data helpers does not require the built library, while
any compute call fails loudly when it is missing.
"""

__all__ = ["Context", "LDDMM", "objgrd", "multiplyKernel", "dqKernel", "varifold",
           "getElmIfo", "computeNodePosition", "Problem"]


def __getattr__(name):
    if name == "Problem":
        from .problem import Problem
        return Problem
    if name in __all__:
        from . import api
        return getattr(api, name)
    raise AttributeError(name)
