"""Helpers of the drop-in `epcq` package (reference: epcq/utils.py)."""


def _get_c_extension():
    """The native module behind epcq (reference epcq/utils.py:2-15).

    The reference returns None and warns when its extension is missing; this
    package has no slow path to fall back to, so a missing CUDA library is an
    error raised at the first call (hashpoint.native.lib()).
    """
    from . import csrc
    return csrc


def is_pow2(x: int):
    return x > 0 and (x & (x - 1)) == 0
