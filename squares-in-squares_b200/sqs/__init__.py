"""sqs -- B200-native engine for packing unit squares in the smallest square.

Python host side of libsqs.so (ctypes; numpy arrays; no PyTorch).  The
modules mirror the reference toolkit's entry points for its hot path:

  sqs.sat        batched FP32 SAT overlap energy + gradient
  sqs.core       certify / evaluate (reference squares.core)
"""
from ._native import Context, SQSError, device_count  # noqa: F401

__all__ = ["Context", "SQSError", "device_count"]
