"""B200-native finite-volume Euler split-solver step (robclu/fluidity hot path).

The compute path is libfluidity_b200.so (hand-written sm_100a CUDA behind the C
ABI of include/fluidity_b200.h).  This package holds the Python side of that
boundary: the ctypes binding (capi), a Python mirror of the reference's
simulator interface (solver), the seeded workload generators (workloads) and
the in-tree build (build).
"""
from . import capi, workloads  # noqa: F401

__all__ = ["capi", "workloads"]
