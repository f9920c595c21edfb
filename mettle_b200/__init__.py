"""mettle_b200 — B200-native (sm_100a) execution path for mettle's offloaded SQL subset.

The product is ``libmettle_cuda.so`` (C ABI in ``include/mettle_cuda.h``):
SQL front-end, planner, executor, serving loop and hand-written CUDA
kernels. This package binds it with ctypes and mirrors the extension's SQL
surface (``gpu_buffer_init``, ``gpu_register_table``, ``gpu_processing``,
``gpu_cache_status``, ``gpu_cache_reset``, ``gpu_rewrite_query`` and the
``gpu_*_scalar`` hooks) on a small host catalog that stands in for DuckDB's.
"""
from ._lib import MettleError, library_path
from .connection import Connection, Request, Result, Rows, Statement

__all__ = ["Connection", "MettleError", "Request", "Result", "Rows", "Statement", "library_path"]
