"""camr_b200: B200-native (sm_100a, FP64) hydro advance of CAMR.

The product is libcamr_b200.so (C ABI, include/camr_b200.h).  This package
builds it (``camr_b200.build``), binds it (``camr_b200.native``), mirrors the
reference's call surface on the host (``camr_b200.hydro``) and generates the
benchmark configurations' initial data (``camr_b200.problems``).
"""
from . import hydro, native, problems  # noqa: F401
from .native import BC, NVAR, CamrError, HydroParams, default_params  # noqa: F401

__all__ = ["native", "problems", "hydro", "BC", "NVAR", "CamrError", "HydroParams",
           "default_params"]
