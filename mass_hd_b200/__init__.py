"""Blackwell (sm_100a) implementation of the MASS lyotropic / nematic /
go-or-grow Model::Step() hot path.

The product is the C-ABI library ``lib/libmass_lb.so`` (include/mass_lb.h)
built from ``csrc/`` and the C++ model plugin in ``host/``; ``lb`` is a
ctypes front-end over the same library.
"""
from .lb import (FIELDS, FP32, FP64, GO_OR_GROW, LYOTROPIC, NEMATIC, Ensemble, Lattice,  # noqa: F401
                 MassLBError, library_path, load_library, make_params)

__all__ = ["FIELDS", "FP32", "FP64", "GO_OR_GROW", "LYOTROPIC", "NEMATIC", "Ensemble",
           "Lattice", "MassLBError", "library_path", "load_library", "make_params"]
