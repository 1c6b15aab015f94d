"""lceqcd_b200: the Monte Carlo hot path of derek-teaney/lceqcd (3D SU(2) +
adjoint Higgs lattice code) as hand-written sm_100a CUDA kernels behind a C ABI
(include/lceqcd_gpu.h, liblceqcd_gpu.so).  This package is the Python mirror
of the reference's subroutine interface over that ABI."""
from .lattice import (Ensemble, GaugeNet, Lattice, Params, SlabLattice, couplings, geometry_tables,
                      params_from_inputfile, read_inputfile)
from ._lib import LceError, load

__all__ = ["Lattice", "Ensemble", "GaugeNet", "Params", "SlabLattice", "couplings", "geometry_tables", "read_inputfile",
           "params_from_inputfile", "LceError", "load"]
