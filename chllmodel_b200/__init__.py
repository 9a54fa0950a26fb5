"""chllmodel_b200: B200-native chiral Lebwohl-Lasher checkerboard Metropolis.

``libchll_mod.so`` (sm_100a CUDA, C ABI in include/chll_mod.h) is a drop-in
for the reference's nvfortran library; ``chllmodel_b200.chll.ChLLSim`` is the
reference's Python host class over it.  Submodules:

  chll         ChLLSim and the ftn_init/ftn_run ctypes prototypes
  lattice      device-resident lattices (handle API)
  batched      many replicas of uneven size in one persistent launch
  workflows    anneal schedules and phase-diagram scans on the batched launch
  observables  S, C_v, chiral susceptibility from FP64 moments
  analysis     shell correlations and structure factor of a lattice's state
  autograd     torch.autograd.Function over the energy adjoint kernel
  distributed  replica sets sharded over ranks
  slab         one lattice split into z-slabs with halo exchange
  build        nvcc build of the shared library
"""
__version__ = "0.1.0"


def load_library():
    from . import _lib

    return _lib.load()
