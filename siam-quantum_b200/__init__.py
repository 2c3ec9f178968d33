"""siam-quantum_b200: B200-native two-electron Fock build (J/K) for Siam Quantum 2.

The product is the CUDA library libsqb200.so behind the C ABI in include/sqb200.h.  This
Python package is the host-side binding used by tests and the benchmark:
  engine     ctypes binding of the C ABI (JKEngine)
  basis      genBasis-order Cartesian Gaussian basis builder (flat arrays for the ABI)
  molecules  seeded workload geometries (water, benzene, C60, random organics)
  scf        device-resident RHF/UHF SCF around the GPU Fock build (SCFJob)
  batch_scf  many molecules' SCF together: batched Fock builds in a CUDA graph (BatchSCF)
  serve      served stream of SCF jobs with continuous batching and HBM admission (Server)
  checkpoint the reference's checkpoint files: read, write, and the projected orbital guess

The directory name is not a Python identifier; import it with `load_package()` from a
checkout root or via importlib (see tests/conftest.py).
"""
from . import basis, batch_scf, checkpoint, engine, molecules, scf, serve  # noqa: F401
from .engine import JKBatch, JKEngine, SQB200Error, load_library  # noqa: F401
