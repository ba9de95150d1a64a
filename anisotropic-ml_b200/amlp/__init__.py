"""anisotropic-ML on B200: rigid-body NEP force evaluation and NVT integration.

Submodules:
  shapes, configs, gsd  -- pure host code (no GPU needed)
  _lib                  -- ctypes binding of libamlp.so (include/amlp.h)
  engine                -- device-resident System driving the library
  build                 -- nvcc build recipe of libamlp.so
"""
__version__ = "0.1.0"
