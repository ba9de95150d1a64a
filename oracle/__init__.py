"""CPU oracle for the nep_simulator hot path.

TEST INFRASTRUCTURE ONLY. This package is the checker: it may be imported by
``tests/``, by ``__graft_entry__.smoke()`` and by the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py``. The product (the ``amlp`` package,
the ``nep_simulator`` drop-in modules and ``libamlp.so``) never imports, links
or calls anything here.

Modules:

* ``nep``      -- numpy restatement of the reference's per-step math in FP32
                  with the reference's operation order, plus FP64 twins and the
                  spherical-harmonic form of the angular descriptor;
* ``adjoint``  -- FP64 pair energy written in torch so that autograd gives the
                  exact force/torque the finite-difference path approximates;
* ``nlist``    -- the reference's own neighbour-list call (scipy cKDTree);
* ``shapes``   -- independent copy of the shape tables;
* ``ref_kernels`` / ``ref_cupy_shim`` -- build recipe that compiles the
  reference's CUDA kernel strings for the host into ``oracle/_ref`` and a
  numpy-backed stand-in for CuPy, used only in the development container to run
  the reference's own Python classes and write ``tests/golden`` fixtures.
"""
