"""CPU oracle for the Wigner2D / Dirac2D split-operator propagators.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package may import this
package; only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` use it, and only as the checker or
as the timed CPU baseline.

Contents
--------
* :mod:`oracle.common`   -- ``%f`` constant rounding, grids, expression eval.
* :mod:`oracle.wigner2d` -- restatement of ``GPU_Wigner2D_FFT.Run`` (Lie step,
  Caldeira-Leggett order-3 and ODM Lindblad damping) and of
  ``GPU_Wigner2D_ODM2.Run``.
* :mod:`oracle.dirac2d`  -- restatement of ``GPU_Dirac2D.Run``.
* :mod:`oracle.strang_notebook` -- the reference's only CPU propagator
  (``CPU_GPU_Wigner2D.ipynb``: real W, Strang V/2-K-V/2), used to pin the
  oracle against the notebook's recorded known answer.
* :mod:`oracle.ref_harness` -- runs the reference's own Python-2 host code
  under a fake PyCUDA whose kernels are the reference's CUDA-C strings compiled
  for the CPU (into ``oracle/_ref/``); produces the golden fixtures.

Parity is pinned by (a) the notebook known answer and (b) golden fixtures
generated by :mod:`oracle.ref_harness` from the reference's own code.
"""
