"""CPU oracle for the fixed-trajectory NUFFT CG-SENSE path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (the ``trajsparsenufft_b200``
package, its C++ host library or its CUDA kernels) imports, links or executes
anything in this directory.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` use it, and there
only as the checker or as the timed CPU baseline, never as the thing measured.

Modules
-------
planner   restatement of the reference pack-once planner and exporter
          (src/nufft_layout_oracle.py, src/export_gpu_case.py,
          src/export_torchkbnufft_gpu_case.py); pinned byte-for-byte against
          golden packs produced by the reference itself (tests/golden/).
kb        complex Kaiser-Bessel interpolation coefficients and deapodization
          (published KB / Beatty mathematics; the reference takes these from
          torchkbnufft 1.5.2, which is not vendored).
nudft     FP64 direct non-uniform DFT with SENSE (the accuracy oracle).
operator  FP64 and FP16x2-emulated SENSE NUFFT operators and the CG-SENSE
          recursion of experiments/production/reference_sparse_solver.py.
"""
