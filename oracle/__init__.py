"""CPU oracle for the dft-zig plane-wave hot path.

TEST INFRASTRUCTURE ONLY.  This package is a plain FP64 numpy restatement of
dft-zig's H|psi>, Davidson ("LOBPCG") eigensolver and band-density code.  It
is imported only by ``tests/``, by ``__graft_entry__.smoke()`` and by the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``, always as the
checker or as the timed CPU baseline, never as part of the product path.
The product (``dft-zig_b200``) never imports it and fails loudly when its
CUDA library is missing.

Every function cites the reference file:line it restates (paths relative to
the dft-zig source tree).  The oracle is pinned against the reference's own
known-answer tests (``tests/golden/``): the 4^3 local-potential KATs
(src/tests.zig:872-1104), the diagonal-operator LOBPCG tests
(src/features/linalg/iterative.zig:80-203), the FFT round trips
(src/features/fft/fft.zig:418-470, src/lib/fft/fftw_fft.zig:176-227), the
spherical Bessel values (src/tests.zig:1245-1318) and the ctrap weights
(src/features/math/radial_integration.zig:18-55).  SCF energies of the
synthetic pseudopotential cells have no reference golden value (the
reference ships no UPF files and cannot be built here), so those
comparisons are parity-unpinned beyond the kernel-level KATs.
"""
