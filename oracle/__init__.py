"""CPU oracle for the s1proc per-burst interferogram chain.

TEST INFRASTRUCTURE ONLY.  This package restates, in float64 NumPy, the
algorithms of the reference project (WWSAR/sentinel_gpu_processor, "s1proc")
for the hot path: geo2rdr (deramp, zero-Doppler geocoding, bilinear
resampling, reramp), crossmul with multilooking, coherence and the Goldstein
filter.  Every function cites the reference file:line it follows.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it, and only as the
checker or the timed CPU baseline.  The product package
(``sentinel_gpu_processor_b200``) never imports it.

Parity pins: the reference ships no tests or golden vectors.  The oracle is
pinned against (a) the reference's own ``orbit.cu``/``bounds.cu`` compiled as
host C++ (``oracle/_ref/libref_geom.so``, built by ``oracle/build_ref.py``)
and (b) outputs of the reference CUDA executables built from the reference
sources and run on a B200, stored under ``tests/golden/`` together with the
script that made them.
"""
