"""CPU oracle for the SOLWEIG per-hour hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in float64 numpy, the reference algorithms that the
CUDA library replaces, so that tests can check the GPU results on the same
seeded inputs.  It is imported only by ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``; the
product package never imports it and fails loudly when its CUDA library is
missing instead of falling back to anything here.

Modules and what they restate (reference paths relative to the reference
project root):

* ``geometry``  shadow sweep (``src/umep_solweig.py:2063-2406``), DSM walls
                (``src/walls.py:24-142``, ``src/kernels/geometry.cu:15-63``) and
                the 153-patch sky view factor (``src/svf.py:19-131``,
                ``src/kernels/geometry.cu:66-172``);
* ``ground``    ground view factors (``src/umep_solweig.py:583-663``, ``:1400-1600``);
* ``radiation`` wave delay, wedge, K/L fluxes and Tmrt
                (``src/umep_solweig.py:345-1398``, ``:1633-1652``);
* ``utci``      the UTCI regression polynomial (``src/kernels/utci.cu``);
* ``step``      the hourly step and the static preparation
                (``src/umep_solweig.py:50-372``, ``src/series.py:197-495``).

Pinning: ``tests/test_oracle_pin.py`` checks these functions against the
reference imported in place (when the reference tree is present) and against
the committed golden fixtures under ``tests/golden/`` on every machine.
"""
