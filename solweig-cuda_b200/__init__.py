"""SOLWEIG on B200: Tmrt and UTCI per pixel-hour with hand-written sm_100a CUDA.

Drop-in modules mirroring the reference's call surfaces:

* ``solweig_cuda_b200.walls``   -- ``calculate_dsm_walls``
* ``solweig_cuda_b200.svf``     -- ``svf_calculator``, ``compute_diffsh``
* ``solweig_cuda_b200.model``   -- ``prepare_model``, ``Solweig_2022a_calc``
* ``solweig_cuda_b200.utci``    -- ``utci_calculator``
* ``solweig_cuda_b200.series``  -- ``run_timeseries``, ``load_meteorology``

Host-only helpers (no GPU needed): ``sun`` (FP64 solar position), ``sky``
(patch layout, Perez luminance), ``synthetic`` (seeded test scenes).

The CUDA library ``libsolweig_b200.so`` is loaded on first use by
``solweig_cuda_b200._lib``; there is no CPU fallback.
"""
__version__ = "0.1.0"
