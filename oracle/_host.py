"""Per-hour FP64 host scalars shared with the product (test infrastructure).

The solar position, clearness index, diffuse split and Perez luminance are
host-side scalar computations of the product (``solweig_cuda_b200.sun`` and
``.sky``) that are pinned bit-exactly against the reference in
``tests/test_host_scalars.py``; the oracle reuses them and restates only the
per-pixel work.
"""
import importlib

sun = importlib.import_module("solweig_cuda_b200.sun")
sky = importlib.import_module("solweig_cuda_b200.sky")
