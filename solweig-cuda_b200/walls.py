"""Drop-in for the DSM wall method of the reference's ``src/walls.py``.

``calculate_dsm_walls`` keeps the reference's signature and returns host
float64 arrays ``(walls, aspect)`` like ``src/walls.py:132-142``: wall height
from the 4-neighbour maximum and the wall aspect from 180 rotated line
templates, both scored on the device; the gradient fallback for walls no
template resolves runs on the host for the few pixels concerned.

The geometry wall method (``src/walls.py:145-332``) rasterises building
polygons with shapely/rasterio; it is not part of this engine.
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import _upload, wall_aspect, wall_heights_device

__all__ = ["calculate_dsm_walls", "calculate_geometry_walls"]


def calculate_dsm_walls(dsm, pixel_size_m, minimum_wall_height_m=3.0, device="cuda"):
    surface = np.asarray(dsm, dtype=np.float64)
    dsm_dev = _upload(surface, np.float64, torch.device(device))
    walls_dev = wall_heights_device(dsm_dev, float(minimum_wall_height_m))
    aspect, walls = wall_aspect(surface, dsm_dev, walls_dev, float(pixel_size_m))
    return walls, aspect


def calculate_geometry_walls(*args, **kwargs):
    raise NotImplementedError(
        "wall_method='geometry' (building polygons via shapely/rasterio) is not provided by "
        "solweig_cuda_b200; use wall_method='dsm'")
