"""Tile windows with halos (the window arithmetic of ``src/tiling.py:29-42``).

``tile_windows`` returns, for a raster of ``height x width`` pixels, the core
and input windows of every tile and the core's position inside its input
window (``output_core``), exactly as ``create_tiles`` plans them; the GDAL/VRT
extraction of the reference is replaced by array slicing (``extract``).
"""
from __future__ import annotations

__all__ = ["tile_windows", "extract"]


def tile_windows(height, width, core=1800, halo=100):
    tiles = []
    for tile_row, row in enumerate(range(0, height, core)):
        for tile_col, col in enumerate(range(0, width, core)):
            core_width, core_height = min(core, width - col), min(core, height - row)
            left, top = max(0, col - halo), max(0, row - halo)
            right, bottom = min(width, col + core_width + halo), min(height, row + core_height + halo)
            tiles.append({
                "tile_id": f"r{tile_row:03d}_c{tile_col:03d}",
                "core_window": [col, row, core_width, core_height],
                "input_window": [left, top, right - left, bottom - top],
                "output_core": [row - top, col - left, core_height, core_width],
            })
    return tiles


def extract(array, tile):
    """The tile's input window of a 2-D array (``srcWin`` of the reference)."""
    left, top, w, h = tile["input_window"]
    return array[top:top + h, left:left + w]
