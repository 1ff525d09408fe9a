"""Command line of the B200 engine, mirroring the reference's ``run.py``.

    python run.py [--case case.json] [--output DIR] [--dtype float32|float64]
                  [--output-core ROW COL ROWS COLS] [--output-chunk-steps N]
                  [--sync-output] [--output-queue-size N] [--no-write] [--progress]
                  [--check] [--form chosen|batched]

Case keys follow the reference's ``examples/case.json`` (paths relative to the
case file; the default case is ``examples/case.json`` beside this file, as in
the reference).  Rasters are ``.npy`` arrays (GeoTIFF where rasterio/GDAL is
installed).  ``case_type: open_data`` needs network downloads and is not
supported; ``core_area_m`` / ``buffer_area_m`` tile the rasters with halos and
every group of tiles runs day by day in one captured graph per day
(``series.run_tiles``).  Under ``torchrun`` each rank takes a share of the
days (one tile) or of the tiles (tiled cases).  ``--dtype float64`` is the
reference's radiation precision switch: every hour runs through the float64
step instead of the batched float32/BF16 form.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
from datetime import datetime
from pathlib import Path

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PATH_KEYS = {"building_dsm_path", "tree_path", "dem_path", "met_file", "building_geometry_path",
             "building_height_path", "landcover_path", "output_path"}
PREPARATION_KEYS = {"case_name", "case_type", "case_size_m", "core_area_m", "buffer_area_m",
                    "resolution_m", "start_date", "end_date"}


def load_case(path):
    """Case dict and preparation settings (``run.py:70-86`` of the reference)."""
    path = Path(path).resolve()
    case = json.loads(path.read_text(encoding="utf-8-sig"))
    settings = {key: case.pop(key) for key in PREPARATION_KEYS if key in case}
    settings.setdefault("case_type", "local")
    settings.setdefault("resolution_m", 1)
    for key in PATH_KEYS & case.keys():
        value = case[key]
        if value is None:
            continue
        entries = value if isinstance(value, list) else [value]
        resolved = [str((path.parent / Path(e).expanduser()).resolve()) for e in entries]
        case[key] = resolved if isinstance(value, list) else resolved[0]
    case.setdefault("async_output", True)
    case.setdefault("output_queue_size", 2)
    case.setdefault("output_chunk_steps", 24)
    return case, settings


def _tile_jobs(case, settings):
    """Tiles of a tiled case (``run.py:113-129`` of the reference): dicts with
    the tile id, the input-window arrays and the output core, for
    ``series.run_tiles``."""
    import numpy as np
    from solweig_cuda_b200.series import load_raster
    from solweig_cuda_b200 import tiling
    res = float(settings.get("resolution_m", 1))
    core, halo = (int(round(settings[k] / res)) for k in ("core_area_m", "buffer_area_m"))
    names = {"building_dsm_path": "dsm", "tree_path": "trees", "dem_path": "dem"}
    if case.get("landcover_path"):
        names["landcover_path"] = "landcover"
    rasters = {names[k]: load_raster(case[k]) for k in names}
    h, w = rasters["dsm"].shape
    jobs = []
    for t in tiling.tile_windows(h, w, core=core, halo=halo):
        job = {"tile_id": t["tile_id"], "output_core": t["output_core"]}
        for k, arr in rasters.items():
            job[k] = np.ascontiguousarray(tiling.extract(arr, t))
        jobs.append(job)
    return jobs


def main(argv=None):
    parser = argparse.ArgumentParser(description="Run SOLWEIG on the GPU for the supplied rasters and forcing.")
    parser.add_argument("--case", type=Path, default=Path(ROOT) / "examples" / "case.json",
                        help="JSON case file (default: examples/case.json beside run.py); paths are relative to it")
    parser.add_argument("--output", type=Path)
    parser.add_argument("--dtype", choices=("float32", "float64"), default="float32",
                        help="radiation precision")
    parser.add_argument("--form", choices=("chosen", "batched"), default="chosen",
                        help="chosen: batched day with tensor-core patch sums; batched: per-hour kernels in a graph")
    parser.add_argument("--output-core", type=int, nargs=4, metavar=("ROW", "COL", "ROWS", "COLS"))
    parser.add_argument("--output-chunk-steps", type=int)
    parser.add_argument("--sync-output", action="store_true")
    parser.add_argument("--output-queue-size", type=int)
    parser.add_argument("--no-write", action="store_true")
    parser.add_argument("--progress", action=argparse.BooleanOptionalAction, default=True)
    parser.add_argument("--check", action="store_true",
                        help="validate case.json and the forcing first (the reference's input_check rules)")
    args = parser.parse_args(argv)
    case_path = args.case.resolve()
    if args.check:
        from solweig_cuda_b200 import input_check
        checked, _ = input_check.check_case(case_path)
        input_check.check_weather(checked["met_file"])
    case, settings = load_case(case_path)
    if settings["case_type"] == "open_data":
        missing = [k for k in ("building_dsm_path", "tree_path", "dem_path", "met_file")
                   if not Path(case[k]).exists()]
        if missing:
            raise SystemExit(f"open_data preparation (network download) is not supported; missing: {missing}")
    if args.output_core is not None:
        case["output_core"] = args.output_core
    if args.output_chunk_steps is not None:
        case["output_chunk_steps"] = args.output_chunk_steps
    if args.sync_output:
        case["async_output"] = False
    if args.output_queue_size is not None:
        case["output_queue_size"] = args.output_queue_size
    output = Path(case.pop("output_path", case_path.parent / "output"))
    output = (args.output or output).resolve()
    import numpy as np
    from solweig_cuda_b200.series import load_meteorology, run_timeseries
    forcing = load_meteorology(case["met_file"])
    case["met_file"] = forcing
    pixel_size = float(settings.get("resolution_m", 1))
    if "core_area_m" in settings:
        if str(case.get("wall_method", "dsm")).strip().lower() != "dsm":
            # the reference's tile jobs crop the DSM, trees, DEM and land cover
            # but not the building-height raster (run.py:113-129)
            raise SystemExit("wall_method='geometry' is not supported for tiled cases")
        from solweig_cuda_b200.series import run_tiles
        known = {"longitude", "latitude", "utc_offset_hours", "site_altitude_m", "output_chunk_steps",
                 "async_output", "output_queue_size", "save_tmrt", "save_kup", "save_kdown", "save_lup",
                 "save_ldown", "save_shadow", "dsm_wall_threshold_m"}
        kwargs = {k: v for k, v in case.items() if k in known}
        run_tiles(_tile_jobs(case, settings), forcing, output, dtype=np.dtype(args.dtype), no_write=args.no_write,
                  progress=args.progress, pixel_size=pixel_size, **kwargs)
    else:
        known = {"building_dsm_path", "tree_path", "dem_path", "met_file", "longitude", "latitude",
                 "landcover_path", "utc_offset_hours", "site_altitude_m", "output_core",
                 "output_chunk_steps", "async_output", "output_queue_size", "save_tmrt", "save_svf",
                 "save_kup", "save_kdown", "save_lup", "save_ldown", "save_shadow", "dsm_wall_threshold_m",
                 "output_valid_mask", "wall_method", "building_geometry_path", "building_height_path",
                 "minimum_wall_height_m", "default_building_height_m", "level_height_m",
                 "minimum_building_height_m", "crs", "geotransform"}
        kwargs = {k: v for k, v in case.items() if k in known}
        run_timeseries(output_path=output, dtype=np.dtype(args.dtype), no_write=args.no_write,
                       progress=args.progress, pixel_size=pixel_size, form=args.form, **kwargs)
    if args.progress and not args.no_write:
        print(f"[{datetime.now():%H:%M:%S}] Results: {output}", flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
