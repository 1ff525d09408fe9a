"""Generate ``building_heights.json`` from the reference itself.

The reference's ``src/walls.py`` imports rasterio and shapely at module level,
which this image lacks, so the module cannot be imported.  Its building-height
rules (``_geometry_positive``, ``_numbers``, ``_length_metres`` and
``building_height``, ``src/walls.py:145-205``) are plain Python, so this
script reads the file, takes exactly those function definitions and the
module constants they use (``_NUMBER_RE``, ``_HEIGHT_KEYS``, ``_LEVEL_KEYS``)
with ``ast``, executes them in a namespace with ``re`` and ``math``, and
records their results on a set of GeoJSON property dicts:

    python tests/golden/make_building_heights.py

(reference tree: ``/root/reference``, override with SOLWEIG_REFERENCE_TREE).
"""
from __future__ import annotations

import ast
import json
import math
import os
import re
from typing import Any, Mapping

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("SOLWEIG_REFERENCE_TREE", "/root/reference")
WANTED = {"_geometry_positive", "_numbers", "_length_metres", "building_height",
          "_NUMBER_RE", "_HEIGHT_KEYS", "_LEVEL_KEYS"}

CASES = [
    {}, {"height": 12}, {"height": "12.5"}, {"height": "12,5 m"}, {"height": "40 ft"},
    {"height": "30'"}, {"height": "10-14"}, {"height": "10 to 16 m"}, {"height": "8;11;9"},
    {"height": "yes"}, {"height": "nan"}, {"height": -3}, {"height": 0}, {"height": 1.2},
    {"height": None}, {"height": "abc"}, {"building:height": "7 m"}, {"est_height": 22.0},
    {"building:part:height": "5"}, {"height": "", "building:levels": 4},
    {"building:levels": "3"}, {"levels": "2-5"}, {"building_levels": "0"}, {"building:levels": -2},
    {"building:levels": "4;6"}, {"height": "none", "levels": 3}, {"height": float("inf")},
    {"height": "1e3"}, {"height": "15 feet"}, {"height": "6.0;x;8 ft"}, {"roof": "flat"},
    {"height": True}, {"building:levels": 1.5}, {"height": "12 m", "building:levels": 40},
]
OPTIONS = [dict(), dict(default_height_m=9.0, level_height_m=3.5, minimum_height_m=4.0),
           dict(default_height_m=1.0, level_height_m=2.0, minimum_height_m=0.5)]


def _reference_namespace():
    source = open(os.path.join(REF, "src", "walls.py"), encoding="utf-8").read()
    tree = ast.parse(source)
    keep = []
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name in WANTED:
            keep.append(node)
        elif isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id in WANTED for t in node.targets):
            keep.append(node)
    module = ast.Module(body=keep, type_ignores=[])
    ns = {"re": re, "math": math, "Any": Any, "Mapping": Mapping}
    exec(compile(module, "src/walls.py", "exec"), ns)
    return ns


def main():
    ns = _reference_namespace()
    records = []
    for props in CASES:
        for opts in OPTIONS:
            records.append({"properties": {k: (repr(v) if isinstance(v, float) and not math.isfinite(v) else v)
                                           for k, v in props.items()},
                            "options": opts, "height": ns["building_height"](props, **opts)})
    lengths = ["12", "12,5", "3 ft", "10 - 12 m", "5 to 7", "a;b", "2;x;3'", "", "-4", "0.5"]
    out = {"building_height": records,
           "length_metres": [{"value": v, "metres": ns["_length_metres"](v)} for v in lengths]}
    path = os.path.join(HERE, "building_heights.json")
    with open(path, "w", encoding="utf-8") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(f"wrote {path}: {len(records)} building heights")


if __name__ == "__main__":
    main()
