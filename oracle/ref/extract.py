"""Build step of the oracle/_ref recipe (test infrastructure only).

Copies named function definitions out of the reference's own CUDA sources into a
generated translation unit under oracle/_ref/ so they can be compiled for the host.
Functions are located by their signature line and closed by brace matching; the
generated file is a build artefact (git-ignored) and is never committed.

    python extract.py <reference root> <out.cpp>

Extracted (paths relative to the reference root):
  src/collisionCheck/spatialHash.cu : isMotionValidSpatialHash   (spatialHash.cu:145-194)
  src/graphs/Graph.cu               : getRegion, getSubRegion    (Graph.cu:99-205)
  src/helper/helper.cu              : readObstaclesFromCSV       (helper.cu:13-39)
"""
import re
import sys
from pathlib import Path

FUNCTIONS = [
    ("src/collisionCheck/spatialHash.cu", r"^__device__ bool isMotionValidSpatialHash\("),
    ("src/graphs/Graph.cu", r"^__host__ __device__ int getRegion\(float\* coord\)"),
    ("src/graphs/Graph.cu", r"^__device__ int getSubRegion\(float\* coord, int r1, float\* minRegion\)"),
    ("src/helper/helper.cu", r"^std::vector<float> readObstaclesFromCSV\("),
]


def extract(path: Path, anchor: str) -> str:
    lines = path.read_text().splitlines()
    pat = re.compile(anchor)
    for start, line in enumerate(lines):
        if pat.search(line):
            break
    else:
        raise SystemExit(f"anchor {anchor!r} not found in {path}")
    depth, seen_open, out = 0, False, []
    for i in range(start, len(lines)):
        out.append(lines[i])
        depth += lines[i].count("{") - lines[i].count("}")
        seen_open = seen_open or "{" in lines[i]
        if seen_open and depth == 0:
            return f'#line {start + 1} "{path}"\n' + "\n".join(out) + "\n"
    raise SystemExit(f"unbalanced braces after {anchor!r} in {path}")


def main() -> None:
    root, out = Path(sys.argv[1]), Path(sys.argv[2])
    parts = [
        "// generated by oracle/ref/extract.py from the reference sources; do not edit\n",
        '#include "statePropagator/statePropagatorSpatialHash.cuh"\n',
        "#include <fstream>\n#include <iostream>\n#include <sstream>\n#include <string>\n#include <vector>\n",
    ]
    for rel, anchor in FUNCTIONS:
        parts.append(extract(root / rel, anchor))
    out.parent.mkdir(parents=True, exist_ok=True)
    out.write_text("".join(parts))


if __name__ == "__main__":
    main()
