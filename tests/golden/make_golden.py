"""Regenerates tests/golden/ from the reference's own test resources.

Run in a container where the reference tree is mounted:

    python tests/golden/make_golden.py <reference checkout>

It copies the reference's test fixtures (gpjson/src/test/resources/, BSD-3
licensed, Copyright (c) 2021 Koen Vlaswinkel) into tests/golden/fixtures/ so
the GPU tests can read them on machines without the reference, and writes
tests/golden/expected.json with the oracle's outputs on each fixture:
newline index, string index and 16 leveled bitmaps (the configuration of
LeveledBitmapsIndexTest.java:32, MAX_NUM_LEVELS), as full arrays for small
fixtures and as SHA-256 digests for the larger ones.
"""

from __future__ import annotations

import hashlib
import json
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from oracle import oracle  # noqa: E402

RESOURCES = "gpjson/src/test/resources"
FIXTURES = [
    "query_gpu_function/simple_single_line.ldjson",
    "query_gpu_function/not_found_in_current_level.ldjson",
    "stages/string_index/simple.txt",
    "stages/string_index/escape_carry.txt",
    "stages/string_index/very_long_string.txt",
    "stages/newline_index/even_positions.txt",
    "stages/newline_index/odd_positions.txt",
    "stages/newline_index/random_data.txt",
    "stages/newline_index/aligned_random_data.txt",
    "stages/leveled_bitmaps_index/simple.json",
    "stages/leveled_bitmaps_index/boundary.json",
]
FULL_ARRAY_LIMIT = 8192  # bytes of input below which arrays are stored in full


def digest(a) -> str:
    return hashlib.sha256(a.tobytes()).hexdigest()


def main(reference_root: str) -> None:
    src_root = Path(reference_root) / RESOURCES
    dst_root = HERE / "fixtures"
    expected = {}
    for rel in FIXTURES:
        src = src_root / rel
        dst = dst_root / rel
        dst.parent.mkdir(parents=True, exist_ok=True)
        shutil.copyfile(src, dst)
        data = dst.read_bytes()
        idx = oracle.Index(data, 16)
        entry = {
            "bytes": len(data),
            "sha256": hashlib.sha256(data).hexdigest(),
            "lines": int(len(idx.newlines)),
            "newline_sha256": digest(idx.newlines),
            "string_sha256": digest(idx.strings),
            "levels16_sha256": digest(idx.levels),
        }
        if len(data) <= FULL_ARRAY_LIMIT:
            entry["newline_index"] = [int(x) for x in idx.newlines]
            entry["string_index"] = [f"{int(x):016x}" for x in idx.strings]
            entry["levels16"] = [[f"{int(x):016x}" for x in row] for row in idx.levels]
        expected[rel] = entry
    (HERE / "expected.json").write_text(json.dumps(expected, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(expected)} fixtures")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout>")
    main(sys.argv[1])
