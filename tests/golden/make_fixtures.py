# SPDX-License-Identifier: Apache-2.0
"""Writes the committed fixtures of tests/golden from the reference's own test data (run in a
checkout that has the reference at EDA_REFERENCE, default /root/reference; the tests only read
the fixtures, so the GPU box needs no reference):

- parity_inputs.npz / parity_expect.json: the inputs of the reference's parity manifest
  (tests/data/parity_v2.json of giorgioangel/eda-cuda), regenerated bit for bit by its
  tests/python/cases.py and checked against the manifest's input_sha256, for every case of at
  most MAX_SAMPLES samples, and per case the call's keywords and the manifest's recorded results
  (decisions, output hashes, conditioning class, sensitivity);
- corpus.npz / corpus.json: the reference's golden corpus (tests/data/golden): x, the recorded
  rows, windows, sifts, sensitivity and conditioning class of each case.
"""

from __future__ import annotations

import hashlib
import json
import math
import os
import sys
from pathlib import Path

import numpy as np

REF = Path(os.environ.get("EDA_REFERENCE", "/root/reference"))
OUT = Path(__file__).resolve().parent
MAX_SAMPLES = 20000
FIELDS = ("n_imfs", "error", "windows", "sifts", "windows_sha256", "sifts_sha256", "y_sha256", "rows_sha256",
          "spacing_sha256", "energy_sha256", "y_shape", "info_shape", "info_axes", "chunks", "conditioning_class",
          "sensitivity", "quick")


def main() -> None:
    sys.path.insert(0, str(REF / "tests" / "python"))
    import cases as C  # the reference's input generator

    manifest = json.loads((REF / "tests" / "data" / "parity_v2.json").read_text())
    want = {e["id"]: e for e in manifest["cases"]}
    inputs, expect = {}, {}
    for case in C.all_cases():
        r = case.recipe
        if math.prod(r.shape) > MAX_SAMPLES:
            continue
        x = case.input()
        assert hashlib.sha256(np.ascontiguousarray(x).tobytes()).hexdigest() == want[case.id]["input_sha256"]
        inputs[case.id] = x
        entry = {k: want[case.id][k] for k in FIELDS if k in want[case.id]}
        entry.update(case.kwargs())
        entry["axes"] = None if r.axes is None else list(r.axes)
        entry["max_chunk"] = r.max_chunk
        entry["shape"] = list(r.shape)
        expect[case.id] = entry
    np.savez_compressed(OUT / "parity_inputs.npz", **inputs)
    (OUT / "parity_expect.json").write_text(json.dumps(
        {"source": "giorgioangel/eda-cuda tests/data/parity_v2.json", "provenance": manifest["provenance"],
         "cases": expect}, indent=0, sort_keys=True))
    gdir = REF / "tests" / "data" / "golden"
    index = json.loads((gdir / "index.json").read_text())
    arrays, meta = {}, {}
    for name in sorted(index["cases"]):
        with np.load(gdir / f"{name}.npz", allow_pickle=False) as z:
            arrays[f"{name}.x"] = z["x"]
            arrays[f"{name}.modes"] = z["modes"]
            meta[name] = {"windows": [int(v) for v in z["windows"]], "sifts": [int(v) for v in z["sifts"]],
                          "sensitivity": float(z["sensitivity"]), "conditioning_class": str(z["conditioning_class"])}
    np.savez_compressed(OUT / "corpus.npz", **arrays)
    (OUT / "corpus.json").write_text(json.dumps(
        {"source": "giorgioangel/eda-cuda tests/data/golden", "cases": meta}, indent=1, sort_keys=True))
    print(f"{len(inputs)} parity cases, {len(meta)} corpus cases")


if __name__ == "__main__":
    main()
