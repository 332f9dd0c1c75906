#!/usr/bin/env python3
"""Generate tests/golden/routing_golden.json by running the reference routing.

Loads ``hybrid/src/fauxce_hybrid/routing.py`` of the reference from
``--reference`` (or the FAUXICE_REFERENCE environment variable: the
reference checkout's root directory) by file path (the module needs only
numpy and scipy) and records, for every case of route_cases.py, either the
raised exception (type and message) or the SHA-256 of the canonical JSON
census, the SHA-256 of the three planes (provisional labels, synthesis mask,
final labels, as C-order bytes) and, for small cases, the census itself.
Run once where the reference is present; the tests need only the JSON file.

Usage: python tests/golden/make_routing_golden.py
"""

from __future__ import annotations

import argparse
import hashlib
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "routing_golden.json")
sys.path.insert(0, HERE)

import route_cases  # noqa: E402


def sha(data: bytes) -> str:
    return hashlib.sha256(data).hexdigest()


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("FAUXICE_REFERENCE"),
                        help="the reference checkout's root directory")
    args = parser.parse_args()
    if not args.reference:
        parser.error("give --reference or set FAUXICE_REFERENCE")
    path = os.path.join(args.reference, "hybrid", "src", "fauxce_hybrid", "routing.py")
    spec = importlib.util.spec_from_file_location("reference_routing", path)
    ref = importlib.util.module_from_spec(spec)
    sys.modules["reference_routing"] = ref
    spec.loader.exec_module(ref)

    results = {}
    for name in route_cases.CASES:
        mask = route_cases.mask(name)
        policy = ref.RoutingPolicy(**route_cases.policy_kwargs(name))
        t0 = time.perf_counter()
        try:
            result = ref.route_at_floor_mask(mask, policy)
        except Exception as exc:  # recorded, not raised
            results[name] = {"error": type(exc).__name__, "message": str(exc),
                             "mask_sha256": sha(mask.tobytes())}
            print(f"{name}: {type(exc).__name__}")
            continue
        doc = ref.serialize_routing_json(result)
        entry = {
            "mask_sha256": sha(mask.tobytes()),
            "json_sha256": sha(doc),
            "provisional_labels_sha256": sha(result.provisional_labels.tobytes()),
            "synthesis_mask_sha256": sha(result.synthesis_mask.tobytes()),
            "final_labels_sha256": sha(result.final_labels.tobytes()),
            "provisional_regions": len(result.provisional_regions),
            "final_regions": len(result.final_regions),
            "synthesis_pixels": result.synthesis_pixel_count,
            "within_synthesis_budget": result.within_synthesis_budget,
        }
        if len(doc) <= 16384:
            entry["json"] = doc.decode("utf-8")
        results[name] = entry
        print(f"{name}: {len(result.provisional_regions)} regions, "
              f"{len(result.final_regions)} final, {time.perf_counter() - t0:.2f} s")
    with open(OUT, "w") as handle:
        json.dump({"reference": "hybrid/src/fauxce_hybrid/routing.py", "cases": results},
                  handle, indent=1, sort_keys=True)
        handle.write("\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
