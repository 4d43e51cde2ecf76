"""Writes batch64_digest.json: a digest of the 64-member batched workload drawn by
h2_b200.batch.draw_batch (seed 1000 + i per member), so that a change of the generator, of
numpy's PCG64 stream or of the drawing order shows up as a test failure.

    python tests/golden/make_batch_spec.py
"""
import hashlib
import json
import os
import struct
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", ".."))

from h2_b200 import batch as B  # noqa: E402


def digest(members):
    out = []
    for m in members:
        h = hashlib.sha256()
        for s in m.hotspots:
            h.update(struct.pack("<i5d", s.die, s.x0, s.x1, s.y0, s.y1, s.q))
        out.append({"index": m.index, "seed": m.seed, "nx": m.nx,
                    "per_die": [sum(1 for s in m.hotspots if s.die == d) for d in range(3)],
                    "q_sum": sum(s.q for s in m.hotspots), "sha256": h.hexdigest()})
    return out


if __name__ == "__main__":
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "batch64_digest.json")
    with open(path, "w") as f:
        json.dump(digest(B.draw_batch(64, 1000)), f, indent=0)
    print(path)
