"""Record the SHA-256 of the model blob that the MJCF compiler makes from
each of the reference's own asset files (assets/*.xml of the reference
repository), into reference_blobs.json.

Run where the reference repository is checked out:
    python tests/golden/make_blob_hashes.py <reference checkout>
(or with PIPPIN_REFERENCE set). The JSON is committed, so that
tests/test_mjcf.py can check the generated workload models against the
reference's assets without a reference checkout.
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from pippin_b200 import mjcf, scenes  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PIPPIN_REFERENCE", "")
OUT = os.path.join(HERE, "reference_blobs.json")


def main():
    if not REF:
        sys.exit("usage: make_blob_hashes.py <reference checkout>  (or set PIPPIN_REFERENCE)")
    out = {}
    for asset in sorted(scenes.REFERENCE_ASSETS):
        blob = mjcf.compile_file(os.path.join(REF, "assets", asset))
        out[asset] = {"sha256": hashlib.sha256(blob).hexdigest(), "bytes": len(blob), "source": f"assets/{asset}"}
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
        fh.write("\n")
    print(f"wrote {OUT} ({len(out)} assets)")


if __name__ == "__main__":
    main()
