"""Extracts the reference's packaged T21 input texts as a fixture for the
format tests: every namelist file and the SST (code 169) and ice-cover
(code 210) .sra files of public/gcm/t21/inputs.json, unchanged, with the
source file's SHA-256. Run it where the reference checkout is available:

    python tests/golden/make_reference_inputs.py /path/to/reference
"""
import gzip
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "reference_inputs_t21.json.gz")
KEEP = ("N032_surf_0169.sra", "N032_surf_0210.sra")


def main(reference):
    raw = open(os.path.join(reference, "public", "gcm", "t21", "inputs.json"), "rb").read()
    files = json.loads(raw)["files"]
    out = {k: v for k, v in sorted(files.items()) if k.endswith("_namelist") or k in KEEP}
    doc = {"source_sha256": hashlib.sha256(raw).hexdigest(), "files": out}
    with gzip.open(OUT, "wt", encoding="utf-8") as f:
        json.dump(doc, f)
    print(OUT, len(out), "files")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_reference_inputs.py <path of the reference checkout>")
    main(sys.argv[1])
