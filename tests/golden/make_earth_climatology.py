"""Extracts the golden boundary fixture from the reference's packaged T21
inputs: the Earth surface-temperature (code 169) and ice-cover (code 210)
climatologies, January to December.

The reference ships them as ExoPlaSim .sra text inside
public/gcm/t21/inputs.json (14 records per code: December before, the twelve
months, January after; each record is 8 header integers and 64 x 32 values).
This script keeps the twelve months as float32 together with the source
file's SHA-256. Run it where the reference checkout is available:

    python tests/golden/make_earth_climatology.py /path/to/reference
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "earth_t21_climatology.npz")
POINTS = 64 * 32


def records(text):
    values = np.array(text.split(), dtype=np.float64)
    rec = values.reshape(-1, 8 + POINTS)
    assert rec.shape[0] == 14, rec.shape
    headers = rec[:, :8].astype(np.int64)
    assert (headers[:, 4] == 64).all() and (headers[:, 5] == 32).all()
    return headers, rec[:, 8:]


def main(reference):
    path = os.path.join(reference, "public", "gcm", "t21", "inputs.json")
    raw = open(path, "rb").read()
    files = json.loads(raw)["files"]
    out = {"source_sha256": np.frombuffer(hashlib.sha256(raw).digest(), dtype=np.uint8)}
    for code, key in (("0169", "sst"), ("0210", "ice")):
        headers, data = records(files[f"N032_surf_{code}.sra"])
        # records 1..12 are months 1..12 (dates YYYY0101 .. YYYY1201)
        assert [(h // 100) % 100 for h in headers[1:13, 2]] == list(range(1, 13))
        out[key] = data[1:13].astype(np.float32)
        out[key + "_dates"] = headers[:, 2]
    np.savez_compressed(OUT, **out)
    print(OUT, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_earth_climatology.py <path of the reference checkout>")
    main(sys.argv[1])
