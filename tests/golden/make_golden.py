"""Extract the reference's golden receiver traces into small committed fixtures.

The reference keeps its experiment results only in its SVN working-copy store:
.svn/wc.db maps each file path to a sha1, and .svn/pristine/<aa>/<sha1>.svn-base
holds the bytes.  The *.hh files are RSF "header + data" files: a text header of
key=value lines, the separator bytes 0x0c 0x0c 0x04, then little-endian float32.

Run once where the reference checkout is available:
    python tests/golden/make_golden.py <reference checkout>
(or with $ECSG_REFERENCE naming the checkout).
Writes tests/golden/<name>.npy (float32, shape (n2, n1): one row per receiver)
and tests/golden/golden_index.json (headers and provenance).
"""
import json
import os
import sqlite3
import sys

import numpy as np

WANT = {
    "rec_eci_test1": "tests/test1-cmp-eci-ii/Fig/tests/test1-cmp-eci-ii/eci/rec_eci_test1.hh",
    "rec_eci_test2": "tests/test1-cmp-eci-ii/Fig/tests/test1-cmp-eci-ii/eci/rec_eci_test2.hh",
    "rec_eci_test3": "tests/test1-cmp-eci-ii/Fig/tests/test1-cmp-eci-ii/eci/rec_eci_test3.hh",
    "rec_ii_test1": "tests/test1-cmp-eci-ii/Fig/tests/test1-cmp-eci-ii/ii/rec_ii_test1.hh",
    "rec_ii_test2": "tests/test1-cmp-eci-ii/Fig/tests/test1-cmp-eci-ii/ii/rec_ii_test2.hh",
    "rec_ii_test3": "tests/test1-cmp-eci-ii/Fig/tests/test1-cmp-eci-ii/ii/rec_ii_test3.hh",
    "geo_eci_test1": "tests/test1-cmp-eci-ii/Fig/tests/test1-cmp-eci-ii/eci/geo_eci_test1.hh",
}


def parse_rsf(blob):
    sep = blob.find(b"\x0c\x0c\x04")
    if sep < 0:
        raise ValueError("no inline data")
    head = blob[:sep].decode("latin-1")
    kv = {}
    for tok in head.replace("\n", " ").replace("\t", " ").split(" "):
        if "=" in tok:
            k, v = tok.split("=", 1)
            kv[k] = v.strip('"')
    data = np.frombuffer(blob[sep + 3:], dtype="<f4")
    n1 = int(kv["n1"])
    n2 = int(kv.get("n2", "1"))
    return kv, data[: n1 * n2].reshape(n2, n1)


def main(ref_root):
    out_dir = os.path.dirname(os.path.abspath(__file__))
    db = sqlite3.connect("file:%s?mode=ro" % os.path.join(ref_root, ".svn", "wc.db"), uri=True)
    index = {}
    for name, rel in WANT.items():
        row = db.execute("select checksum from NODES where local_relpath = ?", (rel,)).fetchone()
        sha = row[0].split("$")[-1]
        path = os.path.join(ref_root, ".svn", "pristine", sha[:2], sha + ".svn-base")
        with open(path, "rb") as fh:
            kv, arr = parse_rsf(fh.read())
        np.save(os.path.join(out_dir, name + ".npy"), arr.astype(np.float32))
        index[name] = {"source": rel, "sha1": sha,
                       "header": {k: kv[k] for k in ("n1", "d1", "o1", "n2") if k in kv}}
    with open(os.path.join(out_dir, "golden_index.json"), "w") as fh:
        json.dump(index, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ECSG_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <reference checkout>  (or set ECSG_REFERENCE)")
    main(ref)
