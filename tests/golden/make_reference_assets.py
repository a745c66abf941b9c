"""Copies the reference's shipped configuration and mesh files used by the
drop-in tests into ``tests/golden/reference_assets/``, gzip-compressed and
unmodified, and writes ``MANIFEST.json`` with each file's origin, size and
SHA-256 of the uncompressed bytes.

The files are FreeFlow's own data (MIT licence with the Commons Clause,
copyright Changyu Hu): two 2D configurations and the two 2D Medit meshes they
name.  They are read from the reference tree (``FFS_REFERENCE_TREE``, by
default /root/reference); the tests only read the copies.

    python tests/golden/make_reference_assets.py
"""
import gzip
import hashlib
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "reference_assets")
REF = os.environ.get("FFS_REFERENCE_TREE", "/root/reference")
FILES = [
    "assets/configs/vortexstreet2d.json",
    "assets/configs/fish2d_lbs_control.json",
    "assets/mesh/fish2d.mesh",
    "assets/mesh/sphere2d.mesh",
]


def main():
    os.makedirs(OUT, exist_ok=True)
    manifest = {"origin": "FreeFlow (changyu-hu/FreeFlow), files copied unmodified",
                "licence": "MIT with Commons Clause (non-commercial use), copyright Changyu Hu",
                "files": {}}
    for rel in FILES:
        with open(os.path.join(REF, rel), "rb") as f:
            data = f.read()
        name = os.path.basename(rel)
        # mtime=0 keeps the compressed bytes reproducible
        with open(os.path.join(OUT, name + ".gz"), "wb") as f:
            f.write(gzip.compress(data, compresslevel=9, mtime=0))
        manifest["files"][name] = {"source": rel, "bytes": len(data), "sha256": hashlib.sha256(data).hexdigest()}
    with open(os.path.join(OUT, "MANIFEST.json"), "w") as f:
        json.dump(manifest, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
