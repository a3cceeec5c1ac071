"""Copies zk-gpu's golden vectors into this repository (run once, on a machine with a checkout of
the reference; the argument is that checkout's tests/golden directory).

    python tests/golden/import_reference_vectors.py <zk-gpu checkout>/tests/golden

The two files are the reference's own fixtures, tests/golden/ntt.json and tests/golden/msm.json,
generated by the reference's tools/golden/gen.mjs with ffjavascript 0.3.1 (bn128) and licensed
MIT OR Apache-2.0 like the reference. They are copied byte for byte; their SHA-256 digests are
pinned here and checked by tests/test_oracle.py.
"""
import hashlib
import pathlib
import shutil
import sys

DST = pathlib.Path(__file__).resolve().parent
FILES = ["ntt.json", "msm.json"]


def digest(path: pathlib.Path) -> str:
    return hashlib.sha256(path.read_bytes()).hexdigest()


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    SRC = pathlib.Path(sys.argv[1])
    if not SRC.is_dir():
        sys.exit(f"reference vectors not found under {SRC}")
    for name in FILES:
        shutil.copyfile(SRC / name, DST / name)
        print(name, digest(DST / name))
