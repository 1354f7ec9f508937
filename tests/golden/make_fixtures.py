"""Regenerates the golden fixtures under tests/golden/ from the reference's
own integration tests (testLB3D.sh, test/<T>/).

For each test T in gyroid, bodyForce, leesEdwards, wettingWall, zouHe the reference
ships a t=0 checkpoint (checkpoint_*, checktopo_*, checkparams_* XDR files),
the input file T.in with its dump_xdr.din override, an obstacle file where
the test uses one, and the FP32 XDR dumps at t=10 (reference/*-t00000010.xdr)
that testLB3D.sh:280-300 compares byte for byte.  This script copies those
data files, gzip-compressed, into tests/golden/T/ so that the tests run
without the reference tree.  Run it from the repository root:

    python tests/golden/make_fixtures.py /path/to/reference
"""
import gzip
import os
import shutil
import sys

TESTS = ["gyroid", "bodyForce", "leesEdwards", "wettingWall", "zouHe"]
HERE = os.path.dirname(os.path.abspath(__file__))


def _copy_gz(src, dst):
    with open(src, "rb") as fi, open(dst + ".gz", "wb") as raw:
        with gzip.GzipFile(filename="", mode="wb", compresslevel=9, fileobj=raw, mtime=0) as fo:
            shutil.copyfileobj(fi, fo)


def main(ref_root):
    for t in TESTS:
        src = os.path.join(ref_root, "test", t)
        dst = os.path.join(HERE, t)
        os.makedirs(dst, exist_ok=True)
        for name in (f"{t}.in", "dump_xdr.din"):
            shutil.copyfile(os.path.join(src, name), os.path.join(dst, name))
        cpdir = os.path.join(src, "checkpoint")
        for name in sorted(os.listdir(cpdir)):
            _copy_gz(os.path.join(cpdir, name), os.path.join(dst, name))
        refdir = os.path.join(src, "reference")
        for name in sorted(os.listdir(refdir)):
            if name.endswith(".xdr"):
                _copy_gz(os.path.join(refdir, name), os.path.join(dst, name))
        for name in sorted(os.listdir(src)):
            if name.endswith(".xdr"):  # obstacle file (wettingWall.wall.xdr)
                _copy_gz(os.path.join(src, name), os.path.join(dst, name))
        print(t, sorted(os.listdir(dst)))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <reference checkout (contains test/)>")
    main(sys.argv[1])
