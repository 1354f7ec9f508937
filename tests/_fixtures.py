"""Loads the reference's golden test cases committed under tests/golden/
(see tests/golden/make_fixtures.py) into plain numpy arrays."""
import gzip
import os

import numpy as np

from lb3d_b200.config import read_input

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Compile-time mixture of each reference test (test/<T>/<T>.cfg FLAGS):
# -DNOSURFACTANT builds are binary.
CASES = {"gyroid": 3, "bodyForce": 3, "leesEdwards": 2, "wettingWall": 2, "zouHe": 3}
FIELDS = {
    "gyroid": ["od", "wd", "sur", "dir", "vel", "arr"],
    "bodyForce": ["od", "wd", "sur", "dir", "vel", "arr"],
    "leesEdwards": ["od", "wd", "vel", "arr"],
    "wettingWall": ["od", "wd", "vel", "arr", "rock"],
    "zouHe": ["od", "wd", "sur", "dir", "vel", "arr"],
}
STAMP = "t00000000-0000000000"


def read_gz(path):
    with gzip.open(path + ".gz", "rb") as f:
        return f.read()


def load_case(name):
    """Returns (params, state) with state = dict(n, db, rock, shear_sum)
    restored as init_cond = 7 does (code/lb3d_io_checkpoint.F90:878-1106,
    then the obstacle file, code/lb3d_ic_rock.F90:50-77)."""
    d = os.path.join(GOLDEN, name)
    nc = CASES[name]
    p = read_input(os.path.join(d, f"{name}.in"), os.path.join(d, "dump_xdr.din"), ncomp=nc)
    nd = 64 if nc == 3 else 39
    raw = read_gz(os.path.join(d, f"checkpoint_{name}_{STAMP}_p000000.xdr"))
    cp = np.frombuffer(raw, ">f8").reshape(p.nx, p.ny, p.nz, nd)  # x outer, z inner
    cp = np.ascontiguousarray(cp.transpose(2, 1, 0, 3)).astype(np.float64)  # -> [z][y][x][nd]
    n = np.ascontiguousarray(cp[..., : 19 * nc].reshape(p.nz, p.ny, p.nx, nc, 19).transpose(3, 4, 0, 1, 2))
    db = np.ascontiguousarray(cp[..., 60:63].transpose(3, 0, 1, 2)) if nc == 3 else None
    rock = np.ascontiguousarray(cp[..., nd - 1])
    topo = read_gz(os.path.join(d, f"checktopo_{name}_{STAMP}.xdr"))
    shear_sum = float(np.frombuffer(topo[24:32], ">f8")[0]) if len(topo) >= 32 else 0.0
    if p.has_rock_file:
        w = np.frombuffer(read_gz(os.path.join(d, p.obs_file.strip())), ">f4")
        rock = (w.reshape(p.nz, p.ny, p.nx) > 0.0).astype(np.float64)
    return p, dict(n=n, db=db, rock=rock, shear_sum=shear_sum)


def load_golden(name, field, t=10):
    d = os.path.join(GOLDEN, name)
    raw = read_gz(os.path.join(d, f"{field}_{name}.reference-t{t:08d}.xdr"))
    return np.frombuffer(raw, ">f4").astype(np.float32)
