"""Generate the golden fixtures of tests/golden/ from the reference's OWN code.

    python tests/golden/make_golden.py          (needs the reference tree and g++)

Builds oracle/_ref/ref_dump (`make -C oracle ref`: the reference's mesh, ogs,
primitives and core sources compiled where they lie, against the host-only
shims of oracle/ref_shim/) and runs it on the cases below, each with the
reference's own command-line keys.  Every record the dump writes (numbering,
CSR, basis, geometric factors, cubature data, and the reference's host ogs
Gather/Scatter applied to seeded vectors) is stored in ref_<name>.npz (the integer records of the full-size case as
SHA-256 digests of their bytes).  The
GPU box has no reference tree: tests read only the committed .npz files.
"""
import hashlib
import os
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_dump")

# name: (Nfields, seed, reference command line, integer records only)
CASES = {
    "hex_3x3x2_p5": (1, 5, "-nx 3 -ny 3 -nz 2 -p 5", False),
    "hex_2x2x2_p7": (1, 7, "-nx 2 -ny 2 -nz 2 -p 7", False),
    "hex_4x3x2_p3_affine": (1, 3, "-nx 4 -ny 3 -nz 2 -p 3 -a", False),
    "hex_3x2x2_p4_nf3": (3, 4, "-nx 3 -ny 2 -nz 2 -p 4", False),
    "hex_2x1x1_p15": (1, 15, "-nx 2 -ny 1 -nz 1 -p 15", False),
    "hex_2x2x2_p1": (1, 1, "-nx 2 -ny 2 -nz 2 -p 1", False),
    # the BP5 p=4 box of 16^3 affine elements (250,047 unknowns): numbering and CSR at full size
    "hex_16x16x16_p4_affine": (1, 0, "-nx 16 -ny 16 -nz 16 -p 4 -a", True),
    # Quad2D boxes (-e Quad; BP6 has Nfields = dim = 2 there)
    "quad_3x2_p4": (1, 4, "-e Quad -nx 3 -ny 2 -p 4", False),
    "quad_4x3_p7_affine": (1, 7, "-e Quad -nx 4 -ny 3 -p 7 -a", False),
    "quad_3x3_p5_nf2": (2, 5, "-e Quad -nx 3 -ny 3 -p 5", False),
    "quad_2x2_p15": (1, 15, "-e Quad -nx 2 -ny 2 -p 15", False),
    "quad_64x48_p6": (1, 0, "-e Quad -nx 64 -ny 48 -p 6", True),
    # Tri2D boxes (-e Tri, affine: two triangles per cell)
    "tri_3x2_p4": (1, 4, "-e Tri -nx 3 -ny 2 -p 4 -a", False),
    "tri_4x3_p7": (1, 7, "-e Tri -nx 4 -ny 3 -p 7 -a", False),
    "tri_2x2_p1": (1, 1, "-e Tri -nx 2 -ny 2 -p 1 -a", False),
    "tri_2x2_p15": (1, 15, "-e Tri -nx 2 -ny 2 -p 15 -a", False),
    "tri_5x4_p3": (1, 3, "-e Tri -nx 5 -ny 4 -p 3 -a", False),
    "tri_96x80_p5": (1, 0, "-e Tri -nx 96 -ny 80 -p 5 -a", True),
    # Tet3D boxes (-e Tet, affine: six tetrahedra per cell)
    "tet_2x2x1_p3": (1, 3, "-e Tet -nx 2 -ny 2 -nz 1 -p 3 -a", False),
    "tet_3x2x2_p4": (1, 4, "-e Tet -nx 3 -ny 2 -nz 2 -p 4 -a", False),
    "tet_2x1x2_p1": (1, 1, "-e Tet -nx 2 -ny 1 -nz 2 -p 1 -a", False),
    "tet_2x2x2_p7": (1, 7, "-e Tet -nx 2 -ny 2 -nz 2 -p 7 -a", False),
    "tet_12x10x8_p3": (1, 0, "-e Tet -nx 12 -ny 10 -nz 8 -p 3 -a", True),
}
INT_RECORDS = {"N", "Nq", "Np", "Nelements", "Nfields", "Ngather", "NgatherGlobal", "cubNq", "GlobalToLocal",
               "rowStartsT", "colIdsT", "rowStartsN", "colIdsN", "gllz", "gllw", "D"}


def read_dump(path):
    out = {}
    b = open(path, "rb").read()
    o = 0
    while o < len(b):
        n, = struct.unpack_from("<I", b, o)
        o += 4
        name = b[o:o + n].decode()
        o += n
        t = chr(b[o])
        o += 1
        c, = struct.unpack_from("<Q", b, o)
        o += 8
        dt = {"i": np.int32, "l": np.int64, "d": np.float64}[t]
        a = np.frombuffer(b, dtype=dt, count=c, offset=o).copy()
        o += c * a.itemsize
        out[name] = a
    return out


def main():
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-s", "-j8", "ref"], check=True)
    only = sys.argv[1:]   # optional name prefixes: regenerate only those cases
    for name, (nf, seed, cli, ints_only) in CASES.items():
        if only and not any(name.startswith(p) for p in only):
            continue
        tmp = os.path.join(ROOT, "oracle", "_ref", name + ".bin")
        subprocess.run([DUMP, tmp, str(nf), str(seed)] + cli.split(), check=True)
        d = read_dump(tmp)
        if name.startswith(("tri", "tet")):   # the simplex BP5 paths use no cubature data
            d = {k: v for k, v in d.items() if not k.startswith("cub")}
        if ints_only:
            # full-size integer records as SHA-256 digests of their little-endian
            # bytes (a bit-exact check without a large fixture), small ones as arrays
            small = {k: v for k, v in d.items() if k in INT_RECORDS and v.size <= 1024}
            for k, v in d.items():
                if k in INT_RECORDS and v.size > 1024:
                    small["sha256_" + k] = np.array(hashlib.sha256(v.astype(v.dtype.newbyteorder("<")).tobytes())
                                                    .hexdigest())
                    small["size_" + k] = np.array(v.size)
            d = small
        d["cli"] = np.array(cli)
        np.savez_compressed(os.path.join(HERE, "ref_%s.npz" % name), **d)
        print("%-26s %s" % (name, ", ".join("%s[%d]" % (k, v.size) for k, v in d.items() if k != "cli")))


if __name__ == "__main__":
    sys.exit(main())
