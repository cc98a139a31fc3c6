"""Regenerate the golden fixtures from the reference's own code.

Builds the reference harnesses under oracle/_ref (oracle/Makefile, target
``ref``: they compile the reference's fem_interface.h/serialization.h, its
SPGrid core and its stiffness-table headers where they lie in the reference
tree) and records their outputs here:

* kat_inputs.bin.gz / kat_outputs.bin.gz: FEMInputs/FEMOutputs blobs written by
  the reference serializer with the values of the reference's interface test;
* kat_inputs.txt / kat_outputs.txt: the reference reader's dump of those blobs;
* spgrid_order.npz: block bases and the page order the reference's page map
  iterates them in, for several grids;
* spgrid_offsets.npz: element offsets and the (4,4,8)-origin level maps;
* stiffness_tables.npy: K_mu, K_la, Km_cell, Kl_cell;
* driver_order.npz: block bases and the order of the optimizer driver's 4x4x4
  page map (the lists its thin/fat/fatter maps hold).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import gzip
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def run(*args, **kw):
    return subprocess.run(list(args), check=True, capture_output=True, text=True, **kw).stdout


def main() -> None:
    run("make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref")
    codec = os.path.join(REF_DIR, "codec_harness")
    spgrid = os.path.join(REF_DIR, "spgrid_harness")
    with tempfile.TemporaryDirectory() as tmp:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        run(codec, "kat", fin, fout)
        for src, name in ((fin, "kat_inputs"), (fout, "kat_outputs")):
            with open(src, "rb") as f, open(os.path.join(HERE, name + ".bin.gz"), "wb") as raw:
                with gzip.GzipFile(fileobj=raw, mode="wb", mtime=0) as g:
                    g.write(f.read())
        with open(os.path.join(HERE, "kat_inputs.txt"), "w") as f:
            f.write(run(codec, "dump-in", fin))
        with open(os.path.join(HERE, "kat_outputs.txt"), "w") as f:
            f.write(run(codec, "dump-out", fout))

        rng = np.random.default_rng(20181201)
        order = {}
        for case, (size, n) in enumerate(((64, 40), (256, 400), (1024, 800))):
            bi = rng.integers(1, size // 4 - 2, n)
            bj = rng.integers(1, size // 4 - 2, n)
            bk = rng.integers(1, size // 8 - 2, n)
            bases = np.unique(np.stack([bi * 4, bj * 4, bk * 8], 1), axis=0)
            bases = bases[rng.permutation(len(bases))].astype(np.int32)
            cf = os.path.join(tmp, "c.txt")
            np.savetxt(cf, bases, fmt="%d")
            out = np.loadtxt(run(spgrid, "order", str(size), cf).splitlines(), dtype=np.int32).reshape(-1, 3)
            order[f"size{case}"] = np.array([size])
            order[f"bases{case}"] = bases
            order[f"ordered{case}"] = out
        np.savez_compressed(os.path.join(HERE, "spgrid_order.npz"), **order)

        coords = np.concatenate([rng.integers(8, 200, (300, 3)), np.array([[8, 8, 8], [9, 9, 9], [15, 15, 15]])]).astype(np.int32)
        cf = os.path.join(tmp, "o.txt")
        np.savetxt(cf, coords, fmt="%d")
        rows = np.array([[int(v) for v in line.split()] for line in run(spgrid, "offsets", cf).splitlines()], dtype=np.int64)
        np.savez_compressed(os.path.join(HERE, "spgrid_offsets.npz"), coords=rows[:, 0:3], offset=rows[:, 3].astype(np.uint64),
                            down=rows[:, 4:7], up=rows[:, 7:10])

        tf = os.path.join(tmp, "t.bin")
        run(spgrid, "tables", tf)
        tables = np.fromfile(tf, np.float64).reshape(4, 576)
        np.save(os.path.join(HERE, "stiffness_tables.npy"), tables)

        # block order of the optimizer driver's 4x4x4 grid (its page-map lists)
        rng4 = np.random.default_rng(20181202)
        order4 = {}
        for case, (size, n) in enumerate(((64, 60), (512, 3000))):
            b = rng4.integers(2, size // 4 - 2, (n, 3))
            bases = np.unique(b * 4, axis=0)
            bases = bases[rng4.permutation(len(bases))].astype(np.int32)
            cf = os.path.join(tmp, "c4.txt")
            np.savetxt(cf, bases, fmt="%d")
            out = np.loadtxt(run(spgrid, "order4", str(size), cf).splitlines(), dtype=np.int32).reshape(-1, 3)
            order4[f"size{case}"] = np.array([size])
            order4[f"bases{case}"] = bases
            order4[f"ordered{case}"] = out
        np.savez_compressed(os.path.join(HERE, "driver_order.npz"), **order4)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
