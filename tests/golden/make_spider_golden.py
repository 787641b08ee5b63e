"""Golden SPIDER particle stacks and the reference's reconstruction from them.

The ctf16 golden dataset (ds_ctf16.npz) is written out as MRC stacks, each
stack is converted to SPIDER by the reference's own writer
(oracle/_ref/convert_probe: read_img + write_img, bsoft/src/rwimg/
rwSPIDER.cpp), the STAR project is pointed at the .spi files, and the
reference's breconstruct reconstructs from them.  spider.npz keeps the .spi
files' bytes, the STAR text and the reference's map.

    python tests/golden/make_spider_golden.py
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from bsoft_b200.io import mrc  # noqa: E402
from tests.helpers import materialize_dataset  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))
OPTIONS = "-interp trilinear -CTF flip"


def main():
    if not os.path.exists(os.path.join(REF, "convert_probe")):
        sys.exit("build the reference first: make -C oracle ref")
    with tempfile.TemporaryDirectory() as d:
        star = materialize_dataset("ctf16", d)
        files = {}
        for m in sorted(glob.glob(os.path.join(d, "*.mrcs"))):
            spi = m[:-5] + ".spi"
            subprocess.run([os.path.join(REF, "convert_probe"), m, spi], check=True)
            with open(spi, "rb") as f:
                files[os.path.basename(spi)] = np.frombuffer(f.read(), dtype=np.uint8)
            os.remove(m)
        with open(star) as f:
            text = f.read().replace(".mrcs", ".spi")
        with open(star, "w") as f:
            f.write(text)
        subprocess.run(f"{REF}/breconstruct {OPTIONS} -threads 2 -recon ref.mrc particles.star", cwd=d, shell=True,
                       check=True, capture_output=True, env=dict(os.environ, OMP_NUM_THREADS="2"))
        vol, _ = mrc.read_volume(os.path.join(d, "ref.mrc"))
    path = os.path.join(OUT, "spider.npz")
    np.savez_compressed(path, star=np.array(text), options=np.array(OPTIONS), map=vol,
                        names=np.array(sorted(files)), **{"file_" + k: v for k, v in files.items()})
    print(path)


if __name__ == "__main__":
    main()
