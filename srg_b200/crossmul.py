"""Interferogram formation on the GPU, as a drop-in for SRG's crossmul program.

  python -m srg_b200.crossmul infile1 infile2 outintfile outampfile length \\
      [valid_lines] [scale=1] [looksac=1] [looksdn=looksac] [mask y/n = y]

Same arguments, defaults and file formats as int/crossmul.f90:25-80 (two
complex64 rasters `length` samples wide in; interferogram and amplitude
rasters of length/looksac samples out, one record per looksdn input lines).
The arithmetic runs in libsrg_bp.so (srg_crossmul_device): both images are
uploaded once, every output line is formed on the device, the two outputs
come back once.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import api


def crossmul_files(fin1: str, fin2: str, figram: str, famp: str, na: int, nvalid: int | None = None,
                   scale: float = 1.0, looksac: int = 1, looksdn: int | None = None,
                   mask: str = "y", device: str = "cuda") -> tuple[int, int]:
    """Run the reference's crossmul on files; returns (output lines, output samples)."""
    import torch
    looksdn = looksac if looksdn is None else looksdn
    nd = os.path.getsize(fin1) // 8 // na                     # crossmul.f90:44-45
    nvalid = nd if nvalid is None else nvalid
    a = np.fromfile(fin1, np.complex64, count=nd * na).reshape(nd, na)
    if os.path.abspath(fin2) != os.path.abspath(fin1):
        b = np.fromfile(fin2, np.complex64, count=nd * na)
        if b.size < nd * na:                                    # a short second file reads as 0
            b = np.concatenate([b, np.zeros(nd * na - b.size, np.complex64)])
        b = b.reshape(nd, na)
    else:
        b = a
    ta = torch.from_numpy(a).to(device)
    tb = ta if b is a else torch.from_numpy(b).to(device)
    ig, am = api.crossmul(ta, tb, looksac=looksac, looksdn=looksdn, scale=scale,
                          mask=(mask.lower() == "y"), nvalid=min(nvalid, nd))
    ig.cpu().numpy().tofile(figram)
    am.cpu().numpy().tofile(famp)
    return ig.shape[0], ig.shape[1]


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) < 5:
        print("usage: crossmul infile1 infile2 outintfile outampfile length "
              "<valid_lines> <scale=1> <looksac> <looksdn> <mask y/n = y>")
        return 1
    fin1, fin2, figram, famp = argv[:4]
    na = int(argv[4])
    nvalid = int(argv[5]) if len(argv) > 5 else None
    scale = float(argv[6]) if len(argv) > 6 else 1.0
    looksac = int(argv[7]) if len(argv) > 7 else 1
    looksdn = int(argv[8]) if len(argv) > 8 else looksac
    mask = argv[9] if len(argv) > 9 else "y"
    n, w = crossmul_files(fin1, fin2, figram, famp, na, nvalid, scale, looksac, looksdn, mask)
    print(f"Lines in output: {n}, interferogram width: {w}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
