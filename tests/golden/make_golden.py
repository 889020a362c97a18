"""Generate the golden fixtures from the reference itself.

Runs the reference CPU backprojection, sentinel/azimuth_compress_cpu.c
compiled unmodified from the reference tree (oracle/_ref/libref_cpu.so, built
by `make -C oracle ref`), on the mini scenes of tests/helpers.py and stores,
per scene:

  * the exact orbit / grid arrays and scalars (the samples are regenerated
    from `sample_seed` by srg_b200.scene.mini_samples, bit for bit);
  * ref_xyz, ref_xyzfit      -- reference setxyz()
  * ref_azoff                -- reference setazoff() on the per-line parabolas
                                of the oracle (the reference does not expose
                                its own; its end-to-end output pins them)
  * ref_pixelint             -- reference pixelint(): unscaled complex64 sums
  * ref_geo                  -- reference azimuth_compress_cpu_() end to end on
                                a zeroed .geo (CPU merge rule), last line of
                                the burst excluded from comparisons (the
                                reference reads an unset parabola there)
  * terms                    -- executed-term count on those inputs.

Usage (where the reference tree is mounted):  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import oracle as O  # noqa: E402
from helpers import MINI_CASES, mini_case  # noqa: E402
from srg_b200 import scene  # noqa: E402


def main():
    O.build(ref=True)
    o = O.Oracle()
    r = O.RefCPU()
    for name, kw in MINI_CASES:
        b = mini_case(name)
        fl, ll, fp, lp = o.limits(b)
        nl = ll - fl + 1
        xyz, fit = r.setxyz(b, fl, nl, fp, lp)
        coef = o.line_coefs(b, fit)
        az = r.setazoff(b, coef, fp, lp)
        pix = r.pixelint(b, xyz, az)
        _, _, terms = o.pixelint(b, xyz, az, gpu_lerp=0, gpu_scale=0)
        geo = r.azimuth_compress_cpu(b)
        arrays = scene.burst_to_arrays(b)
        np.savez_compressed(
            os.path.join(HERE, f"mini_{name}.npz"), sample_seed=np.int64(kw["seed"]),
            limits=np.array([fl, ll, fp, lp], np.int64), ref_xyz=xyz, ref_xyzfit=fit,
            ref_azoff=az, ref_pixelint=pix, ref_geo=geo, terms=np.int64(terms), **arrays)
        print(f"{name}: P={b.rawdatalines} S={b.samples} grid={b.demwidth}x{b.demlength} "
              f"limits={fl, ll, fp, lp} formed={(az > 0).sum()} terms={terms}")


if __name__ == "__main__":
    main()
