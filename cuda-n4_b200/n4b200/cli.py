"""Command line N4 with the options of the reference's ``CUDAN4`` (main.cpp).

    python -m n4b200.cli -i input.nii.gz -o norm.nii.gz [-m mask.nii.gz]
                         [-b bias.nii.gz] [-n 50] [-t 4] [-c 4]
                         [-s shrink] [-l low_value] [-e threshold] [-d device]

-i/-o/-m/-b/-n/-t/-c mean what they mean in ``main.cpp:19-33,49-80``
(input, output, mask, bias-field output, iterations per level, fitting
levels, control points of the first level).  Added: -s shrink factor,
-l low_value (reference default 10), -e convergence threshold (0.001), -d
CUDA device.  Without -m every voxel is in the mask (``main.cpp:138-140``).
"""
from __future__ import annotations

import argparse
import sys

import numpy as np


def build_parser():
    ap = argparse.ArgumentParser(prog="n4b200", description="N4 bias-field correction on B200")
    ap.add_argument("-i", dest="input", required=True, help="input image")
    ap.add_argument("-o", dest="output", required=True, help="bias-corrected output image")
    ap.add_argument("-m", dest="mask", help="mask image (non-zero = foreground)")
    ap.add_argument("-b", dest="bias", help="write the bias field exp(b) here")
    ap.add_argument("-n", dest="iterations", type=int, default=50, help="max iterations per level (50)")
    ap.add_argument("-t", dest="levels", type=int, default=4, help="fitting levels (4)")
    ap.add_argument("-c", dest="control_points", type=int, default=4, help="control points, first level (4)")
    ap.add_argument("-s", dest="shrink", type=int, default=1, help="shrink factor (1)")
    ap.add_argument("-l", dest="low_value", type=float, default=10.0, help="intensity threshold (10)")
    ap.add_argument("-e", dest="threshold", type=float, default=0.001, help="convergence threshold (0.001)")
    ap.add_argument("-d", dest="device", type=int, default=0, help="CUDA device (0)")
    return ap


def main(argv=None) -> int:
    args = build_parser().parse_args(argv)
    import n4b200
    from n4b200 import nifti

    img = nifti.load(args.input)
    mask = None
    if args.mask:
        m = nifti.load(args.mask)
        if m.data.shape != img.data.shape:
            print(f"Size mismatch. im:{img.data.shape[::-1]}, mask:{m.data.shape[::-1]}", file=sys.stderr)
            return 1
        mask = m.data
    p = n4b200.N4Param(NumberOfFittingLevels=args.levels, MaximumNumberOfIterations=args.iterations,
                       NumberOfControlPoints=args.control_points, ShrinkFactor=args.shrink,
                       low_value=args.low_value, ConvergenceThreshold=args.threshold)
    res = n4b200.N4(img.data, mask if mask is not None else np.ones_like(img.data), p,
                    return_bias=bool(args.bias), ctx=n4b200.Context.default(args.device))
    nifti.save(args.output, res.im_normalized, like=img)
    if args.bias:
        nifti.save(args.bias, res.bias_field, like=img)
    r = res.report
    print(f"levels {r['levels']}, iterations {r['iterations']}, final CV "
          f"{[round(c, 6) for c in r['final_cv']]}, path {r['path']} x{r['cluster_size']}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
