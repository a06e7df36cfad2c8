"""Single workloads for kernel profiling, one launch of the kernel of interest
each (run from the repository root)::

    PYTHONPATH=cuda-n4_b200 python -m n4b200.profile_cases c3       # k_n4_grid
    PYTHONPATH=cuda-n4_b200 python -m n4b200.profile_cases c2x4     # k_n4_cluster, k_prologue, k_correct
    PYTHONPATH=cuda-n4_b200 python -m n4b200.profile_cases encoder  # enc::k_igemm
    PYTHONPATH=cuda-n4_b200 python -m n4b200.profile_cases fit      # k_fit_rows_v5
    PYTHONPATH=cuda-n4_b200 python -m n4b200.profile_cases evaluate # k_correct (log field only)

* ``c3``: one 512x512x320 phantom (0.5 mm, 8^3-grid bias N(0, 0.25^2),
  Rician 0.02) through ``n4_run`` at shrink 2 (256x256x160 fitting grid,
  whole-GPU path), 4 levels, <= 50 iterations, convergence 0.001.
* ``c2x4``: four 256x256x176 phantoms (6^3 grid, N(0, 0.25^2), Rician 0.02)
  in one batched run on 6-CTA clusters of 512 threads (the configuration the
  autotuner picks for this workload), shrink 4, 4 levels, convergence 0.001.
* ``encoder``: the warm-start encoder's forward pass over 96 inputs.
* ``fit``: ``FitBspline3D`` of a 256x256x160 field with a float mask on an
  11^3 lattice (the z contraction reads 8 B per voxel).
* ``evaluate``: ``EvaluateBspline3D`` of an 11^3 lattice at 512x512x320 (4 B
  per voxel written) on the default tile (128 rows, 256 threads; the one the
  component autotuner picks for this size when it runs without a profiler).

Every case prints one line and exits 0 on success.
"""
from __future__ import annotations

import sys


def c3():
    import torch
    import n4b200
    from n4b200.warmstart import phantoms_gpu
    im, mk = phantoms_gpu(1, (512, 512, 320), seed=77, sigma=0.02, grid=8, coeff_std=0.25, device="cuda")
    p = n4b200.N4Param(NumberOfFittingLevels=4, MaximumNumberOfIterations=50, ConvergenceThreshold=0.001,
                       low_value=0.0, ShrinkFactor=2)
    r = n4b200.N4(im[0], mk[0], p)
    torch.cuda.synchronize()
    return f"c3 iterations {r.report['iterations']} path {r.report['path']}"


def c2x4():
    import torch
    import n4b200
    from n4b200 import _lib
    from n4b200.warmstart import phantoms_gpu
    im, mk = phantoms_gpu(4, (256, 256, 176), seed=9, sigma=0.02, grid=6, coeff_std=0.25, device="cuda")
    p = n4b200.N4Param(NumberOfFittingLevels=4, MaximumNumberOfIterations=50, ConvergenceThreshold=0.001,
                       low_value=0.0, ShrinkFactor=4)
    p.flags = n4b200.cluster_size_flag(6) | _lib.FLAG_CTA_512
    res = n4b200.N4Batch([(im[i], mk[i]) for i in range(4)], p)
    torch.cuda.synchronize()
    return f"c2x4 iterations {[r.report['iterations'] for r in res]}"


def encoder():
    import torch
    from n4b200.warmstart import load_encoder
    enc = load_encoder(max_batch=96)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = (torch.randn((96, 32, 32, 24), device="cuda", generator=g) * 0.3 - 0.7).to(torch.bfloat16)
    y = enc.predict(x)
    torch.cuda.synchronize()
    return f"encoder out {tuple(y.shape)} mean|y| {float(y.abs().mean()):.4f}"


def fit():
    import torch
    import n4b200
    g = torch.Generator(device="cuda").manual_seed(5)
    field = torch.randn((256, 256, 160), device="cuda", generator=g)
    mask = (torch.rand((256, 256, 160), device="cuda", generator=g) > 0.4).float()
    lat = n4b200.FitBspline3D(field, mask, (11, 11, 11))
    torch.cuda.synchronize()
    return f"fit lattice {tuple(lat.shape)}"


def evaluate():
    import torch
    import n4b200
    ctx = n4b200.Context(0)
    g = torch.Generator(device="cuda").manual_seed(7)
    lat = torch.randn((11, 11, 11), device="cuda", generator=g) * 0.1
    out = n4b200.EvaluateBspline3D(lat, (11, 11, 11), (512, 512, 320), ctx=ctx)
    torch.cuda.synchronize()
    return f"evaluate {tuple(out.shape)}"


CASES = {"c3": c3, "c2x4": c2x4, "encoder": encoder, "fit": fit, "evaluate": evaluate}


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 1 or argv[0] not in CASES:
        print("usage: python -m n4b200.profile_cases {" + ",".join(CASES) + "}", file=sys.stderr)
        return 2
    print(CASES[argv[0]](), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
