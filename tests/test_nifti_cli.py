"""NIfTI-1 I/O (replacing itkLoadVolume.h) and the CUDAN4-style CLI."""
import gzip
import struct

import numpy as np
import pytest

from n4b200 import nifti


@pytest.mark.parametrize("suffix", [".nii", ".nii.gz"])
def test_roundtrip(tmp_path, suffix):
    a = np.random.default_rng(0).normal(size=(7, 5, 3)).astype(np.float32)
    p = tmp_path / f"v{suffix}"
    nifti.save(p, a, spacing=(0.5, 0.6, 0.7))
    img = nifti.load(p)
    assert img.data.shape == (7, 5, 3) and np.array_equal(img.data, a)
    assert img.spacing == pytest.approx((0.5, 0.6, 0.7))
    # the layout of the reference: x (the last C axis) fastest on disk
    raw = gzip.open(p).read() if str(p).endswith(".gz") else open(p, "rb").read()
    nx, ny, nz = struct.unpack("<3h", raw[42:48])
    assert (nx, ny, nz) == (3, 5, 7)
    assert np.array_equal(np.frombuffer(raw, np.float32, count=3, offset=352), a[0, 0, :3])


def test_int16_with_scaling_and_header_copy(tmp_path):
    a = (np.arange(24, dtype=np.int16).reshape(2, 3, 4))
    h = bytearray(348)
    struct.pack_into("<i", h, 0, 348)
    struct.pack_into("<8h", h, 40, 3, 4, 3, 2, 1, 1, 1, 1)
    struct.pack_into("<2h", h, 70, 4, 16)
    struct.pack_into("<8f", h, 76, 1, 2.0, 2.0, 3.0, 1, 1, 1, 1)
    struct.pack_into("<f", h, 108, 352.0)
    struct.pack_into("<2f", h, 112, 0.5, 1.0)
    h[344:348] = b"n+1\0"
    p = tmp_path / "s.nii"
    p.write_bytes(bytes(h) + b"\0" * 4 + a.tobytes())
    img = nifti.load(p)
    assert np.allclose(img.data, a * 0.5 + 1.0)
    out = tmp_path / "o.nii"
    nifti.save(out, img.data, like=img)
    assert nifti.load(out).spacing == pytest.approx((2.0, 2.0, 3.0))


def test_cli_parser_matches_main_cpp_flags():
    from n4b200.cli import build_parser
    a = build_parser().parse_args(["-i", "in.nii", "-o", "out.nii", "-m", "m.nii", "-b", "b.nii",
                                   "-n", "20", "-t", "3", "-c", "5", "-s", "2"])
    assert (a.iterations, a.levels, a.control_points, a.shrink, a.low_value) == (20, 3, 5, 2, 10.0)


@pytest.mark.gpu
def test_cli_end_to_end(cuda, tmp_path):
    import n4b200
    from n4b200.cli import main
    from n4b200.phantom import make_phantom
    ph = make_phantom((32, 32, 24), seed=2)
    nifti.save(tmp_path / "im.nii.gz", ph.im)
    nifti.save(tmp_path / "mask.nii.gz", ph.mask)
    rc = main(["-i", str(tmp_path / "im.nii.gz"), "-o", str(tmp_path / "out.nii.gz"), "-m",
               str(tmp_path / "mask.nii.gz"), "-b", str(tmp_path / "bias.nii.gz"), "-n", "5", "-t", "2",
               "-l", "0"])
    assert rc == 0
    out = nifti.load(tmp_path / "out.nii.gz").data
    p = n4b200.N4Param(NumberOfFittingLevels=2, MaximumNumberOfIterations=5, low_value=0.0)
    ref = n4b200.N4(ph.im, ph.mask, p, return_bias=True)
    assert np.array_equal(out, ref.im_normalized)
    assert np.array_equal(nifti.load(tmp_path / "bias.nii.gz").data, ref.bias_field)
