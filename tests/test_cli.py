"""The FITS command (reference mod/cusmic/__main__.py, src/main.c; tests
test/test_io.py:60-69 and test/test_reference.py:65-123)."""

import numpy as np
import pytest
from click.testing import CliRunner

from cusmic_b200 import fits
from cusmic_b200.__main__ import main
from tests.conftest import assert_bits_equal


def write(path, data, **kw):
    fits.write_fits(path, np.asarray(data), **kw)
    return str(path)


@pytest.mark.parametrize("shape", [None, (2, 3, 3)])
def test_rejects_invalid_images(tmp_path, shape):
    src, out = tmp_path / "invalid.fits", tmp_path / "output.fits"
    if shape is None:
        # a primary HDU without data
        header = "".join(f"{k:<8}= {v:>20}".ljust(80) for k, v in
                         (("SIMPLE", "T"), ("BITPIX", 8), ("NAXIS", 0))) + "END".ljust(80)
        src.write_bytes((header + " " * (-len(header) % 2880)).encode())
    else:
        write(src, np.zeros(shape))
    result = CliRunner().invoke(main, [str(src), str(out), "--maxiter", "0"])
    assert result.exit_code == 1 and "Error:" in result.output
    assert not out.exists()


def test_refuses_existing_output_and_missing_noise(tmp_path):
    src = write(tmp_path / "in.fits", np.ones((5, 5)))
    out = tmp_path / "out.fits"
    out.write_bytes(b"keep")
    result = CliRunner().invoke(main, [src, str(out), "--maxiter", "0"])
    assert result.exit_code == 1 and "already exists" in result.output
    assert out.read_bytes() == b"keep"
    result = CliRunner().invoke(main, [src, str(tmp_path / "new.fits")])
    assert result.exit_code == 2 and "Provide --error or --gain" in result.output
    for options in (["--gain", "1", "--contrast", "nan"], ["--gain", "0"],
                    ["--gain", "1", "--maxiter", "-1"]):
        result = CliRunner().invoke(main, [src, str(tmp_path / "x.fits"), *options])
        assert result.exit_code != 0 and not (tmp_path / "x.fits").exists()


@pytest.mark.gpu
def test_zero_iterations_copy_and_golden_scene(cuda, tmp_path, golden):
    src = write(tmp_path / "input.fits", golden["data"])
    err = write(tmp_path / "error.fits", golden["error"])
    copy = tmp_path / "copy.fits"
    result = CliRunner().invoke(main, [src, str(copy), "--maxiter", "0"])
    assert result.exit_code == 0, result.output
    assert_bits_equal(fits.read_fits(copy)[0], golden["data"])
    assert not fits.read_fits(copy, ext="CRMASK")[0].any()
    out = tmp_path / "clean.fits"
    s = golden["settings"]
    result = CliRunner().invoke(main, [src, str(out), "--error", err,
                                       "--contrast", str(s["contrast"]),
                                       "--cr-threshold", str(s["cr_threshold"]),
                                       "--neighbor-threshold", str(s["neighbor_threshold"]),
                                       "--maxiter", str(s["maxiter"])])
    assert result.exit_code == 0, result.output
    assert "6,518 cosmic-ray pixels" in result.output
    assert_bits_equal(fits.read_fits(out)[0], golden["cleaned"])
    np.testing.assert_array_equal(fits.read_fits(out, ext="CRMASK")[0].astype(bool),
                                  golden["mask"])
    assert fits.verify_checksums(out)


@pytest.mark.gpu
def test_scaled_integer_fits(cuda, oracle, tmp_path):
    """reference test/test_reference.py:85-123: a BSCALE/BZERO int16 image."""
    data = np.ones((9, 9), dtype="int16")
    data[4, 4] = 10000
    cards = [("SIMPLE", "T"), ("BITPIX", 16), ("NAXIS", 2), ("NAXIS1", 9), ("NAXIS2", 9),
             ("BSCALE", 0.1), ("BZERO", 10.2)]
    header = "".join(f"{k:<8}= {v:>20}".ljust(80) for k, v in cards) + "END".ljust(80)
    raw = data.astype(">i2").tobytes()
    src = tmp_path / "scaled.fits"
    src.write_bytes((header + " " * (-len(header) % 2880)).encode() + raw
                    + b"\0" * (-len(raw) % 2880))
    err = write(tmp_path / "error.fits", np.ones((9, 9)))
    pixels = fits.read_fits(src)[0]
    for iterations in (0, 4):
        out = tmp_path / f"out-{iterations}.fits"
        result = CliRunner().invoke(main, [str(src), str(out), "--error", err,
                                           "--maxiter", str(iterations)])
        assert result.exit_code == 0, result.output
        want, mask, _ = oracle.clean_frame(pixels, error=np.ones((9, 9)), maxiter=iterations)
        assert_bits_equal(fits.read_fits(out)[0], want)
        np.testing.assert_array_equal(fits.read_fits(out, ext="CRMASK")[0].astype(bool), mask)
