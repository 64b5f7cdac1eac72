"""FITS I/O (reference src/io.c:21-121, mod/cusmic/io.py:21-58, test/test_io.py,
test/test_io.c).  Inputs are assembled byte by byte here, independently of the
writer under test."""

import gzip

import numpy as np
import pytest

from cusmic_b200 import fits


def card(key, value=None):
    if value is None:
        return f"{key:<80}"
    if isinstance(value, bool):
        v = f"{'T' if value else 'F':>20}"
    elif isinstance(value, str):
        v = f"'{value:<8}'".ljust(20)
    else:
        v = f"{value:>20}"
    return f"{key:<8}= {v}".ljust(80)


def hdu(cards, array):
    text = "".join(cards) + card("END")
    text += " " * (-len(text) % 2880)
    raw = array.astype(array.dtype.newbyteorder(">")).tobytes()
    return text.encode() + raw + b"\0" * (-len(raw) % 2880)


def image_cards(primary, bitpix, shape, extra=()):
    cards = [card("SIMPLE", True)] if primary else [card("XTENSION", "IMAGE")]
    cards += [card("BITPIX", bitpix), card("NAXIS", len(shape))]
    cards += [card(f"NAXIS{i + 1}", n) for i, n in enumerate(reversed(shape))]
    cards += [card("EXTEND", True)] if primary else [card("PCOUNT", 0), card("GCOUNT", 1)]
    return cards + [card(k, v) for k, v in extra]


def test_float64_special_pixels_scaling_and_blank(tmp_path):
    """reference test/test_io.py:27-57 and test/test_io.c:26-97."""
    bits = np.array([0x8000000000000000, 0x7FF0000000000000, 0x7FF8000000001234,
                     0x401C000000000000], dtype="uint64")
    raw = np.array([[1, -32768], [2, 3]], dtype="int16")
    blob = hdu(image_cards(True, -64, (2, 2)), bits.view("float64").reshape(2, 2))
    blob += hdu(image_cards(False, 16, (2, 2), [("EXTNAME", "SCALED"), ("BSCALE", 0.1),
                                                ("BZERO", 10.2), ("BLANK", -32768)]), raw)
    blob += hdu(image_cards(False, 16, (2, 2), [("EXTNAME", "UNSIGNED"), ("BZERO", 32768),
                                                ("BLANK", -32768)]), raw)
    path = tmp_path / "pixels.fits"
    path.write_bytes(blob)

    pixels, _ = fits.read_fits(path, dtype="float64")
    np.testing.assert_array_equal(pixels.view("uint64").ravel(), bits)
    pixels, _ = fits.read_fits(path, dtype="float64", ext="SCALED")
    expected = np.array([0x4024999999999999, 0x7FF8000000000000, 0x4024CCCCCCCCCCCC,
                         0x4025000000000000], dtype="uint64")
    np.testing.assert_array_equal(pixels.view("uint64").ravel(), expected)
    pixels, _ = fits.read_fits(path, dtype="float64", ext="UNSIGNED")
    assert np.isnan(pixels[0, 1])
    np.testing.assert_array_equal(pixels[[0, 1, 1], [0, 0, 1]], [32769, 32770, 32771])


def test_blank_round_trip(tmp_path):
    """reference test/test_io.py:11-24: BLANK becomes NaN and is not written back."""
    data = np.array([[1, 2], [3, -32768]], dtype="int16")
    src, out = tmp_path / "input.fits", tmp_path / "output.fits"
    src.write_bytes(hdu(image_cards(True, 16, (2, 2), [("BLANK", -32768)]), data))
    pixels, header = fits.read_fits(src, dtype="float64")
    assert np.isnan(pixels[1, 1]) and header["BLANK"] == -32768
    fits.write_fits(out, pixels, np.zeros(data.shape, dtype=bool), header=header)
    again, h2 = fits.read_fits(out)
    np.testing.assert_array_equal(again.view("u8"), pixels.view("u8"))
    assert "BLANK" not in h2
    assert not fits.read_fits(out, ext="CRMASK")[0].any()
    assert fits.verify_checksums(out)


def test_primary_without_data_reads_first_extension(tmp_path):
    data = np.arange(6, dtype=">f8").reshape(2, 3)
    blob = hdu([card("SIMPLE", True), card("BITPIX", 8), card("NAXIS", 0),
                card("EXTEND", True)], np.zeros(0, np.uint8))
    blob += hdu(image_cards(False, -64, (2, 3), [("EXTNAME", "SCI")]), data)
    path = tmp_path / "ext.fits.gz"
    path.write_bytes(gzip.compress(blob))
    pixels, header = fits.read_fits(path)
    np.testing.assert_array_equal(pixels, data)
    assert header["EXTNAME"] == "SCI"


def test_writer_refuses_overwrite_and_keeps_history(tmp_path):
    out = tmp_path / "o.fits"
    header = fits.Header([("OBJECT", "M31", "target")])
    header.add_history("Cosmic rays removed with cusmic")
    fits.write_fits(out, np.ones((3, 4)), np.eye(3, 4, dtype=bool), header=header)
    with pytest.raises(FileExistsError):
        fits.write_fits(out, np.ones((3, 4)))
    with pytest.raises(ValueError):
        fits.write_fits("!" + str(tmp_path / "y.fits"), np.ones((2, 2)))
    pixels, h = fits.read_fits(out)
    assert h["OBJECT"] == "M31" and h["BITPIX"] == -64
    assert any(k == "HISTORY" and "cusmic" in v for k, v, _ in h.cards)
    np.testing.assert_array_equal(fits.read_fits(out, ext="CRMASK")[0], np.eye(3, 4))
    assert fits.verify_checksums(out)


def ones_add(a, b):
    s = a + b
    return (s & 0xFFFFFFFF) + (s >> 32)


def test_checksum_encoding_property():
    """The 16 characters, read back in word order, add (ones' complement) to the
    encoded value plus the '0000000000000000' placeholder they replace."""
    placeholder = fits.checksum32(b"0" * 16)
    for value in (0, 1, 0x12345678, 0xDEADBEEF, 0x7FFFFFFF, 0xFFFFFFFE):
        text = fits.encode_checksum(value)
        assert len(text) == 16 and text.isalnum()
        unrotated = (text[1:] + text[:1]).encode()
        assert fits.checksum32(unrotated) == ones_add(value, placeholder)
