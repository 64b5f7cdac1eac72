"""Regenerate tests/golden/fixture_512.npz from the reference's golden FITS files.

The reference ships a 512 x 512 scene cleaned by lacosmic 1.4.0
(test/data/{input,error,reference}.fits.gz, settings contrast=1,
cr_threshold=5, neighbor_threshold=5, maxiter=4, error map, mirror border;
reference test/test_reference.py:43-62, test/mkref.py:12-25).  Those files
cannot travel with the tests, so this script stores what the tests need:

* ``input``: the float64 pixels (little-endian);
* ``error``: the error map, which is the integer constant 5 (checked);
* ``mask_bits``: the CRMASK extension, bit-packed row-major;
* ``masked_values``: the cleaned pixels at masked positions (the only pixels
  that differ from the input, checked);
* ``cleaned_sha256``: SHA-256 of the full cleaned float64 array.

Usage: ``python tests/golden/make_golden.py REFERENCE_TEST_DATA_DIR`` (the
reference's ``test/data`` directory).
"""

import gzip
import hashlib
import sys
from pathlib import Path

import numpy as np

BLOCK = 2880
DTYPES = {-64: ">f8", -32: ">f4", 8: "u1", 16: ">i2", 32: ">i4", 64: ">i8"}


def read_hdus(path):
    """Minimal FITS reader: primary array and IMAGE extensions, BSCALE/BZERO."""
    raw = gzip.open(path).read()
    pos, hdus = 0, []
    while pos < len(raw):
        cards = {}
        while True:
            block = raw[pos:pos + BLOCK]
            pos += BLOCK
            end = False
            for i in range(BLOCK // 80):
                card = block[i * 80:(i + 1) * 80].decode("ascii")
                key = card[:8].strip()
                if key == "END":
                    end = True
                    break
                if card[8:10] == "= ":
                    cards[key] = card[10:].split("/")[0].strip().strip("'").strip()
            if end:
                break
        bitpix, naxis = int(cards["BITPIX"]), int(cards["NAXIS"])
        shape = [int(cards[f"NAXIS{i}"]) for i in range(naxis, 0, -1)]
        count = int(np.prod(shape)) if naxis else 0
        nbytes = count * abs(bitpix) // 8
        data = None
        if count:
            data = np.frombuffer(raw[pos:pos + nbytes], dtype=DTYPES[bitpix]).reshape(shape)
            scale, zero = float(cards.get("BSCALE", 1)), float(cards.get("BZERO", 0))
            if scale != 1 or zero != 0:
                data = data * scale + zero
        pos += -(-nbytes // BLOCK) * BLOCK
        hdus.append((cards, data))
    return hdus


def main(src):
    src = Path(src)
    data = read_hdus(src / "input.fits.gz")[0][1].astype("<f8")
    error = read_hdus(src / "error.fits.gz")[0][1]
    ref = read_hdus(src / "reference.fits.gz")
    cleaned = ref[0][1].astype("<f8")
    crmask = [d for c, d in ref[1:] if c.get("EXTNAME") == "CRMASK"][0].astype(bool)
    assert error.dtype.kind == "i" and np.all(error == 5), "error map is not constant 5"
    differ = cleaned.view("u8") != data.view("u8")
    assert np.array_equal(differ, crmask), "cleaned pixels differ outside the mask"
    out = Path(__file__).with_name("fixture_512.npz")
    np.savez_compressed(
        out,
        input=data,
        error=np.float64(5.0),
        mask_bits=np.packbits(crmask.ravel()),
        masked_values=cleaned[crmask],
        cleaned_sha256=np.frombuffer(hashlib.sha256(cleaned.tobytes()).digest(), "u1"),
        settings=np.array([1.0, 5.0, 5.0, 4.0]),  # contrast, cr, neighbor, maxiter
    )
    print(out, out.stat().st_size, "bytes;", int(crmask.sum()), "masked pixels")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference test/data directory>")
    main(sys.argv[1])
