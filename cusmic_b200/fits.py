"""FITS images on the host, without astropy or CFITSIO.

Mirrors the reference's FITS layer (``mod/cusmic/io.py:21-58``,
``src/io.c:21-121``): reading applies BSCALE/BZERO (multiply, then add) and
turns integer BLANK values into NaN; IEEE pixels are returned bit for bit.
Writing stores float64 pixels in the primary HDU (structural, scaling and
BLANK keywords regenerated or dropped, other cards copied), an optional uint8
``CRMASK`` image extension, and DATASUM/CHECKSUM keywords on every HDU using
the FITS checksum convention.  Existing files are never overwritten unless
asked.  Gzip-compressed inputs are read transparently.
"""

import gzip
from pathlib import Path

import numpy as np

BLOCK = 2880
CARD = 80
_DTYPES = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}
_BITPIX = {np.dtype("uint8"): 8, np.dtype("int16"): 16, np.dtype("int32"): 32,
           np.dtype("int64"): 64, np.dtype("float32"): -32, np.dtype("float64"): -64}
_STRUCTURAL = {"SIMPLE", "XTENSION", "BITPIX", "NAXIS", "EXTEND", "PCOUNT", "GCOUNT",
               "CHECKSUM", "DATASUM", "END"}


class Header:
    """Ordered FITS header cards: (keyword, value, comment)."""

    def __init__(self, cards=None):
        self.cards = list(cards or [])

    def copy(self):
        return Header(list(self.cards))

    def _find(self, key):
        key = key.upper()
        for i, (k, _, _) in enumerate(self.cards):
            if k == key:
                return i
        return -1

    def __contains__(self, key):
        return self._find(key) >= 0

    def __getitem__(self, key):
        i = self._find(key)
        if i < 0:
            raise KeyError(key)
        return self.cards[i][1]

    def get(self, key, default=None):
        i = self._find(key)
        return default if i < 0 else self.cards[i][1]

    def __setitem__(self, key, value):
        i = self._find(key)
        if i >= 0:
            self.cards[i] = (key.upper(), value, self.cards[i][2])
        else:
            self.cards.append((key.upper(), value, ""))

    def pop(self, key, default=None):
        i = self._find(key)
        if i < 0:
            return default
        return self.cards.pop(i)[1]

    def add_history(self, text):
        self.cards.append(("HISTORY", text, ""))


def _parse_value(raw):
    raw = raw.strip()
    if raw.startswith("'"):
        out, i = [], 1
        while i < len(raw):
            if raw[i] == "'":
                if i + 1 < len(raw) and raw[i + 1] == "'":
                    out.append("'")
                    i += 2
                    continue
                break
            out.append(raw[i])
            i += 1
        return "".join(out).rstrip(), raw[i + 1:]
    value, slash, comment = raw.partition("/")
    comment = slash + comment
    value = value.strip()
    if value == "T":
        return True, comment
    if value == "F":
        return False, comment
    try:
        return int(value), comment
    except ValueError:
        pass
    try:
        return float(value.replace("D", "E")), comment
    except ValueError:
        return value, comment


def _parse_header(raw, pos):
    cards = []
    while True:
        block = raw[pos:pos + BLOCK]
        if len(block) < BLOCK:
            raise ValueError("truncated FITS header")
        pos += BLOCK
        for i in range(0, BLOCK, CARD):
            card = block[i:i + CARD].decode("ascii", errors="replace")
            key = card[:8].strip()
            if key == "END":
                return Header(cards), pos
            if not key:
                continue
            if card[8:10] == "= ":
                value, rest = _parse_value(card[10:])
                comment = rest.strip()
                cards.append((key, value, comment[1:].strip() if comment.startswith("/")
                              else comment))
            else:
                cards.append((key, card[8:].rstrip(), ""))


def _data_size(header):
    """(shape, padded byte size) of an HDU's data unit."""
    bitpix, naxis = int(header["BITPIX"]), int(header.get("NAXIS", 0))
    shape = tuple(int(header[f"NAXIS{i}"]) for i in range(naxis, 0, -1))
    count = int(np.prod(shape)) if naxis else 0
    nbytes = abs(bitpix) // 8 * int(header.get("GCOUNT", 1)) * (
        int(header.get("PCOUNT", 0)) + count) if naxis else 0
    return shape, -(-nbytes // BLOCK) * BLOCK


def _hdus(raw):
    pos, out = 0, []
    while pos < len(raw):
        if not raw[pos:pos + CARD].strip(b" \0"):
            break
        header, pos = _parse_header(raw, pos)
        shape, padded = _data_size(header)
        data = None
        if shape and int(np.prod(shape)):
            data = np.frombuffer(raw, dtype=_DTYPES[int(header["BITPIX"])],
                                 count=int(np.prod(shape)), offset=pos).reshape(shape)
        pos += padded
        out.append((header, data))
    return out


def _read_bytes(path):
    with open(path, "rb") as f:
        raw = f.read()
    if raw[:2] == b"\x1f\x8b":
        raw = gzip.decompress(raw)
    return raw


def read_fits(path, dtype=None, *, ext=None):
    """Return (native-endian pixels, Header) of a FITS image HDU.

    ``ext`` selects an extension by EXTNAME (str) or index (int); by default
    the primary HDU, or the first extension when the primary has no data.
    """
    hdus = _hdus(_read_bytes(path))
    if isinstance(ext, str):
        matches = [h for h in hdus if str(h[0].get("EXTNAME", "")).upper() == ext.upper()]
        if not matches:
            raise KeyError(f"{path}: no extension {ext}")
        header, data = matches[0]
    elif ext is not None:
        header, data = hdus[ext]
    else:
        header, data = hdus[0]
        if data is None and len(hdus) > 1:
            header, data = hdus[1]
    if data is None:
        raise ValueError(f"{path}: the FITS image has no data")
    scale = header.get("BSCALE", 1)
    zero = header.get("BZERO", 0)
    blank = header.get("BLANK") if data.dtype.kind in "iu" else None
    if scale != 1 or zero != 0 or blank is not None:
        missing = data == blank if blank is not None else None
        pixels = data.astype("float64")
        pixels *= scale
        pixels += zero
        if missing is not None:
            pixels[missing] = np.nan
    else:
        pixels = data.astype(data.dtype.newbyteorder("="), copy=True)
    return pixels.astype(dtype or pixels.dtype, copy=False), header


# --- checksums (FITS checksum convention: 32-bit ones' complement sums) ---

def checksum32(buf, start=0):
    """Ones' complement sum of big-endian 32-bit words (length a multiple of 4)."""
    words = np.frombuffer(buf, dtype=">u4").astype(np.uint64)
    total = int(words.sum()) + start
    while total >> 32:
        total = (total & 0xFFFFFFFF) + (total >> 32)
    return total


_EXCLUDE = set(range(0x3A, 0x41)) | set(range(0x5B, 0x61))


def encode_checksum(value):
    """16-character ASCII encoding of a 32-bit checksum value.

    Each byte is split into four characters near ASCII '0' + byte / 4 (the
    remainder going to the first), pairs are nudged apart until none falls on
    ASCII punctuation (keeping their sum), the 4 x 4 characters are
    interleaved byte-major, and the string is rotated right by one.
    """
    asc = [0] * 16
    for i in range(4):
        byte = (value >> (24 - 8 * i)) & 0xFF
        quotient, remainder = byte // 4 + 0x30, byte % 4
        ch = [quotient] * 4
        ch[0] += remainder
        changed = True
        while changed:
            changed = False
            for j in (0, 2):
                while ch[j] in _EXCLUDE or ch[j + 1] in _EXCLUDE:
                    ch[j] += 1
                    ch[j + 1] -= 1
                    changed = True
        for j in range(4):
            asc[4 * j + i] = ch[j]
    return "".join(chr(asc[(i + 15) % 16]) for i in range(16))


# --- writing ---

def _format_value(value):
    if isinstance(value, bool):
        return f"{'T' if value else 'F':>20}"
    if isinstance(value, (int, np.integer)):
        return f"{int(value):>20}"
    if isinstance(value, (float, np.floating)):
        text = repr(float(value)).upper()
        if "E" not in text and "." not in text and text not in ("NAN", "INF", "-INF"):
            text += ".0"
        return f"{text:>20}"
    text = "'" + str(value).replace("'", "''").ljust(8) + "'"
    return f"{text:<20}"


def _card(key, value, comment=""):
    if key in ("HISTORY", "COMMENT", ""):
        card = f"{key:<8}{str(value)}"
    else:
        card = f"{key:<8}= {_format_value(value)}"
        if comment:
            card += f" / {comment}"
    return card[:CARD].ljust(CARD)


def _header_bytes(cards):
    text = "".join(_card(*c) for c in cards) + "END".ljust(CARD)
    pad = -len(text) % BLOCK
    return (text + " " * pad).encode("ascii")


def _data_bytes(array):
    raw = np.ascontiguousarray(array).astype(array.dtype.newbyteorder(">"), copy=False).tobytes()
    return raw + b"\0" * (-len(raw) % BLOCK)


def _hdu(cards, array):
    data = _data_bytes(array)
    datasum = checksum32(data)
    cards = cards + [("DATASUM", str(datasum), "data unit checksum"),
                     ("CHECKSUM", "0" * 16, "HDU checksum")]
    header = _header_bytes(cards)
    total = checksum32(header, datasum)
    cards[-1] = ("CHECKSUM", encode_checksum(~total & 0xFFFFFFFF), "HDU checksum")
    return _header_bytes(cards) + data


def _image_cards(array, primary, extend=False):
    bitpix = _BITPIX[np.dtype(array.dtype).newbyteorder("=")]
    cards = [("SIMPLE", True, "conforms to FITS standard")] if primary else \
        [("XTENSION", "IMAGE", "Image extension")]
    cards += [("BITPIX", bitpix, ""), ("NAXIS", array.ndim, "")]
    cards += [(f"NAXIS{i + 1}", n, "") for i, n in enumerate(reversed(array.shape))]
    if primary:
        cards.append(("EXTEND", bool(extend), ""))
    else:
        cards += [("PCOUNT", 0, ""), ("GCOUNT", 1, "")]
    return cards


def write_fits(path, data, mask=None, *, header=None, overwrite=False):
    """Write float pixels (+ an optional uint8 CRMASK); refuse overwrites."""
    path = Path(path)
    if str(path).startswith("!"):
        raise ValueError("Choose a new output filename")
    pixels = np.asarray(data.cpu() if hasattr(data, "cpu") else data)
    cards = _image_cards(pixels, True, extend=mask is not None)
    if header is not None:
        drop = {"BSCALE", "BZERO"} | ({"BLANK"} if pixels.dtype.kind == "f" else set())
        cards += [c for c in header.cards
                  if c[0] not in _STRUCTURAL and c[0] not in drop
                  and not c[0].startswith("NAXIS") and c[0] != "EXTNAME"]
    out = _hdu(cards, pixels)
    if mask is not None:
        flags = np.asarray(mask.cpu() if hasattr(mask, "cpu") else mask).astype(np.uint8)
        mcards = _image_cards(flags, False) + [("EXTNAME", "CRMASK", "")]
        out += _hdu(mcards, flags)
    mode = "wb" if overwrite else "xb"
    with open(path, mode) as f:
        f.write(out)


def verify_checksums(path):
    """True when every HDU sums to negative zero (all ones)."""
    raw = _read_bytes(path)
    pos = 0
    ok = True
    while pos < len(raw):
        header, end = _parse_header(raw, pos)
        _, padded = _data_size(header)
        if "CHECKSUM" in header:
            ok &= checksum32(raw[pos:end + padded]) == 0xFFFFFFFF
        pos = end + padded
    return ok
