"""Minimal FITS image reader/writer (primary HDU, BITPIX -32/-64), enough for SKIRT's frame
outputs (*_total.fits, *_statsK.fits) and for writing the tracer's own images."""
import numpy as np

BLOCK = 2880


def read(path):
    """Returns (data, header dict) of the primary HDU; data has shape (NAXIS3, NAXIS2, NAXIS1)."""
    with open(path, "rb") as f:
        raw = f.read()
    hdr = {}
    pos = 0
    while True:
        block = raw[pos:pos + BLOCK].decode("ascii")
        pos += BLOCK
        done = False
        for i in range(0, BLOCK, 80):
            card = block[i:i + 80]
            key = card[:8].strip()
            if key == "END":
                done = True
                break
            if card[8:10] == "= ":
                val = card[10:].split("/")[0].strip()
                if val.startswith("'"):
                    val = val.strip("'").strip()
                else:
                    try:
                        val = int(val)
                    except ValueError:
                        try:
                            val = float(val)
                        except ValueError:
                            pass
                hdr[key] = val
        if done:
            break
    bitpix = hdr["BITPIX"]
    naxis = hdr["NAXIS"]
    shape = tuple(hdr[f"NAXIS{i}"] for i in range(naxis, 0, -1))
    dtype = {-32: ">f4", -64: ">f8", 32: ">i4", 16: ">i2", 8: "u1"}[bitpix]
    n = int(np.prod(shape))
    data = np.frombuffer(raw, dtype=dtype, count=n, offset=pos).reshape(shape).astype(np.float64)
    return data, hdr


def write(path, data, extra=None):
    """Writes a float64 image cube (nz, ny, nx) or (ny, nx) as a primary HDU."""
    data = np.asarray(data, dtype=np.float64)
    cards = ["SIMPLE  = T", "BITPIX  = -64", f"NAXIS   = {data.ndim}"]
    for i, s in enumerate(reversed(data.shape)):
        cards.append(f"NAXIS{i + 1:<3d}= {s}")
    for k, v in (extra or {}).items():
        cards.append(f"{k[:8]:<8s}= {v!r}" if isinstance(v, str) else f"{k[:8]:<8s}= {v}")
    cards.append("END")
    header = "".join(c.ljust(80)[:80] for c in cards)
    header = header.ljust(((len(header) + BLOCK - 1) // BLOCK) * BLOCK)
    body = data.astype(">f8").tobytes()
    body += b"\0" * ((-len(body)) % BLOCK)
    with open(path, "wb") as f:
        f.write(header.encode("ascii") + body)
