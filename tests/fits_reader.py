"""Minimal FITS binary-table reader (numpy) for checking the library's
HEALPix products without healpy or astropy."""
import numpy as np

_TYPES = {"E": ">f4", "D": ">f8", "J": ">i4", "K": ">i8", "I": ">i2", "B": "u1"}


def _header(buf, pos):
    cards = {}
    order = []
    while True:
        block = buf[pos:pos + 2880].decode("ascii")
        pos += 2880
        for i in range(0, 2880, 80):
            c = block[i:i + 80]
            key = c[:8].strip()
            if key == "END":
                return cards, order, pos
            if c[8:10] == "= ":
                v = c[10:]
                if v.lstrip().startswith("'"):
                    s = v.lstrip()[1:]
                    val = s[:s.index("'")].rstrip()
                else:
                    v = v.split("/")[0].strip()
                    if v in ("T", "F"):
                        val = v == "T"
                    else:
                        try:
                            val = int(v)
                        except ValueError:
                            val = float(v)
                cards[key] = val
                order.append(key)


def read_table(path):
    """Return (header dict, {column name: flat array}) of the first BINTABLE."""
    buf = open(path, "rb").read()
    _, _, pos = _header(buf, 0)
    hdr, _, pos = _header(buf, pos)
    assert hdr["XTENSION"] == "BINTABLE"
    nrows, width, nf = hdr["NAXIS2"], hdr["NAXIS1"], hdr["TFIELDS"]
    fields = []
    for i in range(1, nf + 1):
        form = hdr["TFORM%d" % i]
        rep = int(form[:-1]) if len(form) > 1 else 1
        fields.append((hdr["TTYPE%d" % i], _TYPES[form[-1]], rep))
    dt = np.dtype([(n, t, (r,)) for n, t, r in fields])
    assert dt.itemsize == width
    data = np.frombuffer(buf, dtype=dt, count=nrows, offset=pos)
    return hdr, {n: data[n].reshape(-1).astype(np.dtype(t).newbyteorder("=")) for n, t, _ in fields}


def write_mask(path, values, nside, ordering="NESTED", per_row=1024, code="E"):
    """A one-column HEALPix mask table (as healpy writes one) for file_inmask."""
    import numpy as np
    dt = {"E": ">f4", "D": ">f8", "J": ">i4", "B": "u1"}[code]
    v = np.asarray(values).astype(dt)
    per_row = min(per_row, v.size)
    assert v.size % per_row == 0
    nrow = v.size // per_row

    def hdr(cards):
        s = "".join(c.ljust(80)[:80] for c in cards + ["END"])
        return (s + " " * ((2880 - len(s) % 2880) % 2880)).encode("ascii")

    def kv(k, val):
        if isinstance(val, str):
            val = "'" + val.ljust(8) + "'"
        elif isinstance(val, bool):
            val = ("T" if val else "F").rjust(20)
        else:
            val = str(val).rjust(20)
        return k.ljust(8) + "= " + val

    prim = hdr([kv("SIMPLE", True), kv("BITPIX", 8), kv("NAXIS", 0), kv("EXTEND", True)])
    ext = hdr([kv("XTENSION", "BINTABLE"), kv("BITPIX", 8), kv("NAXIS", 2),
               kv("NAXIS1", per_row * v.itemsize), kv("NAXIS2", nrow), kv("PCOUNT", 0),
               kv("GCOUNT", 1), kv("TFIELDS", 1), kv("TTYPE1", "MASK"),
               kv("TFORM1", "%d%s" % (per_row, code)), kv("PIXTYPE", "HEALPIX"),
               kv("ORDERING", ordering), kv("NSIDE", nside)])
    data = v.tobytes()
    data += b"\0" * ((2880 - len(data) % 2880) % 2880)
    with open(path, "wb") as f:
        f.write(prim + ext + data)
