"""Pure-Python TIFF writer and reader for the map-loading tests: an
independent implementation of the TIFF 6.0 layout (strips or tiles,
uncompressed / LZW / PackBits / Deflate, predictors 1-3, either byte order,
BigTIFF) used to produce synthetic maps and to decode the reference's
fixtures a second way."""
import struct
import zlib

import numpy as np


# ---- compression ----
def lzw_encode(data: bytes) -> bytes:
    """TIFF LZW (MSB-first codes, Clear 256, EOI 257, early code-width change)."""
    out_bits = []

    def put(code, width):
        out_bits.append((code, width))

    table = {bytes([j]): j for j in range(256)}
    nxt, width = 258, 9
    put(256, width)
    w = b""
    for byte in data:
        wc = w + bytes([byte])
        if wc in table:
            w = wc
            continue
        put(table[w], width)
        table[wc] = nxt
        nxt += 1
        # the encoder widens when the next code no longer fits; its decoder,
        # one table entry behind, widens one code early
        if nxt >= (1 << width) and width < 12:
            width += 1
        if nxt >= 4094:  # leave room: clear and start over
            put(256, width)
            table = {bytes([j]): j for j in range(256)}
            nxt, width = 258, 9
        w = bytes([byte])
    if w:
        put(table[w], width)
        nxt += 1
        if nxt >= (1 << width) and width < 12:
            width += 1
    put(257, width)
    acc, nacc, buf = 0, 0, bytearray()
    for code, wd in out_bits:
        acc = (acc << wd) | code
        nacc += wd
        while nacc >= 8:
            nacc -= 8
            buf.append((acc >> nacc) & 0xFF)
    if nacc:
        buf.append((acc << (8 - nacc)) & 0xFF)
    return bytes(buf)


def lzw_decode(data: bytes) -> bytes:
    table = [bytes([j]) for j in range(256)] + [b"", b""]
    width, pos, out, prev = 9, 0, bytearray(), None
    nbits = len(data) * 8
    while pos + width <= nbits:
        code = 0
        for k in range(width):
            code = (code << 1) | ((data[(pos + k) >> 3] >> (7 - ((pos + k) & 7))) & 1)
        pos += width
        if code == 257:
            break
        if code == 256:
            table = table[:258]
            width, prev = 9, None
            continue
        if prev is None:
            entry = table[code]
        elif code < len(table):
            entry = table[code]
            table.append(prev + entry[:1])
        else:
            entry = prev + prev[:1]
            table.append(entry)
        out += entry
        prev = entry
        if len(table) + 1 >= (1 << width) and width < 12:
            width += 1
    return bytes(out)


def packbits_encode(data: bytes) -> bytes:
    out, i = bytearray(), 0
    while i < len(data):
        j = i
        while j + 1 < len(data) and data[j + 1] == data[i] and j - i < 127:
            j += 1
        if j > i:  # a run of j - i + 1 equal bytes
            out += bytes([(257 - (j - i + 1)) & 0xFF, data[i]])
            i = j + 1
        else:
            k = i
            while k < len(data) and k - i < 128 and not (k + 1 < len(data) and data[k + 1] == data[k]):
                k += 1
            k = max(k, i + 1)
            out += bytes([k - i - 1]) + data[i:k]
            i = k
    return bytes(out)


def compress(raw: bytes, compression: int) -> bytes:
    if compression == 1:
        return raw
    if compression == 5:
        return lzw_encode(raw)
    if compression in (8, 32946):
        return zlib.compress(raw)
    if compression == 32773:
        return packbits_encode(raw)
    raise ValueError(compression)


# ---- prediction (encoder side) ----
def predict(block: np.ndarray, predictor: int, big: bool) -> bytes:
    """block: [rows, cols] samples; returns the encoded bytes in file order."""
    rows, cols = block.shape
    isz = block.dtype.itemsize
    order = ">" if big else "<"
    if predictor == 3:
        be = block.astype(block.dtype.newbyteorder(">"))
        out = bytearray()
        for r in range(rows):
            b = np.frombuffer(be[r].tobytes(), dtype=np.uint8).reshape(cols, isz).T.reshape(-1)
            d = np.diff(b.astype(np.int16), prepend=0).astype(np.uint8)
            d[0] = b[0]
            out += d.tobytes()
        return bytes(out)
    if predictor == 2:
        u = block.view(np.dtype("u%d" % isz))
        d = u.copy()
        d[:, 1:] = u[:, 1:] - u[:, :-1]
        return d.astype(d.dtype.newbyteorder(order)).tobytes()
    return block.astype(block.dtype.newbyteorder(order)).tobytes()


# ---- writer ----
SAMPLE_FORMAT = {"u": 1, "i": 2, "f": 3}


def write_tiff(path, arr, compression=1, predictor=1, big=False, bigtiff=False, tile=None, rows_per_strip=None,
               nodata=None, photometric=1, sample_format=True, spp=1):
    arr = np.ascontiguousarray(arr)
    h, w = arr.shape
    isz = arr.dtype.itemsize
    o = ">" if big else "<"
    blocks = []
    if tile:
        tw, th = tile
        for ty in range(0, h, th):
            for tx in range(0, w, tw):
                blk = np.zeros((th, tw), dtype=arr.dtype)
                part = arr[ty:ty + th, tx:tx + tw]
                blk[:part.shape[0], :part.shape[1]] = part
                blocks.append(compress(predict(blk, predictor, big), compression))
    else:
        rps = rows_per_strip or h
        for y in range(0, h, rps):
            blocks.append(compress(predict(arr[y:y + rps], predictor, big), compression))
    tags = [(256, 4, [w]), (257, 4, [h]), (258, 3, [isz * 8] * spp), (259, 3, [compression])]
    if photometric is not None:
        tags.append((262, 3, [photometric]))
    tags.append((277, 3, [spp]))
    if predictor != 1:
        tags.append((317, 3, [predictor]))
    if sample_format:
        tags.append((339, 3, [SAMPLE_FORMAT[arr.dtype.kind]] * spp))
    if tile:
        tags += [(322, 3, [tile[0]]), (323, 3, [tile[1]])]
    else:
        tags.append((278, 4, [rows_per_strip or h]))
    if nodata is not None:
        tags.append((42113, 2, nodata.encode() + b"\0"))
    # layout: header, image data, then the IFD and its out-of-line values
    head = 16 if bigtiff else 8
    data = bytearray()
    offsets, counts = [], []
    for b in blocks:
        offsets.append(head + len(data))
        counts.append(len(b))
        data += b
        if len(data) % 2:
            data += b"\0"
    off_type = 16 if bigtiff else 4
    tags.append((324 if tile else 273, off_type, offsets))
    tags.append((325 if tile else 279, off_type, counts))
    tags.sort(key=lambda t: t[0])
    ifd_off = head + len(data)
    entry_size, count_fmt, inline = (20, "Q", 8) if bigtiff else (12, "I", 4)
    nfmt = "Q" if bigtiff else "H"
    ifd_len = struct.calcsize(o + nfmt) + entry_size * len(tags) + (8 if bigtiff else 4)
    extra = bytearray()
    entries = bytearray()
    fmts = {2: "s", 3: "H", 4: "I", 16: "Q"}
    for tag, typ, vals in tags:
        if typ == 2:
            payload, count = bytes(vals), len(vals)
        else:
            payload, count = struct.pack(o + fmts[typ] * len(vals), *vals), len(vals)
        if len(payload) <= inline:
            field = payload + b"\0" * (inline - len(payload))
        else:
            where = ifd_off + ifd_len + len(extra)
            extra += payload
            if len(extra) % 2:
                extra += b"\0"
            field = struct.pack(o + ("Q" if bigtiff else "I"), where)
        entries += struct.pack(o + "HH" + count_fmt, tag, typ, count) + field
    ifd = struct.pack(o + nfmt, len(tags)) + entries + b"\0" * (8 if bigtiff else 4)
    bom = b"MM" if big else b"II"
    if bigtiff:
        header = bom + struct.pack(o + "HHHQ", 43, 8, 0, ifd_off)
    else:
        header = bom + struct.pack(o + "HI", 42, ifd_off)
    with open(path, "wb") as f:
        f.write(header + data + ifd + extra)


# ---- reader (strips; the reference fixtures' layout) ----
def read_tiff_strips(path):
    b = open(path, "rb").read()
    o = "<" if b[:2] == b"II" else ">"
    assert struct.unpack(o + "H", b[2:4])[0] == 42
    (off,) = struct.unpack(o + "I", b[4:8])
    (n,) = struct.unpack(o + "H", b[off:off + 2])
    tags = {}
    sizes = {1: 1, 2: 1, 3: 2, 4: 4, 5: 8, 12: 8, 16: 8}
    fmts = {1: "B", 3: "H", 4: "I", 16: "Q"}
    for j in range(n):
        e = b[off + 2 + 12 * j: off + 14 + 12 * j]
        tag, typ, cnt = struct.unpack(o + "HHI", e[:8])
        if typ not in fmts:
            continue
        sz = sizes[typ] * cnt
        raw = e[8:8 + sz] if sz <= 4 else b[struct.unpack(o + "I", e[8:12])[0]:][:sz]
        tags[tag] = struct.unpack(o + fmts[typ] * cnt, raw)
    w, h, bits, comp = tags[256][0], tags[257][0], tags[258][0], tags.get(259, (1,))[0]
    fmt = tags.get(339, (1,))[0]
    pred = tags.get(317, (1,))[0]
    dt = np.dtype({(1, 32): "u4", (3, 64): "f8", (3, 32): "f4", (1, 16): "u2", (1, 8): "u1"}[(fmt, bits)])
    rps = tags.get(278, (h,))[0]
    out = bytearray()
    for so, sc in zip(tags[273], tags[279]):
        chunk = b[so:so + sc]
        raw = {1: lambda c: c, 5: lzw_decode, 8: zlib.decompress}[comp](chunk)
        rows = min(rps, h - len(out) // (w * dt.itemsize))
        raw = raw[:rows * w * dt.itemsize]
        a = np.frombuffer(raw, dtype=dt.newbyteorder(o)).reshape(rows, w)
        if pred == 2:
            u = a.view(np.dtype(dt.newbyteorder(o).str.replace("f", "u")))
            a = np.cumsum(u.astype(u.dtype.newbyteorder("=")), axis=1, dtype=u.dtype.newbyteorder("=")).view(
                dt.newbyteorder("="))
        out += np.ascontiguousarray(a, dtype=dt.newbyteorder("=")).tobytes()
    return np.frombuffer(bytes(out), dtype=dt.newbyteorder("=")).reshape(h, w)
