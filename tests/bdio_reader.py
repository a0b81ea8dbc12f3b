"""An independent BDIO reader for the tests: parses a file written by
qed2d/bdio.py word by word with `struct`, without using that module, so the
writer is checked against the layout as written down rather than against
itself.  Layout (little-endian): a header (magic 0x7FFBD07E, version << 16 |
header bytes, dirinfo1, dirinfo2, creation and modification times, five
NUL-terminated strings), then records whose first word has bit 0 set: bit 3
long (64-bit word) or short (32-bit), bits 4-7 format, 8-11 user info, 12- the
data length in bytes."""
import struct


def read_bdio(path):
    data = open(path, "rb").read()
    magic, w1 = struct.unpack_from("<II", data, 0)
    assert magic == 0x7FFBD07E, hex(magic)
    version, hlen = w1 >> 16, w1 & 0xFFFF
    body = data[8:8 + hlen]
    dir1, dir2, ctime, mtime = struct.unpack_from("<IIII", body, 0)
    strings = body[16:].split(b"\0")
    assert strings[-1] == b"" and len(strings) == 6, strings
    header = {"version": version, "dirinfo": (dir1, dir2), "ctime": ctime, "mtime": mtime,
              "cuser": strings[0].decode(), "muser": strings[1].decode(), "chost": strings[2].decode(),
              "mhost": strings[3].decode(), "protocol": strings[4].decode()}
    pos, records = 8 + hlen, []
    while pos < len(data):
        (w,) = struct.unpack_from("<I", data, pos)
        assert w & 1, f"record word without bit 0 at {pos}"
        long = bool(w & 8)
        if long:
            (w,) = struct.unpack_from("<Q", data, pos)
            pos += 8
        else:
            pos += 4
        fmt, uinfo, length = (w >> 4) & 0xF, (w >> 8) & 0xF, w >> 12
        records.append({"fmt": fmt, "uinfo": uinfo, "long": long, "data": data[pos:pos + length]})
        pos += length
    assert pos == len(data), "trailing bytes"
    return header, records
