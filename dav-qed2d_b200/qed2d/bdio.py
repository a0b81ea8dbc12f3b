"""BDIO output of the mc and master-field drivers (main/MC.jl:87-100, 140-152;
main/master_field.jl:87-131), host-side Python.

The reference writes these files with BDIO.jl, a third-party package that is
neither part of the reference tree nor pinned in its Manifest.  This module
writes the BDIO container as the BDIO format is published (the ALPHA
collaboration's BDIO C library and its format note): a file header followed by
records, each record a header word and its data, optionally followed by an MD5
checksum record.  Byte compatibility with BDIO.jl has NOT been checked: no BDIO
implementation is available where this was built.  The layout written, all
words little-endian, is:

  file header   uint32  0x7FFBD07E (magic; bit 0 clear marks a header)
                uint32  (1 << 16) | n   (format version 1; n = bytes of the header after this word)
                uint32  dirinfo1 = 0, uint32 dirinfo2 = 0
                uint32  creation time, uint32 modification time (Unix seconds)
                user\\0 user\\0 host\\0 host\\0 protocol\\0   (created by / last modified by,
                                                     created on / last modified on, the
                                                     protocol text given to BDIO_open)
  record        short: uint32 = 1 | fmt << 4 | uinfo << 8 | length << 12           (length < 2^20)
                long:  uint64 = 1 | 1 << 3 | fmt << 4 | uinfo << 8 | length << 12  (length < 2^52)
                then `length` bytes of data
  hash record   a short record, fmt BIN_GENERIC, uinfo 7, 20 bytes: uint32 HASH_MAGIC and
                the MD5 digest of the data of the record just closed

The drivers call it in the order the reference calls BDIO.jl: BDIO_open ->
BDIOWriter(...), BDIO_start_record! -> start_record, BDIO_write! -> write,
BDIO_write_hash! -> write_hash, BDIO_close! -> close."""
import hashlib
import os
import struct
import time

import numpy as np

MAGIC = 0x7FFBD07E
VERSION = 1
HASH_MAGIC = 1515784845
HASH_UINFO = 7

# record formats (BDIO_BIN_GENERIC ... BDIO_ASC_XML)
BIN_GENERIC, ASC_EXEC, BIN_INT32BE, BIN_INT32LE, BIN_INT64BE, BIN_INT64LE = 0x0, 0x1, 0x2, 0x3, 0x4, 0x5
BIN_F32BE, BIN_F32LE, BIN_F64BE, BIN_F64LE, ASC_GENERIC, ASC_XML = 0x6, 0x7, 0x8, 0x9, 0xA, 0xB


def record_word(fmt, uinfo, length, long):
    """The header word of a record (an int; 4 bytes short, 8 bytes long)."""
    if not (0 <= fmt < 16 and 0 <= uinfo < 16):
        raise ValueError("BDIO format and user info are 4-bit fields")
    if length < 0 or length >= (1 << (52 if long else 20)):
        raise ValueError(f"BDIO record of {length} bytes does not fit a {'long' if long else 'short'} record")
    return 1 | (int(bool(long)) << 3) | (fmt << 4) | (uinfo << 8) | (length << 12)


class BDIOWriter:
    """A BDIO file opened for writing (mode "w" of BDIO_open)."""

    def __init__(self, path, protocol, user="", host="", now=None):
        self.fh = open(path, "wb")
        t = int(time.time() if now is None else now) & 0xFFFFFFFF
        strings = b"".join(s.encode() + b"\0" for s in (user, user, host, host, protocol))
        body = struct.pack("<IIII", 0, 0, t, t) + strings
        self.fh.write(struct.pack("<II", MAGIC, (VERSION << 16) | len(body)) + body)
        self._rec = None   # (file offset of the header word, fmt, uinfo, long, md5, length)

    def start_record(self, fmt, uinfo, long=False):
        self._finish()
        pos = self.fh.tell()
        self.fh.write(b"\0" * (8 if long else 4))   # patched when the record is closed
        self._rec = [pos, fmt, uinfo, bool(long), hashlib.md5(), 0]

    def write(self, data):
        """Append bytes, or a NumPy array in little-endian order of its elements
        (float64 for F64LE records), to the open record."""
        if self._rec is None:
            raise RuntimeError("BDIO: write outside a record")
        if isinstance(data, (bytes, bytearray)):
            b = bytes(data)
        else:
            a = np.asarray(data)
            b = np.ascontiguousarray(a, dtype=a.dtype.newbyteorder("<")).tobytes()
        self.fh.write(b)
        self._rec[4].update(b)
        self._rec[5] += len(b)

    def write_hash(self):
        """Close the open record and append its MD5 checksum record."""
        if self._rec is None:
            raise RuntimeError("BDIO: no record to hash")
        digest = self._rec[4].digest()
        self._finish()
        self.fh.write(struct.pack("<I", record_word(BIN_GENERIC, HASH_UINFO, 20, False)))
        self.fh.write(struct.pack("<I", HASH_MAGIC) + digest)

    def _finish(self):
        if self._rec is None:
            return
        pos, fmt, uinfo, long, _, length = self._rec
        end = self.fh.tell()
        self.fh.seek(pos)
        self.fh.write(struct.pack("<Q" if long else "<I", record_word(fmt, uinfo, length, long)))
        self.fh.seek(end)
        self._rec = None

    def close(self):
        self._finish()
        self.fh.flush()
        os.fsync(self.fh.fileno())
        self.fh.close()


def open_run_file(name, s, infile, title, n4):
    """The first two records both drivers write (main/MC.jl:87-100,
    main/master_field.jl:87-101): the input file's bytes (ASC_GENERIC, uinfo 1)
    and F64LE [L1, L2, beta, n4] (uinfo 2), each long and hashed."""
    L1, L2 = s["Lattice"]["size"]
    beta = float(s["Lattice"]["beta"])
    run = s["Run"]
    fb = BDIOWriter(name + ".bdio", title, user=str(run.get("user", "")), host=str(run.get("host", "")))
    fb.start_record(ASC_GENERIC, 1, True)
    with open(infile, "rb") as fh:
        fb.write(fh.read())
    fb.write_hash()
    fb.start_record(BIN_F64LE, 2, True)
    fb.write(np.array([L1, L2, beta, n4], dtype=np.float64))
    fb.write_hash()
    return fb
