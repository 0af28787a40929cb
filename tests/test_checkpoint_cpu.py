"""Checkpoint container on the CPU: the header of a file laid out by hand as the
C ABI documents it (the data model of HDF5Writer::writeCheckpoint,
hdf5_io.cpp:166-233, plus the block geometry) reads back through
granite_ccz4_checkpoint_header; wrong magic, version, field count, truncation
and a too-small block array are rejected. No GPU is touched."""
import struct

import pytest

import granite_b200 as gb

MAGIC = b"GRNB200\0"


def write_file(path, blocks, step=7, time=1.25, level_times=(1.25, 1.25), matter=0, version=1, nvars=22,
               truncate=False):
    head = struct.pack("<8sII6id", MAGIC, version, 4096, step, len(blocks), nvars, len(level_times), matter, 0,
                       time)
    head += struct.pack(f"<{len(level_times)}d", *level_times)
    for (n, lo, hi, lev, bid) in blocks:
        head += struct.pack("<4i3d3d2i", *n, 4, *lo, *hi, lev, bid)
    if truncate:
        head = head[:-10]
    with open(path, "wb") as f:
        f.write(head)


BLOCKS = [((16, 16, 16), (-8.0, -8.0, -8.0), (8.0, 8.0, 8.0), 0, 0),
          ((22, 16, 16), (-6.0, -4.0, -4.0), (5.0, 4.0, 4.0), 1, 1000)]


def test_header_round_trip(tmp_path):
    p = tmp_path / "ck.bin"
    write_file(p, BLOCKS)
    h = gb.checkpoint_header(str(p))
    assert h["step"] == 7 and h["time"] == 1.25 and not h["has_matter"]
    got = [(b.ncells, b.lo, b.hi, b.level, b.id) for b in h["blocks"]]
    assert got == BLOCKS


@pytest.mark.parametrize("kw", [dict(version=2), dict(nvars=21), dict(truncate=True)])
def test_bad_headers_rejected(tmp_path, kw):
    p = tmp_path / "bad.bin"
    write_file(p, BLOCKS, **kw)
    with pytest.raises(gb.GraniteError):
        gb.checkpoint_header(str(p))


def test_wrong_magic_and_small_array(tmp_path):
    p = tmp_path / "m.bin"
    with open(p, "wb") as f:
        f.write(b"HDF\x89" + b"\0" * 200)
    with pytest.raises(gb.GraniteError):
        gb.checkpoint_header(str(p))
    write_file(p, BLOCKS)
    lib = gb.load_library()
    import ctypes as C
    n = C.c_int()
    one = (gb._BlockDesc * 1)()
    assert lib.granite_ccz4_checkpoint_header(str(p).encode(), None, None, None, one, 1, C.byref(n)) == -8
    assert n.value == 2
