"""Float32 TIFF output (ms_write_tiff_f32): parsed back with a minimal reader
and checked against the fields the reference GUI writes
(CUDA Simulation GUI/MainWindow.xaml.cs:697-707) and the data."""
import struct

import numpy as np
import pytest


def read_tiff_f32(path):
    b = open(path, "rb").read()
    assert b[:4] == b"II*\x00"
    ifd = struct.unpack_from("<I", b, 4)[0]
    n = struct.unpack_from("<H", b, ifd)[0]
    tags = {}
    for i in range(n):
        tid, typ, cnt = struct.unpack_from("<HHI", b, ifd + 2 + 12 * i)
        val = struct.unpack_from("<H" if typ == 3 else "<I", b, ifd + 2 + 12 * i + 8)[0]
        tags[tid] = val
    assert struct.unpack_from("<I", b, ifd + 2 + 12 * n)[0] == 0
    nx, ny = tags[256], tags[257]
    data = np.frombuffer(b, "<f4", nx * ny, tags[273]).reshape(ny, nx)
    return tags, data


def test_write_tiff_f32(tmp_path):
    from cudamultislice_b200 import write_tiff

    a = np.random.default_rng(3).standard_normal((37, 53)).astype(np.float32)
    p = str(tmp_path / "x.tiff")
    write_tiff(p, a)
    tags, d = read_tiff_f32(p)
    assert tags[258] == 32 and tags[339] == 3 and tags[277] == 1  # 32-bit IEEE float, one sample
    assert tags[259] == 1 and tags[262] == 1 and tags[274] == 1 and tags[284] == 1  # raw, MinIsBlack, top-left
    assert tags[278] == 37 and tags[279] == 37 * 53 * 4  # one strip
    assert np.array_equal(d, a)


def test_write_tiff_errors(tmp_path):
    from cudamultislice_b200 import MultisliceError, write_tiff

    with pytest.raises(MultisliceError):
        write_tiff(str(tmp_path / "missing_dir" / "x.tiff"), np.zeros((4, 4)))
