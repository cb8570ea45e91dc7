""".npz reading (host side): archive listing, member extraction, deflate,
ZIP64 and CRC checks, against archives written by NumPy's own writer and
Python's zipfile -- the reader semantics of ferray-io/src/npz/mod.rs."""
import io
import struct
import zipfile

import numpy as np
import pytest

import ferray_b200 as fg


def savez(compressed=False, **arrays):
    buf = io.BytesIO()
    (np.savez_compressed if compressed else np.savez)(buf, **arrays)
    return buf.getvalue()


@pytest.mark.parametrize("compressed", [False, True])
def test_names_and_members_match_zipfile(compressed):
    # mod.rs:219-240 (savez_and_load) / :242-256 (savez_compressed_and_load)
    a = np.array([1.0, 2.0, 3.0])
    b = np.array([[1, 2], [3, 4]], np.int32)
    data = savez(compressed, a=a, b=b)
    assert fg.npz_names(data) == ["a", "b"]
    zf = zipfile.ZipFile(io.BytesIO(data))
    for name in ("a", "b"):
        raw = fg.npz_read(data, name)
        assert raw == zf.read(name + ".npy")
    dt, shape, fortran, off = fg.npy_parse(fg.npz_read(data, "a"))
    assert dt == np.float64 and shape == (3,) and not fortran


def test_repeated_gets_and_missing_key():
    # mod.rs:258-266 (npz_missing_key) and :268-285 (lazy get then get)
    data = savez(a=np.arange(4.0), b=np.ones((2, 3), np.float32))
    for _ in range(3):
        assert fg.npz_read(data, "b") == fg.npz_read(data, "b")
        assert len(fg.npz_read(data, "a")) > 0
    with pytest.raises(fg.FerrayError):
        fg.npz_read(data, "nonexistent")


def test_empty_archive():
    # mod.rs:287-296 (npz_empty)
    assert fg.npz_names(savez()) == []


def test_member_without_npy_suffix_is_listed_but_not_readable():
    # mod.rs:130-133 strips ".npy" for names(); get() reads "<name>.npy" only
    buf = io.BytesIO()
    with zipfile.ZipFile(buf, "w") as zf:
        f = io.BytesIO()
        np.save(f, np.arange(3.0))
        zf.writestr("raw", f.getvalue())
        zf.writestr("x.npy", f.getvalue())
    data = buf.getvalue()
    assert fg.npz_names(data) == ["raw", "x"]
    with pytest.raises(fg.FerrayError):
        fg.npz_read(data, "raw")
    assert fg.npz_read(data, "x") == zipfile.ZipFile(io.BytesIO(data)).read("x.npy")


def test_zip64_records(monkeypatch):
    """ZIP64 end record, locator and central-directory extra fields (forced
    by lowering zipfile's limit, as archives above 4 GiB get them)."""
    monkeypatch.setattr(zipfile, "ZIP64_LIMIT", 1)
    a = np.arange(10, dtype=np.int16)
    for method in (zipfile.ZIP_STORED, zipfile.ZIP_DEFLATED):
        buf = io.BytesIO()
        with zipfile.ZipFile(buf, "w", compression=method, allowZip64=True) as zf:
            f = io.BytesIO()
            np.save(f, a)
            zf.writestr("a.npy", f.getvalue())
            zf.writestr("b.npy", f.getvalue())
        data = buf.getvalue()
        assert b"PK\x06\x06" in data and b"PK\x06\x07" in data  # the ZIP64 records are there
        assert fg.npz_names(data) == ["a", "b"]
        assert fg.npz_read(data, "b") == zipfile.ZipFile(io.BytesIO(data)).read("b.npy")


def test_crc_and_truncation_are_errors():
    data = bytearray(savez(a=np.arange(64.0)))
    zf = zipfile.ZipFile(io.BytesIO(bytes(data)))
    info = zf.getinfo("a.npy")
    nlen, elen = struct.unpack("<HH", data[info.header_offset + 26:info.header_offset + 30])
    payload = info.header_offset + 30 + nlen + elen
    data[payload + info.file_size - 1] ^= 0x5A  # last payload byte
    with pytest.raises(fg.FerrayError, match="CRC"):
        fg.npz_read(bytes(data), "a")
    good = savez(a=np.arange(64.0))
    for cut in (10, len(good) // 2, len(good) - 1):
        with pytest.raises(fg.FerrayError):
            fg.npz_names(good[:cut])
    with pytest.raises(fg.FerrayError):
        fg.npz_names(b"not a zip archive at all, just bytes" * 3)
