"""The .vxq loader's host side, without a GPU: footer and block checks,
CRC-32/IEEE, RLE and dictionary structure, corruption detection and the
row-group rule, through vexq_vxq_verify (which decodes every column but
uploads nothing). Files come from the writer restatement in
oracle/vxq_writer.py; the cases follow storage/storage_test.go (empty file,
CRC corruption, footer truncation, string dictionaries) and
internal/encoding/crc_test.go."""
from __future__ import annotations

import ctypes as C
import os
import struct

import numpy as np
import pytest

from oracle import vxq_writer as VW
from vexq_b200 import abi
from vexq_b200.table import HostTable, bool_column, date_column, float_column, int_column, string_column


def mixed_table(n: int, rg: int, seed: int) -> HostTable:
    """Every column type, NULLs in four of them, NaN and ±0 in the floats."""
    rng = np.random.default_rng(seed)
    iv = rng.integers(-(1 << 40), 1 << 40, n)
    fv = np.rint(rng.uniform(-1e4, 1e4, n)) / 100.0
    fv[rng.choice(n, min(3, n), replace=False)] = np.nan
    fv[rng.choice(n, min(4, n), replace=False)] = -0.0
    dv = (8036 + rng.integers(0, 2500, n)).astype(np.int32)
    bv = rng.integers(0, 2, n)
    sidx = rng.integers(0, 7, n)
    v_int = rng.random(n) > 0.1
    v_str = rng.random(n) > 0.05
    v_bool = rng.random(n) > 0.2
    v_date = rng.random(n) > 0.02
    modes = ["AIR", "FOB", "MAIL", "RAIL", "REG AIR", "SHIP", "TRUCK"]
    cols = [int_column("i", iv, v_int), float_column("f", fv), date_column("d", dv, v_date),
            string_column("s", sidx, modes, n, rg, v_str), bool_column("b", bv, v_bool),
            int_column("k", np.arange(n, dtype=np.int64))]
    return HostTable(cols, n, rg)


def verify(path):
    s = abi.VxqSummary()
    rc = abi.load().vexq_vxq_verify(os.fsencode(str(path)), C.byref(s))
    return rc, s, abi.load().vexq_last_error().decode()


def rewrite(path, at: int, data: bytes):
    b = bytearray(open(path, "rb").read())
    b[at:at + len(data)] = data
    open(path, "wb").write(bytes(b))


def test_crc32_check_value():
    # the published CRC-32/IEEE check value; the library's own CRC is checked
    # against it through every verified file below
    assert VW.crc32(b"123456789") == 0xCBF43926
    assert VW.crc32(b"") == 0


def test_round_trip_summary(tmp_path):
    n, rg = 4096 * 3 + 1500, 4096  # a last row group of 1,500 rows: a partial block
    t = mixed_table(n, rg, 1)
    p = tmp_path / "t.vxq"
    VW.write_vxq(str(p), t)
    rc, s, err = verify(p)
    assert rc == abi.OK, err
    assert (s.nrows, s.ncols, s.n_rg, s.rg_rows) == (n, 6, 4, rg)
    assert s.null_columns == 4  # i, d, s, b
    assert 0 < s.bytes_checked < os.path.getsize(p)


def test_row_groups_not_a_multiple_of_eight(tmp_path):
    t = mixed_table(100 * 5 + 37, 100, 2)
    p = tmp_path / "t.vxq"
    VW.write_vxq(str(p), t)
    rc, s, err = verify(p)
    assert rc == abi.OK, err
    assert (s.nrows, s.n_rg, s.rg_rows) == (537, 6, 100)


def test_empty_file(tmp_path):
    t = HostTable([int_column("x", np.zeros(0, np.int64))], 0, 65536)
    p = tmp_path / "e.vxq"
    VW.write_vxq(str(p), t)
    rc, s, err = verify(p)
    assert rc == abi.OK, err
    assert (s.nrows, s.ncols, s.n_rg) == (0, 1, 0)


def test_block_crc_corruption(tmp_path):
    # storage_test.go TestCRCCorruption: a 100-row int64 row group, byte 100
    # flipped (inside the first block's bitmap and values)
    t = HostTable([int_column("x", np.zeros(100, np.int64))], 100, 100)
    p = tmp_path / "c.vxq"
    VW.write_vxq(str(p), t)
    b = open(p, "rb").read()
    rewrite(p, 100, bytes([b[100] ^ 0xFF]))
    rc, _, err = verify(p)
    assert rc == abi.ECORRUPT and "checksum mismatch" in err and "col=x" in err, (rc, err)


def test_footer_truncation_and_magic(tmp_path):
    t = mixed_table(3000, 1024, 3)
    p = tmp_path / "f.vxq"
    VW.write_vxq(str(p), t)
    good = open(p, "rb").read()
    open(p, "wb").write(good[:-1])  # TestFooterCorruption
    rc, _, err = verify(p)
    assert rc == abi.ECORRUPT and "bad magic" in err, (rc, err)
    open(p, "wb").write(good[:-4] + b"VXQ2")
    rc, _, err = verify(p)
    assert rc == abi.ECORRUPT and "bad magic" in err, (rc, err)
    body_len = struct.unpack("<q", good[-12:-4])[0]
    at = len(good) - 16 - body_len + 9  # inside the footer body
    open(p, "wb").write(good[:at] + bytes([good[at] ^ 1]) + good[at + 1:])
    rc, _, err = verify(p)
    assert rc == abi.ECORRUPT and "checksum mismatch" in err, (rc, err)
    open(p, "wb").write(good[:-12] + struct.pack("<q", len(good)) + b"VXQ1")  # footer longer than the file
    rc, _, err = verify(p)
    assert rc == abi.ECORRUPT and "corrupt footer" in err, (rc, err)
    open(p, "wb").write(b"")
    rc, _, err = verify(p)
    assert rc == abi.ECORRUPT


def test_dictionary_corruption(tmp_path):
    t = mixed_table(2048, 1024, 4)
    p = tmp_path / "d.vxq"
    meta = VW.write_vxq(str(p), t)
    sec = meta[1].cols[3]  # column "s", row group 1
    at = sec.offset + sec.dict_off + 4 + 2  # inside the offsets
    b = open(p, "rb").read()
    rewrite(p, at, bytes([b[at] ^ 0x10]))
    rc, _, err = verify(p)
    assert rc == abi.ECORRUPT and "unmarshal dict" in err and "rg=1" in err, (rc, err)


def _patch_block(p, off: int, size: int, patch):
    """Rewrites a block through `patch` (a bytearray of it without its CRC)
    and seals it with a fresh CRC, so only the structure checks can object."""
    b = bytearray(open(p, "rb").read())
    blk = bytearray(b[off:off + size - 4])
    patch(blk)
    b[off:off + size] = VW.with_crc(bytes(blk))
    open(p, "wb").write(bytes(b))


def test_string_code_out_of_range(tmp_path):
    t = mixed_table(2048, 1024, 5)
    p = tmp_path / "s.vxq"
    meta = VW.write_vxq(str(p), t)
    sec = meta[0].cols[3]
    valid = t.columns[3].valid_mask(t.nrows)
    row = int(np.flatnonzero(valid[:1024])[0])

    def patch(blk):
        blk[VW.BITMAP_BYTES + 4 * row:VW.BITMAP_BYTES + 4 * row + 4] = struct.pack("<I", 7)  # 7 entries: codes 0..6
    _patch_block(p, sec.offset, VW.BITMAP_BYTES + 1024 * 4 + 4, patch)
    rc, _, err = verify(p)
    assert rc == abi.ECORRUPT and "dictionary code out of range" in err, (rc, err)


def test_bool_runs_must_cover_the_block(tmp_path):
    t = mixed_table(1024, 1024, 6)
    p = tmp_path / "b.vxq"
    meta = VW.write_vxq(str(p), t)
    sec = meta[0].cols[4]
    runs = struct.unpack("<I", open(p, "rb").read()[sec.offset:sec.offset + 4])[0]

    def patch(blk):
        ln = struct.unpack("<I", blk[4:8])[0]
        blk[4:8] = struct.pack("<I", ln - 1)  # the runs now cover 1,023 rows
    _patch_block(p, sec.offset, 4 + 5 * runs + 4, patch)
    rc, _, err = verify(p)
    assert rc == abi.ECORRUPT and "rle bool" in err, (rc, err)


def test_uneven_row_groups_are_refused(tmp_path):
    t = mixed_table(300, 100, 7)
    p = tmp_path / "u.vxq"
    VW.write_vxq(str(p), t, rg_sizes=[100, 150, 50])
    rc, _, err = verify(p)
    assert rc == abi.ENOTSUP and "row group 1" in err, (rc, err)
    VW.write_vxq(str(p), t, rg_sizes=[150, 150])  # a full last row group is fine
    rc, s, err = verify(p)
    assert rc == abi.OK and (s.n_rg, s.rg_rows) == (2, 150), err


def test_unknown_column_name_is_refused_before_any_device_work(tmp_path):
    t = mixed_table(500, 256, 8)
    p = tmp_path / "n.vxq"
    VW.write_vxq(str(p), t)
    h = C.c_void_p()
    names = (C.c_char_p * 2)(b"i", b"nope")
    rc = abi.load().vexq_table_load_vxq(os.fsencode(str(p)), names, 2, C.byref(h))
    assert rc == abi.EINVAL and "no column named nope" in abi.load().vexq_last_error().decode()
    rc = abi.load().vexq_table_load_vxq(os.fsencode(str(tmp_path / "absent.vxq")), None, 0, C.byref(h))
    assert rc == abi.EINVAL


@pytest.mark.parametrize("nrows", [1, 7, 1023, 1025])
def test_small_tables(tmp_path, nrows):
    t = mixed_table(nrows, 65536, 9)
    p = tmp_path / "m.vxq"
    VW.write_vxq(str(p), t)
    rc, s, err = verify(p)
    assert rc == abi.OK and s.nrows == nrows and s.n_rg == 1, err
