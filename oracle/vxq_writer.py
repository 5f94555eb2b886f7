"""TEST INFRASTRUCTURE ONLY: a restatement of the reference's .vxq writer.

Writes a HostTable as a .vxq file the way storage.Writer does, so tests can
hand the library's loader real files and check what it decodes. Imported by
tests/ only; the product package never imports it.

Layout (storage/writer.go): the magic "VXQ1" (:52-58); per row group, per
column, a section of 1,024-row blocks (storage/format.go:8):
  * INT64 / FLOAT64 / DATE / STRING codes: [128-byte validity bitmap, bits past
    the block's rows zero][rows x value, little-endian][CRC32] (:205-372);
  * BOOL: RLE runs [u32 runs][runs x (u32 length, u8 value)][CRC32], value 0xFF
    for a NULL run (storage/codec.go:253-290);
  * STRING sections end with the row group's dictionary
    [u32 n][n x u32 offset][u32 bytes][bytes][CRC32] (storage/codec.go:82-99),
    codes in first-occurrence order over the row group's non-NULL rows, NULL
    rows coded 0xFFFFFFFF (:374-420);
then the footer body (:423-472) and the trailer [CRC32 u32][body length i64]
["VXQ1"]. Zone-map statistics follow the writer's rules per type (:205-372).
CRC-32/IEEE is zlib's crc32 (the same polynomial and reflection); its value
on b"123456789" is the published check value 0xCBF43926.
"""
from __future__ import annotations

import math
import os
import struct
import sys
import zlib
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from vexq_b200 import abi  # noqa: E402  (type codes only)
from vexq_b200.table import HostTable  # noqa: E402

MAGIC = b"VXQ1"
BLOCK_ROWS = 1024
BITMAP_BYTES = 128
ENC_PLAIN, ENC_RLE, ENC_DICT = 0, 1, 2


def crc32(b: bytes) -> int:
    return zlib.crc32(b) & 0xFFFFFFFF


def with_crc(b: bytes) -> bytes:
    """AppendChecksum (internal/encoding/crc.go:20-25)."""
    return b + struct.pack("<I", crc32(b))


@dataclass
class ColStats:
    """ZoneMap (storage/schema.go:26-35) as the writer fills it."""
    null_count: int = 0
    sum: int = 0          # raw int64 bits
    min: int = 0          # raw uint64 bits
    max: int = 0
    has_min_max: bool = False


@dataclass
class Section:
    offset: int
    length: int
    stats: ColStats
    dict_off: int = 0
    dict_len: int = 0


@dataclass
class RowGroupMeta:
    file_offset: int
    rows: int
    cols: List[Section] = field(default_factory=list)


def _f64_bits(x: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def _i64(x: int) -> int:
    x &= (1 << 64) - 1
    return x - (1 << 64) if x >> 63 else x


def _first_equal(v: np.ndarray, m) -> int:
    """Index of the first element comparing equal to m (the running min/max
    of the writer's strict comparisons stops at the first such element)."""
    return int(np.flatnonzero(v == m)[0])


def _float_stats(v: np.ndarray, nulls: int) -> ColStats:
    """writeFloat64Blocks (storage/writer.go:248-300): sequential sum in row
    order; min/max start at the first non-NULL value and move only on strict
    < / >, so a leading NaN stays and later NaNs are skipped."""
    st = ColStats(null_count=nulls)
    if len(v) == 0:
        st.sum = 0
        return st
    st.sum = _i64(_f64_bits(float(np.add.accumulate(v)[-1])))
    st.has_min_max = True
    first = v[0]
    if math.isnan(first):
        st.min = st.max = _f64_bits(float(first))
        return st
    ok = v[~np.isnan(v)]
    lo, hi = ok.min(), ok.max()
    st.min = _f64_bits(float(ok[_first_equal(ok, lo)]))
    st.max = _f64_bits(float(ok[_first_equal(ok, hi)]))
    return st


def _bitmap(valid: np.ndarray) -> bytes:
    """A block's validity bitmap padded to 128 bytes, bits past its rows zero."""
    b = np.packbits(valid.astype(bool), bitorder="little").tobytes()
    return b + b"\x00" * (BITMAP_BYTES - len(b))


def _rle_bool(vals: np.ndarray, valid: np.ndarray) -> bytes:
    """EncodeRLEBool (storage/codec.go:253-290)."""
    cur = np.where(valid, (vals != 0).astype(np.int32), 0xFF)
    starts = np.flatnonzero(np.r_[True, cur[1:] != cur[:-1]]) if len(cur) else np.zeros(0, np.int64)
    ends = np.r_[starts[1:], len(cur)]
    out = bytearray(struct.pack("<I", len(starts)))
    for s, e in zip(starts, ends):
        out += struct.pack("<IB", int(e - s), int(cur[s]))
    return with_crc(bytes(out))


def _dict_blob(entries: List[bytes]) -> bytes:
    """DictBuilder.Marshal (storage/codec.go:82-99)."""
    out = bytearray(struct.pack("<I", len(entries)))
    off = 0
    for e in entries:
        out += struct.pack("<I", off)
        off += len(e)
    out += struct.pack("<I", off)
    out += b"".join(entries)
    return with_crc(bytes(out))


class _Writer:
    def __init__(self, f):
        self.f = f
        self.off = 0

    def put(self, b: bytes):
        self.f.write(b)
        self.off += len(b)


def _rg_strings(col, table: HostTable, s: int, e: int):
    """Per-row string bytes of rows [s, e) of a STRING column (None = NULL)."""
    valid = col.valid_mask(table.nrows)[s:e]
    codes = col.values[s:e].astype(np.int64)
    raw = col.dict_bytes.tobytes()
    if col.dict_rg_first is not None:  # the table's own per-row-group dictionaries
        k = col.dict_rg_first[np.arange(s, e) // table.rg_rows].astype(np.int64) + codes
    else:
        k = codes
    off = col.dict_str_off.astype(np.int64)
    return [raw[off[k[i]]:off[k[i] + 1]] if valid[i] else None for i in range(e - s)]


def write_vxq(path: str, table: HostTable, rg_rows: Optional[int] = None,
              nullable: Optional[List[bool]] = None, rg_sizes: Optional[List[int]] = None) -> List[RowGroupMeta]:
    """Writes `table` as a .vxq file with row groups of rg_rows rows (the
    table's own by default), or of the row counts in rg_sizes. Returns the
    row-group directory written."""
    rg_rows = rg_rows or table.rg_rows
    n = table.nrows
    if rg_sizes is None:
        rg_sizes = [min(rg_rows, n - s) for s in range(0, n, rg_rows)]
    assert sum(rg_sizes) == n and all(r > 0 for r in rg_sizes)
    bounds = np.r_[0, np.cumsum(rg_sizes)].astype(np.int64)
    metas: List[RowGroupMeta] = []
    with open(path, "wb") as fh:
        w = _Writer(fh)
        w.put(MAGIC)
        for s, e in zip(bounds[:-1].tolist(), bounds[1:].tolist()):
            rg = RowGroupMeta(w.off, e - s)
            for col in table.columns:
                valid = col.valid_mask(n)[s:e]
                start = w.off
                st = ColStats(null_count=int((~valid).sum()))
                dict_off = dict_len = 0
                if col.type == abi.TYPE_STRING:
                    strs = _rg_strings(col, table, s, e)
                    index, entries = {}, []
                    codes = np.empty(e - s, dtype=np.uint32)
                    for i, x in enumerate(strs):
                        if x is None:
                            codes[i] = 0xFFFFFFFF
                            continue
                        c = index.get(x)
                        if c is None:
                            c = index[x] = len(entries)
                            entries.append(x)
                        codes[i] = c
                    if entries:
                        st.has_min_max, st.min, st.max = True, 0, len(entries) - 1
                    vals = codes
                elif col.type == abi.TYPE_BOOL:
                    vals = col.values[s:e]
                else:
                    vals = col.values[s:e]
                    ok = vals[valid]
                    if col.type == abi.TYPE_INT64:
                        if len(ok):
                            st.sum = _i64(int(ok.astype(np.int64).sum(dtype=np.int64)))
                            st.has_min_max = True
                            st.min = int(ok.min()) & ((1 << 64) - 1)
                            st.max = int(ok.max()) & ((1 << 64) - 1)
                    elif col.type == abi.TYPE_FLOAT64:
                        st = _float_stats(ok.astype(np.float64), st.null_count)
                    elif col.type == abi.TYPE_DATE:
                        if len(ok):
                            st.has_min_max = True
                            st.min = int(ok.min()) & 0xFFFFFFFF
                            st.max = int(ok.max()) & 0xFFFFFFFF
                for b0 in range(0, e - s, BLOCK_ROWS):
                    b1 = min(e - s, b0 + BLOCK_ROWS)
                    if col.type == abi.TYPE_BOOL:
                        w.put(_rle_bool(vals[b0:b1], valid[b0:b1]))
                    else:
                        le = {abi.TYPE_INT64: "<i8", abi.TYPE_FLOAT64: "<f8", abi.TYPE_DATE: "<i4",
                              abi.TYPE_STRING: "<u4"}[col.type]
                        w.put(with_crc(_bitmap(valid[b0:b1]) + np.ascontiguousarray(vals[b0:b1]).astype(le).tobytes()))
                if col.type == abi.TYPE_STRING:
                    blob = _dict_blob(entries)
                    dict_off, dict_len = w.off - start, len(blob)
                    w.put(blob)
                rg.cols.append(Section(start, w.off - start, st, dict_off, dict_len))
            metas.append(rg)
        # footer (storage/writer.go:423-472)
        body = bytearray(struct.pack("<I", len(table.columns)))
        for i, col in enumerate(table.columns):
            nm = col.name.encode()
            enc = ENC_DICT if col.type == abi.TYPE_STRING else ENC_RLE if col.type == abi.TYPE_BOOL else ENC_PLAIN
            nl = nullable[i] if nullable is not None else col.validity is not None
            body += struct.pack("<H", len(nm)) + nm + bytes([col.type, enc, 1 if nl else 0])
        body += struct.pack("<I", len(metas))
        for rg in metas:
            body += struct.pack("<qI", rg.file_offset, rg.rows)
            for sec in rg.cols:
                body += struct.pack("<qqqqQQBII", sec.offset, sec.length, sec.stats.null_count, sec.stats.sum,
                                    sec.stats.min, sec.stats.max, 1 if sec.stats.has_min_max else 0,
                                    sec.dict_off, sec.dict_len)
        w.put(bytes(body) + struct.pack("<Iq", crc32(bytes(body)), len(body)) + MAGIC)
    return metas
