"""Host-side columnar tables in the layout vexq's storage layer hands to
TableScan: fixed-width little-endian values, LSB-first validity bitmaps
(1 = valid, storage/codec.go:13-39) and, for STRING columns, per-row-group
dictionaries with codes in first-occurrence order (storage/writer.go:374-420).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import abi

NP_TYPES = {abi.TYPE_INT64: np.int64, abi.TYPE_FLOAT64: np.float64, abi.TYPE_DATE: np.int32,
            abi.TYPE_STRING: np.uint32, abi.TYPE_BOOL: np.uint8}


def pack_validity(valid: Optional[np.ndarray]) -> Optional[np.ndarray]:
    """Bool array (True = valid) → LSB-first bitmap, or None when all valid."""
    if valid is None:
        return None
    valid = np.asarray(valid, dtype=bool)
    if valid.all():
        return None
    return np.packbits(valid, bitorder="little")


@dataclass
class HostColumn:
    name: str
    type: int
    values: np.ndarray                       # per-row values / local dict codes
    validity: Optional[np.ndarray] = None    # packed LSB-first bitmap
    dict_rg_first: Optional[np.ndarray] = None  # uint32, n_rg+1 (None: one global dictionary)
    dict_str_off: Optional[np.ndarray] = None   # uint32, entries+1
    dict_bytes: Optional[np.ndarray] = None     # uint8

    def valid_mask(self, nrows: int) -> np.ndarray:
        if self.validity is None:
            return np.ones(nrows, dtype=bool)
        return np.unpackbits(self.validity, bitorder="little", count=nrows).astype(bool)


def _flatten_dicts(entries: List[bytes]):
    lens = np.fromiter((len(e) for e in entries), dtype=np.int64, count=len(entries))
    off = np.zeros(len(entries) + 1, dtype=np.uint32)
    np.cumsum(lens, out=off[1:])
    data = np.frombuffer(b"".join(entries), dtype=np.uint8) if entries else np.zeros(1, np.uint8)
    return off, data.copy() if len(data) else np.zeros(1, np.uint8)


def string_column(name: str, idx: np.ndarray, universe: Sequence[str], nrows: int, rg_rows: int,
                  valid: Optional[np.ndarray] = None, per_rg: bool = True) -> HostColumn:
    """Dictionary-codes a string column given per-row indices into `universe`.

    per_rg=True reproduces the writer: one dictionary per row group, codes in
    first-occurrence order over the row group's non-NULL rows, NULL rows coded
    0xFFFFFFFF (storage/writer.go:345-378). per_rg=False gives one table-wide
    dictionary (first-occurrence order), for very large generated tables.
    """
    idx = np.asarray(idx, dtype=np.int64)
    uni = [s.encode() for s in universe]
    valid_b = np.ones(nrows, dtype=bool) if valid is None else np.asarray(valid, dtype=bool)
    codes = np.full(nrows, 0xFFFFFFFF, dtype=np.uint32)
    entries: List[bytes] = []
    rg_first = [0]
    lut = np.zeros(len(uni), dtype=np.uint32)
    spans = [(s, min(nrows, s + rg_rows)) for s in range(0, nrows, rg_rows)] if per_rg else [(0, nrows)]
    for s, e in spans:
        v = idx[s:e]
        m = valid_b[s:e]
        vv = v[m]
        if len(vv):
            u, first = np.unique(vv, return_index=True)
            order = u[np.argsort(first, kind="stable")]
        else:
            order = np.zeros(0, dtype=np.int64)
        lut[order] = np.arange(len(order), dtype=np.uint32)
        c = codes[s:e]
        c[m] = lut[vv]
        entries += [uni[i] for i in order]
        rg_first.append(len(entries))
    off, data = _flatten_dicts(entries)
    return HostColumn(name, abi.TYPE_STRING, codes, pack_validity(valid_b),
                      np.asarray(rg_first, dtype=np.uint32) if per_rg else None, off, data)


class HostTable:
    def __init__(self, columns: List[HostColumn], nrows: int, rg_rows: int = abi.ROW_GROUP_ROWS):
        self.columns, self.nrows, self.rg_rows = columns, int(nrows), int(rg_rows)
        for c in columns:
            c.values = np.ascontiguousarray(c.values, dtype=NP_TYPES[c.type])
            assert len(c.values) == nrows, (c.name, len(c.values), nrows)
        self._descs = None

    @property
    def n_rg(self) -> int:
        return (self.nrows + self.rg_rows - 1) // self.rg_rows

    def col_index(self, name: str) -> int:
        return [c.name for c in self.columns].index(name)

    def descs(self):
        """ctypes vexq_column_desc array over this table's (host) buffers."""
        if self._descs is None:
            arr = (abi.ColumnDesc * len(self.columns))()
            keep = []
            for i, c in enumerate(self.columns):
                nm = c.name.encode()
                keep.append(nm)

                def ptr(a):
                    return None if a is None else a.ctypes.data
                nent = len(c.dict_str_off) - 1 if c.dict_str_off is not None else 0
                arr[i] = abi.ColumnDesc(nm, c.type, c.values.ctypes.data, ptr(c.validity),
                                        ptr(c.dict_rg_first), ptr(c.dict_str_off), ptr(c.dict_bytes),
                                        nent)
            self._descs = (arr, keep)
        return self._descs[0]

    def nbytes(self, cols: Optional[Sequence[int]] = None) -> int:
        """Reference physical width of the given columns × rows (storage/format.go:46-57)."""
        w = {abi.TYPE_INT64: 8, abi.TYPE_FLOAT64: 8, abi.TYPE_DATE: 4, abi.TYPE_STRING: 4, abi.TYPE_BOOL: 1}
        cols = range(len(self.columns)) if cols is None else cols
        return sum(w[self.columns[i].type] for i in cols) * self.nrows

    def global_strings(self, col: int) -> np.ndarray:
        """Per-row decoded strings of a STRING column (None for NULL); tests only."""
        c = self.columns[col]
        out = np.empty(self.nrows, dtype=object)
        valid = c.valid_mask(self.nrows)
        raw = c.dict_bytes.tobytes()
        for rg in range(self.n_rg if c.dict_rg_first is not None else 1):
            s = rg * self.rg_rows if c.dict_rg_first is not None else 0
            e = min(self.nrows, s + self.rg_rows) if c.dict_rg_first is not None else self.nrows
            base = int(c.dict_rg_first[rg]) if c.dict_rg_first is not None else 0
            for r in range(s, e):
                if valid[r]:
                    k = base + int(c.values[r])
                    out[r] = raw[c.dict_str_off[k]:c.dict_str_off[k + 1]].decode()
        return out


def int_column(name, values, valid=None) -> HostColumn:
    return HostColumn(name, abi.TYPE_INT64, np.asarray(values, dtype=np.int64), pack_validity(valid))


def float_column(name, values, valid=None) -> HostColumn:
    return HostColumn(name, abi.TYPE_FLOAT64, np.asarray(values, dtype=np.float64), pack_validity(valid))


def date_column(name, values, valid=None) -> HostColumn:
    return HostColumn(name, abi.TYPE_DATE, np.asarray(values, dtype=np.int32), pack_validity(valid))


def bool_column(name, values, valid=None) -> HostColumn:
    return HostColumn(name, abi.TYPE_BOOL, np.asarray(values, dtype=np.uint8), pack_validity(valid))
