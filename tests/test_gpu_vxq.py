"""GPU tests of the .vxq loader: files written by the writer restatement
(oracle/vxq_writer.py) loaded straight into HBM must hold what uploading the
same HostTable holds — every zone map (and the footer's own statistics), the
global dictionaries, and bit-identical query results — and the queries must
match the oracle. Column selection loads a subset in the order asked."""
from __future__ import annotations

import struct

import numpy as np
import pytest

from oracle import refcpu as R
from oracle import vxq_writer as VW
from tests.helpers import assert_float_vs_exact, assert_rows_match
from tests.test_vxq_cpu import mixed_table
from vexq_b200 import abi, datagen as D, plan as P, workloads as W
from vexq_b200.table import HostTable

pytestmark = pytest.mark.gpu


def _zone_tuple(z):
    return (z.null_count, z.sum, z.min, z.max, z.has_min_max)


def _as_f64(bits: int) -> float:
    return struct.unpack("<d", struct.pack("<Q", bits & ((1 << 64) - 1)))[0]


def _bits(rows):
    """Rows with floats as their raw bits (NaN compares equal to itself)."""
    return [tuple(struct.pack("<d", v) if isinstance(v, float) else v for v in r) for r in rows]


def test_loaded_table_equals_the_uploaded_one(gpu_lib, tmp_path):
    X = gpu_lib
    n, rg = 8192 * 4 + 3001, 8192
    host = mixed_table(n, rg, 11)
    p = tmp_path / "m.vxq"
    meta = VW.write_vxq(str(p), host)
    lt = X.GpuTable.from_vxq(str(p))
    ut = X.GpuTable(host)
    try:
        assert lt.num_row_groups() == ut.num_row_groups() == len(meta) == 5
        for c, col in enumerate(host.columns):
            for r in range(len(meta)):
                zl, zu = lt.zone_map(c, r), ut.zone_map(c, r)
                assert _zone_tuple(zl) == _zone_tuple(zu), (col.name, r)
                st = meta[r].cols[c].stats
                # the footer's statistics, written by the writer's rules
                assert (zl.null_count, zl.min, zl.max, bool(zl.has_min_max)) == \
                    (st.null_count, st.min, st.max, st.has_min_max), (col.name, r)
                if col.type == abi.TYPE_INT64:
                    assert zl.sum == st.sum
                if col.type == abi.TYPE_FLOAT64 and not np.isnan(_as_f64(st.sum)):
                    a, b = _as_f64(zl.sum), _as_f64(st.sum)
                    assert abs(a - b) <= 1e-9 * max(1.0, abs(b)), (col.name, r, a, b)
            if col.type == abi.TYPE_STRING:
                assert lt.dict_entries(c) == ut.dict_entries(c)
        plans = [
            P.AggPlan(P.col(2) <= P.lit("1997-06-30"), [3, 4],
                      [P.count_star("n"), P.sum_(P.col(0), "si"), P.min_(P.col(0), "mn"), P.max_(P.col(0), "mx"),
                       P.sum_(P.col(1), "sf"), P.avg(P.col(1), "af"), P.count(P.col(3), "cs")]),
            P.AggPlan(P.and_(P.col(1) > 0.0, P.col(3) == P.lit("MAIL")), [],
                      [P.sum_(P.col(1) * P.col(5), "x"), P.count_star("n")]),
        ]
        rt = R.RefTable(host)
        for plan in plans:
            a = X.GpuHashAggregate(lt, plan)
            b = X.GpuHashAggregate(ut, plan)
            try:
                ga, gb = a.run().rows(), b.run().rows()
            finally:
                a.close()
                b.close()
            assert _bits(ga) == _bits(gb)  # same data, same plan: the same bits
            ref = R.agg(rt, plan, workers=0)
            assert_rows_match(ga, ref.rows(), ordered=True)
            assert_float_vs_exact(ga, ref)
    finally:
        lt.close()
        ut.close()


def test_column_subset_in_the_order_asked(gpu_lib, tmp_path):
    X = gpu_lib
    n, rg = 20000, 4096
    host = mixed_table(n, rg, 12)
    p = tmp_path / "s.vxq"
    VW.write_vxq(str(p), host)
    lt = X.GpuTable.from_vxq(str(p), ["f", "s", "k"])
    sub = HostTable([host.columns[1], host.columns[3], host.columns[5]], n, rg)
    try:
        plan = P.AggPlan(P.col(2) < 15000, [1], [P.sum_(P.col(0), "sf"), P.count_star("n"), P.max_(P.col(2), "mk")])
        op = X.GpuHashAggregate(lt, plan)
        try:
            g = op.run().rows()
        finally:
            op.close()
        ref = R.agg(R.RefTable(sub), plan, workers=0)
        assert_rows_match(g, ref.rows(), ordered=True)
    finally:
        lt.close()


def test_lineitem_file_runs_q1_and_q6_as_uploaded(gpu_lib, tmp_path):
    """A lineitem-shaped file in the reference's 65,536-row row groups."""
    X = gpu_lib
    host = D.lineitem(400_000, seed=5, rg_rows=65536)
    p = tmp_path / "lineitem.vxq"
    VW.write_vxq(str(p), host)
    lt = X.GpuTable.from_vxq(str(p))
    ut = X.GpuTable(host)
    try:
        for plan in (W.q1_plan(), W.q6_plan()):
            a, b = X.GpuHashAggregate(lt, plan), X.GpuHashAggregate(ut, plan)
            try:
                assert _bits(a.run().rows()) == _bits(b.run().rows())
            finally:
                a.close()
                b.close()
    finally:
        lt.close()
        ut.close()


@pytest.mark.parametrize("n", [0, 1])
def test_empty_and_one_row_files(gpu_lib, tmp_path, n):
    """No row groups (a global aggregate over no rows is one row), and one row."""
    X = gpu_lib
    host = mixed_table(n, 65536, 13)
    p = tmp_path / "e.vxq"
    VW.write_vxq(str(p), host)
    t = X.GpuTable.from_vxq(str(p))
    try:
        assert t.num_row_groups() == n
        plan = P.AggPlan(None, [], [P.count_star("n"), P.sum_(P.col(0), "s"), P.max_(P.col(1), "m")])
        op = X.GpuHashAggregate(t, plan)
        try:
            assert_rows_match(op.run().rows(), R.agg(R.RefTable(host), plan, workers=0).rows(), ordered=True)
        finally:
            op.close()
    finally:
        t.close()


def test_row_groups_not_a_multiple_of_eight_rows(gpu_lib, tmp_path):
    """Row groups of 100 rows: blocks start mid-byte in the table's bitmaps,
    so the device writes their validity bit by bit."""
    X = gpu_lib
    host = mixed_table(100 * 7 + 41, 100, 14)
    p = tmp_path / "odd.vxq"
    VW.write_vxq(str(p), host)
    lt, ut = X.GpuTable.from_vxq(str(p)), X.GpuTable(host)
    try:
        for c in range(len(host.columns)):
            for r in range(lt.num_row_groups()):
                assert _zone_tuple(lt.zone_map(c, r)) == _zone_tuple(ut.zone_map(c, r)), (c, r)
        plan = P.AggPlan(None, [3], [P.count(P.col(0), "ci"), P.count(P.col(2), "cd"), P.sum_(P.col(0), "s"),
                                     P.count_star("n")])
        a, b = X.GpuHashAggregate(lt, plan), X.GpuHashAggregate(ut, plan)
        try:
            assert _bits(a.run().rows()) == _bits(b.run().rows())
        finally:
            a.close()
            b.close()
    finally:
        lt.close()
        ut.close()


def test_device_checks_find_corrupt_blocks(gpu_lib, tmp_path):
    """The device CRC check fails a flipped byte; a re-sealed block with a
    code past its row group's dictionary fails the device's code check."""
    X = gpu_lib
    host = mixed_table(5000, 2048, 15)
    p = tmp_path / "bad.vxq"
    meta = VW.write_vxq(str(p), host)
    good = open(p, "rb").read()
    sec = meta[1].cols[5]  # int64 column "k", row group 1: second block
    at = sec.offset + (VW.BITMAP_BYTES + 1024 * 8 + 4) + VW.BITMAP_BYTES + 77
    open(p, "wb").write(good[:at] + bytes([good[at] ^ 0x04]) + good[at + 1:])
    with pytest.raises(abi.VexqError) as e:
        X.GpuTable.from_vxq(str(p))
    assert e.value.status == abi.ECORRUPT and "checksum mismatch" in str(e.value) and "col=k" in str(e.value)
    sec = meta[1].cols[3]  # STRING codes, row group 1 (first block: 1,024 rows)
    valid = host.columns[3].valid_mask(host.nrows)[2048:2048 + 1024]
    row = int(np.flatnonzero(valid)[0])
    b = bytearray(good)
    blk = bytearray(b[sec.offset:sec.offset + VW.BITMAP_BYTES + 1024 * 4])
    blk[VW.BITMAP_BYTES + 4 * row:VW.BITMAP_BYTES + 4 * row + 4] = struct.pack("<I", 1000)
    b[sec.offset:sec.offset + VW.BITMAP_BYTES + 1024 * 4 + 4] = VW.with_crc(bytes(blk))
    open(p, "wb").write(bytes(b))
    with pytest.raises(abi.VexqError) as e:
        X.GpuTable.from_vxq(str(p))
    assert e.value.status == abi.ECORRUPT and "dictionary code out of range" in str(e.value), str(e.value)
    open(p, "wb").write(good)
    X.GpuTable.from_vxq(str(p)).close()
