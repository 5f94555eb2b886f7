"""Python mirror of vexq's operator contract over libvexqcuda's C ABI.

The Go engine would bind the same entry points through cgo; this module gives
tests and the benchmark the reference's shapes:

  GpuTable                     ≈ the uploaded columns a TableScan would read
  GpuHashAggregate             ≈ exec.NewHashAggregate / NewParallelHashAggregate
                                 (exec/aggregate.go:131, exec/parallel.go:78)
  GpuParallelHashJoinAggregate ≈ exec.NewParallelHashJoinAggregate (exec/parallel_join.go:718)
  GpuFilter                    ≈ exec.NewFilter over a TableScan + BoolToSelVecInto
                                 (exec/filter.go:40-78): next() → the scan's batch with
                                 its SelVec; bitmap() for a whole-table selection
  GpuProject                   ≈ exec.NewProject over that filter (exec/project.go:64-128)
  GpuBatch                     many prepared plans in one persistent launch per path class
                               under a captured CUDA graph (no reference counterpart)

Operators implement next() → Batch | None, schema() and close(), with ≤1024
rows per batch and group-insertion order, like exec.Operator (exec/operator.go:28-32).
Every call goes to the CUDA library; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import abi
from .plan import AggPlan, JoinPlan, predicate_arrays, project_arrays
from .table import HostTable

_initialised = False


def init(device: int = 0) -> None:
    global _initialised
    if not _initialised:
        abi.check(abi.load().vexq_init(device, 0))
        _initialised = True


@dataclass
class Vector:
    name: str
    type: int
    values: list          # Python values; None = NULL


@dataclass
class Batch:
    vectors: List[Vector]
    length: int


class GpuTable:
    """Columns uploaded once into HBM (dictionary codes remapped to global codes)."""

    def __init__(self, t: HostTable):
        init()
        self.host = t
        self.h = C.c_void_p()
        abi.check(abi.load().vexq_table_upload(t.descs(), len(t.columns), t.nrows, t.rg_rows, C.byref(self.h)))

    @classmethod
    def from_vxq(cls, path: str, columns: Optional[Sequence[str]] = None) -> "GpuTable":
        """Loads a .vxq file (all columns, or those named, in that order)
        straight into HBM: storage.Open + TableScan's decode for the GPU."""
        init()
        self = cls.__new__(cls)
        self.host = None
        self.h = C.c_void_p()
        names = None
        if columns is not None:
            names = (C.c_char_p * max(len(columns), 1))(*[c.encode() for c in columns])
        abi.check(abi.load().vexq_table_load_vxq(os.fsencode(path), names, 0 if columns is None else len(columns),
                                                 C.byref(self.h)))
        return self

    def num_row_groups(self) -> int:
        v = C.c_int32()
        abi.check(abi.load().vexq_table_num_row_groups(self.h, C.byref(v)))
        return v.value

    def dict_entries(self, col: int) -> List[str]:
        """The global dictionary of a STRING column, in code order."""
        n = C.c_int32()
        abi.check(abi.load().vexq_table_dict_size(self.h, col, C.byref(n)))
        out = []
        for i in range(n.value):
            p, ln = C.c_char_p(), C.c_int32()
            abi.check(abi.load().vexq_table_dict_entry(self.h, col, i, C.byref(p), C.byref(ln)))
            out.append(C.string_at(p, ln.value).decode() if ln.value else "")
        return out

    def zone_map(self, col: int, rg: int) -> abi.ZoneMap:
        z = abi.ZoneMap()
        abi.check(abi.load().vexq_table_zone_map(self.h, col, rg, C.byref(z)))
        return z

    def device_bytes(self) -> int:
        v = C.c_int64()
        abi.check(abi.load().vexq_table_device_bytes(self.h, C.byref(v)))
        return v.value

    def close(self):
        if self.h:
            abi.load().vexq_table_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _decode(t: int, raw: bytes, n: int):
    if t == abi.TYPE_INT64:
        return list(struct.unpack(f"<{n}q", raw))
    if t == abi.TYPE_FLOAT64:
        return list(struct.unpack(f"<{n}d", raw))
    if t == abi.TYPE_DATE:
        return list(struct.unpack(f"<{n}i", raw))
    if t == abi.TYPE_BOOL:
        return [b != 0 for b in raw]
    return list(struct.unpack(f"<{n}I", raw))


class Result:
    """A run's result: Next()-style batches plus device timing. A submitted
    run (lazy) waits for its kernels at its first read, which raises the
    run's error if it failed."""

    def __init__(self, h: C.c_void_p, lazy: bool = False):
        self.h = h
        self._info = None
        if not lazy:
            self.wait()

    def wait(self) -> "Result":
        if self._info is None:
            s = abi.ResultSummary()
            abi.check(abi.load().vexq_result_info(self.h, C.byref(s)))
            self._info = s
        return self

    nrows = property(lambda self: self.wait()._info.nrows)
    ncols = property(lambda self: self.wait()._info.ncols)
    kernel_ms = property(lambda self: self.wait()._info.kernel_ms)
    scan_ms = property(lambda self: self.wait()._info.scan_ms)
    launches = property(lambda self: self.wait()._info.launches)
    rows_scanned = property(lambda self: self.wait()._info.rows_scanned)
    bytes_scanned = property(lambda self: self.wait()._info.bytes_scanned)

    def next(self) -> Optional[Batch]:
        """Operator.Next: ≤1024 rows, None at EOF."""
        bv = abi.BatchView()
        abi.check(abi.load().vexq_result_next(self.h, C.byref(bv)))
        if bv.length == 0:
            return None
        vecs = []
        for c in range(bv.ncols):
            v = bv.cols[c]
            n = bv.length
            width = {abi.TYPE_INT64: 8, abi.TYPE_FLOAT64: 8, abi.TYPE_DATE: 4, abi.TYPE_STRING: 4, abi.TYPE_BOOL: 1}[v.type]
            raw = C.string_at(v.values, n * width)
            bm = C.string_at(v.validity, (n + 7) // 8)
            vals = _decode(v.type, raw, n)
            if v.type == abi.TYPE_STRING:
                off = np.frombuffer(C.string_at(v.dict_str_off, (v.dict_len + 1) * 4), dtype=np.uint32) if v.dict_len else []
                data = C.string_at(v.dict_bytes, int(off[-1])) if v.dict_len else b""
                strs = [data[off[i]:off[i + 1]].decode() for i in range(v.dict_len)]
                vals = [strs[x] if x < len(strs) else "" for x in vals]
            vals = [vals[i] if (bm[i >> 3] >> (i & 7)) & 1 else None for i in range(n)]
            vecs.append(Vector(v.name.decode() if v.name else "", v.type, vals))
        return Batch(vecs, bv.length)

    def collect(self):
        """All rows as columns (lists), draining next()."""
        cols: List[list] = [[] for _ in range(self.ncols)]
        names, types = [""] * self.ncols, [0] * self.ncols
        while True:
            b = self.next()
            if b is None:
                break
            for i, v in enumerate(b.vectors):
                cols[i] += v.values
                names[i], types[i] = v.name, v.type
        self.columns, self.names, self.types = cols, names, types
        return cols

    def rows(self):
        if not hasattr(self, "columns"):
            self.collect()
        return [tuple(c[r] for c in self.columns) for r in range(self.nrows)]

    def close(self):
        if self.h:
            abi.load().vexq_result_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _PlanOp:
    h: C.c_void_p

    def run(self, rg_start: int = 0, rg_end: int = -1) -> Result:
        h = C.c_void_p()
        abi.check(abi.load().vexq_plan_run(self.h, rg_start, rg_end, C.byref(h)))
        return Result(h)

    def submit(self, rg_start: int = 0, rg_end: int = -1) -> Result:
        """vexq_plan_submit: returns once the run's launches are queued; the
        result waits for them at its first read."""
        h = C.c_void_p()
        abi.check(abi.load().vexq_plan_submit(self.h, rg_start, rg_end, C.byref(h)))
        return Result(h, lazy=True)

    def run_host(self, table: HostTable) -> Result:
        """End-to-end form: refills the columns from host buffers, then runs."""
        h = C.c_void_p()
        abi.check(abi.load().vexq_plan_run_host(self.h, table.descs(), len(table.columns), C.byref(h)))
        return Result(h)

    def explain(self) -> str:
        return abi.load().vexq_plan_explain(self.h).decode()

    # shards ----------------------------------------------------------------------
    def run_partial(self, rg_start: int, rg_end: int) -> bytes:
        """This shard's groups, unfinished, as bytes (vexq_plan_run_partial)."""
        L = abi.load()
        part = C.c_void_p()
        abi.check(L.vexq_plan_run_partial(self.h, rg_start, rg_end, C.byref(part)))
        try:
            ptr, ln = C.c_void_p(), C.c_int64()
            abi.check(L.vexq_partial_serialize(part, C.byref(ptr), C.byref(ln)))
            return C.string_at(ptr, ln.value)
        finally:
            L.vexq_partial_free(part)

    def merge_partials(self, parts) -> Result:
        """The finished result of shard partials, folded in list order."""
        L = abi.load()
        hs = []
        try:
            for b in parts:
                h = C.c_void_p()
                buf = C.create_string_buffer(b, len(b))
                abi.check(L.vexq_partial_deserialize(self.h, buf, len(b), C.byref(h)))
                hs.append(h)
            arr = (C.c_void_p * max(len(hs), 1))(*[h.value for h in hs])
            out = C.c_void_p()
            abi.check(L.vexq_partial_merge(self.h, arr, len(hs), C.byref(out)))
            return Result(out)
        finally:
            for h in hs:
                L.vexq_partial_free(h)

    def autotune(self, retune: bool = False):
        """(choice, best ms): radix bits for a join (0 = global table), the
        shared-memory group cache in KB for a dense aggregate, -1 otherwise."""
        ch, ms = C.c_int32(), C.c_double()
        abi.check(abi.load().vexq_plan_autotune(self.h, abi.PLAN_RETUNE if retune else 0, C.byref(ch), C.byref(ms)))
        return ch.value, ms.value

    def set_stream(self, stream_ptr: int) -> None:
        """Runs on a caller-owned cudaStream_t (0 restores the plan's own)."""
        abi.check(abi.load().vexq_plan_set_stream(self.h, C.c_void_p(stream_ptr or None)))

    # exec.Operator contract -------------------------------------------------------
    def next(self) -> Optional[Batch]:
        if getattr(self, "_result", None) is None:
            self._result = self.run()
        return self._result.next()

    def close(self):
        if getattr(self, "_result", None) is not None:
            self._result.close()
            self._result = None
        if self.h:
            abi.load().vexq_plan_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _set_having(h, plan):
    hv = getattr(plan, "having", None)
    if hv is None:
        return
    _, nodes, nn, ch, nc, root, visible = hv
    abi.check(abi.load().vexq_plan_set_having(h, nodes, nn, ch, nc, root, visible))


class GpuHashAggregate(_PlanOp):
    """Filter → (Project) → HashAggregate over one table; also stands in for
    ParallelHashAggregate (numWorkers/morselSize have no GPU meaning)."""

    def __init__(self, table: GpuTable, plan: AggPlan):
        self.table, self.plan = table, plan
        self.h = C.c_void_p()
        abi.check(abi.load().vexq_agg_plan_create(table.h, C.byref(plan.desc), C.byref(self.h)))
        _set_having(self.h, plan)

    def zone_prune(self) -> List[int]:
        n = self.table.host.n_rg
        m = (C.c_uint8 * max(n, 1))()
        abi.check(abi.load().vexq_zone_prune(self.h, m, n))
        return [int(m[i]) for i in range(n)]


class GpuParallelHashJoinAggregate(_PlanOp):
    def __init__(self, build: GpuTable, probe: GpuTable, plan: JoinPlan):
        self.build, self.probe, self.plan = build, probe, plan
        self.h = C.c_void_p()
        abi.check(abi.load().vexq_join_plan_create(build.h, probe.h, C.byref(plan.desc), C.byref(self.h)))
        _set_having(self.h, plan)


@dataclass
class SelBatch:
    """The batch Filter.Next returns: the scan's vectors (physical rows) with
    the selection vector installed; length = len(sel)."""
    vectors: List[Vector]
    physical: int
    sel: List[int]
    rg: int
    row0: int

    @property
    def length(self) -> int:
        return len(self.sel)


def _view_values(v, n: int):
    width = {abi.TYPE_INT64: 8, abi.TYPE_FLOAT64: 8, abi.TYPE_DATE: 4, abi.TYPE_STRING: 4, abi.TYPE_BOOL: 1}[v.type]
    vals = _decode(v.type, C.string_at(v.values, n * width), n) if n else []
    bm = C.string_at(v.validity, (n + 7) // 8) if n else b""
    if v.type == abi.TYPE_STRING:
        off = np.frombuffer(C.string_at(v.dict_str_off, (v.dict_len + 1) * 4), dtype=np.uint32) if v.dict_len else []
        data = C.string_at(v.dict_bytes, int(off[-1])) if v.dict_len else b""
        strs = [data[off[i]:off[i + 1]].decode() for i in range(v.dict_len)]
        vals = [strs[x] if x < len(strs) else "" for x in vals]
    return [vals[i] if (bm[i >> 3] >> (i & 7)) & 1 else None for i in range(n)]


class GpuFilter:
    """exec.Filter over a table's scan. next() streams 1024-row blocks with
    device-built SelVecs (vexq_filter_open/next); bitmap() returns a
    whole-range selection bitmap (vexq_filter_run)."""

    def __init__(self, table: GpuTable, predicate, rg_start: int = 0, rg_end: int = -1):
        self.table, self.predicate = table, predicate
        self.rg_start, self.rg_end = rg_start, rg_end
        self._arena, self.nodes, self.nn, self.ch, self.nc, self.root = predicate_arrays(predicate)
        self.h = C.c_void_p()

    def open(self) -> None:
        if not self.h:
            abi.check(abi.load().vexq_filter_open(self.table.h, self.nodes, self.nn, self.ch, self.nc, self.root,
                                                  self.rg_start, self.rg_end, C.byref(self.h)))

    def next(self) -> Optional[SelBatch]:
        """Filter.Next: the next block with at least one kept row, None at EOF."""
        self.open()
        fb = abi.FilterBatch()
        abi.check(abi.load().vexq_filter_next(self.h, C.byref(fb)))
        if fb.length == 0:
            return None
        vecs = []
        for c in range(fb.ncols):
            v = fb.cols[c]
            vecs.append(Vector(v.name.decode() if v.name else "", v.type, _view_values(v, fb.physical)))
        return SelBatch(vecs, fb.physical, list(fb.sel[:fb.length]), fb.rg, fb.row0)

    def stats(self):
        """(rows kept, blocks scanned, device ms of open)"""
        self.open()
        s, b, ms = C.c_int64(), C.c_int64(), C.c_double()
        abi.check(abi.load().vexq_filter_stats(self.h, C.byref(s), C.byref(b), C.byref(ms)))
        return s.value, b.value, ms.value

    def close(self):
        if self.h:
            abi.load().vexq_filter_close(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bitmap(self, row_start: int = 0, row_end: int = -1):
        n = (self.table.host.nrows if row_end < 0 else row_end) - row_start
        out = (C.c_uint8 * max((n + 7) // 8, 1))()
        cnt = C.c_int64()
        abi.check(abi.load().vexq_filter_run(self.table.h, self.nodes, self.nn, self.ch, self.nc, self.root,
                                             row_start, row_end, out, C.byref(cnt)))
        return bytes(out)[:(n + 7) // 8], cnt.value

    @staticmethod
    def selvec(bits: bytes, nrows: int, block: int) -> List[int]:
        buf = (C.c_uint8 * len(bits)).from_buffer_copy(bits) if bits else (C.c_uint8 * 1)()
        sel = (C.c_uint16 * abi.BLOCK_ROWS)()
        n = C.c_int32()
        abi.check(abi.load().vexq_selvec_from_bits(buf, nrows, block, sel, C.byref(n)))
        return list(sel[:n.value])


class GpuProject:
    """exec.Project over Filter(TableScan): the named expressions of the kept
    rows, materialised on the device in row order (no SelVec on the output)."""

    def __init__(self, table: GpuTable, exprs, names=None, predicate=None, rg_start: int = 0, rg_end: int = -1):
        self.table = table
        self._arena, self.nodes, self.nn, self.ch, self.nc, self.root, roots = project_arrays(predicate, exprs)
        self.roots = (C.c_int32 * len(roots))(*roots)
        names = names or [f"col{i}" for i in range(len(roots))]
        self._names = [n.encode() for n in names]
        self.names = (C.c_char_p * len(roots))(*self._names)
        self.n = len(roots)
        self.rg_start, self.rg_end = rg_start, rg_end

    def run(self) -> Result:
        h = C.c_void_p()
        abi.check(abi.load().vexq_project_run(self.table.h, self.nodes, self.nn, self.ch, self.nc, self.root,
                                              self.roots, self.names, self.n, self.rg_start, self.rg_end, C.byref(h)))
        return Result(h)


class GpuBatch:
    """Many prepared plans executed together: one persistent launch per path
    class, replayed from a captured CUDA graph on every exec()."""

    def __init__(self, ops, autotune: bool = False):
        self.ops = list(ops)  # keeps the plans (and their tables) alive
        n = len(self.ops)
        arr = (C.c_void_p * max(n, 1))(*[op.h for op in self.ops])
        self.h = C.c_void_p()
        abi.check(abi.load().vexq_batch_create(arr, n, abi.BATCH_AUTOTUNE if autotune else 0, C.byref(self.h)))

    def exec(self) -> List[Result]:
        n = len(self.ops)
        outs = (C.c_void_p * max(n, 1))()
        abi.check(abi.load().vexq_batch_exec(self.h, outs))
        return [Result(C.c_void_p(outs[i])) for i in range(n)]

    def stats(self):
        """(device ms of the replay, ms of its kernels alone, bytes scanned, rows scanned)"""
        ms, km, b, r = C.c_double(), C.c_double(), C.c_int64(), C.c_int64()
        abi.check(abi.load().vexq_batch_stats(self.h, C.byref(ms), C.byref(km), C.byref(b), C.byref(r)))
        return ms.value, km.value, b.value, r.value

    def explain(self) -> str:
        return abi.load().vexq_batch_explain(self.h).decode()

    def close(self):
        if self.h:
            abi.load().vexq_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
