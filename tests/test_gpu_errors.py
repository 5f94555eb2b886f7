"""GPU tests of the error paths the C ABI promises, made on the host (no
device fault): cancellation before a run, a serving wait that times out,
and a device allocation that fails. The reference's counterparts: a
cancelled context ends a parallel query with ctx.Err()
(exec/scan.go:201-203, exec/parallel_join.go:430-476: the first error wins),
and every failure reaches the caller as the query's error."""
from __future__ import annotations

import ctypes as C

import pytest

from vexq_b200 import abi, datagen as D, workloads as W

from tests.helpers import assert_rows_match

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tables(gpu_lib):
    X = gpu_lib
    li = X.GpuTable(D.lineitem(300_000, seed=41, rg_rows=65536))
    o, i = X.GpuTable(D.orders(100_000, seed=42)), X.GpuTable(D.items(400_000, 100_000, seed=43))
    return X, li, o, i


def _run_status(op):
    h = C.c_void_p()
    st = abi.load().vexq_plan_run(op.h, 0, -1, C.byref(h))
    if st == abi.OK:
        abi.load().vexq_result_free(h)
    return st


def test_cancel_before_run(tables):
    X, li, o, i = tables
    for op in (X.GpuHashAggregate(li, W.q1_plan()), X.GpuParallelHashJoinAggregate(o, i, W.q3_plan())):
        try:
            ref = op.run().rows()
            abi.check(abi.load().vexq_cancel(op.h))
            assert _run_status(op) == abi.ECANCELED
            # the flag is consumed by the run it ended: the next run completes
            assert_rows_match(op.run().rows(), ref, ordered=True, rtol=0.0)
        finally:
            op.close()


def test_server_wait_times_out_on_queued_ticket(tables):
    X, li, o, i = tables
    ops = [X.GpuParallelHashJoinAggregate(o, i, W.q3_plan()) for _ in range(2)]
    L = abi.load()
    try:
        ref = ops[0].run().rows()
        srv = C.c_void_p()
        abi.check(L.vexq_server_start(1 << 36, 1, 1, abi.SERVE_NO_BATCH, C.byref(srv)))
        try:
            tickets = []
            for k in range(8):
                tk = C.c_int64()
                abi.check(L.vexq_server_submit(srv, ops[k % 2].h, C.byref(tk)))
                tickets.append(tk.value)
            h = C.c_void_p()
            # one worker, one slot: the last ticket waits behind seven joins
            assert L.vexq_server_wait(srv, tickets[-1], 0, C.byref(h)) == abi.ETIMEDOUT
            assert not h.value
            done, out = C.c_int32(), C.c_void_p()
            abi.check(L.vexq_server_poll(srv, tickets[-1], C.byref(done), C.byref(out)))
            for tk in tickets:
                abi.check(L.vexq_server_wait(srv, tk, 120000, C.byref(h)))
                assert_rows_match(X.Result(h).rows(), ref, ordered=True, rtol=0.0)
        finally:
            abi.check(L.vexq_server_stop(srv))
    finally:
        for op in ops:
            op.close()


def _free_bytes():
    """Device bytes the library holds (tables, plans, workspaces)."""
    v = C.c_int64()
    abi.check(abi.load().vexq_debug_live_device_bytes(C.byref(v)))
    return v.value


@pytest.mark.parametrize("kind", ["q1", "q3"])
def test_injected_allocation_failure(tables, kind):
    """A device allocation fails at each point of a plan's first run in turn:
    the run returns VEXQ_ENOMEM, the same plan's next run is correct, and
    destroying the plan gives every byte back."""
    import gc
    X, li, o, i = tables
    L = abi.load()

    def make():
        if kind == "q1":
            return X.GpuHashAggregate(li, W.q1_plan())
        return X.GpuParallelHashJoinAggregate(o, i, W.q3_plan())

    warm = make()
    ref = warm.run().rows()  # kernels compiled and loaded once
    warm.close()
    failed = 0
    try:
        for after in range(0, 40):
            gc.collect()
            base = _free_bytes()  # everything but the plan made next
            op = make()
            abi.check(L.vexq_debug_fail_alloc(after))
            st = _run_status(op)
            abi.check(L.vexq_debug_fail_alloc(-1))
            if st == abi.OK:
                op.close()
                break  # the run needs fewer allocations than `after`
            assert st == abi.ENOMEM, (after, st, L.vexq_last_error())
            assert b"injected" in L.vexq_last_error()
            failed += 1
            # the plan that failed stays usable: its next run allocates again
            assert_rows_match(op.run().rows(), ref, ordered=True, rtol=0.0)
            op.close()
            gc.collect()
            assert _free_bytes() == base, f"device memory not returned after a failure at allocation {after}"
        assert failed >= 1
        op = make()
        try:
            assert_rows_match(op.run().rows(), ref, ordered=True, rtol=0.0)
        finally:
            op.close()
    finally:
        L.vexq_debug_fail_alloc(-1)
