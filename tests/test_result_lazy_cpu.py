"""CPU test of the Python result wrapper over vexq_plan_submit: a submitted
result reads its summary (vexq_result_info, the call that waits for the run)
only at its first read, once, and a failed run's status is raised there; a
plain run's result reads it at once. A fake library stands in for
libvexqcuda, so no device is needed."""
from __future__ import annotations

import ctypes as C

import pytest

from vexq_b200 import abi, exec as X


class FakeLib:
    def __init__(self, status=0):
        self.info_calls = 0
        self.freed = 0
        self.status = status

    def vexq_result_info(self, h, out):
        self.info_calls += 1
        if self.status:
            return self.status
        s = C.cast(out, C.POINTER(abi.ResultSummary)).contents
        s.nrows, s.ncols, s.launches, s.kernel_ms, s.scan_ms = 6, 10, 1, 0.06, 0.059
        s.rows_scanned, s.bytes_scanned = 6_000_000, 264_000_000
        return 0

    def vexq_result_free(self, h):
        self.freed += 1
        return 0

    def vexq_last_error(self):
        return b"the scan kernel reported error flags 4"


@pytest.fixture
def fake(monkeypatch):
    lib = FakeLib()
    monkeypatch.setattr(abi, "load", lambda: lib)
    return lib


def test_submitted_result_waits_at_first_read_once(fake):
    r = X.Result(C.c_void_p(1), lazy=True)
    assert fake.info_calls == 0
    assert r.nrows == 6 and r.kernel_ms == 0.06 and r.bytes_scanned == 264_000_000
    assert r.launches == 1 and r.ncols == 10 and r.scan_ms == 0.059 and r.rows_scanned == 6_000_000
    assert fake.info_calls == 1
    r.close()
    assert fake.freed == 1


def test_plain_result_reads_at_once(fake):
    r = X.Result(C.c_void_p(2))
    assert fake.info_calls == 1
    assert r.nrows == 6
    assert fake.info_calls == 1
    r.close()


def test_failed_run_raises_at_first_read(monkeypatch):
    lib = FakeLib(status=abi.EDEVICE)
    monkeypatch.setattr(abi, "load", lambda: lib)
    r = X.Result(C.c_void_p(3), lazy=True)  # submit itself succeeded
    for _ in range(2):  # every read returns the run's status
        with pytest.raises(abi.VexqError) as e:
            r.wait()
        assert e.value.status == abi.EDEVICE and "error flags" in str(e.value)
    r.close()
