"""One call at a time per backend, as the reference's bindings enforce
(cpp/python/native_call.hpp:19-84): the native calls release the GIL, so a
call from a second thread while one runs must raise RuntimeError("native
object is in use by another thread") rather than race on the context.
Checked with a stand-in for the native library, on the CPU."""

import threading

import pytest

from microsimulator_b200 import abi
from microsimulator_b200 import backend as backend_module


class BlockingLibrary:
    """msb_set_relaxation blocks until released; the rest return at once."""

    def __init__(self):
        self.entered = threading.Event()
        self.release = threading.Event()
        self.nested = None

    def msb_context_create(self, device, handle):
        handle._obj.value = 1
        return abi.OK

    def msb_context_destroy(self, handle):
        return abi.OK

    def msb_last_error(self, handle):
        return b""

    def msb_set_relaxation(self, handle, form):
        if self.nested is not None:
            self.nested()
        self.entered.set()
        self.release.wait(10)
        return abi.OK

    def msb_set_warm_start(self, handle, mode):
        return abi.OK


@pytest.fixture
def library(monkeypatch):
    fake = BlockingLibrary()
    monkeypatch.setattr(abi, "load_library", lambda path=None: fake)
    return fake


def test_second_thread_is_refused_while_a_call_runs(library):
    backend = backend_module.B200Backend(0)
    worker = threading.Thread(target=backend.set_relaxation, args=(1,))
    worker.start()
    try:
        assert library.entered.wait(10)
        with pytest.raises(RuntimeError, match="native object is in use by another thread"):
            backend.set_warm_start(0)
        with pytest.raises(RuntimeError, match="native object is in use by another thread"):
            backend.close()
    finally:
        library.release.set()
        worker.join(10)
    assert not worker.is_alive()
    backend.set_warm_start(0)  # idle again
    backend.close()


def test_nested_calls_on_one_thread_proceed(library):
    backend = backend_module.B200Backend(0)
    calls = []
    library.nested = lambda: calls.append(backend.set_warm_start(0))
    library.release.set()
    backend.set_relaxation(1)
    assert calls == [None]
    backend.close()


def test_busy_error_is_a_native_runtime_error(library):
    backend = backend_module.B200Backend(0)
    worker = threading.Thread(target=backend.set_relaxation, args=(1,))
    worker.start()
    try:
        assert library.entered.wait(10)
        with pytest.raises(abi.NativeError) as caught:
            backend.info()
        assert caught.value.status == abi.ERR_RUNTIME
    finally:
        library.release.set()
        worker.join(10)
    backend.close()


def test_every_public_method_is_guarded():
    for name, member in vars(backend_module.B200Backend).items():
        if callable(member) and not name.startswith("_") and not isinstance(member, (staticmethod, classmethod)):
            assert hasattr(member, "__wrapped__"), name
