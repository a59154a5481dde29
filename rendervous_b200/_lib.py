"""cffi binding of libvrt.so (include/vrt.h).

The declarations are read from the header itself (between its CDEF markers),
so the Python side and the C ABI cannot drift apart.  Loading fails loudly
when the library is missing: there is no CPU fallback for any operator.
"""
from __future__ import annotations

import os
import threading

import cffi
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvrt.so")
HEADER = os.path.join(_HERE, "..", "include", "vrt.h")

_lock = threading.Lock()
_state: dict = {}


class VrtError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"vrt error {status} ({status_string(status)}){': ' + what if what else ''}")


def cdef_text() -> str:
    text = open(HEADER).read()
    return text.split("/* CDEF-BEGIN */")[1].split("/* CDEF-END */")[0]


def ffi_lib():
    """(ffi, lib); raises if libvrt.so has not been built."""
    with _lock:
        if "lib" not in _state:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `python -m rendervous_b200.build` "
                    "(there is no CPU fallback)")
            ffi = cffi.FFI()
            ffi.cdef(cdef_text())
            _state["ffi"] = ffi
            _state["lib"] = ffi.dlopen(LIB_PATH)
        return _state["ffi"], _state["lib"]


def status_string(status: int) -> str:
    try:
        ffi, lib = ffi_lib()
        return ffi.string(lib.vrt_status_string(int(status))).decode()
    except Exception:  # pragma: no cover - only while the library is unavailable
        return "?"


def check(status: int, what: str = "") -> None:
    if status != 0:
        raise VrtError(int(status), what)


def fptr(t: torch.Tensor | None):
    ffi, _ = ffi_lib()
    if t is None:
        return ffi.NULL
    assert t.dtype == torch.float32, t.dtype
    return ffi.cast("float *", t.data_ptr())


def stream_handle(device: torch.device):
    ffi, _ = ffi_lib()
    return ffi.cast("void *", torch.cuda.current_stream(device).cuda_stream)


class Context:
    """One vrt_context (device scratch: work queue, counters, error word) per device."""

    def __init__(self, device: int):
        ffi, lib = ffi_lib()
        out = ffi.new("vrt_context **")
        with torch.cuda.device(device):
            check(lib.vrt_context_create(device, out), "vrt_context_create")
        self.ptr = out[0]
        self.device = device

    def sync(self) -> dict:
        """Waits for the current stream; returns and clears the device counters.
        Raises VrtError if a kernel recorded an error."""
        ffi, lib = ffi_lib()
        c = ffi.new("vrt_counters *")
        with torch.cuda.device(self.device):
            st = lib.vrt_context_sync(self.ptr, stream_handle(torch.device("cuda", self.device)), c)
        counters = dict(paths=int(c.paths), vertices=int(c.vertices), steps=int(c.steps), lookups=int(c.lookups),
                        reds=int(c.reds), albedo_lookups=int(c.albedo_lookups), status=int(c.status),
                        detail=int(c.detail))
        check(st, "device-side error recorded by a kernel")
        return counters


_contexts: dict = {}


def context(device: torch.device | int | None = None) -> Context:
    if device is None:
        device = torch.cuda.current_device()
    if isinstance(device, torch.device):
        device = device.index if device.index is not None else torch.cuda.current_device()
    with _lock:
        if device not in _contexts:
            _contexts[device] = None
    if _contexts[device] is None:
        _contexts[device] = Context(device)
    return _contexts[device]


def exported_symbols() -> list:
    """Names of the functions declared between the header's CDEF markers."""
    import re
    return re.findall(r"\b(vrt_[a-z0-9_]+)\s*\(", cdef_text())
