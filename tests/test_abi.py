"""The C ABI library: it loads, exports every function that
include/creature_engine.h declares, and its structs have the layouts the
reference's #[repr(C)] types have. No GPU call is made."""
import ctypes as C
import re
from pathlib import Path

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200 import api

HEADER = Path(__file__).resolve().parents[1] / "include" / "creature_engine.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ce_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = ce.lib()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(api.EXPORTED) <= set(names)


def test_header_compiles_as_c11_and_cpp17(tmp_path):
    """The header is what a cgo / ctypes / JNI binding includes: it must
    stand alone in C and C++ (every type declared before its first use)."""
    import shutil
    import subprocess
    src = tmp_path / "use.c"
    src.write_text('#include "creature_engine.h"\nint main(void) { return 0; }\n')
    for tool, std in (("gcc", "-std=c11"), ("g++", "-std=c++17")):
        if shutil.which(tool) is None:
            continue
        cmd = [tool, std, "-Wall", "-Werror", "-fsyntax-only", "-I", str(HEADER.parent)]
        if tool == "g++":
            cmd += ["-x", "c++"]
        proc = subprocess.run(cmd + [str(src)], capture_output=True, text=True)
        assert proc.returncode == 0, proc.stderr[-2000:]


def test_struct_layouts():
    # Params: 25 words and two rungs of 8 (shaders/creature.cu:66-103).
    assert C.sizeof(api.Params) == 25 * 4 + 2 * 32
    # Result: 19 floats (src/creature_kernel.rs:17-91).
    assert ce.RESULT_DTYPE.itemsize == 76
    # Genes (src/evolution.rs:41-50, 58-80, 209-243).
    assert api.NODE_DTYPE.itemsize == 16
    assert api.BONE_DTYPE.itemsize == 28
    assert api.MUSCLE_DTYPE.itemsize == 52


def test_errors_are_reported_without_a_gpu():
    lib = ce.lib()
    h = C.c_void_p()
    status = lib.ce_submit(None, None, None, None)
    assert status == ce.CE_ERR_INVALID
    assert b"null" in lib.ce_last_error()
    assert lib.ce_free_slots(None) == 0
    assert lib.ce_allocated_bytes(None) == 0
    del h


def test_failure_entry_points_reject_null_handles_without_a_gpu():
    lib = ce.lib()
    assert lib.ce_inject_fault(None, 1, ce.CE_ERR_DEVICE) == ce.CE_ERR_INVALID
    assert lib.ce_wait(None, 0) == ce.CE_ERR_INVALID
    assert lib.ce_release_idle(None) == ce.CE_ERR_INVALID
    t, n, busy = C.c_uint64(), C.c_size_t(), C.c_double()
    assert lib.ce_poll(None, 0, C.byref(t), None, 0, C.byref(n), C.byref(busy)) == ce.CE_ERR_INVALID
    assert lib.ce_close(None) == ce.CE_OK
    h = C.c_void_p()
    assert lib.ce_open(0, None, None) == ce.CE_ERR_INVALID
    # With no GPU (or a device ordinal that does not exist) the open fails
    # with a status and a message, never a crash.
    st = lib.ce_open(1000, None, C.byref(h))
    assert st != ce.CE_OK and not h.value
    assert lib.ce_last_error()
