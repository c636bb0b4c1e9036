"""The C ABI: header <-> library symbols, loading without a GPU, error paths that need no device."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "ps2cuda.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(ps[23]_[a-z_0-9]+)\s*\(", text, re.M)))


def test_header_declares_the_context_and_kernel_entry_points():
    names = declared_functions()
    for n in ("ps2_create", "ps2_load_patch", "ps2_run_to_convergence", "ps2_download", "ps2_topofit",
              "ps2_grid_accumulate", "ps2_clap_filter_grid", "ps2_random_coherence_histogram"):
        assert n in names


def test_library_builds_loads_and_exports_every_declared_symbol(cuda_lib):
    for name in declared_functions():
        assert hasattr(cuda_lib, name), name


def test_python_binding_lists_every_symbol():
    from pystamps_b200 import _lib

    assert sorted(_lib.EXPORTED) == declared_functions()


def _field_names(struct):
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    body = text[text.index("typedef struct " + struct):text.index("} " + struct + ";")]
    body = body[body.index("{") + 1:]
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        for part in decl.split(","):
            names.append(re.findall(r"[A-Za-z_][A-Za-z_0-9]*", part)[-1])
    return names


def test_struct_layouts_match_header():
    from pystamps_b200 import _lib

    for struct, cls in (("ps2_patch_desc", _lib.PatchDesc), ("ps2_outputs", _lib.Outputs),
                        ("ps2_iter_stats", _lib.IterStats), ("ps3_reestimate_desc", _lib.S3Desc),
                        ("ps3_reestimate_out", _lib.S3Out)):
        assert _field_names(struct) == [f for f, _ in cls._fields_], struct


def test_invalid_arguments_are_rejected_before_any_device_work(cuda_lib):
    # NULL inputs fail with PS2_ERR_INVALID_ARG and a message; no GPU is touched
    rc = cuda_lib.ps2_topofit(None, None, 0, ctypes.c_double(1.0), ctypes.c_int64(1), ctypes.c_int64(1), None, None,
                              None, None)
    assert rc == -1
    assert b"invalid" in cuda_lib.ps2_last_error()
    rc = cuda_lib.ps2_grid_accumulate(None, None, ctypes.c_int64(1), ctypes.c_int64(1), ctypes.c_int64(1),
                                      ctypes.c_int64(1), None)
    assert rc == -1
    rc = cuda_lib.ps2_load_patch(None, None)
    assert rc == -1


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from pystamps_b200 import _lib

    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setenv("PS2CUDA_LIB", str(tmp_path / "nope.so"))
    with pytest.raises(_lib.BackendUnavailableError):
        _lib.lib()


def test_stage3_reestimate_rejects_bad_descriptors_without_a_device(cuda_lib):
    from pystamps_b200 import _lib

    d = _lib.S3Desc()
    o = _lib.S3Out()
    d.n_sel, d.n_ifg, d.clap_win, d.n_fit = 1, 4, 24, 4
    assert cuda_lib.ps3_reestimate(ctypes.byref(d), ctypes.byref(o), 0) == -4  # clap_win must be 32
    d.clap_win, d.n_fit = 32, 0
    assert cuda_lib.ps3_reestimate(ctypes.byref(d), ctypes.byref(o), 0) == -1
    assert b"n_fit" in cuda_lib.ps2_last_error()
