"""The C-ABI library loads and exports every function include/*.h declares."""
import ctypes
import re

from helpers import ROOT


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(v(?:gpu|host)_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_headers_declare_entry_points():
    names = declared_functions()
    assert "vgpu_create" in names and "vhost_load" in names and "vgpu_run" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from vulture_b200 import _native

    lib = ctypes.CDLL(str(_native.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"
    assert set(_native.EXPORTS) <= set(declared_functions())


def test_oracle_library_loads():
    from vcpu import _load

    L = _load()
    for pre in ("vcpu64_", "vcpu32_"):
        for fn in ("create", "run", "read_td", "read_dft", "read_field", "write_field", "destroy"):
            assert hasattr(L, pre + fn)


def test_engine_reports_missing_device_without_exiting():
    """vgpu_create returns an error code (never exits) when no sm_100 device is
    visible; with a device present it must succeed instead."""
    import vulture_b200 as vb
    from conftest import gpu_available
    from helpers import stage_case

    m = vb.Mesh(stage_case("hardsrc_ez"))
    if gpu_available():
        g = vb.GpuRun(m)
        g.close()
    else:
        from vulture_b200._native import NativeError

        try:
            vb.GpuRun(m)
        except NativeError as e:
            assert e.code in (-4, -3)
        else:
            raise AssertionError("engine created without a GPU")
