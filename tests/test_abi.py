"""CPU checks of the drop-in boundary: the library loads, exports every function the header declares, and reports
errors as statuses (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess

import pytest
import torch

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ryoanji_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return re.findall(r"RYO_API\s+[\w\s\*]+?\b(ryo_\w+)\s*\(", text)


def test_header_declares_functions():
    names = declared_functions()
    assert len(names) >= 30
    assert "ryo_traverse_f32" in names and "ryo_treebuilder_update_f32" in names


def test_library_exports_every_declared_symbol():
    from ryoanji_b200._abi import LIB_PATH, SIGNATURES
    lib = C.CDLL(LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name
    # the Python bindings cover the whole header
    assert set(declared_functions()) == set(SIGNATURES)


def test_only_c_abi_is_exported():
    from ryoanji_b200._abi import LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True).stdout
    exported = [l.split()[-1] for l in out.splitlines() if " T " in l]
    assert exported and all(n.startswith("ryo_") for n in exported), [n for n in exported if not n.startswith("ryo_")]


def test_status_strings_and_version():
    import ryoanji_b200 as ryo
    assert ryo.lib.ryo_version() == b"0.1.0"
    assert ryo.lib.ryo_status_string(0) == b"ok"
    assert b"stack" in ryo.lib.ryo_status_string(4)
    assert ryo.lib.ryo_status_string(ryo._abi.ERR_INTERNAL) == b"internal error"
    assert ryo.lib.ryo_status_string(ryo._abi.ERR_INTERNAL + 1) == b"unknown status"
    assert ryo.bh_max_target_size() == 64
    assert ryo.stack_size(1000) == 0


def test_bad_arguments_return_status_not_crash():
    import ryoanji_b200 as ryo
    assert ryo.lib.ryo_ctx_create(0, None) == 2
    assert ryo.lib.ryo_read_bh_stats(None, None) == 2
    assert ryo.lib.ryo_treebuilder_create(None, 64, None) == 2
    args = [None, None, 1] + [None] * 15 + [1.0, 0, None, None, None, None, None, None, None]
    assert ryo.lib.ryo_traverse_f32(*args) == 2


def test_direct_sums_check_ranges_before_any_launch():
    """targets past the body count, replicas without a box and negative shells are refused on the host"""
    import ryoanji_b200 as ryo
    fake = C.c_void_p(16)  # never dereferenced: the checks come first
    arrays = [fake] * 9
    assert ryo.lib.ryo_direct_sum_f32(0, 10, 5, None, 0, *arrays, None) == 2
    assert ryo.lib.ryo_direct_sum_f32(0, 5, 5, None, 1, *arrays, None) == 2
    assert ryo.lib.ryo_direct_sum_f64(6, 5, 10, None, 0, *arrays, None) == 2
    assert ryo.lib.ryo_direct_targets_f64(fake, 4, *[fake] * 5, 10, 1.0, None, -1, *[fake] * 4, None) == 2
    assert b"replicas" in ryo.lib.ryo_ctx_last_error(None)


def test_sort_rejects_counts_beyond_32_bits():
    """the sort's digit offsets are 32-bit: 2^32 keys are refused before any pointer is used or kernel launched"""
    import ryoanji_b200 as ryo
    fake = C.c_void_p(16)  # never dereferenced: the count check comes first
    n = 1 << 32
    st = ryo.lib.ryo_sort_by_key(fake, fake, n, fake, fake, fake, ryo.lib.ryo_sort_by_key_temp_bytes(n), None)
    assert st == 2
    assert b"2^32" in ryo.lib.ryo_ctx_last_error(None)


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_context_without_device_fails_cleanly():
    import ryoanji_b200 as ryo
    h = C.c_void_p()
    st = ryo.lib.ryo_ctx_create(0, C.byref(h))
    assert st != 0 and not h.value
    assert len(ryo.lib.ryo_ctx_last_error(None)) > 0


def test_cpp_shim_headers_compile():
    """the C++ drop-in headers (reference signatures) compile against the C ABI"""
    shim = os.path.join(ROOT, "include", "ryoanji_b200", "ryoanji.hpp")
    if not os.path.exists(shim):
        pytest.skip("no C++ shim")
    src = f'#include "{shim}"\nint main() {{ return 0; }}\n'
    r = subprocess.run(["/usr/bin/g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), "-x",
                        "c++", "-"], input=src, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_cpp_shim_links_and_reports_errors(tmp_path):
    """a C++ caller of the drop-in header links against the library; without a device, creating a context throws
    ryo::Error with the no-device status instead of exiting"""
    from ryoanji_b200._abi import LIB_PATH
    src = tmp_path / "caller.cpp"
    src.write_text(r'''
#include "ryoanji_b200/ryoanji.hpp"
#include <cstdio>
int main() {
    if (ryo::bhMaxTargetSize() != 64 || ryo::stackSize(1000) != 0) return 2;
    // the cstone primitives: sizes and empty inputs need no device
    if (ryo::sortByKeyTempStorage<uint64_t, unsigned>(1000) != ryo_sort_by_key_temp_bytes(1000)) return 6;
    ryo::sortByKey<unsigned>(nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0);
    ryo::sequence(nullptr, 0, 0);
    ryo::Box<float> box(-1.f, 1.f);
    if (box.lx() != 2.f || box.boundaryX() != ryo::BoundaryType::open) return 3;
    try { ryo::Context ctx(0); return 4; }
    catch (const ryo::Error& e) { std::printf("%d %s\n", int(e.status), e.what()); return e.status == RYO_ERR_NO_DEVICE || e.status == RYO_ERR_CUDA ? 0 : 5; }
}
''')
    exe = tmp_path / "caller"
    libdir = os.path.dirname(LIB_PATH)
    r = subprocess.run(["/usr/bin/g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L", libdir, "-lryoanji_b200", f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True)
    assert run.returncode == 0, (run.returncode, run.stdout, run.stderr)


def test_public_api_is_exported():
    """every name in ryoanji_b200.__all__ exists, and every public function and class of the package is listed"""
    import inspect
    import ryoanji_b200 as ryo
    missing = [n for n in ryo.__all__ if not hasattr(ryo, n)]
    assert not missing, missing
    own = [n for n, v in vars(ryo).items() if not n.startswith("_") and (inspect.isfunction(v) or inspect.isclass(v))
           and getattr(v, "__module__", "") == ryo.__name__]
    assert set(own) <= set(ryo.__all__), set(own) - set(ryo.__all__)


def test_compat_demo_flow_compiles_and_links(tmp_path):
    """the reference demo's flow in the reference's own spellings (cstone::, ryoanji::, execution::Gpu) builds against
    ryoanji_b200/compat.hpp and this library, for all three type sets"""
    from ryoanji_b200._abi import LIB_PATH
    exe = tmp_path / "demo_flow"
    libdir = os.path.dirname(LIB_PATH)
    r = subprocess.run(["/usr/bin/g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I",
                        "/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "demo_flow.cpp"), "-o", str(exe),
                        "-L", libdir, "-lryoanji_b200", "-L", "/usr/local/cuda/lib64", "-lcudart",
                        f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
