"""The C-ABI library loads and exports every function the public header declares (no GPU)."""
import ctypes
import os
import subprocess

from cosmicscanner_b200 import _abi


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    declared = _abi.declared_functions()
    assert len(declared) >= 19
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, missing
    # every declared function also has a ctypes signature in the Python binding
    assert sorted(_abi._SIGNATURES) == declared


def test_exported_symbols_are_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for name in _abi.declared_functions():
        assert name in exported, name


def test_version_and_error_without_device_work():
    lib = _abi.load()
    assert b"sm_100a" in lib.cs_version()
    # argument validation happens before any device work
    handle = ctypes.c_void_p()
    rc = lib.cs_genotypes_create(None, 0, 4, 1, ctypes.byref(handle))
    assert rc == _abi.CS_ERR_FORMAT
    assert b"too small" in lib.cs_last_error()
    bad = (ctypes.c_uint8 * 4)(0x6C, 0x1B, 0x00, 0)
    rc = lib.cs_genotypes_create(bad, 4, 4, 1, ctypes.byref(handle))
    assert rc == _abi.CS_ERR_FORMAT
    assert b"SNP-major" in lib.cs_last_error()
    rc = lib.cs_genotypes_create(bad, 4, 0, 1, ctypes.byref(handle))
    assert rc == _abi.CS_ERR_INVALID_ARGUMENT


def test_package_fails_loudly_without_library(tmp_path):
    missing = os.path.join(tmp_path, "nope.so")
    try:
        _abi.load(missing)
    except RuntimeError as e:
        assert "no CPU fallback" in str(e)
    else:
        raise AssertionError("load of a missing library must raise")


def test_cpp_facade_compiles_links_and_reports_errors(tmp_path):
    """include/cosmicscanner_b200.hpp compiles against the header, links against the library
    and turns a status code into the reference's exception types (no device work)."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "facade.cpp"
    src.write_text(r'''
#include "cosmicscanner_b200.hpp"
#include <cstdio>
int main() {
    unsigned char bad[4] = {0x6C, 0x1B, 0x00, 0};
    try {
        cs::Genotypes::from_bed(bad, 4, 4, 1);
        return 1;
    } catch (const std::runtime_error& e) {
        std::printf("%s\n", e.what());
    }
    try {
        cs::Genotypes::from_bed(bad, 4, 0, 1);
        return 2;
    } catch (const std::invalid_argument& e) {
        std::printf("invalid: %s\n", e.what());
    }
    cs_vce_options o = cs::StcgVce::default_options();
    cs::MvEigenVce mv;
    if (mv.options().max_iter != 1000 || mv.options().tol != 1e-8) return 4;
    try {
        cs::GrmBuilder grm;
        cs::EigenVce vce;
        vce.prepare({1.0}, {}, 0, grm);  // no GRM computed yet
        return 5;
    } catch (const std::invalid_argument& e) {
        std::printf("invalid: %s\n", e.what());
    } catch (const std::runtime_error& e) {
        std::printf("error: %s\n", e.what());
    }
    return (o.mc_samples == 20 && o.pcg_tol == 1e-10 && o.probe_seed == 20250101ull) ? 0 : 3;
}
''')
    exe = tmp_path / "facade"
    lib_dir = os.path.dirname(_abi.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(root, "include"), str(src),
                    "-o", str(exe), "-L", lib_dir, "-lcosmicscanner_b200",
                    f"-Wl,-rpath,{lib_dir}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "SNP-major" in out.stdout and "invalid:" in out.stdout
