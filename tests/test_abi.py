"""The C-ABI library: exports, host-side argument handling and loud failure
without a GPU.  No integration runs here (that needs a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

import galpy_b200
from galpy_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "galpy_cuda.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = "\n".join(ln for ln in txt.splitlines() if not ln.lstrip().startswith("typedef"))
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    names = header_functions()
    assert "integrateFullOrbit_cuda" in names and "galpy_cuda_integrate_device" in names
    for n in names:
        assert hasattr(lib, n), n
    # and the Python binding knows every one of them
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_abi_version_and_record_size():
    lib = _lib.lib()
    assert lib.galpy_cuda_abi_version() == 2
    # type + table offset, scalars, gamma* table, binade table, two exponent
    # tables, single-precision copies of the gamma* and binade tables
    assert lib.galpy_cuda_comp_size() == (8 + 16 * 8 + 32 * 12 * 8 + 8 * 12 * 8 + 32 * 8 + 64 * 8
                                          + 32 * 12 * 4 + 8 * 12 * 4)


def test_compile_potential_host_only(golden):
    buf, n = galpy_b200.compile_potential((golden["mw14_type"], golden["mw14_args"]))
    assert n == 3 and buf.size == 3 * _lib.lib().galpy_cuda_comp_size()
    rec = buf.reshape(3, -1)
    assert rec[:, :4].view(np.int32).ravel().tolist() == [15, 5, 9]
    with pytest.raises(galpy_b200.PotentialNotSupported):  # TwoPowerSphericalPotential
        galpy_b200.compile_potential(([42], [1.0, 1.0, 1.5, 3.5]))


def test_scf_continuation_records():
    """An SCF expansion compiles to its record and continuation records
    (type -100) holding its coefficients; the count is the launch's ncomp.
    Time-dependent SCF coefficients are not carried."""
    import timedep_pots as TP

    pt, pa = TP.potential("scf_nonaxi")
    size = _lib.lib().galpy_cuda_comp_size()
    buf, n = galpy_b200.compile_potential((pt, pa))
    N, L = 6, 5
    payload = (L * (L + 1) // 2) * N * 2 + 6 * L * (N - 1)
    per = (size - 8) // 8
    assert n == 1 + -(-payload // per) and buf.size == n * size
    types = buf.reshape(n, -1)[:, :4].view(np.int32).ravel().tolist()
    assert types == [24] + [-100] * (n - 1)
    pt2, pa2 = TP.potential("scf_axi+mn")
    buf2, n2 = galpy_b200.compile_potential((pt2, pa2))
    assert buf2.reshape(n2, -1)[:, :4].view(np.int32).ravel().tolist() == [24, -100, 5]
    tdep = pa.copy()
    tdep[5] = 3.0  # Nt > 0: coefficients interpolated in time
    with pytest.raises(galpy_b200.PotentialNotSupported):
        galpy_b200.compile_potential((pt, tdep))


def test_signatures_of_component_lists():
    """MWPotential2014's exact list gets the compile-time kernels; lists
    without an ellipsoidal component the lighter run-time list; any list with
    one the full run-time list."""
    sig = _lib.lib().galpy_cuda_signature

    def s(types):
        t = np.ascontiguousarray(types, np.int32)
        return sig(len(t), t.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))

    assert s([15, 5, 9]) == 1
    assert s([15, 9, 5]) == 2 and s([13]) == 2 and s([5, 19, 29]) == 2
    for ell in (21, 22, 23, 30, 37, 38, 43):
        assert s([ell]) == 0 and s([15, 5, ell]) == 0
    # DehnenBar (time-dependent) and SCF: the full run-time list
    assert s([15, 5, 9, 1]) == 0 and s([24]) == 0 and s([24, 5]) == 0


def _no_gpu():
    return _lib.lib().galpy_cuda_device_count() == 0


def test_fails_loudly_without_gpu(mw14):
    if not _no_gpu():
        pytest.skip("a GPU is present")
    yo = np.array([[1.0, 0.1, 1.1, 0.0, 0.0, 0.0]])
    with pytest.raises(galpy_b200.CudaError) as e:
        galpy_b200.integrateFullOrbit_cuda(mw14, yo, np.linspace(0, 1, 11), "dop853_cuda")
    assert e.value.code == _lib.ERR_NODEVICE


def test_unsupported_method_is_reported(mw14):
    lib = _lib.lib()
    yo = np.array([[1.0, 0.1, 1.1, 0.0, 0.0, 0.0]])
    t = np.linspace(0, 1, 11)
    res = np.zeros((1, 11, 6))
    err = np.zeros(1, np.int32)
    pt = np.ascontiguousarray(mw14[0], np.int32)
    pa = np.ascontiguousarray(mw14[1], np.float64)
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    for code in (7, 8, -1):  # ias15 (galpy falls back) and codes galpy does not have
        rc = lib.integrateFullOrbit_cuda(1, yo.ctypes.data_as(dp), 11, t.ctypes.data_as(dp), 0, 3,
                                         pt.ctypes.data_as(ip), pa.ctypes.data_as(dp), None,
                                         -9999.99, -27.6, -27.6, res.ctypes.data_as(dp),
                                         err.ctypes.data_as(ip), code, _lib.CALLBACK(), None)
        assert rc in (_lib.ERR_METHOD, _lib.ERR_NODEVICE)


def test_parse_integrator_and_tolerances():
    assert galpy_b200.parse_integrator("symplec4_cuda") == 3
    assert galpy_b200.parse_integrator("DOP853_CUDA") == 6
    assert galpy_b200.parse_integrator("leapfrog_c") == 0
    assert galpy_b200.parse_integrator("rk4") == 1
    assert galpy_b200.parse_integrator("dopr54_cuda") == 5
    assert galpy_b200.parse_integrator("symplec6_c") == 4
    assert galpy_b200.parse_integrator("rk6") == 2
    with pytest.raises(ValueError):
        galpy_b200.parse_integrator("ias15_cuda")
    r, a = galpy_b200.parse_tol(None, 1e-10)
    assert r == pytest.approx(-12 * np.log(10)) and a == pytest.approx(np.log(1e-10))


def test_package_has_no_cpu_path():
    """The package never imports the oracle and has no CPU integrator."""
    pkg = os.path.join(ROOT, "galpy_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h")):
                txt = open(os.path.join(dirpath, f)).read()
                for needle in ("import oracle", "from oracle", "liboracle", "oracle/",
                               "libgalpy_ref", "oracle_integrate"):
                    assert needle not in txt, (f, needle)


def test_autotune_candidates_and_keys():
    from galpy_b200 import autotune

    dop = autotune.candidates("dop853_cuda")
    assert all(c["threads_per_orbit"] == 1 and c["schedule"] == "longest_first" for c in dop)
    assert {(c["block_size"], c["variant"]) for c in dop} == {(128, 0), (128, 1)}
    assert {c["block_size"] for c in autotune.candidates("symplec4_cuda")} == {64, 128}
    k1 = autotune.workload_key("B200", "dop853_cuda", False, "fp64", 1, False, 1 << 20, True)
    k2 = autotune.workload_key("B200", "dop853_cuda", False, "fp64", 1, False, (1 << 20) + 5,
                               True)
    k3 = autotune.workload_key("B200", "dop853_cuda", True, "fp64", 1, False, 1 << 20, True)
    assert k1 != k3 and k1.split("|n~")[0] == k2.split("|n~")[0]


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors of the ABI structs have the header's field offsets
    and sizes (a mismatch would silently misplace arguments)."""
    import subprocess

    structs = {"galpy_cuda_opts": _lib.GalpyCudaOpts, "galpy_cuda_launch": _lib.GalpyCudaLaunch,
               "galpy_cuda_adjoint": _lib.GalpyCudaAdjoint}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} @sizeof %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{name} {fname} %zu\\n", offsetof({name}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(ln.split()[:2]): int(ln.split()[2]) for ln in out if ln}
    for name, cls in structs.items():
        assert got[(name, "@sizeof")] == ctypes.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert got[(name, fname)] == getattr(cls, fname).offset, (name, fname)
