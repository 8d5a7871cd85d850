"""CPU checks of the drop-in boundary: libkwb.so loads, exports every function include/kwb.h
declares, its structs match the ctypes mirror byte for byte, and it reports a missing device as a
status code (no compute call is made without a GPU)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "kwb.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(kwb_\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if not n.endswith("_fn")))


def test_library_exports_every_declared_function():
    import kwave_b200 as kb
    lib = kb.load_library()
    names = declared_functions()
    assert len(names) >= 18, names
    for n in names:
        assert hasattr(lib, n), f"{n} declared in kwb.h but not exported"
    assert lib.kwb_version() == 10000


def test_struct_layouts_match_header():
    import kwave_b200._lib as L
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "kwb.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(kwb_problem), sizeof(kwb_sensor_group),
         offsetof(kwb_sensor_group, directivity_angle), offsetof(kwb_sensor_group, frequency_bandwidth),
         offsetof(kwb_problem, groups), offsetof(kwb_problem, tr), offsetof(kwb_problem, u_signal),
         sizeof(kwb_kernel_times), sizeof(kwb_group_sizes), sizeof(kwb_outputs), offsetof(kwb_problem, p0),
         offsetof(kwb_problem, elastic), offsetof(kwb_problem, cs), offsetof(kwb_problem, alpha_coeff_shear),
         offsetof(kwb_problem, s_signal));
  return 0;
}'''
    with tempfile.TemporaryDirectory() as d:
        cpath, exe = os.path.join(d, "s.c"), os.path.join(d, "s")
        open(cpath, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), cpath, "-o", exe], check=True)
        got = [int(v) for v in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    exp = [C.sizeof(L.Problem), C.sizeof(L.SensorGroup), L.SensorGroup.directivity_angle.offset,
           L.SensorGroup.frequency_bandwidth.offset, L.Problem.groups.offset, L.Problem.tr.offset,
           L.Problem.u_signal.offset, C.sizeof(L.KernelTimes), C.sizeof(L.GroupSizes), C.sizeof(L.Outputs),
           L.Problem.p0.offset, L.Problem.elastic.offset, L.Problem.cs.offset,
           L.Problem.alpha_coeff_shear.offset, L.Problem.s_signal.offset]
    assert got == exp


def test_no_device_is_a_status_not_a_crash():
    import kwave_b200 as kb
    lib = kb.load_library()
    h = C.c_void_p()
    rc = lib.kwb_context_create(0, C.byref(h))
    if rc == 0:
        lib.kwb_context_destroy(h)
        pytest.skip("a CUDA device is present")
    assert rc in (-4, -2)
    assert lib.kwb_last_error(None)
    with pytest.raises(kb.KWaveB200Error):
        kb.Context(0)


def test_missing_library_fails_loudly(tmp_path):
    import kwave_b200._lib as L
    saved = L._lib
    try:
        L._lib = None
        with pytest.raises(L.KWaveB200Error, match="no CPU fallback"):
            L.load_library(str(tmp_path / "libkwb.so"))
    finally:
        L._lib = saved


def test_julia_problem_struct_matches_header():
    """The Julia shim's KwbProblem (no Julia here to run it) lists the header's fields, in order,
    with the same C sizes."""
    import re
    import kwave_b200._lib as L
    src = open(os.path.join(ROOT, "k-wave-julia_b200", "julia", "KWaveB200.jl")).read()
    body = re.search(r"struct KwbProblem\n(.*?)\nend\n", src, re.S).group(1)
    jl = [(m.group(1), m.group(2)) for m in re.finditer(r"^\s*(\w+)::([\w{},]+)", body, re.M)]
    size = {"Int32": 4, "Int64": 8, "Float64": 8, "UInt32": 4, "KwbField": 16, "KwbSignal": 24}

    def jl_size(t):
        m = re.fullmatch(r"NTuple\{(\d+),(\w+)\}", t)
        if m:
            return int(m.group(1)) * size[m.group(2)]
        return 8 if t.startswith("Ptr") else size[t]

    names = [n for n, _ in L.Problem._fields_]
    assert [n for n, _ in jl] == names
    for (n, t), (_, ct) in zip(jl, L.Problem._fields_):
        assert jl_size(t) == C.sizeof(ct), (n, t)
