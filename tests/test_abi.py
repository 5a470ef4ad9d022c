"""CPU checks of the C ABI boundary: the library loads without a GPU and
exports every function include/avionic.h declares, and the Python binding
declares each of them."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "avionic.h")
LIB = os.path.join(ROOT, "avionic_b200", "libavionic_core.so")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(avx_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "avx_solver_run" in names and "avx_cartesian_operator_create" in names
    assert len(names) >= 30


@pytest.mark.skipif(not os.path.exists(LIB), reason="library not built")
def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.skipif(not os.path.exists(LIB), reason="library not built")
def test_python_binding_covers_header():
    from avionic_b200 import _abi
    assert sorted(_abi.SIGNATURES) == declared_functions()


@pytest.mark.skipif(not os.path.exists(LIB), reason="library not built")
def test_cpu_only_entry_points():
    """Entry points that do no device work answer on a CPU-only host."""
    import avionic_b200 as av
    assert av.lib.avx_version().startswith(b"avionic-b200")
    assert abs(av.ellipke(0.5) - 1.3506) < 1e-3
    ds, dt = av.time_space_weights(5.0)
    from oracle import stencils as st
    rds, rdt = st.time_space_weights(5.0)
    assert abs(ds - rds) < 1e-6 and abs(dt - rdt) < 1e-6
    p = av.default_params(av.ICTGV2)
    assert p.maxIt == 500 and abs(p.alpha - 0.6423) < 1e-6 and abs(p.timeSpaceWeight - 6.5) < 1e-6
    with pytest.raises(av.AvionicError):
        av.default_params(av.TGV2_3D)
    with pytest.raises(av.AvionicError):
        av.time_space_weights(-1.0)


STRUCTS = {
    # C type: ctypes mirror name in avionic_b200._abi
    "avx_pd_params": "PDParams",
    "avx_run_stats": "RunStats",
    "avx_coil_params": "CoilParams",
    "avx_request": "Request",
    "avx_completion": "Completion",
}


@pytest.mark.skipif(not os.path.exists(LIB), reason="library not built")
def test_struct_layouts_match_the_header(tmp_path):
    """sizeof and every field offset of the ABI structs, as gcc lays them out
    from include/avionic.h, equal the ctypes mirrors."""
    import shutil
    import subprocess
    from avionic_b200 import _abi
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "avionic.h"', "int main(void) {"]
    for ctype, pyname in STRUCTS.items():
        cls = getattr(_abi, pyname)
        lines.append('printf("%s sizeof %%zu\\n", sizeof(%s));' % (ctype, ctype))
        for fname, _ in cls._fields_:
            cf = "lambda" if fname == "lambda_" else fname
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (ctype, fname, ctype, cf))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln.strip():
            c, f, v = ln.split()
            got[(c, f)] = int(v)
    for ctype, pyname in STRUCTS.items():
        cls = getattr(_abi, pyname)
        assert got[(ctype, "sizeof")] == ctypes.sizeof(cls), ctype
        for fname, _ in cls._fields_:
            assert got[(ctype, fname)] == getattr(cls, fname).offset, (ctype, fname)


def test_generators_import_without_the_library():
    """The numpy problem generators (and so the CPU reference arm of the
    bench) run in a process that never loads libavionic_core.so; the first
    library name used through the package loads it."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from avionic_b200 import synth\n"
            "p = synth.small(1)\n"
            "assert 'avionic_b200.api' not in sys.modules\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libavionic_core' not in maps\n"
            "print('ok')\n") % ROOT
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stderr
