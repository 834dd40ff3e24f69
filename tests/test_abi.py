"""The C-ABI library loads and exports every entry point include/*.h declares,
and the ctypes mirrors have the header's layouts (no compute; runs on CPU)."""

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for header in sorted((ROOT / "include").glob("*.h")):
        text = header.read_text()
        for m in re.finditer(r"REFORM_API\s+[\w\s\*]+?\b(\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported(native):
    names = declared_symbols()
    assert {"praq_solve", "praq_default_parameters", "praq_check_interval"} <= names
    missing = [n for n in sorted(names) if not hasattr(native, n)]
    assert not missing, missing


def test_struct_layouts_match_reference_sizes():
    from reformulation_b200 import _native
    # PraqParameters: d, i64, int(+pad), 7 d, i64, 3 d  = 8+8+8+56+8+24
    assert ctypes.sizeof(_native.PraqParameters) == 112
    assert ctypes.sizeof(_native.PraqInstance) == 48
    assert ctypes.sizeof(_native.PraqResult) == 32
    assert ctypes.sizeof(_native.PriaParams) == 9 * 8 + 8 + 4 * 4
    assert ctypes.sizeof(_native.PriaResultInfo) == 32


def test_trace_record_layout_matches_the_header(tmp_path):
    """reform_trace_record (include/reform_trace.h) as compiled by the host C
    compiler has the size and field offsets of the NumPy record type the
    Python backends read the trace into."""
    import shutil
    import subprocess
    import numpy as np
    from reformulation_b200 import _native
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    root = Path(__file__).resolve().parent.parent
    src = tmp_path / "t.c"
    fields = _native.TRACE_DTYPE.names
    src.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"reform_trace.h\"\n"
                   "int main(void) { printf(\"%zu\", sizeof(reform_trace_record));"
                   + "".join(f" printf(\" %zu\", offsetof(reform_trace_record, {f}));" for f in fields)
                   + " return 0; }\n")
    exe = tmp_path / "t"
    subprocess.run([cc, f"-I{root / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got[0] == _native.TRACE_DTYPE.itemsize
    assert got[1:] == [_native.TRACE_DTYPE.fields[f][1] for f in fields]
    assert np.dtype(_native.TRACE_DTYPE).itemsize == 56


def test_default_parameters_and_interval_rule(native):
    from reformulation_b200.praq import Library
    lib = Library()
    p = lib.parameters()
    assert p.tolerance == 1e-8 and p.max_iter == -1 and p.op_steps == 16
    assert abs(p.beta_sufficient - 0.36787944117144233) < 1e-17
    q = lib.parameters(op_steps=0)
    # 3 log2(n / 50k): 50k -> 2 (floor), 400k -> 9, 2M -> 16 (test_solver.cu:238-262)
    assert lib.check_interval(50_000, q) == 2
    assert lib.check_interval(400_000, q) == 9
    assert lib.check_interval(2_000_000, q) == 16
    q.interval_power = 0.5
    assert lib.check_interval(int(50000.0 * 7.38905609893065), q) == 15
