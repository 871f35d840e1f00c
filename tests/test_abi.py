"""The C-ABI library loads, exports every entry point the C headers under include/ declare,
and its host-side topology planning matches the oracle (no GPU needed)."""
import glob
import os
import re

import pytest

import dsdecompx_b200 as dsx
from oracle import Grid

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    """Entry points of every C header under include/ (dsx.h, dsx_shard.h, ...)."""
    names = set()
    for h in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(dsx_[a-z_0-9]+)\s*\(", text))
    return sorted(names - {"dsx_step_callback"})


def test_library_exports_every_declared_symbol():
    lib = dsx.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_errors():
    lib = dsx.lib()
    assert b"sm_100a" in lib.dsx_version()
    with pytest.raises(ValueError, match="dsDecompX: nranks"):
        dsx.plan_topology(0, 0)
    with pytest.raises(ValueError, match="do not match"):
        dsx.plan_topology(8, 0, dims=(3, 1, 1))


CASES = [
    dict(nranks=1, dims=(1, 1, 1)),
    dict(nranks=2, dims=(0, 0, 0)),
    dict(nranks=8, dims=(2, 2, 2)),
    dict(nranks=12, dims=(3, 1, 4), periodic=(True, False, False)),
    dict(nranks=12, dims=(3, 1, 4), periodic=(False, True, False), edges_and_corners=False),
    dict(nranks=64, dims=(4, 4, 4)),
    dict(nranks=256, dims=(8, 8, 4), upper=(400.0, 400.0, 200.0)),
    dict(nranks=6, policy="balanced", upper=(12.0, 8.0, 4.0)),
    dict(nranks=24, policy="dynamic", upper=(3.0, 2.0, 1.0)),
    dict(nranks=16, policy="topology_aware", upper=(1.0, 1.0, 8.0)),
    dict(nranks=7, dims=(0, 0, 0)),
]


@pytest.mark.parametrize("case", CASES)
def test_topology_matches_oracle(case):
    case = dict(case)
    P = case.pop("nranks")
    kw = dict(dims=case.get("dims", (0, 0, 0)), policy=case.get("policy", "manual"),
              lower=(0.0, 0.0, 0.0), upper=case.get("upper", (10.0, 10.0, 10.0)),
              periodic=case.get("periodic", (True, True, True)),
              edges_and_corners=case.get("edges_and_corners", True))
    g = Grid("port", P, kw["dims"], kw["policy"], kw["lower"], kw["upper"], kw["periodic"],
             0.5, kw["edges_and_corners"])
    for r in range(P):
        dims, nbrs = dsx.plan_topology(P, r, **kw)
        assert dims == g.topology(r)[0]
        assert nbrs == g.neighbors(r)


def _mirrors():
    """(C struct name, Python mirror) of every struct that crosses the ABI."""
    import ctypes as C

    from dsdecompx_b200 import sharded
    return [("dsx_domain", dsx._Domain), ("dsx_migration_result", dsx._MigrationResult),
            ("dsx_grid_desc", dsx._GridDesc), ("dsx_field_desc", dsx._FieldDesc),
            ("dsx_grid_view", dsx.GridView), ("dsx_tune_report", dsx.TuneReport),
            ("dsx_segment", dsx.SEGMENT_DTYPE), ("dsx_copy", dsx.COPY_DTYPE),
            ("dsx_transport", sharded._Transport)], C


def test_struct_layouts_match_headers(tmp_path):
    """The ctypes structures and numpy record types of the Python front end
    have the size and field offsets that a C compiler gives the header
    structs (a field added on one side only would shift every later one)."""
    import shutil
    import subprocess
    mirrors, C = _mirrors()
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    layout = {}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "dsx.h"', '#include "dsx_shard.h"',
             "int main(void) {"]
    for name, mirror in mirrors:
        fields = list(mirror.names) if hasattr(mirror, "names") else [f[0] for f in mirror._fields_]
        layout[name] = fields
        lines.append(f'    printf("{name} size %zu\\n", sizeof({name}));')
        for f in fields:
            lines.append(f'    printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    want = {}
    for line in filter(None, out):
        name, what, value = line.split()
        want[(name, what)] = int(value)
    for name, mirror in mirrors:
        if hasattr(mirror, "names"):
            size = mirror.itemsize
            offsets = {f: mirror.fields[f][1] for f in mirror.names}
        else:
            size = C.sizeof(mirror)
            offsets = {f[0]: getattr(mirror, f[0]).offset for f in mirror._fields_}
        assert size == want[(name, "size")], (name, size, want[(name, "size")])
        for f, off in offsets.items():
            assert off == want[(name, f)], (name, f, off, want[(name, f)])


def _noalloc():
    import ctypes as C
    fn = dsx.lib().dsx_migrate_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(dsx._GridDesc), C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                   C.POINTER(C.c_void_p), C.POINTER(C.c_longlong), C.POINTER(C.c_void_p),
                   C.POINTER(C.c_longlong), C.c_void_p, C.c_char_p, C.c_int]
    return fn


def _noalloc_call(nranks, dims, counts, ins, outs, cuts=None, upper=(10.0, 10.0, 10.0)):
    """Calls that the entry point refuses on the host, before any CUDA call."""
    import ctypes as C

    import numpy as np
    desc = dsx._grid_desc(nranks, dims, "manual", (0, 0, 0), upper, (True, True, True),
                          1.0, True, None)
    counts = np.asarray(counts, dtype=np.int64)
    out = np.zeros(max(nranks, 1), dtype=np.int64)
    err = C.create_string_buffer(256)
    cut_arg = None
    if cuts is not None:
        cuts = np.ascontiguousarray(cuts, dtype=np.float64)
        cut_arg = cuts.ctypes.data_as(C.POINTER(C.c_double))
    status = _noalloc()(C.byref(desc), cut_arg, counts.ctypes.data_as(C.POINTER(C.c_longlong)),
                        (C.c_void_p * 13)(*ins), out.ctypes.data_as(C.POINTER(C.c_longlong)),
                        (C.c_void_p * 13)(*outs), None, None, err, 256)
    return status, err.value


def test_noalloc_refuses_overflowing_dims():
    # 3 * 1431655768 * 1 wraps to 8 in 32-bit arithmetic
    status, msg = _noalloc_call(8, (3, 1431655768, 1), [0] * 8, [0] * 13, [0] * 13)
    assert status == -1 and b"dims whose product is nranks" in msg
    status, msg = _noalloc_call(8, (2, 2, 3), [0] * 8, [0] * 13, [0] * 13)
    assert status == -1


def test_noalloc_refuses_overlapping_arrays():
    base = 1 << 40            # never dereferenced: the call refuses first
    ins = [base + 0x100000 * a for a in range(13)]
    outs = [base + 0x4000000 + 0x100000 * a for a in range(13)]
    outs[5] = ins[5] + 64     # output 5 starts inside input 5
    status, msg = _noalloc_call(1, (1, 1, 1), [1000], ins, outs)
    assert status == -1 and b"overlap" in msg
    outs[5] = ins[12]         # aliasing across arrays of different widths
    status, msg = _noalloc_call(1, (1, 1, 1), [1000], ins, outs)
    assert status == -1 and b"overlap" in msg


@pytest.mark.parametrize("cuts", [
    [0.0, 0.0, 10.0, 0.0, 10.0, 0.0, 10.0],     # x cuts not strictly increasing
    [0.0, 11.0, 10.0, 0.0, 10.0, 0.0, 10.0],    # x cuts decrease
    [1.0, 5.0, 10.0, 0.0, 10.0, 0.0, 10.0],     # x cuts do not start at lower
    [0.0, 5.0, 10.0, 0.0, 9.0, 0.0, 10.0],      # y cuts do not end at upper
])
def test_noalloc_refuses_bad_cuts(cuts):
    status, msg = _noalloc_call(2, (2, 1, 1), [0, 0], [0] * 13, [0] * 13, cuts=cuts)
    assert status == -1 and b"strictly increasing and span" in msg


def test_every_library_kernel_waits_for_its_predecessor():
    """The library launches its kernels with programmatic stream serialisation
    (a kernel may become resident while the one before it drains).  That is
    only ordered if every such kernel waits (griddepcontrol.wait, through
    pdl_begin) before it touches memory: each kernel body of dsx_kernels.cu
    must open with pdl_begin(), and every launch there must go through
    pdl_launch (no triple-chevron launch)."""
    src = open(os.path.join(ROOT, "dsdecompx_b200", "csrc", "dsx_kernels.cu")).read()
    code = re.sub(r"//[^\n]*", "", src)
    kernels = 0
    for m in re.finditer(r"__global__[^{;]*?\b(k_\w+)\s*\(", code):
        depth, k = 0, m.end() - 1
        while True:
            depth += {"(": 1, ")": -1}.get(code[k], 0)
            if depth == 0:
                break
            k += 1
        body = code[code.index("{", k) + 1:]
        assert body.lstrip().startswith("pdl_begin();"), m.group(1)
        kernels += 1
    assert kernels >= 20
    assert "<<<" not in code
