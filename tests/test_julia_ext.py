"""The Julia extension (julia/ext/RadiativeViewFactorB200Ext.jl) against the
C header: every struct it passes to ccall must have the C struct's fields,
in order, at the same offsets and with the same size.  Julia lays out an
immutable isbits struct like C (natural alignment), so the offsets follow
from the field types; they are compared with offsetof() of the header
compiled by gcc.  Julia itself is not installed, so the extension's code is
checked here and not run."""
import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
EXT = ROOT / "julia" / "ext" / "RadiativeViewFactorB200Ext.jl"
PATCH = ROOT / "julia" / "patches" / "Assembly_gpu_supports.diff"
HEADER = ROOT / "include" / "rvf_b200.h"

SCALARS = {"Int8": 1, "UInt8": 1, "Int32": 4, "UInt32": 4, "Int64": 8, "UInt64": 8, "Float64": 8, "Float32": 4,
           "Cint": 4, "Csize_t": 8}
STRUCTS = {"RvfMeshDesc": "rvf_mesh_desc", "RvfOptions": "rvf_options", "RvfStats": "rvf_stats",
           "RvfServerOpts": "rvf_server_opts", "RvfRequestInfo": "rvf_request_info",
           "RvfTunedShape": "rvf_tuned_shape", "RvfServerStats": "rvf_server_stats"}


def julia_structs():
    text = EXT.read_text()
    out = {}
    for name, body in re.findall(r"^struct (\w+)\n(.*?)^end", text, re.S | re.M):
        fields = []
        for line in body.splitlines():
            line = line.split("#")[0].strip()
            if line:
                f, t = line.split("::")
                fields.append((f.strip(), t.strip()))
        out[name] = fields
    return out


def size_align(t):
    """(size, alignment) of a Julia field type in C layout."""
    if t in SCALARS:
        return SCALARS[t], SCALARS[t]
    js = julia_structs()
    if t in js:  # a nested struct of the extension
        offs, size = julia_layout(js[t])
        return size, max(size_align(ft)[1] for _, ft in js[t])
    if t.startswith("Ptr{"):
        return 8, 8
    m = re.fullmatch(r"NTuple\{(\d+),\s*(.+)\}", t)
    if m:
        s, a = size_align(m.group(2))
        return int(m.group(1)) * s, a
    raise ValueError(f"unknown field type {t}")


def julia_layout(fields):
    off, align, out = 0, 1, {}
    for f, t in fields:
        s, a = size_align(t)
        off = (off + a - 1) // a * a
        out[f] = off
        off += s
        align = max(align, a)
    return out, (off + align - 1) // align * align


def c_layout(tmp_path, structs):
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', 'int main(void) {']
    for cname, fields in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in fields:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "jl_layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "jl_layout"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        c, f, v = ln.split()
        got[(c, f)] = int(v)
    return got


def test_extension_structs_match_header(tmp_path):
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    js = julia_structs()
    assert set(STRUCTS) <= set(js), set(STRUCTS) - set(js)
    got = c_layout(tmp_path, {STRUCTS[j]: js[j] for j in STRUCTS})
    for jname, cname in STRUCTS.items():
        offs, size = julia_layout(js[jname])
        assert got[(cname, "size")] == size, (jname, size, got[(cname, "size")])
        for f, o in offs.items():
            assert got[(cname, f)] == o, (jname, f, o, got[(cname, f)])


def test_extension_covers_every_c_field():
    """No field of the C structs is missing from the Julia mirror."""
    hdr = HEADER.read_text()
    js = julia_structs()
    for jname, cname in STRUCTS.items():
        end = re.search(r"\}\s*" + cname + ";", hdr).start()
        body = hdr[hdr.rindex("typedef struct {", 0, end) + len("typedef struct {"):end]
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        names = []
        for decl in body.split(";"):  # "const type* a, b, c[4]" -> a, b, c
            if decl.strip():
                names += [re.search(r"(\w+)\s*(?:\[\w+\])?\s*$", v).group(1) for v in decl.split(",")]
        assert names == [f for f, _ in js[jname]], (jname, names)


def test_extension_uses_the_hook_and_trait():
    text = EXT.read_text()
    assert "register_gpu_hook!" in text and "_GPU_HOOK_REF[]" in text
    assert "_gpu_supports(::B200Backend" in text
    patch = PATCH.read_text()
    assert patch.startswith("--- a/src/Assembly.jl\n+++ b/src/Assembly.jl\n")
    assert "+_gpu_supports(backend, feature::Symbol) = false" in patch
