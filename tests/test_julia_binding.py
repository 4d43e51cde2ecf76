"""The Julia binding (julia/H2GPU.jl, julia/H2GPURules.jl) and the patch that adds par="gpu" to the
reference (julia/par_gpu.patch), checked without Julia: every ccall names a function declared in
include/h2g.h and passes as many argument types as the declaration has parameters, every exported
entry of the header that the drop-in needs has a stub, and the patch's hunks only add lines, with
hunk headers consistent with their contents."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = [os.path.join(ROOT, "julia", f) for f in ("H2GPU.jl", "H2GPURules.jl")]


def _header_arity():
    text = open(os.path.join(ROOT, "include", "h2g.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(h2g_\w+)\s*\(([^)]*)\)\s*;", text):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else len(params.split(","))
    return out


def _balanced(text, i):
    """The text of the parenthesised group that starts at text[i] == '('."""
    depth = 0
    for j in range(i, len(text)):
        depth += {"(": 1, ")": -1}.get(text[j], 0)
        if depth == 0:
            return text[i + 1:j]
    raise ValueError("unbalanced")


def _stubs(text):
    for m in re.finditer(r"ccall\(\(:(\w+)\s*,\s*libh2g\)\s*,\s*\w+\s*,\s*", text):
        types = _balanced(text, m.end())
        n = 0 if not types.strip() else len([t for t in types.split(",") if t.strip()])
        yield m.group(1), n


def test_ccall_stubs_match_the_header():
    arity = _header_arity()
    stubs = [st for f in JL for st in _stubs(open(f).read())]
    assert len(stubs) >= 15
    for name, n in stubs:
        assert name in arity, name
        assert n == arity[name], (name, n, arity[name])
    names = {n for n, _ in stubs}
    for needed in ("h2g_PBiCGSTAB", "h2g_CG", "h2g_SolveSOR", "h2g_create", "h2g_destroy", "h2g_set_grid",
                   "h2g_set_fields", "h2g_pbicgstab", "h2g_transient", "h2g_calrhs", "h2g_adjoint",
                   "h2g_calcrk_noalloc", "h2g_last_error"):
        assert needed in names, needed


def test_rrule_uses_the_binding():
    text = open(JL[1]).read()
    assert "function ChainRulesCore.rrule(::typeof(hotspot_norm)" in text
    assert "adjoint_gradient" in text and "using ..H2GPU" in text


def test_patch_only_adds_lines():
    lines = open(os.path.join(ROOT, "julia", "par_gpu.patch")).read().splitlines()
    start = next(i for i, l in enumerate(lines) if l.startswith("--- a/"))
    files, shift, hunks = [], 0, 0
    i = start
    while i < len(lines):
        l = lines[i]
        if l.startswith("--- a/"):
            assert lines[i + 1] == "+++ b/" + l[6:]
            files.append(l[6:])
            shift = 0
            i += 2
            continue
        m = re.match(r"@@ -(\d+),0 \+(\d+)(?:,(\d+))? @@$", l)
        assert m, l
        old, new, count = int(m.group(1)), int(m.group(2)), int(m.group(3) or 1)
        assert new == old + 1 + shift  # added after line `old`, shifted by the earlier hunks
        body = lines[i + 1:i + 1 + count]
        assert len(body) == count and all(b.startswith("+") for b in body)
        shift += count
        hunks += 1
        i += 1 + count
    assert files == ["src/heat3ds.jl", "src/NonUniform.jl"] and hunks == 4
    text = "\n".join(lines)
    assert "Main.H2GPU.PBiCGSTAB!" in text and "Main.H2GPU.CG!" in text and 'par=="gpu"' in text
