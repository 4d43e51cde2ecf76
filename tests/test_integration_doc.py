"""The Julia ccall stubs in INTEGRATION.md against include/h2g.h (no Julia here): every stub names
a declared function and passes as many argument types as the declaration has parameters."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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


def _stubs():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    for m in re.finditer(r"ccall\(\((:|fn)(\w*)\s*,\s*libh2g\)\s*,\s*\w+\s*,\s*", text):
        types = _balanced(text, m.end())
        n = 0 if not types.strip() else len([t for t in types.split(",") if t.strip()])
        yield (m.group(2) if m.group(1) == ":" else None), n


def test_ccall_stubs_match_the_header():
    arity = _header_arity()
    stubs = list(_stubs())
    assert len(stubs) >= 10
    for name, n in stubs:
        if name is None:  # the stub that picks h2g_PBiCGSTAB or h2g_CG at run time
            assert n == arity["h2g_PBiCGSTAB"] == arity["h2g_CG"]
            continue
        assert name in arity, name
        assert n == arity[name], (name, n, arity[name])
