"""The Rust declarations written out for the reference crate name entry points
that include/cpm.h declares, with the same number of parameters."""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _c_decls() -> dict:
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "cpm.h").read_text(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(cpm_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def _rust_decls() -> dict:
    text = (ROOT / "INTEGRATION.md").read_text()
    out = {}
    for m in re.finditer(r"pub fn (cpm_[a-z0-9_]+)\(([^)]*)\)", text):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if not args else args.count(",") + 1
    return out


def test_rust_declarations_match_the_c_header():
    c, rust = _c_decls(), _rust_decls()
    assert len(rust) >= 20
    for name, nargs in rust.items():
        assert name in c, name
        assert nargs == c[name], (name, nargs, c[name])
