"""The Rust declarations for the reference crate's `cuda` feature (include/cpm_ffi.rs) name entry
points that include/cpm.h declares, with the same number of parameters."""
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
    text = re.sub(r"//[^\n]*", "", (ROOT / "include" / "cpm_ffi.rs").read_text())
    out = {}
    for m in re.finditer(r"pub fn (cpm_[a-z0-9_]+)\(([^)]*)\)", text):
        args = m.group(2).strip().rstrip(",")
        out[m.group(1)] = 0 if not args else args.count(",") + 1
    return out


def test_rust_declarations_match_the_c_header():
    c, rust = _c_decls(), _rust_decls()
    assert len(rust) >= 20
    for name, nargs in rust.items():
        assert name in c, name
        assert nargs == c[name], (name, nargs, c[name])


def test_rust_file_declares_every_reference_facing_entry_point():
    rust = _rust_decls()
    for name in ("cpm_mesh_deposit", "cpm_mesh_interpolate3", "cpm_fft3", "cpm_poisson_accel", "cpm_tree_accel",
                 "cpm_sim_create", "cpm_sim_step_host", "cpm_sim_get_state", "cpm_sim_destroy"):
        assert name in rust, name
