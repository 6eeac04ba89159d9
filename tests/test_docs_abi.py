"""The binding a maintainer would add stays in step with the C ABI: every
entry point declared in include/scxpca.h appears in INTEGRATION.md's Rust
`extern "C"` block, and nothing there is missing from the header."""

import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _names(text):
    return set(re.findall(r"\b(scxpca_[a-z0-9_]+)\s*\(", text))


def test_rust_block_covers_the_header():
    header = _names((ROOT / "include" / "scxpca.h").read_text())
    doc = (ROOT / "INTEGRATION.md").read_text()
    m = re.search(r'extern "C" \{(.*?)\n\}', doc, re.S)
    assert m, "INTEGRATION.md has no Rust extern block"
    rust = set(re.findall(r"pub fn (scxpca_[a-z0-9_]+)\s*\(", m.group(1)))
    assert header - rust == set(), f"declared but not bound: {sorted(header - rust)}"
    assert rust - header == set(), f"bound but not declared: {sorted(rust - header)}"
