"""Regenerate tests/golden/*.json from the reference's own test fixtures.

Reads the Rust test source of ArcInstitute/scx (the CSR fixture
``test_csr_10x5`` and the small QR/SVD matrices of scx-accel/src/pca/cpu.rs
tests) as text and writes them, with exact dense FP64 PCA answers computed by
numpy, to ``reference_fixtures.json``.  Run in a container that has the
reference checkout:

    python tests/golden/make_golden.py /path/to/scx

The committed JSON is what the tests read; nothing at test time touches the
reference tree.
"""

from __future__ import annotations

import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _vec(text: str) -> list[float]:
    return [float(t) for t in re.findall(r"-?\d+(?:\.\d+)?", text)]


def extract(cpu_rs: str) -> dict:
    m = re.search(r"fn test_csr_10x5\(\) -> ScxCsr \{(.*?)\n    \}", cpu_rs, re.S)
    if not m:
        raise SystemExit("test_csr_10x5 not found")
    body = m.group(1)
    vecs = re.findall(r"vec!\[(.*?)\]", body, re.S)
    shape = tuple(int(x) for x in re.search(r"\((\d+),\s*(\d+)\)", body).groups())
    indptr, indices, data = (_vec(v) for v in vecs[:3])
    out = {"csr_10x5": {"source": "scx-accel/src/pca/cpu.rs:2326-2339 (test_csr_10x5)",
                        "shape": list(shape), "indptr": [int(x) for x in indptr],
                        "indices": [int(x) for x in indices], "data": data}}
    m = re.search(r"fn test_qr_orthonormal\(\) \{\s*let data = vec!\[(.*?)\];", cpu_rs, re.S)
    out["qr_4x2"] = {"source": "scx-accel/src/pca/cpu.rs:2447-2461 (test_qr_orthonormal)",
                     "rows": 4, "cols": 2, "data": _vec(m.group(1))}
    m = re.search(r"fn test_svd_basic\(\) \{\s*let data = vec!\[(.*?)\];", cpu_rs, re.S)
    out["svd_3x2"] = {"source": "scx-accel/src/pca/cpu.rs:2463-2479 (test_svd_basic)",
                      "rows": 3, "cols": 2, "data": _vec(m.group(1))}
    m = re.search(r"fn test_qr_and_svd_on_row_major_slice\(\) \{.*?let data = vec!\[(.*?)\];",
                  cpu_rs, re.S)
    out["rowmajor_4x3"] = {"source": "scx-accel/src/pca/cpu.rs:2481-2514 "
                                     "(test_qr_and_svd_on_row_major_slice)",
                           "rows": 4, "cols": 3, "data": _vec(m.group(1))}
    return out


def exact_answers(fx: dict) -> dict:
    c = fx["csr_10x5"]
    n, g = c["shape"]
    dense = np.zeros((n, g))
    for r in range(n):
        for p in range(c["indptr"][r], c["indptr"][r + 1]):
            dense[r, c["indices"][p]] += c["data"][p]
    ans = {}
    for center in (True, False):
        x = dense - dense.mean(axis=0) if center else dense
        s = np.linalg.svd(x, compute_uv=False)
        ans["centered" if center else "uncentered"] = {
            "singular_values": s.tolist(),
            "variance_explained": (s ** 2 / (n - 1)).tolist(),
            "total_var": float(np.sum(x * x) / (n - 1)),
        }
    return ans


def main(ref_root: str) -> None:
    cpu_rs = (Path(ref_root) / "scx-accel/src/pca/cpu.rs").read_text()
    fx = extract(cpu_rs)
    fx["csr_10x5"]["exact"] = exact_answers(fx)
    (HERE / "reference_fixtures.json").write_text(json.dumps(fx, indent=1))
    print("wrote", HERE / "reference_fixtures.json")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
