"""Regenerate tests/golden/reference_pins.json from the reference's own tests.

The reference (rust_umap v1.1.4) cannot be built here (no Rust toolchain), so
its known-answer tests are the golden vectors.  This script reads them as
text from the reference checkout and records:
  * find_ab_params bit patterns (rust_umap/src/lib.rs:5781-5795),
  * the smooth_knn_dist self / non-self layouts (lib.rs:6975-7020),
  * the Laplacian-equality edge list (lib.rs:7457-7538),
  * the auto exact/approximate switch cases (lib.rs:5814-5840),
  * the transform thread-count determinism inputs (lib.rs:6193-6236).
Usage: python tests/golden/make_pins.py /path/to/reference
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

if len(sys.argv) != 2:
    raise SystemExit("usage: python tests/golden/make_pins.py <reference checkout>")
ref = Path(sys.argv[1])
src = (ref / "rust_umap/src/lib.rs").read_text()
lines = src.splitlines()


def block(start_pat: str, n: int = 80) -> str:
    for i, line in enumerate(lines):
        if start_pat in line:
            return "\n".join(lines[i:i + n])
    raise SystemExit(f"pattern not found: {start_pat}")


pins: dict = {"source": "rust_umap/src/lib.rs (v1.1.4 tests)"}

ab = block("fn optimized_curve_search_preserves_reference_results", 20)
cases = re.findall(
    r"\(\s*([0-9.]+)(?:_f32)?,\s*([0-9.]+)(?:_f32)?,\s*0x([0-9a-f_]+)(?:_u32)?,\s*0x([0-9a-f_]+)(?:_u32)?\s*\)",
    ab,
)
pins["find_ab_params"] = [
    {"spread": float(s), "min_dist": float(m), "a_bits": int(a.replace("_", ""), 16),
     "b_bits": int(b.replace("_", ""), 16)}
    for s, m, a, b in cases
]

sk = block("fn smooth_knn_dist_handles_rows_without_self_neighbor", 30)
sk2 = block("fn smooth_knn_dist_with_zero_rows_matches_self_and_non_self_layouts", 30)


def vecs(text: str, name: str) -> list:
    m = re.search(name + r"\s*=\s*vec!\[(.*?)\];", text, re.S)
    rows = re.findall(r"vec!\[([^\]]*)\]", m.group(1))
    return [[float(v) for v in row.split(",") if v.strip()] for row in rows]


pins["smooth_knn_cases"] = [
    {"with_self": vecs(sk, "dists_with_self"), "without_self": vecs(sk, "dists_without_self"),
     "k": 3.0, "sigma_tol": 1e-5, "rho_tol": 1e-6},
    {"with_self": vecs(sk2, "dists_with_self"), "without_self": vecs(sk2, "dists_without_self"),
     "k": 3.0, "sigma_tol": 1e-6, "rho_tol": 1e-6},
]

lap = block("fn normalized_laplacian_from_edges_matches_dense_affinity_path", 45)
edges = re.findall(r"head:\s*(\d+),\s*tail:\s*(\d+),\s*weight:\s*([0-9.]+)", lap)
pins["laplacian_edges"] = {"n": 5, "edges": [[int(h), int(t), float(w)] for h, t, w in edges],
                           "tol": 1e-12}

sw = block("fn auto_approximate_knn_delays_crossover_beyond_public_threshold", 30)
pins["ann_switch"] = [
    {"n": int(n.replace("_", "")), "d": int(d), "expect": neg == ""}
    for neg, n, d in re.findall(r"assert!\((!?)should_use_approximate_knn\(&params,\s*([0-9_]+),\s*(\d+)\)\)", sw)
]

det = block("fn transform_head_parallelism_is_thread_count_deterministic", 50)
nums = re.findall(r"optimize_layout_transform\(\s*&mut embedding,\s*&base_embedding,\s*&edges,\s*(\d+),\s*([0-9._]+),\s*([0-9._]+),\s*([0-9._]+),\s*(\d+),\s*([0-9._]+),\s*(\d+)", det)
e, a, b, alpha, neg, rep, seed = nums[0]
pins["transform_determinism"] = {
    "n_heads": 64, "n_tail": 128, "edges_per_head": 12, "n_epochs": int(e),
    "a": float(a.replace("_", "")), "b": float(b.replace("_", "")), "alpha": float(alpha),
    "neg_rate": int(neg), "repulsion": float(rep), "seed": int(seed),
}

out = Path(__file__).resolve().parent / "reference_pins.json"
out.write_text(json.dumps(pins, indent=1) + "\n")
print(out)
