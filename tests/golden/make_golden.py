"""Generates the golden fixtures under tests/golden/ from the reference project.

Run in a container where the reference tree is mounted (it reads it, never writes it):

    python tests/golden/make_golden.py <root of the reference project>

Outputs (committed; the tests read only these files, never the reference tree):

  known_answers.json   the worked examples of the reference API documents, parsed from
                       the fenced code blocks of each example section:
                       docs/zh/sgetrf.md, sgetrs.md, sgetri.md, spotrs.md,
                       spotrf_batched.md, smatinv_batched.md, cpotrf_batched.md
  basic_lu_cases.json  the deterministic matrices of the reference's native LU test
                       (test/sgetrf/real_lu_test_impl.h:62-118, FillInput/PrepareMatrix),
                       restated here with the INFO each case must produce (:149)
  solve_lu.npz         seeded LU factors (LAPACK sgetrf), right-hand sides and the solution
                       the reference's own numpy solver computes
                       (test/utils/lu_verify_utils.py:172-192, solve_lu), for trans 0 and 1
  complex_lu.npz       the reference's complex LU data recipes with LAPACK's pivots, the
                       solutions of its numpy LU solver (trans 0, 1, 2) and numpy inverses
  cholesky_cpu_ratios.npz  seeded SPD matrices (the reference runner's recipe,
                       test/cholesky/runner.py:265-272) with the FP32-LAPACK residual
                       ratios of the reference judge (test/cholesky/lapack_residual.py:64-86)
"""

import json
import re
import sys
from pathlib import Path

import numpy as np
from scipy.linalg import lapack

OUT = Path(__file__).resolve().parent
NUMBER = re.compile(r"(?<![A-Za-z_\d.])-?\d+(?:\.\d+)?(?:[eE]-?\d+)?")


def example_blocks(doc):
    """Numbers of each fenced block inside the document's example section."""
    lines = Path(doc).read_text(encoding="utf-8").splitlines()
    start = next(i for i, line in enumerate(lines) if "示例" in line and line.strip().startswith("-"))
    blocks, current, inside = [], [], False
    for line in lines[start + 1 :]:
        if line.startswith("## "):
            break
        if line.strip().startswith("```"):
            if inside:
                blocks.append([float(x) for x in NUMBER.findall(" ".join(current))])
                current = []
            inside = not inside
            continue
        if inside:
            current.append(line)
    return blocks


def known_answers(ref):
    docs = Path(ref) / "docs" / "zh"
    out = {}
    b = example_blocks(docs / "sgetrf.md")
    out["sgetrf_4x4"] = {"a": b[0], "lu": b[1], "ipiv": [int(v) for v in b[2]], "source": "docs/zh/sgetrf.md"}
    b = example_blocks(docs / "sgetrs.md")
    out["sgetrs_4x4"] = {
        "lu": b[0],
        "ipiv": [int(v) for v in b[1]],
        "b": b[2],
        "x": b[3],
        "source": "docs/zh/sgetrs.md",
    }
    b = example_blocks(docs / "sgetri.md")
    out["sgetri_4x4"] = {"a": b[0], "lu": b[1], "inverse": b[2], "ipiv": [1, 2, 3, 4], "source": "docs/zh/sgetri.md"}
    b = example_blocks(docs / "spotrs.md")
    out["spotrs_4x4"] = {"a": b[0], "l": b[1], "b": b[2], "x": b[3], "source": "docs/zh/spotrs.md"}
    b = example_blocks(docs / "spotrf_batched.md")
    out["spotrf_batched_4x4"] = {"a": [b[0], b[1]], "l": [b[2], b[3]], "source": "docs/zh/spotrf_batched.md"}
    b = example_blocks(docs / "smatinv_batched.md")
    # Two 2x2 matrices printed side by side, row by row: [a00 a01 | b00 b01; a10 a11 | b10 b11].
    side = lambda v: ([v[0], v[1], v[4], v[5]], [v[2], v[3], v[6], v[7]])
    out["smatinv_2x2"] = {"a": list(side(b[0])), "inverse": list(side(b[1])), "source": "docs/zh/smatinv_batched.md"}
    b = example_blocks(docs / "cpotrf_batched.md")
    out["cpotrf_batched_4x4"] = {
        "a": [b[0], b[1]],
        "l": [b[2], b[3]],
        "layout": "row-major (re, im) pairs",
        "source": "docs/zh/cpotrf_batched.md",
    }
    b = example_blocks(docs / "cgetrs.md")
    out["cgetrs_4x4"] = {
        "lu": b[0],
        "ipiv": [int(v) for v in b[1]],
        "b": b[2],
        "x": b[3],
        "layout": "row-major (re, im) pairs",
        "source": "docs/zh/cgetrs.md",
    }
    return out


def basic_lu_cases():
    """FillInput/PrepareMatrix of real_lu_test_impl.h for the factor mode (row-major data)."""
    cases = []
    for m, n, batch, pivot, singular in [(7, 5, 1, True, False), (3, 3, 1, False, False), (2, 2, 1, True, False),
                                         (3, 3, 1, True, True), (32, 32, 8, True, False)]:
        mats = []
        for b in range(batch):
            bad = singular and b == 0
            a = np.zeros((m, n), dtype=np.float32)
            for r in range(m):
                for c in range(n):
                    if r == c:
                        a[r, c] = 0.0 if (bad and r == 1) else float(n + r + b + 2)
                    elif bad:
                        a[r, c] = 0.0
                    else:
                        a[r, c] = 0.25
            if pivot and m > 1 and not bad:
                a[[0, 1], :] = a[[1, 0], :]
            mats.append(a.tolist())
        cases.append({"m": m, "n": n, "pivot": pivot, "a": mats,
                      "info": [2 if (singular and b == 0) else 0 for b in range(batch)]})
    return cases


def solve_lu_vectors(ref):
    sys.path.insert(0, str(Path(ref) / "test" / "utils"))
    from lu_verify_utils import solve_lu  # the reference's own numpy solver

    rng = np.random.default_rng(20261203)
    out = {}
    for n, nrhs in [(8, 1), (33, 3), (64, 1), (64, 4)]:
        a = rng.normal(size=(n, n)).astype(np.float32)
        lu, piv, info = lapack.sgetrf(a)
        assert info == 0
        b = rng.normal(size=(n, nrhs)).astype(np.float32)
        for trans in (0, 1):
            x = solve_lu(lu.astype(np.float64), b.astype(np.float64), piv.astype(np.int64), trans)
            key = f"n{n}_r{nrhs}_t{trans}"
            out[key + "_lu"] = lu.astype(np.float32)
            out[key + "_ipiv"] = (piv + 1).astype(np.int32)
            out[key + "_b"] = b
            out[key + "_x"] = np.asarray(x, dtype=np.float64)
    return out


def complex_lu_vectors(ref):
    """The reference's complex LU data recipes (test/cgetrf/data/gen_data.py: integer parts
    1..10; test/cgetrs/data/gen_data.py: a dominant shuffled diagonal, seed 149;
    test/cgetri_batched/data/gen_data.py: N(0,1) parts with a raised diagonal, seed 42) with
    LAPACK's complex64 pivots and the solutions of the reference's own numpy LU solver
    (test/utils/lu_verify_utils.py:174-191, solve_lu, trans 0 / 1 / 2)."""
    sys.path.insert(0, str(Path(ref) / "test" / "utils"))
    from lu_verify_utils import solve_lu  # the reference's own numpy solver

    out = {}
    for m, n in [(32, 32), (48, 64), (64, 48), (128, 128)]:
        rng = np.random.RandomState(149)
        a = rng.randint(1, 11, size=(m, n * 2)).astype(np.float32).view(np.complex64)
        lu, piv, info = lapack.cgetrf(a)
        assert info == 0
        out[f"getrf_m{m}_n{n}_a"] = a
        out[f"getrf_m{m}_n{n}_lapack_ipiv"] = (piv + 1).astype(np.int32)
    for n, nrhs in [(4, 1), (32, 32), (65, 3)]:
        rng = np.random.RandomState(149)
        a = (rng.randint(1, 11, size=(n, n)) + 1j * rng.randint(1, 11, size=(n, n))).astype(np.complex64)
        for i in range(n):
            row = np.sum(np.abs(a[i, :])) - np.abs(a[i, i])
            a[i, i] = row + rng.rand() * 10 + 1j * rng.rand() * 10
        rng.shuffle(a)
        b = (rng.randn(n, nrhs) + 1j * rng.randn(n, nrhs)).astype(np.complex64)
        lu, piv, info = lapack.cgetrf(a)
        assert info == 0
        key = f"getrs_n{n}_r{nrhs}"
        out[key + "_lu"] = lu.astype(np.complex64)
        out[key + "_ipiv"] = (piv + 1).astype(np.int32)
        out[key + "_b"] = b
        for trans in (0, 1, 2):
            x = solve_lu(lu.astype(np.complex128), b.astype(np.complex128), piv.astype(np.int64), trans)
            out[f"{key}_x{trans}"] = np.asarray(x, dtype=np.complex128)
    for n, count in [(48, 2), (3, 2), (32, 4)]:
        np.random.seed(42)
        a = np.random.randn(count, n, n).astype(np.float32) + 1j * np.random.randn(count, n, n).astype(np.float32)
        for q in range(count):
            for i in range(n):
                row = np.sum(np.abs(a[q, i, :])) - np.abs(a[q, i, i])
                a[q, i, i] = (row + np.random.rand() * 10) * (1 + 1j)
        a = a.astype(np.complex64)
        out[f"inverse_n{n}_a"] = a
        out[f"inverse_n{n}_golden"] = np.stack([np.linalg.inv(a[q]).astype(np.complex64) for q in range(count)])
    return out


def cholesky_ratios(ref):
    sys.path.insert(0, str(Path(ref) / "test" / "cholesky"))
    from lapack_residual import paired  # the reference judge

    out = {}
    for n in (1, 8, 9, 17, 32, 33, 64, 65):
        rng = np.random.default_rng(950 + n)
        r = rng.normal(size=(5, n, n)) / np.sqrt(n)
        a = (r @ r.transpose(0, 2, 1) + np.eye(n) * 2).astype(np.float32)
        b = rng.normal(size=(5, n, 1)).astype(np.float32)
        ratios = []
        for q in range(5):
            f, _ = lapack.spotrf(np.array(a[q], order="F"), lower=True)
            ratios.append(
                [paired("spotrf", a[q], np.tril(f), False)["ratio_cpu"],
                 paired("spotrs", a[q], lapack.spotrs(f, np.array(b[q], order="F"), lower=True)[0], False,
                        b[q])["ratio_cpu"]])
        out[f"n{n}_a"] = a
        out[f"n{n}_b"] = b
        out[f"n{n}_ratio_cpu"] = np.array(ratios)
    return out


def main(ref):
    (OUT / "known_answers.json").write_text(json.dumps(known_answers(ref), indent=1))
    (OUT / "basic_lu_cases.json").write_text(json.dumps(basic_lu_cases()))
    np.savez_compressed(OUT / "solve_lu.npz", **solve_lu_vectors(ref))
    np.savez_compressed(OUT / "cholesky_cpu_ratios.npz", **cholesky_ratios(ref))
    np.savez_compressed(OUT / "complex_lu.npz", **complex_lu_vectors(ref))
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <root of the reference project>")
    main(sys.argv[1])
