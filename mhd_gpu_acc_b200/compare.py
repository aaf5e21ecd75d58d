"""Compare the field CSVs of two run directories (the role of the reference's
scripts/compare_runs.py, same pass rule and exit codes).

    python -m mhd_gpu_acc_b200.compare DIR_A DIR_B [--tol 1e-10] [--rtol 1e-6]
                                       [--fields rho,p] [--verbose]

Files are paired by their path relative to each directory.  Per pair: maximum
and mean absolute difference, maximum relative difference |a-b| / max(|a|,|b|)
(0 where both are 0), RMS difference, plus the relative L1 sum|a-b| / sum|b|.
A pair passes when max_abs <= tol or max_rel <= rtol.
Exit status: 0 all pairs pass, 1 some pair fails, 2 usage / IO error (no
common files, unreadable file, shape mismatch).
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np


def load(path: str) -> np.ndarray:
    return np.loadtxt(path, delimiter=",", dtype=np.float64, ndmin=2)


def csv_files(root: str) -> dict[str, str]:
    out = {}
    for d, _, files in os.walk(root):
        for f in files:
            if f.endswith(".csv"):
                p = os.path.join(d, f)
                out[os.path.relpath(p, root)] = p
    return out


def field_of(rel: str) -> str:
    return os.path.splitext(os.path.basename(rel))[0].rsplit("_", 1)[-1]


def stats(a: np.ndarray, b: np.ndarray) -> dict:
    d = np.abs(a - b)
    m = np.maximum(np.abs(a), np.abs(b))
    rel = np.divide(d, m, out=np.zeros_like(d), where=m > 0)
    den = np.abs(b).sum()
    return {"max_abs": float(d.max()), "mean_abs": float(d.mean()), "max_rel": float(rel.max()),
            "rms": float(np.sqrt((d * d).mean())), "rel_l1": float(d.sum() / den) if den > 0 else float(d.sum())}


def compare(dir_a: str, dir_b: str, tol: float = 1e-10, rtol: float = 1e-6, fields=None, verbose=False,
            out=sys.stdout) -> int:
    fa, fb = csv_files(dir_a), csv_files(dir_b)
    common = sorted(set(fa) & set(fb))
    if fields:
        common = [r for r in common if field_of(r) in fields]
    if not common:
        print("no common CSV files", file=out)
        return 2
    worst = 0
    for rel in common:
        try:
            a, b = load(fa[rel]), load(fb[rel])
        except (OSError, ValueError) as e:
            print(f"{rel}: cannot read: {e}", file=out)
            return 2
        if a.shape != b.shape:
            print(f"{rel}: shape {a.shape} vs {b.shape}", file=out)
            return 2
        s = stats(a, b)
        ok = s["max_abs"] <= tol or s["max_rel"] <= rtol
        worst = max(worst, 0 if ok else 1)
        if verbose or not ok:
            print(f"{'PASS' if ok else 'FAIL'} {rel}: max_abs {s['max_abs']:.3e} mean_abs {s['mean_abs']:.3e} "
                  f"max_rel {s['max_rel']:.3e} rms {s['rms']:.3e} rel_l1 {s['rel_l1']:.3e}", file=out)
    only = sorted(set(fa) ^ set(fb))
    if only and verbose:
        print(f"{len(only)} files present on one side only", file=out)
    print(f"{len(common)} pairs compared: {'PASS' if worst == 0 else 'FAIL'}", file=out)
    return worst


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("dir_a")
    ap.add_argument("dir_b")
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--rtol", type=float, default=1e-6)
    ap.add_argument("--fields", default=None, help="comma-separated field names")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    for d in (a.dir_a, a.dir_b):
        if not os.path.isdir(d):
            print(f"not a directory: {d}")
            return 2
    return compare(a.dir_a, a.dir_b, a.tol, a.rtol, a.fields.split(",") if a.fields else None, a.verbose)


if __name__ == "__main__":
    sys.exit(main())
