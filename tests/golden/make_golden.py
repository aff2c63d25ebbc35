"""Regenerate the golden fixtures under tests/golden/ from the reference tree.

Reads the reference's own recorded test data (read-only, this container only):
  tests/fileread/runs/mld_mat.mtx  (4096x4096 2D 5-point Laplacian, 20224 nnz)
  tests/fileread/runs/mld_rhs.mtx  (right-hand side)
  tests/fileread/runs/mld_sol.mtx  (reference solution; ||A sol - rhs||/||rhs|| ~ 1.4e-10)
and stores them as a compressed CSR npz, so that the tests do not need the
reference tree at run time.

Usage:  python tests/golden/make_golden.py /path/to/reference
"""
import os
import sys

import numpy as np
import scipy.io
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    runs = os.path.join(ref_root, "tests", "fileread", "runs")
    a = sp.csr_matrix(scipy.io.mmread(os.path.join(runs, "mld_mat.mtx"), spmatrix=True))
    a.sum_duplicates()
    a.sort_indices()
    rhs = np.asarray(scipy.io.mmread(os.path.join(runs, "mld_rhs.mtx"))).ravel()
    sol = np.asarray(scipy.io.mmread(os.path.join(runs, "mld_sol.mtx"))).ravel()
    out = os.path.join(HERE, "fileread_fixture.npz")
    np.savez_compressed(out, irp=a.indptr.astype(np.int32), ja=a.indices.astype(np.int32),
                        val=a.data.astype(np.float64), rhs=rhs, sol=sol)
    r = np.linalg.norm(a @ sol - rhs) / np.linalg.norm(rhs)
    print(f"wrote {out}: n={a.shape[0]} nnz={a.nnz} relres(sol)={r:.3e}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/reference")
    main(sys.argv[1])
