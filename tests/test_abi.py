"""CPU: the C-ABI library loads, exports every declared entry point, and
rejects bad calls on the host side without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mld[gp]_[a-z0-9_]+)\s*\(", txt)))


@pytest.mark.parametrize("header", ["mldg.h", "mld_prec.h", "mldg_test.h"])
def test_library_exports_every_declared_symbol(mld, header):
    lib = mld.lib()
    names = _declared(header)
    assert len(names) >= (1 if header == "mldg_test.h" else 8)
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/{header} but not exported"


def test_null_handle_errors(mld):
    lib = mld.lib()
    assert lib.mldg_upload_level(None, 0, None) == 30
    assert lib.mldg_finalize(None, 1, 0) == 30
    assert lib.mldg_apply(None, None, None, b"N", 1, 0, 0) == 30
    assert lib.mldg_last_error(None) == b"null handle"
    lib.mldg_destroy(None)  # no-op


def test_host_mirror_set_and_build_errors(mld):
    p = mld.MldPrec()
    with pytest.raises(mld.MldError) as e:
        p.set("SMOOTHER_TYPE", "BJAC")          # set before init
    assert e.value.code == 3111
    p.init("ML")
    with pytest.raises(mld.MldError):
        p.set("NO_SUCH_KEY", 1)
    a = mld.gen_pde3d(6, 1)
    # the reference's ML default (FBGS smoother, ILU coarse solve) builds
    p.hierarchy_build(a)
    assert p.nlev >= 1
    # a smoother without a GPU apply is refused with the keyword named
    p.set("SMOOTHER_TYPE", "AS")
    with pytest.raises(mld.MldError) as e:
        p.hierarchy_build(a)
    assert "SMOOTHER_TYPE" in str(e.value)
    p.init("ML")
    p.set("SMOOTHER_TYPE", "BJAC")
    p.set("ML_CYCLE", "NO_SUCH_CYCLE")
    with pytest.raises(mld.MldError) as e:
        p.hierarchy_build(a)
    assert "ML_CYCLE" in str(e.value)
    with pytest.raises(mld.MldError) as e:
        p.apply(np.zeros(a.nrows))
    assert e.value.code == mld.ERR_NOT_BUILT


def test_host_mirror_descr_and_levels(mld):
    p = mld.MldPrec()
    p.init("ML")
    p.set("SMOOTHER_TYPE", "JACOBI")
    p.set("SMOOTHER_SWEEPS", 2)
    p.set("SMOOTHER_DAMPING", 0.8)
    p.set("MIN_COARSE_SIZE", 100)
    p.hierarchy_build(mld.gen_pde3d(12, 1))
    assert p.nlev >= 2
    info = p.level_info(1)
    assert info["n"] == info["naggr"] and info["nnzP"] == info["nnzR"]


def test_kappa_generator_is_symmetric_and_matches_constant_case(mld):
    idim = 6
    k = np.ones(idim ** 3)
    a = mld.gen_kappa3d(idim, k)
    b = mld.gen_pde3d(idim, 1, (1, 1, 1, 0, 0, 0, 0))
    assert np.array_equal(a.irp, b.irp) and np.array_equal(a.ja, b.ja)
    assert np.allclose(a.val, b.val, rtol=1e-14)
    rng = np.random.default_rng(0)
    a2 = mld.gen_kappa3d(idim, np.exp(rng.normal(size=idim ** 3)))
    import scipy.sparse as sp
    m = sp.csr_matrix((a2.val, a2.ja, a2.irp))
    assert abs(m - m.T).max() <= 1e-9 * abs(m).max()


def test_krylov_batch_rejects_mismatched_lists(mld):
    # checked on the host before any handle is touched
    with pytest.raises(ValueError):
        mld.krylov_batch("FCG", [object(), object()], [np.ones(4)])
    with pytest.raises(ValueError):
        mld.krylov_batch("FCG", [object()], [np.ones(4)], [np.ones(4), np.ones(4)])


def test_header_compiles_as_c99_and_links(mld, tmp_path):
    """include/mldg.h as a C caller sees it: a C99 program that includes the
    header, links libmldgpu.so and checks the host-side error paths (null
    handle, error text), with no GPU."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    mld.lib()  # built
    src = tmp_path / "abi_c99.c"
    src.write_text(r'''
#include <stdio.h>
#include <string.h>
#include "mldg.h"
int main(void) {
  mldg_level_desc d;
  memset(&d, 0, sizeof d);
  if (mldg_upload_level(NULL, 0, &d) != MLDG_ERR_ARG) return 1;
  if (mldg_finalize(NULL, 1, MLDG_PREC_FP64) != MLDG_ERR_ARG) return 2;
  if (mldg_apply(NULL, NULL, NULL, 'N', 1, 0, MLDG_MEM_HOST) != MLDG_ERR_ARG) return 3;
  if (mldg_krylov(NULL, 1, NULL, NULL, NULL, 1e-10, 10, NULL, NULL, MLDG_MEM_HOST) != MLDG_ERR_ARG) return 4;
  if (strcmp(mldg_last_error(NULL), "null handle") != 0) return 5;
  mldg_destroy(NULL);
  puts("c99 ok");
  return 0;
}
''')
    exe = tmp_path / "abi_c99"
    libdir = os.path.join(ROOT, "mld2p4-2_b200")
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I",
                        os.path.join(ROOT, "include"), str(src), "-o", str(exe), "-L", libdir,
                        "-lmldgpu", f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "c99 ok" in r.stdout, (r.returncode, r.stdout, r.stderr)


def test_fortran_constants_match_header():
    """Every named constant of the Fortran binding (mldg_cbind.f90) has the
    value the C header defines, and every MLDG_PREC_ / MLDG_SMOOTHER_ /
    MLDG_ERR_ constant of the header is bound."""
    h = open(os.path.join(ROOT, "include", "mldg.h")).read()
    defs = {k: int(v) for k, v in re.findall(r"#define\s+(MLDG_[A-Z0-9_]+)\s+(-?\d+)\b", h)}
    f = open(os.path.join(ROOT, "mld2p4-2_b200", "fortran", "mldg_cbind.f90")).read()
    params = {k: int(v) for k, v in re.findall(r"parameter\s*::\s*(MLDG_[A-Z0-9_]+)\s*=\s*(-?\d+)", f)}
    assert params, "no constants found in mldg_cbind.f90"
    for k, v in params.items():
        assert k in defs and defs[k] == v, (k, v, defs.get(k))
    for k in defs:
        if k.startswith(("MLDG_PREC_", "MLDG_SMOOTHER_", "MLDG_ERR_")):
            assert k in params, f"{k} not bound in mldg_cbind.f90"
