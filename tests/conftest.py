"""Shared fixtures: the product package (loaded by path: its directory name,
mld2p4-2_b200, is not an identifier) and the C test oracle."""
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def load_package():
    name = "mld2p4_2_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = os.path.join(ROOT, "mld2p4-2_b200")
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def mld():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


S3 = 1.0 / np.sqrt(3.0)
# -Lap u + (1/sqrt3)(u_x+u_y+u_z): coefficients a1,a2,a3,b1,b2,b3,c
ISO = (1.0, 1.0, 1.0, S3, S3, S3, 0.0)
ANISO = (1.0, 1.0, 0.01, S3, S3, S3, 0.0)


def oracle_params(orc, smoother="BJAC", sweeps=1, damp=1.0, coarse_sweeps=4, mcs=2000):
    sm = {"BJAC": orc.BJAC, "JACOBI": orc.JACOBI, "FBGS": orc.FBGS}[smoother]
    return orc.default_params(smoother=sm, sweeps_pre=sweeps, sweeps_post=sweeps,
                              jac_damp=damp, coarse_solver=orc.BJAC,
                              coarse_sweeps=coarse_sweeps, min_coarse_size=mcs)


def upload_oracle_hierarchy(mld, orc, oprec, use_graphs=True, precision=0, autotune=True):
    """Upload the oracle's (reference-algorithm) hierarchy through the C ABI."""
    h = mld.Hierarchy(use_graphs=use_graphs, autotune=autotune)
    for l in range(oprec.nlev):
        info = oprec.level_info(l)
        def conv(m):
            return None if m is None else mld.CSR(m.irp, m.ja, m.val, ncols=m.ncols)
        kind = info["smoother"]
        tri = kind in (orc.BJAC, orc.FBGS)
        d = oprec.level_vec(l, "d") if tri else oprec.level_vec(l, "dinv")
        h.upload_level(
            l, conv(oprec.level_csr(l, "A")),
            P=conv(oprec.level_csr(l, "P")) if l else None,
            R=conv(oprec.level_csr(l, "R")) if l else None,
            ND=conv(oprec.level_csr(l, "ND")) if info["nnzND"] else None,
            L=conv(oprec.level_csr(l, "L")) if tri else None,
            U=conv(oprec.level_csr(l, "U")) if tri else None,
            d=d, smoother=kind, sweeps_pre=info["sweeps_pre"], sweeps_post=info["sweeps_pre"],
            damping=info["damp"])
    h.finalize(oprec.nlev, precision)
    return h
