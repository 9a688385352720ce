"""Shared fixtures.  The package directory `crystallographicfft.jl_b200/` is not a
valid Python identifier, so it is registered as `crystallographicfft_b200` here;
the native library is built in-tree first when it is missing."""
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "crystallographicfft.jl_b200")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_package():
    name = "crystallographicfft_b200"
    if name in sys.modules:
        return sys.modules[name]
    lib = os.path.join(PKG_DIR, "libcfft_b200.so")
    if not os.path.exists(lib):
        spec_b = importlib.util.spec_from_file_location("cfft_build", os.path.join(PKG_DIR, "build.py"))
        mod_b = importlib.util.module_from_spec(spec_b)
        spec_b.loader.exec_module(mod_b)
        mod_b.build()
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def cf():
    return load_package()


@pytest.fixture(scope="session")
def O():
    from oracle import krfft_oracle

    return krfft_oracle


def to_oracle_ops(O, ops):
    return [O.SymOp(op.R, op.t) for op in ops]


def oracle_group(cf, O, sg, N):
    """Operations of group `sg` from the oracle's own Hall-symbol table, shifted by the
    oracle's find_optimal_shift.  Returns (ops, ops_s) in the library's SymOp form (what
    a caller hands the plan) and the oracle's shifted ops, so the field, the truth and
    the plan all rest on operations that the library under test did not produce."""
    dim = len(N)
    oops = O.get_ops(sg, dim, N)
    _, oops_s = O.find_optimal_shift(oops, N)
    lib = lambda ops: [cf.SymOp(op.R, op.t) for op in ops]
    return lib(oops), lib(oops_s), oops_s


@pytest.fixture(scope="session")
def prep(cf, O):
    """Per-group fixtures like test/runtests.jl:111-127: shifted ops, spectral ASU,
    seeded symmetric field (numpy generator)."""
    cache = {}

    def get(sg, N, seed=42):
        key = (sg, tuple(N), seed)
        if key not in cache:
            dim = len(N)
            ops, ops_s, oops = oracle_group(cf, O, sg, N)
            spec = cf.calc_spectral_asu(ops_s, dim, N)
            u = O.make_symmetric(oops, N, seed=seed)
            cache[key] = dict(ops=ops, ops_s=ops_s, spec=spec, oops=oops, u=u)
        return cache[key]

    return get


def oracle_shifted_ops(cf, sg, N):
    """The library-form shifted operations of oracle_group (oracle imported here)."""
    from oracle import krfft_oracle as O

    return oracle_group(cf, O, sg, N)[1]


def q_plan(cf, p, path, ds, lattice, **kw):
    """An M2Q / M7 plan (plan_m2_q / plan_m7_scft, src/q_fused_krfft.jl:83,822) on the
    prep fixture's (oracle) operations, so its Q tables compare with the oracle's."""
    return cf.KRFFTPlan(p["spec"], p["ops_s"], N=p["spec"].N, ds=ds, lattice=lattice, path=path, **kw)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
