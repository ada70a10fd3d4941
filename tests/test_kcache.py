"""On-disk K cache (no GPU: the column builder is the oracle's C restatement,
standing in for the GPU build): resume after an interrupted build, reload
without solving, and separate entries for different keys."""
import os
import sys
import types

import numpy as np
import pytest

from conftest import ROOT, load_package

sys.path.insert(0, ROOT)


def _kcache():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "eqd_kcache", os.path.join(ROOT, "earthquakediffinitive.jl_b200", "kcache.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.fixture(scope="module")
def small():
    from oracle.fault import FaultElasticity as OracleFE, cube_grids
    from oracle.cref import CRefStiffness
    eqd = load_package()
    gm, gp = cube_grids(11)
    ofe = OracleFE(gm, gp, 2.0, 1.0, l_f=0.4)
    ref = CRefStiffness(ofe)
    K = ref.columns(np.arange(2 * ofe.nf), rtol=1e-12, nthreads=1)[0]
    fe = types.SimpleNamespace(grids=eqd.cube_grids(11), lam=2.0, mu=1.0, l_f=0.4, nf=ofe.nf,
                               rs=types.SimpleNamespace(rtol=1e-12))
    return fe, ref, K


def test_resume_and_reload(tmp_path, small):
    kc = _kcache()
    fe, ref, K_ref = small
    calls = []

    def build(cols):
        calls.append((int(cols[0]), int(cols[-1]) + 1))
        if len(calls) == 3:
            raise KeyboardInterrupt  # the build stops part way
        return ref.columns(cols, rtol=1e-12, nthreads=1)[0]

    with pytest.raises(KeyboardInterrupt):
        kc.cached_fault_stiffness(fe, str(tmp_path), block=16, build=build)
    entry = kc.KCache(str(tmp_path), kc.cache_key(fe), fe.nf, 16)
    assert len(entry.done) == 2 and not entry.complete()
    calls.clear()
    K = kc.cached_fault_stiffness(fe, str(tmp_path), block=16, build=build)
    assert calls == [(32, 48), (48, 50)]              # only the missing blocks
    assert np.array_equal(K, K_ref)
    calls.clear()
    K2 = kc.cached_fault_stiffness(fe, str(tmp_path), block=16, build=build)
    assert calls == [] and np.array_equal(K2, K_ref)   # loaded, nothing solved


def test_keys_separate_entries(tmp_path, small):
    kc = _kcache()
    fe, ref, _ = small
    other = types.SimpleNamespace(**{**fe.__dict__, "mu": 1.5})
    assert kc.key_digest(kc.cache_key(fe)) != kc.key_digest(kc.cache_key(other))
    a = kc.KCache(str(tmp_path), kc.cache_key(fe), fe.nf)
    b = kc.KCache(str(tmp_path), kc.cache_key(other), fe.nf)
    assert a.dir != b.dir
    with pytest.raises(ValueError):
        a.put((0, 16), np.zeros((2 * fe.nf, 15)))      # wrong block shape
