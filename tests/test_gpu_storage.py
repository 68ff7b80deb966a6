"""On-disk cache of the built intermediates (nw_save_intermediates / nw_load_intermediates; the
counterpart of the reference's wicks.bin / wicks.meta cache, src/nonorthogonalwicks/storage.rs):
a context that loads the cache evaluates every pair bit-identically to the context that built
it (H, S, the zero-overlap counts and, after nw_update_fock, F + S), on a system with both pair
layouts (m = 0 and m > 0 reference pairs); a cache of another system, a corrupted or truncated
metadata file and a missing file are rejected."""
import numpy as np
import pytest

import nociwick
from nociwick import lib as L
from nociwick import synthetic as sy

pytestmark = pytest.mark.gpu


def _system(seed=5):
    return sy.make_system(12, 3, 3, 3, 24, seed=seed, k_scale=0.3, zero_pairs=[(0, 1, 1, 0)], enuc=0.2)


def _engine(system):
    return nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8)


def test_cache_round_trip_is_bit_identical(tmp_path):
    system = _system()
    basis = sy.sd_basis(12, 3, 3, 3, orders=(1, 2, 3))
    pairs = sy.sample_pairs(basis, 50000, seed=4, distinct_parents=False)
    rng = np.random.default_rng(1)
    fa = rng.standard_normal((12, 12))
    fa = fa + fa.T
    fb = fa + 0.1 * np.eye(12)
    slab, meta = tmp_path / "wicks.bin", tmp_path / "wicks.meta"
    with _engine(system).build() as w:
        w.set_basis(basis)
        hs = w.eval_pairs(pairs)
        m = w.zero_counts()
        w.update_fock(fa, fb)
        fs = w.eval_fs_pairs(pairs)
        w.save(slab, meta)
    assert m.sum() > 0 and (m == 0).any()    # both layouts are in the cache
    with _engine(system).load(slab, meta) as w:
        w.set_basis(basis)
        assert np.array_equal(w.zero_counts(), m)
        assert np.array_equal(w.eval_pairs(pairs), hs)
        w.update_fock(fa, fb)
        assert np.array_equal(w.eval_fs_pairs(pairs), fs)


def test_cache_rejects_other_system_and_damaged_files(tmp_path):
    system = _system()
    slab, meta = tmp_path / "wicks.bin", tmp_path / "wicks.meta"
    with _engine(system).build() as w:
        w.save(slab, meta)
    other = _system(seed=6)                               # same geometry, other integrals
    with _engine(other) as w:
        with pytest.raises(L.NwError) as e:
            w.load(slab, meta)
        assert e.value.status == 1
    raw = bytearray(meta.read_bytes())
    bad = tmp_path / "bad.meta"
    raw[200] ^= 0xFF                                      # one flipped byte: the metadata hash fails
    bad.write_bytes(bytes(raw))
    short = tmp_path / "short.meta"
    short.write_bytes(meta.read_bytes()[:100])
    with _engine(system) as w:
        for m in (bad, short):
            with pytest.raises(L.NwError) as e:
                w.load(slab, m)
            assert e.value.status == 1
        with pytest.raises(L.NwError) as e:
            w.load(tmp_path / "missing.bin", meta)
        assert e.value.status == 7
        w.load(slab, meta)                                # the intact cache still loads
