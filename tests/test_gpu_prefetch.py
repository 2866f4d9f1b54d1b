"""asohf_prefetch_particles: an upload of the prefetched host arrays takes
the staged copy, and the store (and what is computed from it) is the same as
after a plain upload; an upload of other arrays ignores the staged copy."""
import numpy as np
import pytest
import torch

from asohf_b200 import api, grid, synth

pytestmark = pytest.mark.gpu


def _pinned(s):
    return [torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
            for a in (s.x, s.y, s.z, s.vx, s.vy, s.vz, s.m, s.id)]


def _store(a):
    return [np.asarray(v).copy() for v in a.download_particles()]


def test_prefetched_upload_equals_plain(gpu_lib):
    s1, s2 = synth.generate("tiny"), synth.generate("small")
    h1, h2 = _pinned(s1), _pinned(s2)
    cfg = s1.cfg
    radx, dx = grid.malla(cfg.nx, np.float32(cfg.lado0))
    cos = grid.cosmology(cfg.h, cfg.omega_m, cfg.zeta)
    ref = api.Asohf(0)
    ref.upload_particles(*h1)
    want = _store(ref)
    want_npe = ref.sort_dm_particles_localdensity(cfg.nx, dx, cos["rodo"], cos["re0"])
    want_sorted = _store(ref)

    a = api.Asohf(0)
    a.upload_particles(*h2)          # a store to be replaced
    a.prefetch_particles(*h1)        # staged beside it
    a.upload_particles(*h1)          # takes the staged copy
    assert all(np.array_equal(x, y) for x, y in zip(_store(a), want))
    npe = a.sort_dm_particles_localdensity(cfg.nx, dx, cos["rodo"], cos["re0"])
    assert np.array_equal(np.asarray(npe), np.asarray(want_npe))
    assert all(np.array_equal(x, y) for x, y in zip(_store(a), want_sorted))
    # back to back: the arrays handed back become the next staging store
    for _ in range(3):
        a.prefetch_particles(*h1)
        a.upload_particles(*h1)
        assert all(np.array_equal(x, y) for x, y in zip(_store(a), want))


def test_other_arrays_ignore_the_staged_copy(gpu_lib):
    """An upload of other arrays copies them and leaves the staged copy for
    its own upload.  The staging store handed over can have another capacity
    than the set the sorts permute into: a later, larger plain upload must
    still find both sets large enough (the species sort permutes the whole
    store)."""
    s1, s2 = synth.generate("tiny"), synth.generate("small")
    h1, h2 = _pinned(s1), _pinned(s2)
    cfg = s2.cfg
    radx, dx = grid.malla(cfg.nx, np.float32(cfg.lado0))
    cos = grid.cosmology(cfg.h, cfg.omega_m, cfg.zeta)
    ref1, ref2 = api.Asohf(0), api.Asohf(0)
    ref1.upload_particles(*h1)
    ref2.upload_particles(*h2)
    want1, want2 = _store(ref1), _store(ref2)
    want_npe = ref2.sort_dm_particles_localdensity(cfg.nx, dx, cos["rodo"], cos["re0"])
    want_sorted = _store(ref2)

    a = api.Asohf(0)
    a.upload_particles(*h1)          # store sets sized for the small snapshot
    a.prefetch_particles(*h2)        # a larger staging store
    a.upload_particles(*h1)          # not the prefetched arrays: a plain copy
    assert all(np.array_equal(x, y) for x, y in zip(_store(a), want1))
    a.prefetch_particles(*h1)        # replaces the staged copy, same staging store
    a.upload_particles(*h1)          # takes it: the store now has the larger capacity
    assert all(np.array_equal(x, y) for x, y in zip(_store(a), want1))
    a.upload_particles(*h2)          # plain, larger than the other set
    assert all(np.array_equal(x, y) for x, y in zip(_store(a), want2))
    npe = a.sort_dm_particles_localdensity(cfg.nx, dx, cos["rodo"], cos["re0"])
    assert np.array_equal(np.asarray(npe), np.asarray(want_npe))
    assert all(np.array_equal(x, y) for x, y in zip(_store(a), want_sorted))
