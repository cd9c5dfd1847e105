"""The brick pool (sparse brick path) on the host: the behaviour the reference's
own topology test checks (FluxFX_Source/native/bricks_test.cpp): idempotent
activation, neighbours both ways, LIFO slot reuse, coordinate limits, 20,000
randomized operations against a dictionary model with constant metadata, pool
exhaustion, and atomic box activation."""
import random

import pytest

from fluxfx_b200 import _native as N
from fluxfx_b200.backend.sparse import BrickPool, seed_faces, solve_mask


def test_activation_neighbors_and_slot_reuse():
    t = BrickPool(64)
    center = t.activate((0, 0, 0))
    assert center == t.activate((0, 0, 0))
    east = t.activate((1, 0, 0))
    assert t.neighbors((0, 0, 0))[1] == east and t.neighbors((1, 0, 0))[0] == center
    assert t.deactivate((1, 0, 0)) and t.neighbors((0, 0, 0))[1] == -1
    assert t.activate((-1, 0, 0)) == east          # the removed slot is handed out next
    corner = (1048575, -1048576, 0)
    t.activate(corner)
    assert t.neighbors(corner)[1] == -1
    with pytest.raises(N.FfxError, match='coordinates'):
        t.activate((1048576, 0, 0))
    t.close()


def test_randomized_operations_match_a_dictionary():
    t = BrickPool(64)
    meta = t.stats()['metadata_bytes']
    model = {}
    rng = random.Random(78)
    for _ in range(20000):
        c = (rng.randrange(8) - 4, rng.randrange(8) - 4, rng.randrange(8) - 4)
        if rng.random() < 0.5:
            if len(model) < 64 or c in model:
                model[c] = t.activate(c)
            else:
                with pytest.raises(N.FfxError, match='exhausted'):
                    t.activate(c)
        else:
            assert t.deactivate(c) == (model.pop(c, None) is not None)
        st = t.stats()
        assert st['active'] == len(model) and st['metadata_bytes'] == meta
    for c, slot in model.items():
        assert t.lookup(c) == slot
        x, y, z = c
        adjacent = [(x - 1, y, z), (x + 1, y, z), (x, y - 1, z), (x, y + 1, z), (x, y, z - 1), (x, y, z + 1)]
        assert t.neighbors(c) == [model.get(a, -1) for a in adjacent]
    slots, coords = t.active()
    assert sorted(slots) == sorted(model.values())
    assert {tuple(coords[s]) for s in slots} == set(model)
    t.close()


def test_box_activation_is_atomic():
    box = BrickPool(8)
    box.activate_box((0, 0, 0), (2, 2, 2))
    assert box.stats()['active'] == 8
    with pytest.raises(N.FfxError, match='exhausted'):
        box.activate_box((1, 0, 0), (2, 2, 2))
    assert box.stats()['active'] == 8 and box.lookup((2, 0, 0)) == -1
    with pytest.raises(N.FfxError, match='exceeds pool capacity'):
        BrickPool(4).activate_box((0, 0, 0), (3, 1, 2))
    with pytest.raises(N.FfxError, match='capacity'):
        BrickPool(0)
    box.close()


def test_seeded_velocity_lives_beside_the_solve_region():
    n = 32
    for mode in (0, 1, 2):
        solve = solve_mask(n, mode)
        faces = seed_faces(n, mode)
        for a, f in enumerate(faces):
            shape = [n, n, n]
            shape[2 - a] += 1
            assert f.shape == tuple(shape)
            walls = [slice(None)] * 3
            walls[2 - a] = 0
            assert not f[tuple(walls)].any()
        assert solve.sum() > 0 and any(f.any() for f in faces)
    # mode 1: faces of axis 0 lie in the rows of the central box, and x from n/4 to 3n/4
    u = seed_faces(n, 1)[0]
    lo, hi = n // 4, 3 * n // 4
    assert not u[:lo].any() and not u[hi:].any() and not u[:, :lo].any() and not u[:, hi:].any()
    assert not u[:, :, :lo].any() and not u[:, :, hi + 1:].any() and u[lo:hi, lo:hi, lo:hi + 1].any()


def test_arena_alignment_budget_reuse_and_handles():
    """The reference's arena test (FluxFX_Source/native/arena_test.cpp) restated."""
    from fluxfx_b200.backend.sparse import Arena
    a = Arena(1024)
    x, y, z = a.allocate(1), a.allocate(257), a.allocate(256)
    assert a.stats()['used'] == 1024 and a.get(y)[:2] == (256, 512)
    with pytest.raises(N.FfxError, match='exhausted'):
        a.allocate(1)
    a.release(y)
    fresh = a.allocate(500)
    assert fresh != y and a.get(fresh)[0] == 256
    with pytest.raises(N.FfxError, match='unknown'):
        a.get(y)
    for h in (x, z, fresh):
        a.release(h)
    st = a.stats()
    assert st['used'] == 0 and st['largest_free'] == 1024 and st['peak'] == 1024
    other = Arena(1024)
    foreign = other.allocate(1)
    with pytest.raises(N.FfxError, match='foreign'):
        a.release(foreign)
    with pytest.raises(N.FfxError, match='multiple of 256'):
        Arena(1000)
    rng = random.Random(110)
    stress = Arena(65536)
    ids = []
    for _ in range(3000):
        if ids and rng.random() < 0.5:
            stress.release(ids.pop(rng.randrange(len(ids))))
        else:
            try:
                ids.append(stress.allocate(1 + rng.randrange(2048)))
            except N.FfxError:
                pass
        spans = sorted(stress.get(h)[:2] for h in ids)
        assert all(o % 256 == 0 and o + b <= 65536 for o, b in spans)
        assert all(o1 + b1 <= o2 for (o1, b1), (o2, _) in zip(spans, spans[1:]))
        assert sum(b for _, b in spans) == stress.stats()['used']
    for h in ids:
        stress.release(h)
    assert stress.stats()['largest_free'] == 65536
