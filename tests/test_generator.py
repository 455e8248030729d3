"""Seeded scene generator: determinism, the biaxial sample's confinement geometry and a short
oracle run that stays bounded."""
import numpy as np

from conftest import input_checksum


def small_biaxial(seed=5):
    from melody2d_b200 import generator as g
    return g.biaxial_scene(seed=seed, n_discs=12, n_border=32, n_interior=80, workers=1)


def test_biaxial_is_deterministic():
    from melody2d_b200 import generator as g
    a, b = g.flatten(small_biaxial()), g.flatten(small_biaxial())
    assert input_checksum(a) == input_checksum(b)
    assert input_checksum(a) != input_checksum(g.flatten(small_biaxial(seed=6)))


def test_biaxial_walls_close_the_sample():
    """Walls span the plates' full height and the plates the walls' travel, so no grain can leave
    through a corner; plate/wall pairs use a zero-stiffness law."""
    sc = small_biaxial()
    W, H = sc.meta["box"]
    bot, top, left, right = sc.bodies[-4:]
    for wall in (left, right):
        assert wall.nodes[:, 1].min() <= bot.nodes[:, 1].min() + 1e-12
        assert wall.nodes[:, 1].max() >= top.nodes[:, 1].max() - 1e-12
    for plate in (bot, top):
        assert plate.nodes[:, 0].min() < 0 and plate.nodes[:, 0].max() > W
    names = [m[0] for m in sc.materials]
    assert ("Steel", "Steel") in [(l[0], l[1]) for l in sc.laws]
    steel = [l for l in sc.laws if l[0] == l[1] == "Steel"][0]
    assert steel[2] == 0 and steel[4][0] == 0.0
    rho_steel = sc.materials[names.index("Steel")][2][0]
    assert rho_steel == 7800.0 * sc.meta["mass_factor"]


def test_biaxial_oracle_run_stays_bounded(oracle_built):
    from melody2d_b200 import generator as g
    from oracle.pyoracle import Oracle
    sc = small_biaxial()
    flat = g.flatten(sc)
    o = Oracle(flat)
    o.step(400)
    st = o.node_state()
    assert np.isfinite(st).all()
    W, H = sc.meta["box"]
    assert np.abs(st[:, 0:2]).max() < 0.05 * W        # displacements stay small over 400 steps
    assert (o.contacts()["fx"] != 0).sum() > 0


def _shm_blocks():
    import os
    return {f for f in os.listdir("/dev/shm") if f.startswith("psm_")} if os.path.isdir("/dev/shm") else set()


def test_shared_sample_pipeline_matches_direct_generation():
    """Samples built by spawn workers and handed over through shared memory are the arrays the
    generator gives in this process; kept samples stay readable until released, the others are
    released after their creation, and no block is left behind."""
    from melody2d_b200 import generator as g
    seeds = [11, 12, 13]
    before = _shm_blocks()
    created, kept, meta = g.build_batch_samples(seeds, input_checksum, workers=2, create_threads=2, keep=[1])
    templates = g.DiscTemplates(list(range(32, 97)), workers=1)
    for i, s in enumerate(seeds):
        sc = g.batch_sample_scene(s, templates)
        assert created[i] == input_checksum(g.flatten(sc))
        assert meta[i][1] == sc.dt
    assert set(kept) == {1}
    assert input_checksum(kept[1].flat) == created[1]
    kept[1].release()
    assert _shm_blocks() <= before


def test_share_flat_round_trip():
    from melody2d_b200 import generator as g
    flat = {"a": np.arange(10000, dtype=np.float64), "b": np.arange(7, dtype=np.int32), "c": 2.5}
    sf = g.SharedFlat(g.share_flat(flat))
    np.testing.assert_array_equal(sf.flat["a"], flat["a"])
    np.testing.assert_array_equal(sf.flat["b"], flat["b"])
    assert sf.flat["c"] == 2.5 and sf.nbytes == sum(np.asarray(v).nbytes for v in flat.values())
    sf.release()
