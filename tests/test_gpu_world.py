"""World periodic-boundary interface through the Python surface, restating the
semantics of the reference's test/test_PBC_interface.py: construction and
set_pbc with valid and invalid (repetitions, mastergrid) pairs, the mastergrid
derived from the bounding grid of the magnets when set_pbc gets none, magnets
outside the mastergrid, the mastergrid / pbc_repetitions setters and unset_pbc.
Error types follow the reference (ValueError or TypeError for bad values,
IndexError for grids that do not fit).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CS = (1.0, 1.0, 1.0)


def _valid(mpx):
    G = mpx.Grid
    return [((0, 0, 0), G((0, 0, 0))),
            ((3, 0, 0), G((64, 0, 0), (2, 1, 0))),
            ((0, 1, 0), G((0, 48, 0), (0, 3, 5))),
            ((0, 0, 2), G((0, 0, 16), (4, 0, 1))),
            ((1, 2, 3), G((32, 16, 8), (0, 2, 0)))]


def _invalid(mpx):
    G = mpx.Grid
    return [((-2, 0, 0), G((16, 0, 0))),       # negative repetitions
            ((0, 0, -1), G((0, 0, 4))),
            ((1.5, 0, 0), G((8, 1, 1))),       # not integers
            ((1, 1), G((2, 2, 2))),            # two dimensions
            ((0, 0, 0), G((0, 12, 0))),        # periodic size without repetitions
            ((2, 0, 0), G((0, 0, 0))),         # repetitions without a periodic size
            ((1, 0, 2), G((0, 0, 32)))]


def test_world_pbc_construction_and_set_pbc(mpx):
    world = mpx.World(CS)
    assert tuple(world.pbc_repetitions) == (0, 0, 0) and world.mastergrid == mpx.Grid((0, 0, 0))
    for rep, mg in _valid(mpx):
        w = mpx.World(CS, rep, mg)
        assert tuple(w.pbc_repetitions) == rep and w.mastergrid == mg
        w = mpx.World(CS)
        w.set_pbc(rep, mg)
        assert tuple(w.pbc_repetitions) == rep and w.mastergrid == mg
    for rep, mg in _invalid(mpx):
        with pytest.raises((ValueError, TypeError)):
            mpx.World(CS, rep, mg)
        with pytest.raises((ValueError, TypeError)):
            mpx.World(CS).set_pbc(rep, mg)


def _bounds(grids):
    lo = np.min([g.origin for g in grids], axis=0)
    hi = np.max([np.add(g.origin, g.size) for g in grids], axis=0)
    return lo, hi


@pytest.mark.parametrize("rep", [(1, 1, 2), (0, 2, 1), (3, 0, 0), (0, 0, 0)])
def test_set_pbc_derives_mastergrid_from_magnets(mpx, rep):
    G = mpx.Grid
    grids = [G((6, 3, 1), (-2, 0, 0)), G((2, 5, 2), (4, 9, 3))]
    world = mpx.World(CS)
    for g in grids:
        mpx.Ferromagnet(world, g)
    lo, hi = _bounds(grids)
    assert world.bounding_grid == G(tuple(int(v) for v in hi - lo), tuple(int(v) for v in lo))
    world.set_pbc(rep)
    size = tuple(int(hi[i] - lo[i]) if rep[i] else 0 for i in range(3))
    assert tuple(world.pbc_repetitions) == rep
    assert world.mastergrid == G(size, tuple(int(v) for v in lo))


def test_pbc_errors_for_grids_that_do_not_fit(mpx):
    G = mpx.Grid
    with pytest.raises(IndexError):  # no magnets: no bounding grid to derive a mastergrid from
        mpx.World(CS).set_pbc((2, 1, 1))
    with pytest.raises(IndexError):
        mpx.World(CS).bounding_grid
    world = mpx.World(CS, pbc_repetitions=(1, 1, 1), mastergrid=G((4, 4, 2)))
    for origin in [(-1, 0, 0), (0, 3, 0), (0, 0, 2)]:
        with pytest.raises(IndexError):
            mpx.Ferromagnet(world, G((2, 2, 1), origin))
    mpx.Ferromagnet(world, G((4, 4, 2)))
    with pytest.raises(IndexError):
        world.set_pbc((1, 1, 1), G((2, 2, 2)))
    with pytest.raises(IndexError):
        world.mastergrid = G((2, 4, 2))


def test_mastergrid_and_repetition_setters(mpx):
    G = mpx.Grid
    world = mpx.World(CS, pbc_repetitions=(0, 2, 1), mastergrid=G((0, 8, 4)))
    world.mastergrid = G((0, 2, 3))
    assert world.mastergrid == G((0, 2, 3))
    with pytest.raises(ValueError):  # periodic along x without repetitions along x
        world.mastergrid = G((3, 0, 3))
    world = mpx.World(CS, pbc_repetitions=(2, 1, 3), mastergrid=G((6, 5, 4)))
    world.pbc_repetitions = (1, 3, 2)
    assert tuple(world.pbc_repetitions) == (1, 3, 2)
    for bad in [(0, 1, 1), (1, 1, 0), (-1, 1, 1), (1, 2.5, 1)]:
        with pytest.raises((ValueError, TypeError)):
            world.pbc_repetitions = bad
    world = mpx.World(CS, pbc_repetitions=(1, 1, 2), mastergrid=G((40, 20, 10), (-3, 5, 2)))
    world.unset_pbc()
    assert tuple(world.pbc_repetitions) == (0, 0, 0) and world.mastergrid == G((0, 0, 0))
