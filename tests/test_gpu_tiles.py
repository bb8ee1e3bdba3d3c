"""Stencil tile autotuner: every tile shape of the flow-flux sweeps and every k-chunk of the
marching viscous kernels gives bit-identical states (a tile decides which block computes a point,
not how), and the tuner's timed choice is one of the candidates and leaves the solution unchanged."""
import numpy as np
import pytest

from ocfd_b200 import abi, cases, solver

pytestmark = pytest.mark.gpu

CHOICES = [
    [0, 0, 0, 16, 16, 0, 0, 0, 0],  # everything on one stream
    [1, 1, 1, 8, 32, 0, 0, 0, 1],
    [2, 2, 2, 64, 8, 1, 0, 1, 3],  # both side streams
    [1, 2, 0, 3, 5, 0, 1, 0, 2],  # k chunks that do not divide nz; species chain on a third stream
    [0, 1, 2, 16, 0, 1, 1, 1, 1],  # per-cell k_visc_div, stored metric arrays everywhere
]


def _case(kind):
    if kind == "flatplate":
        return cases.flatplate(nx=40, ny=24, nz=12, scheme="HYBRID", lx=0.01, ly=0.004, y1=2e-5)
    if kind == "isotropic":
        return cases.isotropic(n=16, scheme="WENO7", flux_splitting=abi.SPLIT_LLF)
    return cases.jet(nx=24, ny=16, nz=16)


def _run(c, choice=None, tune=False, steps=2):
    g = solver.Solver(c)
    g.init_state()
    tuned = None
    if choice is not None:
        g.set_tiles(choice)
        expect = list(choice) if solver.lib().ocfd_gpu_is_separable() else choice[:5] + [1, 1, 1] + choice[8:]
        assert g.tiles() == expect
    if tune:
        tuned = g.autotune(reps=2)
    for s in range(steps):
        g.tt = s * c.dt
        g.step(c.dt, c.if_reaction, c.nsub)
    st = g.download_state()
    g.close()
    return st, tuned


@pytest.mark.parametrize("kind", ["flatplate", "isotropic", "jet"])
def test_tile_choices_are_bit_identical(kind):
    c = _case(kind)
    ref, _ = _run(c)
    for choice in CHOICES[1:]:
        st, _ = _run(c, choice)
        for a, b in zip(ref, st):
            assert np.array_equal(a, b), (kind, choice)


def test_autotune_choice_and_solution():
    c = _case("flatplate")
    ref, _ = _run(c)
    st, (choice, ms) = _run(c, tune=True)
    assert choice[0] in (0, 1, 2) and choice[1] in (0, 1, 2) and choice[2] in (0, 1, 2)
    assert choice[3] in (8, 16, 32, 64) and choice[4] in (0, 8, 16, 32, 64)
    assert all(x in (0, 1) for x in choice[5:]) and len(choice) == 9
    assert all(t > 0 for t in ms[:25]), ms  # viscous separable case: every candidate timed
    assert ms[25:27] == [-1.0, -1.0]  # one species: no species chain to place
    for d in range(3):
        assert ms[3 * d + choice[d]] == min(ms[3 * d:3 * d + 3])
    for a, b in zip(ref, st):
        assert np.array_equal(a, b)


def test_autotune_places_the_species_chain():
    """the reacting jet: the tuner times a stage's right-hand sides with the species chain in order
    and on the third stream, keeps the faster, and leaves the solution as it was"""
    c = _case("jet")
    ref, _ = _run(c)
    st, (choice, ms) = _run(c, tune=True)
    assert choice[8] in (0, 1, 2, 3)
    assert ms[25] > 0 and ms[26] > 0
    assert bool(choice[8] & 2) == (ms[26] < ms[25])
    for a, b in zip(ref, st):
        assert np.array_equal(a, b)


def test_autotune_remembers_the_configuration():
    c = _case("isotropic")
    g = solver.Solver(c)
    g.init_state()
    first, _ = g.autotune(reps=2)
    g.set_tiles([0, 0, 0, 16, 16, 0, 0, 0, 1])
    again, ms = g.autotune(reps=0)  # cached: applied without timing
    assert again == first and all(t == -1.0 for t in ms)
    assert g.tiles() == first
    g.close()


def test_bad_tile_choice_is_rejected():
    c = _case("isotropic")
    g = solver.Solver(c)
    g.init_state()
    for bad in ([3, 0, 0, 16, 16], [0, -1, 0, 16, 16], [0, 0, 0, 0, 16], [0, 0, 0, 16, -1], [0, 0, 0, 16, 16, 2],
                [0, 0, 0, 16, 16, 0, 0, 0, 4], [0, 0, 0, 16, 16, 0, 0, 0, -1]):
        with pytest.raises(solver.OcfdError):
            g.set_tiles(bad)
    g.close()
