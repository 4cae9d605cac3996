"""The FP64 CPU oracle against the reference's own known-answer tests (CPU only)."""
import math

import numpy as np
import pytest

import oracle as O


def two_points():
    return np.array([[0.0, 0, 0], [1, 0, 0]]), np.ones(2)


def test_bb_two_point_force():
    # test/unit/physics/test_bond_based.jl:154-179
    X, V = two_points()
    p = O.point_params(O.BB, 1.5, 1.0, E=210e9)
    b = O.OracleBody(O.BB, X, V, [p], fp_point=np.zeros(2, np.uint8))
    b.pos[1, 0] = 1.0015
    b.force_density()
    E, d = 210e9, 1.5
    b12 = 18 * E / (3 * (1 - 2 * 0.25)) / (math.pi * d ** 4) * 1.0015 * 0.0015 / 1.0015 * 1.0
    assert b.b_int[0, 0] == pytest.approx(b12, rel=1e-12)
    assert b.b_int[1, 0] == pytest.approx(-b12, rel=1e-12)
    assert np.all(b.b_int[:, 1:] == 0)


def test_osb_two_point_force(golden):
    # test/unit/physics/test_ordinary_state_based.jl:3-29
    X, V = two_points()
    p = O.point_params(O.OSB, 1.5, 1.0, E=210e9, nu=0.25, Gc=1.0)
    b = O.OracleBody(O.OSB, X, V, [p], fp_point=np.zeros(2, np.uint8))
    b.pos[1, 0] = 1.0015
    b.force_density()
    assert b.b_int[0, 0] == pytest.approx(golden["osb_two_point_b12"], rel=1e-14)
    assert b.b_int[1, 0] == pytest.approx(-golden["osb_two_point_b12"], rel=1e-14)


def test_osb_interface_force(golden):
    # test/unit/physics/test_ordinary_state_based.jl:31-61 (ParameterHandler semantics)
    X, _ = two_points()
    pa = O.point_params(O.OSB, 1.5, 1.0, E=105e9, nu=0.25, Gc=1.0)
    pb = O.point_params(O.OSB, 1.5, 1.0, E=210e9, nu=0.25, Gc=1.0)
    b = O.OracleBody(O.OSB, X, np.array([1.0, 2.0]), [pa, pb], pid=[0, 1],
                     fp_point=np.zeros(2, np.uint8))
    b.pos[1, 0] = 1.0015
    b.force_density()
    assert b.b_int[0, 0] == pytest.approx(golden["osb_interface_b1"], rel=1e-14)
    assert b.b_int[1, 0] == pytest.approx(-golden["osb_interface_b2"], rel=1e-14)


def tetra_nhp():
    X = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [2, 2, 2]])
    p = O.point_params(O.CMAT, 1.5, 1.0, E=1.0, nu=0.25, Gc=1.0)
    return O.OracleBody(O.CMAT, X, np.ones(5), [p], cmodel=O.NHPENALTY,
                        fp_point=np.zeros(5, np.uint8))


def test_correspondence_nhp_regression(golden):
    # test/unit/physics/test_correspondence.jl:35-55
    b = tetra_nhp()
    b.pos[1, 0] += 0.0015
    b.force_density()
    bi = b.b_int
    assert np.all(bi[4] == 0)
    assert np.all(np.abs(bi.sum(axis=0)) < 1e-12 * np.abs(bi).max())
    assert bi[0] == pytest.approx(golden["c_nhp_b_int_1"], rel=1.5e-8)
    assert bi[1, 0] == pytest.approx(golden["c_nhp_b_int_12"], rel=1.5e-8)
    assert bi[2, 1] == pytest.approx(golden["c_nhp_b_int_23"], rel=1.5e-8)
    assert bi[1, 0] < 0 < bi[0, 0]


def test_epsilon_c(golden):
    # test/unit/physics/test_bond_based.jl:25-40
    p = O.point_params(O.BB, 2.0, 1.0, E=1.0, nu=0.25, Gc=1.0)
    assert p.epsc == pytest.approx(golden["bb_epsilon_c"], rel=1e-15)
    assert (p.G, p.K, p.lambda_, p.mu) == pytest.approx((0.4, 0.6666666666666666, 0.4, 0.4))
    with pytest.raises(ValueError):
        O.point_params(O.BB, 2.0, 1.0, E=1.0, nu=0.26, Gc=1.0)


def test_timestep_two_point():
    # test/unit/time_solvers/test_velocity_verlet.jl:40-71
    X, V = two_points()
    p = O.point_params(O.BB, 1.5, 1.0, E=1.0, Gc=1.0)
    b = O.OracleBody(O.BB, X, V, [p])
    bc = 18 * 1 / (3 * (1 - 2 * 0.25)) / (math.pi * 1.5 ** 4)
    assert b.stable_timestep(0.7) == pytest.approx(0.7 * math.sqrt(2 / bc), abs=2.3e-16)


def test_bond_lists_tetra():
    # test/unit/discretization/test_bond_system.jl:1-69
    X = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    off, nbr, L, fp = O.find_bonds(X, 2.0)
    assert off.tolist() == [0, 3, 6, 9, 12]
    assert nbr.tolist() == [1, 2, 3, 0, 2, 3, 0, 1, 3, 0, 1, 2]
    r2 = math.sqrt(2)
    assert L.tolist() == [1, 1, 1, 1, r2, r2, 1, r2, r2, 1, r2, r2]
    assert fp.all()


def test_storage_bond_count(golden):
    # test/unit/physics/test_bond_based.jl:3-23: 4x4x4 lattice with horizon 2 -> every
    # point bonds with the 63 others
    g = (np.arange(4) - 1.5) * 0.25
    X = np.array([[x, y, z] for z in g for y in g for x in g])
    off, nbr, L, fp = O.find_bonds(X, 2.0)
    assert len(nbr) == golden["bb_storage_bond_count"]
    assert np.all(np.diff(off) == 63)


def test_precrack_damage():
    # test/unit/discretization/test_predefined_cracks.jl:35-75: damage 2/3, pattern 1,0,0
    X = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    p = O.point_params(O.BB, 2.0, 1.0, E=1.0, Gc=1.0)
    b = O.OracleBody(O.BB, X, np.array([1.1, 1.2, 1.3, 1.4]), [p])
    b.break_bonds([0, 1], [2, 3])
    b.calc_damage()
    assert b.bond_active[:6].tolist() == [1, 0, 0, 1, 0, 0]
    assert b.damage[:2] == pytest.approx([2 / 3, 2 / 3])
    assert b.n_active[:2].tolist() == [1, 1]
    # filter mode (update_dmg=false): the bonds are deleted, damage stays 0
    a = np.array([1, 1, 0, 0], np.uint8)
    off, nbr, L, fp = O.find_bonds(X, 2.0, cracks=[(a, 1 - a)])
    assert off.tolist() == [0, 1, 2, 3, 4]
    assert nbr.tolist() == [1, 0, 3, 2]


def test_invariants_zero_force_and_momentum():
    # test/materials/test_force_density.jl:5-40 on the oracle
    n = 6
    dx = 1.0 / n
    g = (np.arange(n) - (n - 1) / 2) * dx
    X = np.array([[x, y, z] for z in g for y in g for x in g])
    V = np.full(len(X), dx ** 3)
    for mat in (O.BB, O.OSB, O.CMAT):
        p = O.point_params(mat, 3.015 * dx, 7850.0, E=210e9, **({} if mat == O.BB else {"nu": 0.25}), Gc=2.7)
        b = O.OracleBody(mat, X, V, [p], fp_point=np.zeros(len(X), np.uint8))
        b.force_density()
        assert np.abs(b.b_int).max() < 1e-12 * 210e9 * n
        u = 1e-4 * np.sin(np.pi * 3 * X[:, [1, 2, 0]]) + X @ np.array([[0.01, 0.003, 0], [0, -0.005, 0], [0, 0, 0]]).T
        b.pos[:] = X + u
        b.force_density()
        total = (b.b_int * V[:, None]).sum(axis=0)
        scale = (np.abs(b.b_int) * V[:, None]).sum(axis=0)
        assert np.all(np.abs(total) < 1e-10 * scale)


def test_oracle_threads_match_serial():
    # the chunked scatter of the threads backend changes only the summation order
    n = 8
    dx = 1.0 / n
    g = (np.arange(n) - (n - 1) / 2) * dx
    X = np.array([[x, y, z] for z in g for y in g for x in g])
    V = np.full(len(X), dx ** 3)
    p = O.point_params(O.OSB, 3.015 * dx, 7850.0, E=210e9, nu=0.25, Gc=2.7)
    u = 1e-3 * np.sin(np.pi * 3 * X[:, [1, 2, 0]])
    res = []
    for th in (1, 4):
        O.set_threads(th)
        b = O.OracleBody(O.OSB, X, V, [p], fp_point=np.zeros(len(X), np.uint8))
        b.pos[:] = X + u
        b.force_density()
        res.append(b.b_int.copy())
    O.set_threads(1)
    assert np.allclose(res[0], res[1], rtol=1e-12, atol=1e-9 * np.abs(res[0]).max())
