"""GPU edge cases of the plain WCSPH step against the oracle, bit for bit.

The reference step (crates/pe-fluid/src/wcsph.rs:326-347) has no special
cases for them, so neither does the oracle: a world without particles, a
world of boundary samples only
(no fluid moves, every density is the boundary's own), a single fluid
particle without neighbours in free fall inside the wall shell, and a
neighbour-cell union larger than the list build's shared-memory stage (the
build's slow path, flagged by STATUS_SLOW_UNION; also through the PBF and
DFSPH steps, whose list modes keep every candidate or every boundary
candidate). A particle that leaves the
dense grid domain makes the step return PE_ERR_BOUNDS with STATUS_DOMAIN set
(the reference's sparse grid has no domain); a non-positive dt is PE_ERR_ARG.
"""
import numpy as np
import pytest

import oracle as O
import physics_engine_rs as pe
from helpers import assert_bits_equal

pytestmark = pytest.mark.gpu

RHO0, DX = 1000.0, 0.02
PE_ERR_BOUNDS, PE_ERR_ARG = 2, 3


def _params():
    prm = pe.WcsphParams.water(RHO0, 20.0, (0.0, 0.0, -9.81))
    prm.adapt_sound_speed = False
    op = O.water_params(RHO0, 20.0, (0.0, 0.0, -9.81), materialize=False)
    op.adapt_sound_speed = 0
    return prm, op


def _scenes(h, build):
    mass = pe.mass_from_spacing(RHO0, DX, 3)
    ps = pe.Particles(3, RHO0, mass, h)
    os_ = O.Scene(3, RHO0, mass, h)
    for s in (ps, os_):
        build(s)
    return ps, os_


def _compare(w, o, what):
    assert_bits_equal(w.positions(), o.x(), f"{what} x")
    assert_bits_equal(w.velocities(), o.v(), f"{what} v")
    assert_bits_equal(w.densities(), o.rho(), f"{what} rho")
    assert_bits_equal(w.pressures(), o.p(), f"{what} p")
    assert_bits_equal(w.boundary_forces(), o.boundary_force(), f"{what} boundary force")
    assert w.t == o.t


def test_boundary_only_world_is_static_and_bit_exact():
    ps, os_ = _scenes(2 * DX, lambda s: s.fill_box_boundary((0.0, 0.0, 0.0), (0.3, 0.2, 0.2), DX, 1))
    prm, op = _params()
    w = pe.WcsphWorld(ps, prm)
    o = O.World(os_, op)
    x0 = w.positions().copy()
    for _ in range(5):
        w.step(1e-4)
        o.step(1e-4)
    _compare(w, o, "boundary only")
    assert_bits_equal(w.positions(), x0, "boundary samples do not move")
    assert w.status() == 0
    w.close()


def test_single_fluid_particle_free_fall_bit_exact():
    def build(s):
        s.push_fluid((0.15, 0.1, 0.3), (0.1, -0.05, 0.0))
        s.fill_box_boundary((0.0, 0.0, 0.0), (0.3, 0.2, 0.4), DX, 1)

    ps, os_ = _scenes(2 * DX, build)
    prm, op = _params()
    w = pe.WcsphWorld(ps, prm)
    o = O.World(os_, op)
    for _ in range(40):
        w.step(1e-3)
        o.step(1e-3)
    _compare(w, o, "single particle")
    x, v = w.positions(), w.velocities()
    i = int(np.argmax(np.abs(v[:, 2])))  # the one fluid particle is the only mover
    assert v[i, 2] < 0.0 and x[i, 2] < 0.3
    w.close()


def test_union_beyond_the_stage_takes_the_slow_path_bit_exact():
    # 22^3 boundary samples 0.002 m apart with h = 0.02: the block sits in
    # 2 x 2 x 2 cells of 0.04 m, so a cell's 27-cell union (10,648 + the fluid)
    # exceeds the 5,888-entry shared-memory stage. Eight fluid particles sit
    # inside it, so the slow path's lists (built per particle from global
    # memory, the lower ones by repeated selection) stay short.
    h, s = 0.02, 0.002
    g = (0.1 + s * np.arange(22)).tolist()

    def build(sc):
        for x in g:
            for y in g:
                for z in g:
                    sc.push_boundary((x, y, z), s ** 3)
        for k in range(8):
            sc.push_fluid((0.111 + 0.004 * (k & 1), 0.113 + 0.004 * ((k >> 1) & 1), 0.117 + 0.004 * (k >> 2)))

    mass = pe.mass_from_spacing(RHO0, s, 3)
    ps = pe.Particles(3, RHO0, mass, h)
    os_ = O.Scene(3, RHO0, mass, h)
    build(ps)
    build(os_)
    prm, op = _params()
    w = pe.WcsphWorld(ps, prm)
    o = O.World(os_, op)
    w.step(1e-6)
    o.step(1e-6)
    _compare(w, o, "slow path")
    assert w.status() & pe.STATUS_SLOW_UNION
    assert w.status() & ~pe.STATUS_SLOW_UNION == 0
    w.close()


def test_leaving_the_grid_domain_is_an_error():
    def build(s):
        s.push_fluid((0.15, 0.1, 0.1), (0.0, 0.0, 0.0))
        s.push_fluid((0.15, 0.1, 0.16), (2000.0, 0.0, 0.0))
        s.fill_box_boundary((0.0, 0.0, 0.0), (0.3, 0.2, 0.2), DX, 1)

    ps, _ = _scenes(2 * DX, build)
    prm, _ = _params()
    w = pe.WcsphWorld(ps, prm)
    with pytest.raises(pe.PeError) as e:
        w.step(-1e-4)
    assert e.value.code == PE_ERR_ARG
    with pytest.raises(pe.PeError) as e:
        w.step(1e-3)  # 2 m in one step: far past the domain's margin
    assert e.value.code == PE_ERR_BOUNDS
    assert w.status() & pe.STATUS_DOMAIN
    w.close()


def test_empty_world_steps():
    ps, os_ = _scenes(2 * DX, lambda s: None)
    prm, op = _params()
    w = pe.WcsphWorld(ps, prm)
    o = O.World(os_, op)
    w.step(1e-4)
    w.run(1e-4, 7)
    o.step(1e-4)
    o.run(1e-4, 7)
    assert w.t == o.t
    assert w.positions().shape == (0, 3) and w.densities().shape == (0,)
    assert w.status() == 0
    w.close()


def _dense_block(sc, s):
    """22^3 boundary samples s apart around eight fluid particles."""
    g = (0.1 + s * np.arange(22)).tolist()
    for x in g:
        for y in g:
            for z in g:
                sc.push_boundary((x, y, z), s ** 3)
    for k in range(8):
        sc.push_fluid((0.111 + 0.004 * (k & 1), 0.113 + 0.004 * ((k >> 1) & 1), 0.117 + 0.004 * (k >> 2)))


def test_pbf_slow_path_bit_exact():
    """PBF's lists (every candidate kept during the iterations) through the
    slow path: poly6 support h = 0.02 m, so the block spans ~3^3 cells."""
    h, s = 0.02, 0.002
    mass = pe.mass_from_spacing(RHO0, s, 3)
    ps, os_ = pe.Particles(3, RHO0, mass, h), O.Scene(3, RHO0, mass, h)
    _dense_block(ps, s)
    _dense_block(os_, s)
    p = pe.PbfParams(iterations=2, art_pressure_k=0.0)
    q = O.pbf_default_params()
    for k in pe.PbfParams._FIELDS:
        v = getattr(p, k)
        if k == "gravity":
            q.gravity[:] = v
        else:
            setattr(q, k, int(v) if isinstance(v, bool) else v)
    w, o = pe.PbfWorld(ps, p), O.PbfWorld(os_, q)
    w.step(1e-6)
    o.step(1e-6)
    assert_bits_equal(w.positions(), o.x(), "pbf slow path x")
    assert_bits_equal(w.velocities(), o.v(), "pbf slow path v")
    assert_bits_equal(w.densities(), o.rho(), "pbf slow path rho")
    assert w.status() & pe.STATUS_SLOW_UNION
    w.close()


def test_dfsph_slow_path_bit_exact():
    """DFSPH's visit lists (boundary candidates kept) and the boundary slots'
    ascending fluid lists through the slow path."""
    h, s = 0.02, 0.002
    mass = pe.mass_from_spacing(RHO0, s, 3)
    ps, os_ = pe.Particles(3, RHO0, mass, h), O.Scene(3, RHO0, mass, h)
    _dense_block(ps, s)
    _dense_block(os_, s)
    p = pe.DfsphParams(adaptive_dt=False, particle_diameter=s, max_density_iters=3, max_divergence_iters=3)
    q = O.dfsph_default_params()
    q.kernel = p.kernel
    q.max_density_iters, q.max_divergence_iters = p.max_density_iters, p.max_divergence_iters
    q.density_error_tol, q.divergence_error_tol = p.density_error_tol, p.divergence_error_tol
    q.gravity[:] = p.gravity
    q.xsph_epsilon, q.particle_diameter, q.cfl_lambda = p.xsph_epsilon, p.particle_diameter, p.cfl_lambda
    q.adaptive_dt, q.warm_start = int(p.adaptive_dt), int(p.warm_start)
    for a, k in enumerate(pe.DfsphParams._SLIPS):
        v = getattr(p, k)
        q.has_slip[a] = 0 if v is None else 1
        q.slip[a] = 0.0 if v is None else v
    q.solver_omega, q.max_velocity_correction = p.solver_omega, p.max_velocity_correction
    w, o = pe.DfsphWorld(ps, p), O.DfsphWorld(os_, q)
    w.step(1e-6)
    o.step(1e-6)
    assert_bits_equal(w.positions(), o.x(), "dfsph slow path x")
    assert_bits_equal(w.velocities(), o.v(), "dfsph slow path v")
    assert_bits_equal(w.densities(), o.rho(), "dfsph slow path rho")
    assert_bits_equal(w.boundary_forces(), o.boundary_force(), "dfsph slow path boundary force")
    assert w.last_iterations() == o.iterations()
    assert w.status() & pe.STATUS_SLOW_UNION
    w.close()


def test_widely_spread_indices_sort_in_three_passes_bit_exact():
    """A fluid block whose original indices are spread over 400,000 (one
    particle in 200 is fluid; the rest are boundary samples of a plane far
    below), so the widest cell union's fluid indices span 314,000 > 2^18
    (19 bits) and the list build's radix sort takes three 9-bit passes. The lower lists (ascending original index) order the force sums,
    so the step is bit-exact only if the sort is right. The list stage is
    sized from the unions at creation with a small margin; the first step's
    unions (the lattice's particles leave cell faces) may outgrow it, so that
    step may take the slow path (an informational status bit) while the world
    grows the stage; the second step must run every cell on the staged path."""
    n_total, every = 400_000, 200
    side = int(np.ceil(np.sqrt(n_total)))
    fl = [(0.1 + DX * (k % 12), 0.1 + DX * ((k // 12) % 12), 0.1 + DX * (k // 144)) for k in range(n_total // every)]

    def build(sc):
        f = b = 0
        for k in range(n_total):
            if k % every == 0:
                sc.push_fluid(fl[f])
                f += 1
            else:
                sc.push_boundary((DX * (b % side), DX * (b // side), -3.0), DX ** 3)
                b += 1

    ps, os_ = _scenes(2 * DX, build)
    prm, op = _params()
    w = pe.WcsphWorld(ps, prm)
    o = O.World(os_, op)
    w.step(1e-4)
    o.step(1e-4)
    assert w.status() & ~pe.STATUS_SLOW_UNION == 0
    w.clear_status()
    w.step(1e-4)
    o.step(1e-4)
    _compare(w, o, "spread indices")
    assert w.status() == 0
    w.close()
