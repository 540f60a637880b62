"""The reference's host test cases (test/test.cpp), written once against a solver-neutral driver.

Each ``case_*`` function builds the scenario of one reference test, runs it through ``runner`` (the
CPU oracle or the CUDA library, see ``OracleRunner`` / ``GpuRunner`` in the test modules) and
checks the golden values the reference test checks, looked up by ``test/test.cpp`` line number.
"""

from __future__ import annotations

import numpy as np

from scenarios import (add_boundary_dirichlet, add_dirichlet_at, agents_from_rows, assert_float_eq,
                       biorobots_microenv, default_microenv, golden, golden_vector, index_field, mesh,
                       set_default_agent_values)

f32 = np.float32


def _view(dens, scn):
    X, Y, Z = scn.grid
    return np.asarray(dens).reshape(Z, Y, X, scn.S)


# ---------------------------------------------------------------------------------------------
# diffusion (test/test.cpp:33-244)

def case_diffusion_uniform(runner, dims):
    if dims == 1:
        scn = default_microenv(mesh(1, (80, 0, 0), (20, 0, 0)))
        l0, l1 = 59, 60
    elif dims == 2:
        scn = default_microenv(mesh(2, (800, 800, 0), (20, 20, 0)))
        l0, l1 = 85, 86
    else:
        scn = default_microenv(mesh(3, (200, 200, 200), (20, 20, 20)))
        l0, l1 = 111, 112
    r = runner(scn)
    r.diffusion()
    d = _view(r.densities(), scn)
    assert_float_eq(d[..., 0], golden(l0), f"D{dims}_uniform s0")
    assert_float_eq(d[..., 1], golden(l1), f"D{dims}_uniform s1")


def case_diffusion_random(runner, dims):
    bmax = {1: (60, 0, 0), 2: (60, 60, 0), 3: (60, 60, 60)}[dims]
    scn = biorobots_microenv(mesh(dims, bmax, (20, 20, 20)))
    scn.densities = index_field(scn)
    r = runner(scn)
    r.diffusion()
    expected = golden_vector(f"host_diffusion_solver.D{dims}_random")
    assert_float_eq(r.densities(), np.array(expected), f"D{dims}_random")


# ---------------------------------------------------------------------------------------------
# interior Dirichlet (test/test.cpp:246-505)

def case_dirichlet_one_cond(runner, dims):
    if dims == 1:
        scn = default_microenv(mesh(1, (100, 0, 0), (20, 0, 0)))
        add_dirichlet_at(scn, [(2, 0, 0)], [1])
        r = runner(scn)
        r.diffusion()
        d = _view(r.densities(), scn)[0, 0]
        for x in range(scn.grid[0]):
            assert_float_eq(d[x, 0], golden(268) if x == 2 else golden(270), f"x={x} s0")
            assert_float_eq(d[x, 1], golden(271), f"x={x} s1")
        return
    if dims == 2:
        scn = default_microenv(mesh(2, (60, 60, 0), (20, 20, 0)))
        add_dirichlet_at(scn, [(1, 1, 0)], [10])
        r = runner(scn)
        r.diffusion()
        d = _view(r.densities(), scn)[0]
        assert_float_eq(d[..., 1], golden(298), "s1")
        for y in range(3):
            for x in range(3):
                if x == 1 and y == 1:
                    exp = golden(309)
                elif abs(x - 1) == 1 and abs(y - 1) == 1:
                    exp = golden(312)
                elif abs(x - 1) == 1 and y == 1:
                    exp = golden(315)
                else:
                    exp = golden(318)
                assert_float_eq(d[y, x, 0], exp, f"({x},{y}) s0")
        return
    scn = default_microenv(mesh(3, (60, 60, 60), (20, 20, 20)))
    add_dirichlet_at(scn, [(1, 1, 1)], [1000])
    r = runner(scn)
    r.diffusion()
    d = _view(r.densities(), scn)
    assert_float_eq(d[..., 1], golden(345), "s1")
    s0 = d[..., 0]  # [z][y][x]
    for z in (0, 2):
        for (x, y, line) in ((0, 0, 353), (1, 0, 354), (2, 0, 355), (0, 1, 357), (1, 1, 358), (2, 1, 359),
                             (0, 2, 361), (1, 2, 362), (2, 2, 363)):
            assert_float_eq(s0[z, y, x], golden(line), f"({x},{y},{z})")
    for (x, y, line) in ((0, 0, 366), (1, 0, 367), (2, 0, 368), (0, 1, 370), (1, 1, 371), (2, 1, 372),
                         (0, 2, 374), (1, 2, 375), (2, 2, 376)):
        assert_float_eq(s0[1, y, x], golden(line), f"({x},{y},1)")


def case_dirichlet_multiple_cond(runner, dims):
    if dims == 1:
        scn = default_microenv(mesh(1, (100, 0, 0), (20, 0, 0)))
        add_dirichlet_at(scn, [(0, 0, 0), (4, 0, 0)], [1, 1])
        r = runner(scn)
        r.diffusion()
        d = _view(r.densities(), scn)[0, 0]
        for x in range(scn.grid[0]):
            assert_float_eq(d[x, 0], golden(401) if x in (0, 4) else golden(403), f"x={x} s0")
            assert_float_eq(d[x, 1], golden(404), f"x={x} s1")
        return
    if dims == 2:
        scn = default_microenv(mesh(2, (60, 60, 0), (20, 20, 0)))
        add_dirichlet_at(scn, [(0, 0, 0), (1, 0, 0), (2, 0, 0)], [10, 10, 10])
        r = runner(scn)
        r.diffusion()
        d = _view(r.densities(), scn)[0]
        assert_float_eq(d[..., 1], golden(431), "s1")
        for y in range(3):
            exp = golden(440) if y == 0 else (golden(443) if y == 1 else golden(446))
            assert_float_eq(d[y, :, 0], exp, f"y={y} s0")
        return
    scn = default_microenv(mesh(3, (60, 60, 60), (20, 20, 20)))
    add_dirichlet_at(scn, [(x, y, 1) for y in range(3) for x in range(3)], [1000] * 9)
    r = runner(scn)
    r.diffusion()
    d = _view(r.densities(), scn)
    assert_float_eq(d[..., 1], golden(483), "s1")
    for z in (0, 2):
        assert_float_eq(d[z, :, :, 0], golden(494), f"z={z} s0")
    assert_float_eq(d[1, :, :, 0], golden(503), "z=1 s0")


# ---------------------------------------------------------------------------------------------
# gradient (test/test.cpp:507-664)

def case_gradient(runner, dims):
    if dims == 1:
        scn = default_microenv(mesh(1, (100, 0, 0), (20, 0, 0)))
        n = scn.grid[0]
        dens = np.zeros((n, 2))
        for x in range(n):
            dens[x, 0] = x * x
            dens[n - 1 - x, 1] = x * x
        scn.densities = dens.reshape(-1)
        r = runner(scn)
        r.gradient()
        g = np.asarray(r.gradients()).reshape(n, 2)  # [x][s][d=1]
        for line, (s, x) in zip(range(533, 538), [(0, 0), (0, 1), (0, 2), (0, 3), (0, 4)]):
            assert_float_eq(g[x, s], golden(line), f"line {line}")
        for line, (s, x) in zip(range(539, 544), [(1, 4), (1, 3), (1, 2), (1, 1), (1, 0)]):
            assert_float_eq(g[x, s], golden(line), f"line {line}")
        return
    if dims == 2:
        scn = default_microenv(mesh(2, (100, 100, 0), (20, 20, 0)))
        get = lambda x, y, s: (x + y) * (x + y) + s  # noqa: E731
        X, Y, _ = scn.grid
        scn.densities = np.array([get(x, y, s) for y in range(Y) for x in range(X) for s in range(2)], float)
        r = runner(scn)
        r.gradient()
        g = np.asarray(r.gradients()).reshape(Y, X, 2, 2)  # [y][x][s][d]
        for x in range(X):
            for y in range(Y):
                xu, xd = x + (0 if x == X - 1 else 1), x - (0 if x == 0 else 1)
                xdiv = 20.0 if x in (0, X - 1) else 40.0
                yu, yd = y + (0 if y == Y - 1 else 1), y - (0 if y == 0 else 1)
                ydiv = 20.0 if y in (0, Y - 1) else 40.0
                for s in range(2):
                    assert_float_eq(g[y, x, s, 0], (get(xu, y, s) - get(xd, y, s)) / xdiv, "gx")
                    assert_float_eq(g[y, x, s, 1], (get(x, yu, s) - get(x, yd, s)) / ydiv, "gy")
        return
    scn = default_microenv(mesh(3, (100, 100, 100), (20, 20, 20)))
    get = lambda x, y, z, s: (x + y + z) * (x + y + z) + s  # noqa: E731
    X, Y, Z = scn.grid
    scn.densities = np.array([get(x, y, z, s) for z in range(Z) for y in range(Y) for x in range(X)
                              for s in range(2)], float)
    r = runner(scn)
    r.gradient()
    g = np.asarray(r.gradients()).reshape(3, Z, Y, X, 2)  # [d][z][y][x][s]
    for x in range(X):
        for y in range(Y):
            for z in range(Z):
                def nb(i, n):
                    return i + (0 if i == n - 1 else 1), i - (0 if i == 0 else 1), (20.0 if i in (0, n - 1) else 40.0)
                xu, xd, xdiv = nb(x, X)
                yu, yd, ydiv = nb(y, Y)
                zu, zd, zdiv = nb(z, Z)
                for s in range(2):
                    assert_float_eq(g[0, z, y, x, s], (get(xu, y, z, s) - get(xd, y, z, s)) / xdiv, "gx")
                    assert_float_eq(g[1, z, y, x, s], (get(x, yu, z, s) - get(x, yd, z, s)) / ydiv, "gy")
                    assert_float_eq(g[2, z, y, x, s], (get(x, y, zu, s) - get(x, y, zd, s)) / zdiv, "gz")


# ---------------------------------------------------------------------------------------------
# boundary Dirichlet precedence (test/test.cpp:666-810)

def case_dirichlet_boundaries(runner, dims):
    scn = default_microenv(mesh(dims, (100, 100, 100), (20, 20, 20)))
    add_boundary_dirichlet(scn, 0, True, 4)
    add_boundary_dirichlet(scn, 0, False, 5)
    if dims >= 2:
        add_boundary_dirichlet(scn, 1, True, 6)
        add_boundary_dirichlet(scn, 1, False, 7)
    if dims >= 3:
        add_boundary_dirichlet(scn, 2, True, 8)
        add_boundary_dirichlet(scn, 2, False, 9)
    r = runner(scn)
    r.dirichlet()
    X, Y, Z = scn.grid
    d = _view(r.densities(), scn)
    for z in range(Z):
        for y in range(Y):
            for x in range(X):
                if dims == 3 and z == 0:
                    exp = 8
                elif dims == 3 and z == Z - 1:
                    exp = 9
                elif dims >= 2 and y == 0:
                    exp = 6
                elif dims >= 2 and y == Y - 1:
                    exp = 7
                elif x == 0:
                    exp = 4
                elif x == X - 1:
                    exp = 5
                else:
                    exp = 1
                assert_float_eq(d[z, y, x, 0], exp, f"({x},{y},{z}) s0")
                assert_float_eq(d[z, y, x, 1], 1, f"({x},{y},{z}) s1")


# ---------------------------------------------------------------------------------------------
# agents (test/test.cpp:812-1214)

def _agent_scn(dims, bmax, internalized):
    scn = default_microenv(mesh(dims, bmax, (20, 20, 20)))
    scn.time_step = 0.01
    scn.compute_internalized = internalized
    return scn


def case_agents_simple(runner, dims, internalized, recompute):
    bmax = {1: (60, 20, 20), 2: (60, 60, 20), 3: (60, 60, 60)}[dims]
    scn = _agent_scn(dims, bmax, internalized)
    rows = []
    set_default_agent_values(rows, 0, 1000, (10, 10, 10), dims)
    set_default_agent_values(rows, 400, 1000, (30, 30, 30), dims)
    set_default_agent_values(rows, 800, 1000, (50, 50, 50), dims)
    scn.agents = agents_from_rows(rows, 2, dims)
    r = runner(scn)

    # expected lines per dims: (internalized a1..a3 first call, densities first call, second call)
    base = {1: 850, 2: 925, 3: 1000}[dims]
    dbase = {1: 860, 2: 935, 3: 1010}[dims]

    def at(d, i):
        return _dens_at(d, scn, i)

    r.secretion(True)
    if internalized:
        I = np.asarray(r.internalized()).reshape(3, 2)
        for k, line in enumerate((base, base + 3, base + 6)):
            assert_float_eq(I[k, 0], golden(line), f"a{k + 1} s0")
            assert_float_eq(I[k, 1], golden(line + 1), f"a{k + 1} s1")
    d = r.densities()
    for k, line in enumerate((dbase, dbase + 3, dbase + 6)):
        assert_float_eq(at(d, k)[0], golden(line), f"voxel {k} s0")
        assert_float_eq(at(d, k)[1], golden(line + 1), f"voxel {k} s1")

    r.secretion(recompute)
    if internalized:
        I = np.asarray(r.internalized()).reshape(3, 2)
        for k, line in enumerate((base + 23, base + 26, base + 29)):
            assert_float_eq(I[k, 0], golden(line), f"a{k + 1} s0 (2nd)")
            assert_float_eq(I[k, 1], golden(line + 1), f"a{k + 1} s1 (2nd)")
    d = r.densities()
    for k, line in enumerate((dbase + 23, dbase + 26, dbase + 29)):
        assert_float_eq(at(d, k)[0], golden(line), f"voxel {k} s0 (2nd)")
        assert_float_eq(at(d, k)[1], golden(line + 1), f"voxel {k} s1 (2nd)")


def _dens_at(d, scn, i):
    X, Y, Z = scn.grid
    v = np.asarray(d).reshape(Z, Y, X, scn.S)
    if scn.dims == 1:
        return v[0, 0, i]
    if scn.dims == 2:
        return v[0, i, i]
    return v[i, i, i]


def expected_internalized_1d(scn, dens, I):
    """test/utils.cpp:134-162 in float arithmetic: I -= (vv*-den*D + num)/(1+den) + fac."""
    a = scn.agents
    vv = f32(scn.voxel_volume)
    dt = f32(scn.time_step)
    out = np.array(I, dtype=np.float32).reshape(a.count, scn.S)
    dv = np.asarray(dens, np.float32).reshape(-1, scn.S)
    for i in range(a.count):
        for s in range(scn.S):
            S_, T_, U_, N_ = (f32(a.secretion_rates[i, s]), f32(a.saturation_densities[i, s]),
                              f32(a.uptake_rates[i, s]), f32(a.net_export_rates[i, s]))
            vol = f32(a.volumes[i])
            num = f32(f32(f32(S_ * T_) * dt) * vol)
            den = f32(f32(f32(f32(S_ + U_) * dt) * vol) / vv)
            fac = f32(N_ * dt)
            x = int(f32(f32(a.positions[i, 0]) / f32(scn.voxel_shape[0])))
            D = dv[x, s]
            term = f32(f32(f32(f32(vv * f32(-den)) * D) + num) / f32(1 + den))
            out[i, s] = f32(out[i, s] - f32(term + fac))
    return out


def expected_densities_1d(scn, dens):
    """test/utils.cpp:164-202 in float arithmetic, sums in agent order.

    The agent-to-voxel match uses the truncating voxel index of src/mesh.cpp:35-53.  The
    reference's helper compares ``position / dx == x`` in floating point (test/utils.cpp:185),
    which is never true for agents at voxel centres, so as written it matches no agent."""
    a = scn.agents
    vv = f32(scn.voxel_volume)
    dt = f32(scn.time_step)
    dv = np.asarray(dens, np.float32).reshape(-1, scn.S)
    out = np.zeros_like(dv)
    for s in range(scn.S):
        for x in range(scn.grid[0]):
            num = den = fac = f32(0)
            for i in range(a.count):
                if int(f32(f32(a.positions[i, 0]) / f32(scn.voxel_shape[0]))) == x:
                    S_, T_, U_, N_ = (f32(a.secretion_rates[i, s]), f32(a.saturation_densities[i, s]),
                                      f32(a.uptake_rates[i, s]), f32(a.net_export_rates[i, s]))
                    vol = f32(a.volumes[i])
                    num = f32(num + f32(f32(f32(f32(S_ * T_) * dt) * vol) / vv))
                    den = f32(den + f32(f32(f32(f32(S_ + U_) * dt) * vol) / vv))
                    fac = f32(fac + f32(f32(N_ * dt) / vv))
            out[x, s] = f32(f32(f32(dv[x, s] + num) / f32(1 + den)) + fac)
    return out.reshape(-1)


def case_agents_conflict(runner, internalized, recompute, big=False):
    """Expected values use the field from before each call.  The reference computes its expected
    densities after the call, from the already-updated field (test/test.cpp:1097-1105,
    1120-1128); with its voxel match (see ``expected_densities_1d``) that check compares the field
    with itself.  The formula of test/utils.cpp:164-202 is kept and applied to the pre-call field;
    its sums associate differently from the solver's ballot sums, so with 50 agents per voxel the
    bound is relative (1e-6) rather than 4 ULPs."""
    if big:
        # test/test.cpp:1131-1214: 50 agents at the centre of each of 100 voxels
        scn = _agent_scn(1, (2000, 20, 20), internalized)
        rows = []
        for i in range(scn.grid[0]):
            for _ in range(50):
                set_default_agent_values(rows, 0, 500, (i * 20 + 20 / 2.0, 0, 0), 1)
    else:
        # test/test.cpp:1043-1129
        scn = _agent_scn(1, (60, 20, 20), internalized)
        rows = []
        set_default_agent_values(rows, 0, 500, (10, 0, 0), 1)
        set_default_agent_values(rows, 600, 1000, (30, 0, 0), 1)
        set_default_agent_values(rows, 1100, 1500, (30, 0, 0), 1)
        set_default_agent_values(rows, 1600, 2000, (50, 0, 0), 1)
        set_default_agent_values(rows, 2100, 2500, (50, 0, 0), 1)
        set_default_agent_values(rows, 2600, 3000, (50, 0, 0), 1)
    scn.agents = agents_from_rows(rows, 2, 1)
    r = runner(scn)
    A = scn.agents.count

    dens0 = r.densities()
    exp_I = expected_internalized_1d(scn, dens0, np.zeros(A * 2))
    def check_dens(actual, expected, what):
        if big:
            a = np.asarray(actual, np.float64)
            e = np.asarray(expected, np.float64)
            err = float(np.max(np.abs(a - e) / np.abs(e)))
            assert err < 1e-6, f"{what}: rel err {err}"
        else:
            assert_float_eq(actual, expected, what)

    r.secretion(True)
    if internalized:
        assert_float_eq(np.asarray(r.internalized()).reshape(A, 2), exp_I, "internalized (1st)")
    check_dens(r.densities(), expected_densities_1d(scn, dens0), "densities (1st)")

    dens1 = r.densities()
    exp_I = expected_internalized_1d(scn, dens1, exp_I)
    r.secretion(recompute)
    if internalized:
        assert_float_eq(np.asarray(r.internalized()).reshape(A, 2), exp_I, "internalized (2nd)")
    check_dens(r.densities(), expected_densities_1d(scn, dens1), "densities (2nd)")
