"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No dataset is involved: every array is drawn from numpy's PCG64 generator
with a fixed seed (seed + instance index), so a workload is reproducible.

    plain_2d         1000x1000 um, dx 20 (50x50x1), one O2-like substrate
                     (D 1e5, decay 0.1, Dirichlet 38, init 38), 500 cells in a
                     disc of r 200, radius 8.41, uptake 10, repulsion 10,
                     adhesion 0.4, relative max adhesion 1.25; mechanics
                     voxel 30 um; dt 0.01 / 0.1 min
    plain_3d         3000^3 um, dx 20 (150^3), 4 substrates (D log-uniform
                     1e3..1e5, decay U[0,1], Dirichlet targets U[0,40]),
                     200k cells uniform in a sphere of r 1200, radius
                     N(8.4, 0.5), secretion/uptake U[0,10]
    batched_2d       256 instances, side U{32..256}, 1-3 substrates,
                     100-20k cells uniform over the domain
    batched_3d       64 instances, side U{40..120}, 2 substrates (O2-like
                     D 1e5 decay 0.1; drug D log-U[1e3,5e4] decay U[0,0.5]),
                     1k-100k cells in a central sphere of radius
                     0.4 * side * dx (the radius is not given by the
                     configuration; this choice is ours), repulsion U[5,20],
                     adhesion U[0,1] per instance
    serving_requests Poisson arrivals (20/s), 70% 2-D side 64-256, 30% 3-D
                     side 40-100, 1-4 substrates, 500-50k cells, drug D
                     log-U[1e3,1e5], uptake U[0,20], 600-6000 steps
"""
import numpy as np

from . import (F_ADHESION, F_POS_X, F_POS_Y, F_POS_Z, F_RADIUS, F_REL_MAX_ADH, F_REPULSION, F_TOTAL_VOL,
               F_VOXEL_IDX, INST_REFRESH_VOXELS, NUM_FIELDS, Instance, make_grid, make_substrates,
               mech_params_for_domain)

DT_DIFF = 0.01
DT_MECH = 0.1


def voxel_index(x, y, z, grid):
    """Microenvironment::voxelIndex (src/microenvironment.mm:176-184), FP32."""
    f = np.float32

    def axis(p, lo, h, n):
        q = (np.asarray(p, f) - f(lo)) / f(h)
        q = np.where(np.isfinite(q), q, 0).astype(np.float64)
        i = np.trunc(np.clip(q, -2.0 ** 31, 2.0 ** 31 - 1)).astype(np.int64)
        return np.clip(i, 0, n - 1)
    i = axis(x, grid.x_min, grid.dx, grid.nx)
    j = axis(y, grid.y_min, grid.dy, grid.ny)
    k = axis(z, grid.z_min, grid.dz, grid.nz)
    return (k * grid.nx * grid.ny + j * grid.nx + i).astype(np.uint32)


def make_soa(pos, radius, rep, adh, relmax, grid, max_cells=None):
    n = len(radius)
    mc = max_cells or max(n, 1)
    soa = np.zeros(NUM_FIELDS * mc, np.float32)
    for a, f in enumerate((F_POS_X, F_POS_Y, F_POS_Z)):
        soa[f * mc:f * mc + n] = pos[:, a]
    soa[F_RADIUS * mc:F_RADIUS * mc + n] = radius
    soa[F_TOTAL_VOL * mc:F_TOTAL_VOL * mc + n] = (4.0 / 3.0) * np.pi * np.asarray(radius, np.float64) ** 3
    soa[F_REPULSION * mc:F_REPULSION * mc + n] = rep
    soa[F_ADHESION * mc:F_ADHESION * mc + n] = adh
    soa[F_REL_MAX_ADH * mc:F_REL_MAX_ADH * mc + n] = relmax
    vox = voxel_index(pos[:, 0], pos[:, 1], pos[:, 2], grid)
    soa[F_VOXEL_IDX * mc:F_VOXEL_IDX * mc + n] = vox.view(np.float32)
    return soa


def _disc(rng, n, r, cx, cy):
    rr = r * np.sqrt(rng.random(n))
    th = rng.random(n) * 2 * np.pi
    return np.stack([cx + rr * np.cos(th), cy + rr * np.sin(th), np.zeros(n)], 1).astype(np.float32)


def _ball(rng, n, r, c):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    rr = r * rng.random(n) ** (1.0 / 3.0)
    return (np.asarray(c) + v * rr[:, None]).astype(np.float32)


def _box(rng, n, lo, hi, two_d):
    p = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    if two_d:
        p[:, 2] = 0.0
    return p


def instance(grid, subs_params, pos, radius, rep, adh, relmax, sec, upt, sat, ne=None, init=None,
             two_d=True, z_span=(-10.0, 10.0), flags=0):
    """An Instance over 'grid' with cells at 'pos' (domain = grid box)."""
    S = len(subs_params)
    n = len(radius)
    x0, y0 = grid.x_min, grid.y_min
    x1, y1 = x0 + grid.nx * grid.dx, y0 + grid.ny * grid.dy
    if two_d:
        z0, z1 = z_span
    else:
        z0, z1 = grid.z_min, grid.z_min + grid.nz * grid.dz
    mech = mech_params_for_domain(x0, x1, y0, y1, z0, z1, two_d, DT_MECH)
    soa = make_soa(pos, radius, rep, adh, relmax, grid)
    init_vals = np.array([p[3] for p in subs_params] if init is None else init, np.float32)
    return Instance(grid, make_substrates(subs_params), mech, DT_MECH, initial_values=init_vals, soa=soa,
                    n_cells=n, soa_max=max(n, 1), sec=sec, upt=upt, sat=sat,
                    ne=np.zeros(n * S) if ne is None else ne, flags=flags)


def plain_2d(seed=1234, n_cells=500):
    rng = np.random.default_rng(seed)
    grid = make_grid(50, 50, 1, 1, dx=20.0, dt=DT_DIFF, x_min=-500.0, y_min=-500.0, z_min=-10.0)
    subs = [(1e5, 0.1, True, 38.0)]
    pos = _disc(rng, n_cells, 200.0, 0.0, 0.0)
    n = n_cells
    return instance(grid, subs, pos, np.full(n, 8.41, np.float32), 10.0, 0.4, 1.25,
                    sec=np.zeros(n), upt=np.full(n, 10.0), sat=np.full(n, 38.0))


def plain_3d(seed=1235, n_cells=200_000, side=150):
    rng = np.random.default_rng(seed)
    L = side * 20.0
    grid = make_grid(side, side, side, 4, dx=20.0, dt=DT_DIFF, x_min=-L / 2, y_min=-L / 2, z_min=-L / 2)
    D = np.exp(rng.uniform(np.log(1e3), np.log(1e5), 4))
    lam = rng.uniform(0, 1, 4)
    T = rng.uniform(0, 40, 4)
    subs = [(float(D[s]), float(lam[s]), True, float(T[s])) for s in range(4)]
    pos = _ball(rng, n_cells, 1200.0 * side / 150, (0.0, 0.0, 0.0))
    n = n_cells
    radius = np.clip(rng.normal(8.4, 0.5, n), 5.0, 12.0).astype(np.float32)
    return instance(grid, subs, pos, radius, 10.0, 0.4, 1.25,
                    sec=rng.uniform(0, 10, n * 4), upt=rng.uniform(0, 10, n * 4), sat=np.tile(T, n),
                    two_d=False)


def batched_2d(n_instances=256, seed=1236, max_cells=20_000, min_cells=100):
    out = []
    for i in range(n_instances):
        rng = np.random.default_rng(seed + i)
        side = int(rng.integers(32, 257))
        S = int(rng.integers(1, 4))
        L = side * 20.0
        grid = make_grid(side, side, 1, S, dx=20.0, dt=DT_DIFF, x_min=0.0, y_min=0.0, z_min=-10.0)
        D = np.exp(rng.uniform(np.log(1e3), np.log(1e5), S))
        lam = rng.uniform(0, 1, S)
        T = rng.uniform(0, 40, S)
        subs = [(float(D[s]), float(lam[s]), True, float(T[s])) for s in range(S)]
        n = int(rng.integers(min_cells, max_cells + 1))
        pos = _box(rng, n, 0.0, L, True)
        out.append(instance(grid, subs, pos, np.full(n, 8.41, np.float32), 10.0, 0.4, 1.25,
                            sec=np.zeros(n * S), upt=np.tile(np.r_[10.0, rng.uniform(0, 1, S - 1)], n),
                            sat=np.tile(T, n)))
    return out


def _batched_3d_spec(i, seed, min_cells, max_cells, side_range):
    """Scalar parameters of batched_3d instance i and its generator (the
    per-cell arrays are drawn from the same generator afterwards)."""
    rng = np.random.default_rng(seed + i)
    side = int(rng.integers(side_range[0], side_range[1] + 1))
    drug_D = float(np.exp(rng.uniform(np.log(1e3), np.log(5e4))))
    drug_lam = float(rng.uniform(0, 0.5))
    target = float(rng.uniform(0, 10))
    n = int(rng.integers(min_cells, max_cells + 1))
    return rng, side, drug_D, drug_lam, target, n


def batched_3d_work(n_instances=64, seed=1237, min_cells=1_000, max_cells=100_000, side_range=(40, 120)):
    """Algorithmic bytes of one mechanics period (10 diffusion sub-steps + 1
    mechanics step) per batched_3d instance, from its parameters alone:
    3 sweeps x 8 B per voxel-substrate, secretion 8 + 24 S B per cell, per
    sub-step; mechanics 136 B per cell.  Used to shard instances across GPUs
    without drawing their cells."""
    out = []
    for i in range(n_instances):
        _, side, _, _, _, n = _batched_3d_spec(i, seed, min_cells, max_cells, side_range)
        S = 2
        out.append(10 * (24 * S * side ** 3 + (8 + 24 * S) * n) + 136 * n)
    return out


def batched_3d(n_instances=64, seed=1237, min_cells=1_000, max_cells=100_000, side_range=(40, 120), only=None,
               flags=INST_REFRESH_VOXELS):
    """The batched 3-D configuration; 'only' restricts it to the given
    instance indices (a shard), each drawn exactly as in the full set.
    flags: instance flags.  By default INST_REFRESH_VOXELS: voxel indices
    are recomputed from the positions after every mechanics step (so the
    secretion order is rebuilt), the path's own rule; flags=0 keeps the
    reference's indices, which it refreshes only at phenotype steps."""
    out = []
    for i in (range(n_instances) if only is None else only):
        rng, side, drug_D, drug_lam, target, n = _batched_3d_spec(i, seed, min_cells, max_cells, side_range)
        L = side * 20.0
        grid = make_grid(side, side, side, 2, dx=20.0, dt=DT_DIFF)
        subs = [(1e5, 0.1, True, 38.0), (drug_D, drug_lam, True, target)]
        pos = _ball(rng, n, 0.4 * L, (L / 2, L / 2, L / 2))
        radius = np.clip(rng.normal(8.4, 0.5, n), 5.0, 12.0).astype(np.float32)
        rep = float(rng.uniform(5, 20))
        adh = float(rng.uniform(0, 1))
        upt = np.stack([np.full(n, 10.0), rng.uniform(0, 2, n)], 1).ravel()
        out.append(instance(grid, subs, pos, radius, rep, adh, 1.25, sec=np.zeros(n * 2), upt=upt,
                            sat=np.tile([38.0, 0.0], n), two_d=False, flags=flags))
    return out


def serving_requests(horizon_s=60.0, rate=20.0, seed=1238, cell_range=(500, 50_000), steps_range=(600, 6000),
                     side2d=(64, 256), side3d=(40, 100)):
    """[(arrival_time_s, Instance, n_steps)] with Poisson arrivals."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    k = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > horizon_s:
            break
        r = np.random.default_rng(seed * 7919 + k)
        k += 1
        two_d = r.random() < 0.7
        S = int(r.integers(1, 5))
        side = int(r.integers(side2d[0], side2d[1] + 1)) if two_d else int(r.integers(side3d[0], side3d[1] + 1))
        L = side * 20.0
        grid = make_grid(side, side, 1 if two_d else side, S, dx=20.0, dt=DT_DIFF, z_min=-10.0 if two_d else 0.0)
        drug_D = np.exp(r.uniform(np.log(1e3), np.log(1e5), S - 1))
        subs = [(1e5, 0.1, True, 38.0)] + [(float(drug_D[s]), float(r.uniform(0, 0.5)), True, 0.0)
                                           for s in range(S - 1)]
        n = int(r.integers(cell_range[0], cell_range[1] + 1))
        if two_d:
            pos = _disc(r, n, 0.4 * L, L / 2, L / 2)
        else:
            pos = _ball(r, n, 0.4 * L, (L / 2, L / 2, L / 2))
        upt = r.uniform(0, 20, n * S)
        inst = instance(grid, subs, pos, np.full(n, 8.41, np.float32), 10.0, 0.4, 1.25, sec=np.zeros(n * S),
                        upt=upt, sat=np.zeros(n * S), two_d=two_d)
        steps = int(r.integers(steps_range[0], steps_range[1] + 1))
        out.append((t, inst, steps))
    return out
