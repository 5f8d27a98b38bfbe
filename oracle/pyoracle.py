"""ctypes bindings for the CPU oracle (TEST INFRASTRUCTURE).

Loads oracle/liboracle.so (FP64 restatement, FP32 reference-exact mode),
oracle/libport.so (multi-threaded FP32 port used as the CPU baseline) and,
when it was built, oracle/_ref/libpcg_ref.so (the reference's own shader and
secretion code compiled for the CPU).  Only tests, the smoke check and the
CPU-baseline leg of bench.py import this module.

Array conventions follow the reference: density is float32 [s][k][j][i];
the cell SoA is float32 [field * max_cells + cell] with 28 fields
(shaders/types.h:74-102); per-cell per-substrate rates are float64
[cell * S + s] (src/cell_data.cpp:380-394).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

OR_FP64 = 0
OR_FP32_REF = 1

F_POS_X, F_POS_Y, F_POS_Z = 0, 1, 2
F_VEL_X, F_VEL_Y, F_VEL_Z = 3, 4, 5
F_PREV_VX, F_PREV_VY, F_PREV_VZ = 6, 7, 8
F_RADIUS, F_NUCLEAR_RAD, F_TOTAL_VOL, F_NUCLEAR_VOL = 9, 10, 11, 12
F_REPULSION, F_ADHESION, F_REL_MAX_ADH = 13, 14, 15
F_PRESSURE = 22
F_CELL_TYPE, F_CUR_PHASE, F_IS_ALIVE, F_VOXEL_IDX, F_MECH_VOXEL = 23, 24, 25, 26, 27
NUM_FIELDS = 28


class Grid(C.Structure):
    """GridParams (shaders/types.h:23-37)."""
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
                ("n_substrates", C.c_uint32), ("dx", C.c_float), ("dy", C.c_float),
                ("dz", C.c_float), ("dt", C.c_float), ("x_min", C.c_float),
                ("y_min", C.c_float), ("z_min", C.c_float), ("_pad0", C.c_float)]


class Substrate(C.Structure):
    """SubstrateParams (shaders/types.h:40-48)."""
    _fields_ = [("diffusion_coefficient", C.c_float), ("decay_rate", C.c_float),
                ("supply_rate", C.c_float), ("target_value", C.c_float),
                ("dirichlet_enabled", C.c_uint32), ("dirichlet_consistent", C.c_uint32),
                ("_pad", C.c_float * 2)]


class Mech(C.Structure):
    """MechanicsParams (shaders/types.h:51-61)."""
    _fields_ = [("dt", C.c_float), ("cell_cell_repulsion", C.c_float),
                ("cell_cell_adhesion", C.c_float), ("max_interaction_distance", C.c_float),
                ("mechanics_voxel_size", C.c_float), ("mech_grid_nx", C.c_uint32),
                ("mech_grid_ny", C.c_uint32), ("mech_grid_nz", C.c_uint32)]


class Sim(C.Structure):
    _fields_ = [("grid", Grid), ("subs", C.POINTER(Substrate)), ("mech", Mech),
                ("dt_mechanics", C.c_float), ("refresh_voxels", C.c_int), ("pos64", C.POINTER(C.c_double))]


def make_grid(nx, ny, nz, S, dx=20.0, dt=0.01, x_min=0.0, y_min=0.0, z_min=0.0, dy=None, dz=None):
    return Grid(nx, ny, nz, S, dx, dy if dy is not None else dx, dz if dz is not None else dx,
                dt, x_min, y_min, z_min, 0.0)


def make_subs(params):
    """params: list of (D, decay, dirichlet_enabled, target[, consistent])."""
    arr = (Substrate * max(1, len(params)))()
    for s, p in enumerate(params):
        D, lam, dirichlet, T = p[:4]
        arr[s].dirichlet_consistent = 1 if len(p) > 4 and p[4] else 0
        arr[s].diffusion_coefficient = D
        arr[s].decay_rate = lam
        arr[s].supply_rate = 0.0
        arr[s].target_value = T
        arr[s].dirichlet_enabled = 1 if dirichlet else 0
    return arr


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


_F32, _F64, _U32, _U8 = C.c_float, C.c_double, C.c_uint32, C.c_uint8


def build():
    """Compile the oracle libraries in place (make in oracle/)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class _Lib:
    def __init__(self, path):
        self.path = path
        self.lib = C.CDLL(path)


_oracle = None
_port = None
_ref = None


def oracle():
    global _oracle
    if _oracle is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        lib.or_nbr_hash.restype = C.c_uint32
        _oracle = lib
    return _oracle


def port():
    global _port
    if _port is None:
        path = os.path.join(HERE, "libport.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        lib.port_num_threads.restype = C.c_int
        _port = lib
    return _port


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libpcg_ref.so"))


def ref():
    global _ref
    if _ref is None:
        _ref = C.CDLL(os.path.join(HERE, "_ref", "libpcg_ref.so"))
    return _ref


# ---------------------------------------------------------------- diffusion

def sweeps(density, grid, subs, mode=OR_FP64):
    assert density.dtype == np.float32 and density.flags.c_contiguous
    oracle().or_diffusion_sweeps(_p(density, _F32), C.byref(grid), subs, C.c_int(mode))


def sweep_axis(density, grid, subs, axis, mode=OR_FP64):
    oracle().or_sweep_axis(_p(density, _F32), C.byref(grid), subs, C.c_int(axis), C.c_int(mode))


def dirichlet(density, grid, subs):
    oracle().or_apply_dirichlet(_p(density, _F32), C.byref(grid), subs)


def gradients(density, grid):
    n = density.size
    gx = np.zeros(n, np.float32)
    gy = np.zeros(n, np.float32)
    gz = np.zeros(n, np.float32)
    oracle().or_gradients(_p(density, _F32), C.byref(grid), _p(gx, _F32), _p(gy, _F32), _p(gz, _F32))
    return gx, gy, gz


# ---------------------------------------------------------------- secretion

def secretion(density, grid, voxel, volume, sec, upt, sat, ne, active=None, dt=0.01, lib=None):
    n = len(voxel)
    voxel = np.ascontiguousarray(voxel, np.uint32)
    volume = np.ascontiguousarray(volume, np.float32)
    sec, upt, sat, ne = (np.ascontiguousarray(a, np.float64) for a in (sec, upt, sat, ne))
    act = None if active is None else np.ascontiguousarray(active, np.uint8)
    oracle().or_secretion(_p(density, _F32), C.byref(grid), _U32(n), _p(voxel, _U32), _p(volume, _F32),
                          _p(sec, _F64), _p(upt, _F64), _p(sat, _F64), _p(ne, _F64),
                          None if act is None else _p(act, _U8), _F64(dt))


# ---------------------------------------------------------------- mechanics

def mech_params(x_min, x_max, y_min, y_max, z_min, z_max, use_2d, dt_mech=0.1):
    m = Mech()
    oracle().or_mech_params(_F32(x_min), _F32(x_max), _F32(y_min), _F32(y_max), _F32(z_min),
                            _F32(z_max), C.c_int(1 if use_2d else 0), _F32(dt_mech), C.byref(m))
    return m


def mech_nvox(m):
    return m.mech_grid_nx * m.mech_grid_ny * m.mech_grid_nz


def mech_bin(soa, max_cells, n, m, origin):
    key = np.zeros(max(n, 1), np.uint32)
    oracle().or_mech_bin(_p(soa, _F32), _U32(max_cells), _U32(n), C.byref(m), _F32(origin[0]),
                         _F32(origin[1]), _F32(origin[2]), _p(key, _U32))
    return key[:n]


def mech_sort(key, m):
    n = len(key)
    V = mech_nvox(m)
    key = np.ascontiguousarray(key, np.uint32)
    order = np.zeros(max(n, 1), np.uint32)
    start = np.zeros(V + 1, np.uint32)
    oracle().or_mech_sort(_p(key, _U32), _U32(n), _U32(V), _p(order, _U32), _p(start, _U32))
    return order[:n], start


def mech_forces(soa, max_cells, n, m, key, order, start):
    cnt = np.zeros(max(n, 1), np.uint32)
    hsh = np.zeros(max(n, 1), np.uint32)
    scale = np.zeros(max(n, 1), np.float64)
    key = np.ascontiguousarray(key, np.uint32)
    oracle().or_mech_forces(_p(soa, _F32), _U32(max_cells), _U32(n), C.byref(m), _p(key, _U32),
                            _p(order, _U32), _p(start, _U32), _p(cnt, _U32), _p(hsh, _U32),
                            _p(scale, _F64))
    return cnt[:n], hsh[:n], scale[:n]


def mech_integrate(soa, max_cells, n, m, origin, dt, pos64=None):
    """AB2 in place; with pos64 (3 * max_cells doubles) on FP64 master
    positions (or_mech_integrate_master)."""
    if pos64 is None:
        oracle().or_mech_integrate(_p(soa, _F32), _U32(max_cells), _U32(n), C.byref(m), _F32(origin[0]),
                                   _F32(origin[1]), _F32(origin[2]), _F32(dt))
        return
    assert pos64.dtype == np.float64 and pos64.size >= 3 * max_cells
    oracle().or_mech_integrate_master(_p(soa, _F32), _U32(max_cells), _U32(n), C.byref(m), _F32(origin[0]),
                                      _F32(origin[1]), _F32(origin[2]), _F32(dt), _p(pos64, _F64))


def voxel_refresh(soa, max_cells, n, grid):
    oracle().or_voxel_refresh(_p(soa, _F32), _U32(max_cells), _U32(n), C.byref(grid))


def _opt(a, t):
    return None if a is None else _p(a, t)


def cells_remove(soa, max_cells, n, S, sec, upt, sat, ne, active, indices):
    """or_cells_remove, in place; returns the new count."""
    lib = oracle()
    lib.or_cells_remove.restype = C.c_uint32
    idx = np.ascontiguousarray(indices, np.uint32)
    return lib.or_cells_remove(_p(soa, _F32), _U32(max_cells), _U32(n), _U32(S), _opt(sec, _F64), _opt(upt, _F64),
                               _opt(sat, _F64), _opt(ne, _F64), _opt(active, _U8), _p(idx, _U32), _U32(idx.size))


def master_positions(soa, max_cells):
    """FP64 master positions equal to the SoA's FP32 positions."""
    return np.ascontiguousarray(soa[:3 * max_cells], np.float64).copy()


def nbr_hash(j):
    return oracle().or_nbr_hash(_U32(j))


def run(grid, subs, mech, dt_mech, density, soa, max_cells, n, sec, upt, sat, ne, active, steps,
        accum=0.0, refresh=False, motility=None, seed=0, mot_step=0, layout=0, pos64=None):
    """The main loop (or_run).  With a motility state (motility_state), the
    motility phase runs between forces and integrate and the state is
    updated in place; returns (accumulator, next motility step) then.
    pos64 (3 * max_cells doubles, updated in place): FP64 master positions
    for the AB2 update (master_positions() gives the starting masters)."""
    if pos64 is not None:
        assert pos64.dtype == np.float64 and pos64.size >= 3 * max_cells and pos64.flags.c_contiguous
    sim = Sim(grid, C.cast(subs, C.POINTER(Substrate)), mech, dt_mech, 1 if refresh else 0,
              None if pos64 is None else _p(pos64, _F64))
    acc = C.c_double(accum)
    sec, upt, sat, ne = (np.ascontiguousarray(a, np.float64) for a in (sec, upt, sat, ne))
    act = None if active is None else np.ascontiguousarray(active, np.uint8)
    args = (C.byref(sim), _p(density, _F32), _p(soa, _F32), _U32(max_cells), _U32(n),
            _p(sec, _F64), _p(upt, _F64), _p(sat, _F64), _p(ne, _F64),
            None if act is None else _p(act, _U8), C.c_int(steps), C.byref(acc))
    if motility is None:
        oracle().or_run(*args)
        return acc.value
    m = _mot_struct(motility)
    ms = C.c_uint64(mot_step)
    oracle().or_run_motile(*args, C.byref(m), C.c_uint64(seed), C.byref(ms), C.c_int(layout))
    return acc.value, ms.value


# ---------------------------------------------------------------- FP32 port

def port_sweeps(density, grid, subs):
    port().port_diffusion_sweeps(_p(density, _F32), C.byref(grid), subs)


def port_dirichlet(density, grid, subs):
    port().port_apply_dirichlet(_p(density, _F32), C.byref(grid), subs)


def port_secretion(density, grid, voxel, volume, sec, upt, sat, ne, active=None, dt=0.01):
    n = len(voxel)
    act = None if active is None else np.ascontiguousarray(active, np.uint8)
    port().port_secretion(_p(density, _F32), C.byref(grid), _U32(n), _p(voxel, _U32), _p(volume, _F32),
                          _p(sec, _F64), _p(upt, _F64), _p(sat, _F64), _p(ne, _F64),
                          None if act is None else _p(act, _U8), _F64(dt))


def port_mech_step(soa, max_cells, n, m, origin, dt, scratch=None):
    V = mech_nvox(m)
    if scratch is None:
        scratch = (np.zeros(max(n, 1), np.uint32), np.zeros(max(n, 1), np.uint32), np.zeros(V + 1, np.uint32))
    key, order, start = scratch
    port().port_mech_step(_p(soa, _F32), _U32(max_cells), _U32(n), C.byref(m), _F32(origin[0]),
                          _F32(origin[1]), _F32(origin[2]), _F32(dt), _p(key, _U32), _p(order, _U32),
                          _p(start, _U32))
    return scratch


def port_threads(n=None):
    if n is not None:
        port().port_set_threads(C.c_int(n))
    return port().port_num_threads()


# ---------------------------------------------------------------- reference (compiled from the reference tree)

def ref_sweeps(density, grid, subs, threads=1):
    ref().ref_simulate_diffusion_decay(_p(density, _F32), C.byref(grid), subs, C.c_int(threads))


def ref_sweep_x(density, grid, subs):
    ref().ref_sweep_x(_p(density, _F32), C.byref(grid), subs)


def ref_sweep_y(density, grid, subs):
    ref().ref_sweep_y(_p(density, _F32), C.byref(grid), subs)


def ref_dirichlet(density, grid, subs):
    ref().ref_apply_dirichlet(_p(density, _F32), C.byref(grid), subs)


def ref_secretion(density, grid, voxel, volume, sec, upt, sat, ne, dt=0.01):
    n = len(voxel)
    voxel = np.ascontiguousarray(voxel, np.uint32)
    volume = np.ascontiguousarray(volume, np.float32)
    sec, upt, sat, ne = (np.ascontiguousarray(a, np.float64) for a in (sec, upt, sat, ne))
    ref().ref_process_secretion(_p(density, _F32), C.byref(grid), _U32(n), _p(voxel, _U32),
                                _p(volume, _F32), _p(sec, _F64), _p(upt, _F64), _p(sat, _F64),
                                _p(ne, _F64), _F64(dt))


def ref_forces(soa, max_cells, n, m, origin, threads=1):
    """Runs the reference's clear/build/compute_forces kernels; returns the
    hash (counts, cells[V*64])."""
    V = mech_nvox(m)
    counts = np.zeros(V, np.uint32)
    cells = np.zeros(V * 64, np.uint32)
    mg = Grid(m.mech_grid_nx, m.mech_grid_ny, m.mech_grid_nz, 0, m.mechanics_voxel_size,
              m.mechanics_voxel_size, m.mechanics_voxel_size, 0.0, origin[0], origin[1], origin[2], 0.0)
    ref().ref_compute_forces(_p(soa, _F32), _U32(max_cells), _U32(n), C.byref(m), C.byref(mg),
                             _p(counts, _U32), _p(cells, _U32), C.c_int(threads))
    return counts, cells


def ref_cells_remove(soa, max_cells, n, S, sec, upt, sat, ne, indices):
    """The reference's CellData::removeCell in phase-3 order, in place;
    returns the new count (rate arrays of max_cells * S)."""
    lib = ref()
    lib.ref_remove_cells.restype = C.c_uint32
    idx = np.ascontiguousarray(indices, np.uint32)
    return lib.ref_remove_cells(_p(soa, _F32), _U32(max_cells), _U32(n), _U32(S), _p(sec, _F64), _p(upt, _F64),
                                _p(sat, _F64), _p(ne, _F64), _p(idx, _U32), _U32(idx.size))


def ref_integrate(soa, max_cells, n, m, origin, dt):
    mg = Grid(m.mech_grid_nx, m.mech_grid_ny, m.mech_grid_nz, 0, m.mechanics_voxel_size,
              m.mechanics_voxel_size, m.mechanics_voxel_size, 0.0, origin[0], origin[1], origin[2], 0.0)
    ref().ref_integrate(_p(soa, _F32), _U32(max_cells), _U32(n), C.byref(mg), _F32(dt))


# ---------------------------------------------------------------- motility

MOT_REF, MOT_SUBSTRATE_MAJOR = 0, 1


class MotilityState(C.Structure):
    """or_motility: pointers into the arrays of a motility state dict."""
    _fields_ = [("persistence_time", C.POINTER(C.c_double)), ("elapsed", C.POINTER(C.c_double)),
                ("bias", C.POINTER(C.c_double)), ("vec", C.POINTER(C.c_double)),
                ("is_motile", C.POINTER(C.c_uint32)), ("restrict_2d", C.POINTER(C.c_uint32)),
                ("chemotaxis_index", C.POINTER(C.c_int32)), ("chemotaxis_direction", C.POINTER(C.c_int32)),
                ("sensitivity", C.POINTER(C.c_double)), ("n_sens", C.c_uint32)]


def motility_state(n, n_sens=0):
    """A zeroed motility state (src/motility.cpp:133-152 defaults): persistence
    15, bias 0.5, not motile, 2-D, chemotaxis up the first substrate."""
    st = {"persistence_time": np.full(n, 15.0), "elapsed": np.zeros(n), "bias": np.full(n, 0.5),
          "vec": np.zeros(3 * n), "is_motile": np.zeros(n, np.uint32), "restrict_2d": np.ones(n, np.uint32),
          "chemotaxis_index": np.zeros(n, np.int32), "chemotaxis_direction": np.ones(n, np.int32),
          "sensitivity": np.zeros(n * n_sens) if n_sens else None, "n_sens": n_sens}
    return st


def _mot_struct(st):
    m = MotilityState()
    m.persistence_time = _p(st["persistence_time"], C.c_double)
    m.elapsed = _p(st["elapsed"], C.c_double)
    m.bias = _p(st["bias"], C.c_double)
    m.vec = _p(st["vec"], C.c_double)
    m.is_motile = _p(st["is_motile"], C.c_uint32)
    m.restrict_2d = _p(st["restrict_2d"], C.c_uint32)
    m.chemotaxis_index = _p(st["chemotaxis_index"], C.c_int32)
    m.chemotaxis_direction = _p(st["chemotaxis_direction"], C.c_int32)
    m.sensitivity = _p(st["sensitivity"], C.c_double) if st["sensitivity"] is not None else None
    m.n_sens = st["n_sens"] if st["sensitivity"] is not None else 0
    return m


def uniform(seed, cell, step, k):
    lib = oracle()
    lib.or_uniform.restype = C.c_double
    return lib.or_uniform(C.c_uint64(seed), C.c_uint64(cell), C.c_uint64(step), C.c_uint32(k))


def motility_update(soa, max_cells, n, density, grid, st, dt, seed, step, layout=MOT_REF):
    m = _mot_struct(st)
    oracle().or_motility_update(_p(soa, _F32), _U32(max_cells), _U32(n),
                                _p(density, _F32) if density is not None else None, C.byref(grid), C.byref(m),
                                _F64(dt), C.c_uint64(seed), C.c_uint64(step), C.c_int(layout))


def ref_motility_update(soa, max_cells, n, density, grid, st, dt):
    s = st["sensitivity"]
    ref().ref_update_motility(_p(soa, _F32), _U32(max_cells), _U32(n),
                              _p(density, _F32) if density is not None else None, C.byref(grid),
                              _p(st["persistence_time"], C.c_double), _p(st["elapsed"], C.c_double),
                              _p(st["bias"], C.c_double), _p(st["vec"], C.c_double),
                              _p(st["is_motile"], C.c_uint32), _p(st["restrict_2d"], C.c_uint32),
                              _p(st["chemotaxis_index"], C.c_int32), _p(st["chemotaxis_direction"], C.c_int32),
                              _p(s, C.c_double) if s is not None else None, _U32(st["n_sens"] if s is not None else 0),
                              _F64(dt))


# ---------------------------------------------------------------- .mat snapshots

def ref_write_matlab(soa, max_cells, n, n_types, sec, upt, sat, ne, density, grid, frame, folder):
    sec, upt, sat, ne = (np.ascontiguousarray(a, np.float64) for a in (sec, upt, sat, ne))
    ref().ref_write_matlab(_p(soa, _F32), _U32(max_cells), _U32(n), _U32(n_types), _p(sec, _F64), _p(upt, _F64),
                           _p(sat, _F64), _p(ne, _F64), _p(density, _F32), C.byref(grid), C.c_int(frame),
                           C.c_char_p(folder.encode()))


def read_mat4(path):
    """(name, matrix rows x cols) of a MATLAB v4 file of one full double matrix."""
    raw = open(path, "rb").read()
    typ, rows, cols, imag, nlen = np.frombuffer(raw[:20], np.uint32)
    assert typ == 0 and imag == 0
    name = raw[20:20 + nlen - 1].decode()
    data = np.frombuffer(raw[20 + nlen:], np.float64)
    assert data.size == rows * cols
    return name, data.reshape(cols, rows).T
