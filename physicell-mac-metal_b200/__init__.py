"""Python host mirror of the B200 hot path (ctypes over libpcg.so).

The classes follow the reference's C++ call surface so that tests and tools
read like the reference's own code:

    Microenvironment   src/microenvironment.h:17-83
        simulateDiffusionDecay, applyDirichletBC, applySecretion (batched
        processSecretion, src/cell_phenotype.cpp:526-564), computeGradients,
        getDensity/setDensity (bulk), densityBuffer (read-back)
    Cells              GPU-shared block of CellData (src/cell_data.h:19-244)
    CellMechanics      src/cell_mechanics.h:15-87
        computeForces, integratePositions, update, syncHashPointers ->
        voxelCellCount / voxelCells
    Motility           MotilityData + updateMotility (src/motility.h,
                       src/motility.cpp:179-293)
    Batch, Server      many simulations at once; continuous batching

Every call goes through the C ABI of include/pcg.h.  There is no CPU
fallback: constructing a Context raises when libpcg.so is missing or no
CUDA device is present.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpcg.so")

NUM_FIELDS = 28
(F_POS_X, F_POS_Y, F_POS_Z, F_VEL_X, F_VEL_Y, F_VEL_Z, F_PREV_VX, F_PREV_VY, F_PREV_VZ, F_RADIUS,
 F_NUCLEAR_RAD, F_TOTAL_VOL, F_NUCLEAR_VOL, F_REPULSION, F_ADHESION, F_REL_MAX_ADH, F_MOT_SPEED,
 F_MOT_BIAS, F_MOT_DIR_X, F_MOT_DIR_Y, F_MOT_DIR_Z, F_ONCOPROTEIN, F_PRESSURE, F_CELL_TYPE,
 F_CUR_PHASE, F_IS_ALIVE, F_VOXEL_IDX, F_MECH_VOXEL) = range(28)

PCG_OK = 0
# fields the sub-steps and mechanics steps write (PCG_STEP_WRITTEN_FIELDS)
STEP_WRITTEN_FIELDS = sum(1 << f for f in (0, 1, 2, 3, 4, 5, 6, 7, 8, 22, 26, 27))
# every other field: what a host that owns the phenotype sends (PCG_HOST_OWNED_FIELDS)
HOST_OWNED_FIELDS = ((1 << 28) - 1) & ~STEP_WRITTEN_FIELDS
INST_REFRESH_VOXELS = 1
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_CANCELLED = 0, 1, 2, 3
N_PHASES = 7
PHASES = ("x_sweep", "y_sweep", "z_sweep", "secretion", "bin_sort", "forces", "integrate")


class PcgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"pcg status {status}: {msg}")
        self.status = status


class GridParams(C.Structure):
    """GridParams (shaders/types.h:23-37)."""
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
                ("n_substrates", C.c_uint32), ("dx", C.c_float), ("dy", C.c_float),
                ("dz", C.c_float), ("dt", C.c_float), ("x_min", C.c_float),
                ("y_min", C.c_float), ("z_min", C.c_float), ("_pad0", C.c_float)]


class SubstrateParams(C.Structure):
    """SubstrateParams (shaders/types.h:40-48)."""
    _fields_ = [("diffusion_coefficient", C.c_float), ("decay_rate", C.c_float),
                ("supply_rate", C.c_float), ("target_value", C.c_float),
                ("dirichlet_enabled", C.c_uint32), ("dirichlet_consistent", C.c_uint32),
                ("_pad", C.c_float * 2)]


class MechanicsParams(C.Structure):
    """MechanicsParams (shaders/types.h:51-61)."""
    _fields_ = [("dt", C.c_float), ("cell_cell_repulsion", C.c_float),
                ("cell_cell_adhesion", C.c_float), ("max_interaction_distance", C.c_float),
                ("mechanics_voxel_size", C.c_float), ("mech_grid_nx", C.c_uint32),
                ("mech_grid_ny", C.c_uint32), ("mech_grid_nz", C.c_uint32)]


_F32P = C.POINTER(C.c_float)
_F64P = C.POINTER(C.c_double)
_U32P = C.POINTER(C.c_uint32)
_U8P = C.POINTER(C.c_uint8)
_I32P = C.POINTER(C.c_int32)


class InstanceDesc(C.Structure):
    """pcg_instance_desc (include/pcg.h)."""
    _fields_ = [("grid", GridParams), ("substrates", C.POINTER(SubstrateParams)),
                ("initial_density", _F32P), ("initial_values", _F32P), ("n_cells", C.c_uint32),
                ("cells_soa", _F32P), ("cells_soa_max", C.c_uint32),
                ("secretion", _F64P), ("uptake", _F64P), ("saturation", _F64P), ("net_export", _F64P),
                ("active", _U8P), ("mech", MechanicsParams), ("dt_mechanics", C.c_float),
                ("flags", C.c_uint32)]


class BatchOptions(C.Structure):
    _fields_ = [("use_graphs", C.c_int), ("autotune", C.c_int), ("tune_cache", C.c_char_p),
                ("profile_phases", C.c_int), ("pin_x", C.c_int), ("pin_cols", C.c_int),
                ("disable_planes", C.c_int), ("pin_forces", C.c_int), ("pin_cell_threads", C.c_int)]


class ServeOptions(C.Structure):
    _fields_ = [("budget_bytes", C.c_uint64), ("max_active", C.c_uint32), ("steps_per_tick", C.c_uint32)]


_lib = None

# (name, restype, argtypes) of every entry point in include/pcg.h
_P = C.c_void_p
_SIGS = [
    ("pcg_abi_version", C.c_int, []),
    ("pcg_create", C.c_int, [C.c_int, C.POINTER(_P)]),
    ("pcg_create_on_stream", C.c_int, [C.c_int, _P, C.POINTER(_P)]),
    ("pcg_destroy", C.c_int, [_P]),
    ("pcg_sync", C.c_int, [_P]),
    ("pcg_stream", _P, [_P]),
    ("pcg_last_error_string", C.c_char_p, [_P]),
    ("pcg_kernel_launches", C.c_uint64, [_P]),
    ("pcg_host_alloc", C.c_int, [C.c_size_t, C.POINTER(_P)]),
    ("pcg_host_free", C.c_int, [_P]),
    ("pcg_me_create", C.c_int, [_P, C.POINTER(GridParams), C.POINTER(SubstrateParams), C.POINTER(_P)]),
    ("pcg_me_destroy", C.c_int, [_P]),
    ("pcg_me_fill", C.c_int, [_P, _F32P]),
    ("pcg_me_upload", C.c_int, [_P, _F32P, C.c_size_t]),
    ("pcg_me_download", C.c_int, [_P, _F32P, C.c_size_t]),
    ("pcg_me_diffuse", C.c_int, [_P, C.c_int]),
    ("pcg_me_apply_dirichlet", C.c_int, [_P]),
    ("pcg_me_secrete", C.c_int, [_P, _P, C.c_double]),
    ("pcg_me_step", C.c_int, [_P, _P, C.c_int]),
    ("pcg_me_gradients", C.c_int, [_P, _F32P, _F32P, _F32P, C.c_size_t]),
    ("pcg_me_device_density", C.c_int, [_P, C.POINTER(_F32P), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    ("pcg_cells_create", C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(_P)]),
    ("pcg_cells_destroy", C.c_int, [_P]),
    ("pcg_cells_upload", C.c_int, [_P, _F32P, C.c_uint32, C.c_uint32]),
    ("pcg_cells_download", C.c_int, [_P, _F32P, C.c_uint32]),
    ("pcg_cells_upload_fields", C.c_int, [_P, C.c_uint32, C.c_uint32, _F32P, C.c_uint32]),
    ("pcg_cells_download_fields", C.c_int, [_P, C.c_uint32, C.c_uint32, _F32P, C.c_uint32]),
    ("pcg_cells_set_secretion", C.c_int, [_P, _F64P, _F64P, _F64P, _F64P, _U8P]),
    ("pcg_cells_count", C.c_int, [_P, _U32P]),
    ("pcg_cells_set_voxel_refresh", C.c_int, [_P, _P, C.c_int]),
    ("pcg_cells_remove", C.c_int, [_P, _U32P, C.c_uint32]),
    ("pcg_removal_plan", C.c_int, [C.c_uint32, _U32P, C.c_uint32, _U32P, _U32P, _U32P, _U32P]),
    ("pcg_cells_append", C.c_int, [_P, _F32P, C.c_uint32, C.c_uint32, _F64P, _F64P, _F64P, _F64P, _U8P]),
    ("pcg_cells_download_secretion", C.c_int, [_P, _F64P, _F64P, _F64P, _F64P, _U8P]),
    ("pcg_cells_device_soa", C.c_int, [_P, C.POINTER(_F32P), _U32P]),
    ("pcg_cells_download_positions64", C.c_int, [_P, _F64P, C.c_uint32]),
    ("pcg_mech_create", C.c_int, [_P, C.POINTER(MechanicsParams), C.c_float, C.c_float, C.c_float,
                                  C.c_uint32, C.POINTER(_P)]),
    ("pcg_mech_destroy", C.c_int, [_P]),
    ("pcg_mech_forces", C.c_int, [_P, _P]),
    ("pcg_mech_integrate", C.c_int, [_P, _P, C.c_float]),
    ("pcg_mech_update", C.c_int, [_P, _P, C.c_float]),
    ("pcg_mech_bins", C.c_int, [_P, _U32P, _U32P]),
    ("pcg_mech_total_voxels", C.c_uint32, [_P]),
    ("pcg_mech_set_diagnostics", C.c_int, [_P, C.c_int]),
    ("pcg_mech_neighbor_stats", C.c_int, [_P, _U32P, _U32P]),
    ("pcg_neighbor_hash", C.c_uint32, [C.c_uint32]),
    ("pcg_motility_create", C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(_P)]),
    ("pcg_motility_destroy", C.c_int, [_P]),
    ("pcg_motility_upload", C.c_int, [_P, C.c_uint32, _F64P, _F64P, _F64P, _F64P, _U32P, _U32P, _I32P, _I32P,
                                      _F64P]),
    ("pcg_motility_download", C.c_int, [_P, _F64P, _F64P]),
    ("pcg_motility_update", C.c_int, [_P, _P, _P, C.c_double, C.c_uint64, C.c_uint64, C.c_int]),
    ("pcg_snapshot_create", C.c_int, [_P, C.POINTER(_P)]),
    ("pcg_snapshot_wait", C.c_int, [_P]),
    ("pcg_snapshot_destroy", C.c_int, [_P]),
    ("pcg_snapshot_microenvironment", C.c_int, [_P, _P, C.c_char_p]),
    ("pcg_snapshot_cells", C.c_int, [_P, _P, C.c_uint32, C.c_char_p]),
    ("pcg_snapshot_frame", C.c_int, [_P, _P, _P, C.c_uint32, C.c_char_p, C.c_int]),
    ("pcg_sort_pairs_static", C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                        C.c_int]),
    ("pcg_batch_create", C.c_int, [_P, C.POINTER(InstanceDesc), C.c_uint32, C.POINTER(BatchOptions),
                                   C.POINTER(_P)]),
    ("pcg_batch_destroy", C.c_int, [_P]),
    ("pcg_batch_step", C.c_int, [_P, C.c_int]),
    ("pcg_batch_download_density", C.c_int, [_P, C.c_uint32, _F32P, C.c_size_t]),
    ("pcg_batch_download_cells", C.c_int, [_P, C.c_uint32, _F32P, C.c_uint32]),
    ("pcg_batch_upload_cells", C.c_int, [_P, C.c_uint32, _F32P, C.c_uint32]),
    ("pcg_batch_download_positions64", C.c_int, [_P, C.c_uint32, _F64P, C.c_uint32]),
    ("pcg_batch_upload_all_cells", C.c_int, [_P, _F32P, C.c_uint64]),
    ("pcg_batch_download_all_cells", C.c_int, [_P, _F32P, C.c_uint64]),
    ("pcg_batch_download_all_density", C.c_int, [_P, _F32P, C.c_uint64]),
    ("pcg_batch_download_cell_fields", C.c_int, [_P, _F32P, C.c_uint64, C.c_uint32]),
    ("pcg_batch_upload_cell_fields", C.c_int, [_P, _F32P, C.c_uint64, C.c_uint32]),
    ("pcg_batch_density_layout", C.c_int, [_P, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                           C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("pcg_join", C.c_int, [_P]),
    ("pcg_batch_totals", C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("pcg_batch_sweep_units", C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("pcg_batch_step_launches", C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("pcg_batch_phase_times", C.c_int, [_P, _F32P, C.POINTER(C.c_uint64), C.c_int]),
    ("pcg_batch_set_profile", C.c_int, [_P, C.c_int]),
    ("pcg_batch_set_diagnostics", C.c_int, [_P, C.c_int]),
    ("pcg_batch_mech_bins", C.c_int, [_P, C.c_uint32, _U32P, _U32P, _U32P, _U32P]),
    ("pcg_batch_describe", C.c_char_p, [_P]),
    ("pcg_serve_create", C.c_int, [_P, C.POINTER(ServeOptions), C.POINTER(_P)]),
    ("pcg_serve_destroy", C.c_int, [_P]),
    ("pcg_serve_create_multi", C.c_int, [C.POINTER(_P), C.c_uint32, C.POINTER(ServeOptions), C.POINTER(_P)]),
    ("pcg_serve_cancel", C.c_int, [_P, C.c_uint64]),
    ("pcg_serve_placement", C.c_int, [_P, C.c_uint64, C.POINTER(C.c_int)]),
    ("pcg_serve_submit", C.c_int, [_P, C.POINTER(InstanceDesc), C.c_uint32, C.POINTER(C.c_uint64)]),
    ("pcg_serve_tick", C.c_int, [_P, _U32P, _U32P, _U32P]),
    ("pcg_serve_state", C.c_int, [_P, C.c_uint64, C.POINTER(C.c_int)]),
    ("pcg_serve_fetch", C.c_int, [_P, C.c_uint64, _F32P, C.c_size_t, _F32P, C.c_uint32]),
    ("pcg_serve_request_times", C.c_int, [_P, C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("pcg_serve_totals", C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("pcg_instance_bytes", C.c_uint64, [C.POINTER(InstanceDesc)]),
    ("pcg_debug_alloc_stats", None, [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("pcg_debug_fail_alloc", None, [C.c_uint64]),
    ("pcg_debug_give_up_waits", C.c_int, [_P, C.c_int]),
]


def lib():
    """Load libpcg.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PcgError(-1, f"{LIB_PATH} not built; run __graft_entry__.build() or make in the package")
        L = C.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def removal_plan(n_cells, indices):
    """Host-only moves of a dead-cell compaction: (dest, src, n_final), the
    cell that started at src[k] ends at dest[k]."""
    idx = np.ascontiguousarray(indices, np.uint32)
    dest = np.zeros(max(idx.size, 1), np.uint32)
    src = np.zeros(max(idx.size, 1), np.uint32)
    nm, nf = C.c_uint32(), C.c_uint32()
    st = lib().pcg_removal_plan(n_cells, _u32(idx), idx.size, _u32(dest), _u32(src), C.byref(nm), C.byref(nf))
    if st != PCG_OK:
        raise PcgError(st, "pcg_removal_plan")
    return dest[:nm.value], src[:nm.value], nf.value


def exported_symbols():
    return [s[0] for s in _SIGS]


def _f32(a):
    return a.ctypes.data_as(_F32P) if a is not None else None


def _f64(a):
    return a.ctypes.data_as(_F64P) if a is not None else None


def _u32(a):
    return a.ctypes.data_as(_U32P) if a is not None else None


def _u8(a):
    return a.ctypes.data_as(_U8P) if a is not None else None


def make_grid(nx, ny, nz, S, dx=20.0, dt=0.01, x_min=0.0, y_min=0.0, z_min=0.0, dy=None, dz=None):
    return GridParams(nx, ny, nz, S, dx, dy if dy is not None else dx, dz if dz is not None else dx, dt,
                      x_min, y_min, z_min, 0.0)


def make_substrates(params):
    """params: iterable of (D, decay, dirichlet_enabled, target[, consistent]);
    consistent: the consistent Dirichlet option (pcg_substrate_params)."""
    params = list(params)
    arr = (SubstrateParams * max(1, len(params)))()
    for s, p in enumerate(params):
        D, lam, dirichlet, T = p[:4]
        arr[s].dirichlet_consistent = 1 if len(p) > 4 and p[4] else 0
        arr[s].diffusion_coefficient = D
        arr[s].decay_rate = lam
        arr[s].supply_rate = 0.0
        arr[s].target_value = T
        arr[s].dirichlet_enabled = 1 if dirichlet else 0
    return arr


def mech_params_for_domain(x_min, x_max, y_min, y_max, z_min, z_max, use_2d, dt_mech=0.1, voxel=30.0):
    """CellMechanics::initialize grid rule (src/cell_mechanics.mm:26-41):
    30 um voxels, truncation, at least 1, nz = 1 in 2-D (FP32 arithmetic)."""
    f = np.float32
    vs = f(voxel)

    def n_of(lo, hi):
        return max(1, int(np.uint32(f(f(hi) - f(lo)) / vs)))
    return MechanicsParams(dt_mech, 10.0, 0.4, voxel, voxel, n_of(x_min, x_max), n_of(y_min, y_max),
                           1 if use_2d else n_of(z_min, z_max))


class Context:
    """pcg_ctx: device, CUDA stream, error reporting (replaces MetalContext)."""

    def __init__(self, device=0, stream=None):
        L = lib()
        h = _P()
        st = L.pcg_create(device, C.byref(h)) if stream is None else \
            L.pcg_create_on_stream(device, C.c_void_p(stream), C.byref(h))
        if st != PCG_OK:
            raise PcgError(st, (L.pcg_last_error_string(None) or b"").decode())
        self.h = h
        self.device = device

    def check(self, st):
        if st != PCG_OK:
            raise PcgError(st, (lib().pcg_last_error_string(self.h) or b"").decode())

    def sync(self):
        self.check(lib().pcg_sync(self.h))

    def join(self):
        """Order the context stream after the whole-batch host copies issued so far."""
        self.check(lib().pcg_join(self.h))

    @property
    def stream(self):
        return lib().pcg_stream(self.h)

    @property
    def launches(self):
        return int(lib().pcg_kernel_launches(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().pcg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PinnedArray:
    """numpy view of page-locked host memory from pcg_host_alloc."""

    def __init__(self, shape, dtype=np.float32):
        dtype = np.dtype(dtype)
        n = int(np.prod(shape)) * dtype.itemsize
        p = _P()
        st = lib().pcg_host_alloc(max(n, 1), C.byref(p))
        if st != PCG_OK:
            raise PcgError(st, "pinned allocation failed")
        self.p = p
        buf = (C.c_char * max(n, 1)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    def free(self):
        if self.p:
            self.array = None
            lib().pcg_host_free(self.p)
            self.p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Microenvironment:
    """Microenvironment (src/microenvironment.h:17-83) on the device."""

    def __init__(self, ctx, grid, substrates):
        self.ctx = ctx
        self.grid = grid
        self.S = grid.n_substrates
        self.substrates = substrates
        h = _P()
        ctx.check(lib().pcg_me_create(ctx.h, C.byref(grid), substrates, C.byref(h)))
        self.h = h
        self.n = grid.nx * grid.ny * grid.nz * grid.n_substrates

    def numVoxels(self):
        return self.grid.nx * self.grid.ny * self.grid.nz

    def fill(self, values):
        v = np.ascontiguousarray(values, np.float32)
        self.ctx.check(lib().pcg_me_fill(self.h, _f32(v)))

    def setDensityAll(self, density):
        d = np.ascontiguousarray(density, np.float32).ravel()
        self.ctx.check(lib().pcg_me_upload(self.h, _f32(d), d.size))

    def densityBuffer(self):
        out = np.empty(self.n, np.float32)
        self.ctx.check(lib().pcg_me_download(self.h, _f32(out), out.size))
        return out

    def simulateDiffusionDecay(self, n_steps=1):
        self.ctx.check(lib().pcg_me_diffuse(self.h, n_steps))

    def applyDirichletBC(self):
        self.ctx.check(lib().pcg_me_apply_dirichlet(self.h))

    def applySecretion(self, cells, dt):
        self.ctx.check(lib().pcg_me_secrete(self.h, cells.h, float(dt)))

    def step(self, cells=None, n_steps=1):
        self.ctx.check(lib().pcg_me_step(self.h, cells.h if cells is not None else None, n_steps))

    def computeGradients(self):
        gx = np.empty(self.n, np.float32)
        gy = np.empty(self.n, np.float32)
        gz = np.empty(self.n, np.float32)
        self.ctx.check(lib().pcg_me_gradients(self.h, _f32(gx), _f32(gy), _f32(gz), self.n))
        return gx, gy, gz

    def close(self):
        if getattr(self, "h", None):
            lib().pcg_me_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Cells:
    """The GPU-shared 28-field SoA block of CellData on the device."""

    def __init__(self, ctx, max_cells, n_substrates):
        self.ctx = ctx
        self.S = n_substrates
        self.max_cells = max_cells
        h = _P()
        ctx.check(lib().pcg_cells_create(ctx.h, max_cells, n_substrates, C.byref(h)))
        self.h = h
        self.n = 0

    def upload(self, soa, n_cells, soa_max):
        soa = np.ascontiguousarray(soa, np.float32)
        assert soa.size >= NUM_FIELDS * soa_max
        self.ctx.check(lib().pcg_cells_upload(self.h, _f32(soa), n_cells, soa_max))
        self.n = n_cells

    def download(self, soa_max=None):
        soa_max = soa_max or max(self.n, 1)
        out = np.zeros(NUM_FIELDS * soa_max, np.float32)
        self.ctx.check(lib().pcg_cells_download(self.h, _f32(out), soa_max))
        return out

    def set_voxel_refresh(self, me, on=True):
        """Recompute voxel indices on me's grid after every integrate."""
        self.ctx.check(lib().pcg_cells_set_voxel_refresh(self.h, me.h if me is not None else None, 1 if on else 0))

    def positions64(self):
        """FP64 master positions of the current cells: (3, n) array."""
        n = self.count()
        out = np.zeros(3 * max(n, 1), np.float64)
        self.ctx.check(lib().pcg_cells_download_positions64(self.h, _f64(out), n))
        return out[:3 * n].reshape(3, n)

    def upload_fields(self, first, count, soa, soa_max):
        soa = np.ascontiguousarray(soa, np.float32)
        self.ctx.check(lib().pcg_cells_upload_fields(self.h, first, count, _f32(soa), soa_max))

    def set_secretion(self, sec=None, upt=None, sat=None, ne=None, active=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (sec, upt, sat, ne)]
        act = None if active is None else np.ascontiguousarray(active, np.uint8)
        self._keep = (arrs, act)
        self.ctx.check(lib().pcg_cells_set_secretion(self.h, *[_f64(a) for a in arrs], _u8(act)))

    def download_secretion(self):
        """(secretion, uptake, saturation, net_export, active) of the current cells."""
        k = self.n * self.S
        arrs = [np.zeros(max(k, 1), np.float64) for _ in range(4)]
        act = np.zeros(max(self.n, 1), np.uint8)
        self.ctx.check(lib().pcg_cells_download_secretion(self.h, *[_f64(a) for a in arrs], _u8(act)))
        return tuple(a[:k] for a in arrs) + (act[:self.n],)

    def count(self):
        n = C.c_uint32()
        self.ctx.check(lib().pcg_cells_count(self.h, C.byref(n)))
        self.n = n.value
        return self.n

    def remove(self, indices):
        """Dead-cell compaction (CellData::removeCell for each index in
        descending order, cell_phenotype.cpp:838-844) on the device; returns
        the new count."""
        idx = np.ascontiguousarray(indices, np.uint32)
        self.ctx.check(lib().pcg_cells_remove(self.h, _u32(idx), idx.size))
        return self.count()

    def append(self, soa, count, soa_max, sec=None, upt=None, sat=None, ne=None, active=None):
        """New cells after the current ones (CellData::addCell); returns the new count."""
        soa = np.ascontiguousarray(soa, np.float32)
        assert soa.size >= NUM_FIELDS * soa_max
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (sec, upt, sat, ne)]
        act = None if active is None else np.ascontiguousarray(active, np.uint8)
        self.ctx.check(lib().pcg_cells_append(self.h, _f32(soa), count, soa_max, *[_f64(a) for a in arrs], _u8(act)))
        return self.count()

    def close(self):
        if getattr(self, "h", None):
            lib().pcg_cells_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


MOT_REFERENCE, MOT_SUBSTRATE_MAJOR = 0, 1


class Motility:
    """MotilityData (src/motility.h:10-50) resident on the device, with
    updateMotility (src/motility.cpp:179-293).  'state' is a dict of the
    per-cell arrays: persistence_time, elapsed, bias, vec (3 * n: x, y, z),
    is_motile, restrict_2d, chemotaxis_index, chemotaxis_direction and
    sensitivity (n * S, or None for the single-substrate rule)."""

    def __init__(self, ctx, max_cells, n_substrates=0):
        self.ctx = ctx
        self.S = n_substrates
        h = _P()
        ctx.check(lib().pcg_motility_create(ctx.h, max_cells, n_substrates, C.byref(h)))
        self.h = h
        self.n = 0

    def upload(self, state):
        n = len(state["persistence_time"])
        f64 = lambda k: np.ascontiguousarray(state[k], np.float64)
        arrs = [f64("persistence_time"), f64("elapsed"), f64("bias"), f64("vec"),
                np.ascontiguousarray(state["is_motile"], np.uint32),
                np.ascontiguousarray(state["restrict_2d"], np.uint32),
                np.ascontiguousarray(state["chemotaxis_index"], np.int32),
                np.ascontiguousarray(state["chemotaxis_direction"], np.int32)]
        sens = state.get("sensitivity")
        sens = None if sens is None else np.ascontiguousarray(sens, np.float64)
        ptrs = [_f64(arrs[0]), _f64(arrs[1]), _f64(arrs[2]), _f64(arrs[3]), _u32(arrs[4]), _u32(arrs[5]),
                arrs[6].ctypes.data_as(_I32P), arrs[7].ctypes.data_as(_I32P), _f64(sens) if sens is not None else None]
        self.ctx.check(lib().pcg_motility_upload(self.h, n, *ptrs))
        self.n = n

    def download(self):
        el = np.zeros(max(self.n, 1))
        vec = np.zeros(max(3 * self.n, 3))
        self.ctx.check(lib().pcg_motility_download(self.h, _f64(el), _f64(vec)))
        return el[:self.n], vec[:3 * self.n]

    def update(self, cells, me, dt, seed, step, layout=MOT_REFERENCE):
        self.ctx.check(lib().pcg_motility_update(self.h, cells.h, me.h if me is not None else None, dt,
                                                 C.c_uint64(seed), C.c_uint64(step), layout))

    def close(self):
        if getattr(self, "h", None):
            lib().pcg_motility_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Snapshot:
    """Asynchronous .mat snapshots (writeMatlabSnapshots,
    src/output_writer.cpp:295-452)."""

    def __init__(self, ctx):
        self.ctx = ctx
        h = _P()
        ctx.check(lib().pcg_snapshot_create(ctx.h, C.byref(h)))
        self.h = h

    def microenvironment(self, me, path):
        self.ctx.check(lib().pcg_snapshot_microenvironment(self.h, me.h, str(path).encode()))

    def cells(self, cells, path, n_cell_types=1):
        self.ctx.check(lib().pcg_snapshot_cells(self.h, cells.h, n_cell_types, str(path).encode()))

    def frame(self, me, cells, folder, frame, n_cell_types=1):
        self.ctx.check(lib().pcg_snapshot_frame(self.h, me.h if me is not None else None,
                                                cells.h if cells is not None else None, n_cell_types,
                                                str(folder).encode(), frame))

    def wait(self):
        self.ctx.check(lib().pcg_snapshot_wait(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().pcg_snapshot_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CellMechanics:
    """CellMechanics (src/cell_mechanics.h:15-87) on the device."""

    def __init__(self, ctx, params, origin, max_cells):
        self.ctx = ctx
        self.params = params
        h = _P()
        ctx.check(lib().pcg_mech_create(ctx.h, C.byref(params), origin[0], origin[1], origin[2], max_cells,
                                        C.byref(h)))
        self.h = h

    def totalMechVoxels(self):
        return int(lib().pcg_mech_total_voxels(self.h))

    def computeForces(self, cells):
        self.ctx.check(lib().pcg_mech_forces(self.h, cells.h))

    def integratePositions(self, cells, dt):
        self.ctx.check(lib().pcg_mech_integrate(self.h, cells.h, float(dt)))

    def update(self, cells, dt):
        self.ctx.check(lib().pcg_mech_update(self.h, cells.h, float(dt)))

    def syncHashPointers(self, n_cells):
        """Returns (start[V+1], sorted_cells[n]): voxelCellCount(v) =
        start[v+1]-start[v], voxelCells(v) = sorted_cells[start[v]:start[v+1]]."""
        start = np.zeros(self.totalMechVoxels() + 1, np.uint32)
        cells = np.zeros(max(n_cells, 1), np.uint32)
        self.ctx.check(lib().pcg_mech_bins(self.h, _u32(start), _u32(cells)))
        return start, cells[:n_cells]

    def set_diagnostics(self, on=True):
        self.ctx.check(lib().pcg_mech_set_diagnostics(self.h, 1 if on else 0))

    def neighbor_stats(self, n_cells):
        cnt = np.zeros(max(n_cells, 1), np.uint32)
        hsh = np.zeros(max(n_cells, 1), np.uint32)
        self.ctx.check(lib().pcg_mech_neighbor_stats(self.h, _u32(cnt), _u32(hsh)))
        return cnt[:n_cells], hsh[:n_cells]

    def close(self):
        if getattr(self, "h", None):
            lib().pcg_mech_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Instance:
    """Host-side description of one simulation (keeps its arrays alive)."""

    def __init__(self, grid, substrates, mech, dt_mechanics, density=None, initial_values=None, soa=None,
                 n_cells=0, soa_max=None, sec=None, upt=None, sat=None, ne=None, active=None, flags=0):
        self.grid = grid
        self.substrates = substrates
        self.density = None if density is None else np.ascontiguousarray(density, np.float32)
        self.initial_values = None if initial_values is None else np.ascontiguousarray(initial_values, np.float32)
        self.soa = None if soa is None else np.ascontiguousarray(soa, np.float32)
        self.n_cells = n_cells
        self.soa_max = soa_max if soa_max is not None else n_cells
        self.rates = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (sec, upt, sat, ne)]
        self.active = None if active is None else np.ascontiguousarray(active, np.uint8)
        self.mech = mech
        self.dt_mechanics = dt_mechanics
        self.flags = flags

    def desc(self):
        d = InstanceDesc()
        d.grid = self.grid
        d.substrates = C.cast(self.substrates, C.POINTER(SubstrateParams))
        d.initial_density = _f32(self.density)
        d.initial_values = _f32(self.initial_values)
        d.n_cells = self.n_cells
        d.cells_soa = _f32(self.soa)
        d.cells_soa_max = self.soa_max
        d.secretion, d.uptake, d.saturation, d.net_export = [_f64(a) for a in self.rates]
        d.active = _u8(self.active)
        d.mech = self.mech
        d.dt_mechanics = self.dt_mechanics
        d.flags = self.flags
        return d

    def bytes(self):
        d = self.desc()
        return int(lib().pcg_instance_bytes(C.byref(d)))


class Batch:
    """pcg_batch: many simulations advanced in one graph launch per sub-step
    (per mechanics period where a call covers one)."""

    def __init__(self, ctx, instances, use_graphs=True, autotune=True, tune_cache=None, profile=False,
                 pin_x=0, pin_cols=0, planes=True, pin_forces=0, pin_cell_threads=0):
        """pin_x / pin_cols: launch shape warps * 16 + stages of the x /
        column sweeps instead of the tuned one (0 = tuned).  planes=False:
        x and y sweeps as separate passes even where a plane fits.
        pin_forces: force pass threads * 1000 + queue slots; pin_cell_threads:
        threads per block of the secretion, binning and AB2 kernels (0 =
        tuned)."""
        self.ctx = ctx
        self.instances = list(instances)
        arr = (InstanceDesc * len(self.instances))(*[i.desc() for i in self.instances])
        opt = BatchOptions(1 if use_graphs else 0, 1 if autotune else 0,
                           tune_cache.encode() if tune_cache else None, 1 if profile else 0, pin_x, pin_cols,
                           0 if planes else 1, pin_forces, pin_cell_threads)
        h = _P()
        ctx.check(lib().pcg_batch_create(ctx.h, arr, len(self.instances), C.byref(opt), C.byref(h)))
        self.h = h

    def step(self, n_steps=1):
        self.ctx.check(lib().pcg_batch_step(self.h, n_steps))

    def density(self, i):
        inst = self.instances[i]
        g = inst.grid
        out = np.empty(g.nx * g.ny * g.nz * g.n_substrates, np.float32)
        self.ctx.check(lib().pcg_batch_download_density(self.h, i, _f32(out), out.size))
        return out

    def cells(self, i):
        n = self.instances[i].n_cells
        out = np.zeros(NUM_FIELDS * max(n, 1), np.float32)
        self.ctx.check(lib().pcg_batch_download_cells(self.h, i, _f32(out), max(n, 1)))
        return out

    def upload_cells(self, i, soa, soa_max):
        soa = np.ascontiguousarray(soa, np.float32)
        self.ctx.check(lib().pcg_batch_upload_cells(self.h, i, _f32(soa), soa_max))

    def positions64(self, i):
        """Instance i's FP64 master positions: (3, n) array (x, y, z)."""
        n = self.instances[i].n_cells
        out = np.zeros(3 * max(n, 1), np.float64)
        self.ctx.check(lib().pcg_batch_download_positions64(self.h, i, _f64(out), n))
        return out[:3 * n].reshape(3, n)

    def totals(self):
        v, vs, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.ctx.check(lib().pcg_batch_totals(self.h, C.byref(v), C.byref(vs), C.byref(c)))
        return v.value, vs.value, c.value

    def sweep_units(self):
        """(plane_units, all_units): voxel-substrates one sub-step's plane
        launches / all sweep launches cover (8 bytes each)."""
        pu, au = C.c_uint64(), C.c_uint64()
        self.ctx.check(lib().pcg_batch_sweep_units(self.h, C.byref(pu), C.byref(au)))
        return pu.value, au.value

    def layout(self, i):
        """(offset, row_pitch, substrate_pitch, arena_floats) of instance i's density on the device."""
        off, rp, pitch, arena = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.ctx.check(lib().pcg_batch_density_layout(self.h, i, C.byref(off), C.byref(rp), C.byref(pitch),
                                                      C.byref(arena)))
        return off.value, rp.value, pitch.value, arena.value

    def upload_all_cells(self, soa):
        self.ctx.check(lib().pcg_batch_upload_all_cells(self.h, _f32(soa), soa.size))

    def download_all_cells(self, soa):
        self.ctx.check(lib().pcg_batch_download_all_cells(self.h, _f32(soa), soa.size))

    def download_cell_fields(self, soa, mask=None):
        """download_all_cells for the fields in 'mask' (bit f = field f;
        default: the fields the steps write, STEP_WRITTEN_FIELDS)."""
        m = STEP_WRITTEN_FIELDS if mask is None else int(mask)
        self.ctx.check(lib().pcg_batch_download_cell_fields(self.h, _f32(soa), soa.size, m))

    def upload_cell_fields(self, soa, mask=None):
        """upload_all_cells for the fields in 'mask' (default: the fields the
        host owns, HOST_OWNED_FIELDS); the device keeps its other fields."""
        m = HOST_OWNED_FIELDS if mask is None else int(mask)
        self.ctx.check(lib().pcg_batch_upload_cell_fields(self.h, _f32(soa), soa.size, m))

    def download_all_density(self, dens):
        self.ctx.check(lib().pcg_batch_download_all_density(self.h, _f32(dens), dens.size))

    def step_launches(self):
        a, b = C.c_uint64(), C.c_uint64()
        self.ctx.check(lib().pcg_batch_step_launches(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_profile(self, on):
        self.ctx.check(lib().pcg_batch_set_profile(self.h, 1 if on else 0))

    def phase_times(self, reset=True):
        ms = np.zeros(N_PHASES, np.float32)
        n = C.c_uint64()
        self.ctx.check(lib().pcg_batch_phase_times(self.h, _f32(ms), C.byref(n), 1 if reset else 0))
        return dict(zip(PHASES, ms.tolist())), n.value

    def describe(self):
        return (lib().pcg_batch_describe(self.h) or b"").decode()

    def set_diagnostics(self, on=True):
        self.ctx.check(lib().pcg_batch_set_diagnostics(self.h, 1 if on else 0))

    def mech_bins(self, i, stats=False):
        """Instance i after its last mechanics step: (start[V+1],
        sorted_cells[n]) and, with stats (diagnostics on), the neighbour
        counts and hashes by cell."""
        inst = self.instances[i]
        m, n = inst.mech, inst.n_cells
        start = np.zeros(m.mech_grid_nx * m.mech_grid_ny * m.mech_grid_nz + 1, np.uint32)
        order = np.zeros(max(n, 1), np.uint32)
        cnt = np.zeros(max(n, 1), np.uint32) if stats else None
        hsh = np.zeros(max(n, 1), np.uint32) if stats else None
        self.ctx.check(lib().pcg_batch_mech_bins(self.h, i, _u32(start), _u32(order), _u32(cnt), _u32(hsh)))
        if stats:
            return start, order[:n], cnt[:n], hsh[:n]
        return start, order[:n]

    def close(self):
        if getattr(self, "h", None):
            lib().pcg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """pcg_server: continuous batching of simulation requests.  ctx may be
    one Context or a list of them (one per GPU, pcg_serve_create_multi);
    budget_bytes and max_active then apply to each."""

    def __init__(self, ctx, budget_bytes=150e9, max_active=0, steps_per_tick=100):
        ctxs = list(ctx) if isinstance(ctx, (list, tuple)) else [ctx]
        self.ctx = ctxs[0]
        self.ctxs = ctxs
        opt = ServeOptions(int(budget_bytes), max_active, steps_per_tick)
        h = _P()
        arr = (_P * len(ctxs))(*[c.h for c in ctxs])
        self.ctx.check(lib().pcg_serve_create_multi(arr, len(ctxs), C.byref(opt), C.byref(h)))
        self.h = h
        self.requests = {}

    def cancel(self, rid):
        self.ctx.check(lib().pcg_serve_cancel(self.h, rid))

    def placement(self, rid):
        """Index of the context request rid runs on (-1 while queued)."""
        k = C.c_int()
        self.ctx.check(lib().pcg_serve_placement(self.h, rid, C.byref(k)))
        return k.value

    def submit(self, inst, n_steps):
        d = inst.desc()
        rid = C.c_uint64()
        self.ctx.check(lib().pcg_serve_submit(self.h, C.byref(d), n_steps, C.byref(rid)))
        self.requests[rid.value] = inst
        return rid.value

    def tick(self):
        r, q, f = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self.ctx.check(lib().pcg_serve_tick(self.h, C.byref(r), C.byref(q), C.byref(f)))
        return r.value, q.value, f.value

    def state(self, rid):
        s = C.c_int()
        self.ctx.check(lib().pcg_serve_state(self.h, rid, C.byref(s)))
        return s.value

    def fetch(self, rid):
        inst = self.requests[rid]
        g = inst.grid
        dens = np.empty(g.nx * g.ny * g.nz * g.n_substrates, np.float32)
        n = max(inst.n_cells, 1)
        soa = np.zeros(NUM_FIELDS * n, np.float32)
        self.ctx.check(lib().pcg_serve_fetch(self.h, rid, _f32(dens), dens.size, _f32(soa), n))
        return dens, soa

    def times(self, rid):
        a, b = C.c_double(), C.c_double()
        self.ctx.check(lib().pcg_serve_request_times(self.h, rid, C.byref(a), C.byref(b)))
        return a.value, b.value

    def totals(self):
        v, c, b = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.ctx.check(lib().pcg_serve_totals(self.h, C.byref(v), C.byref(c), C.byref(b)))
        return v.value, c.value, b.value

    def close(self):
        if getattr(self, "h", None):
            lib().pcg_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build(verbose=False):
    """Compile libpcg.so in place for sm_100a (make in this directory)."""
    import subprocess
    out = None if verbose else subprocess.DEVNULL
    subprocess.run(["make", "-j8", "-C", HERE], check=True, stdout=out)
