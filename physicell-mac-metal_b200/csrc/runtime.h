// runtime.h — host runtime behind the C ABI: device buffers, the diffusion /
// cell / mechanics engines shared by the single-simulation API, the batch
// and the server, launch-shape selection and the autotuner.
#pragma once

#include <atomic>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "pcg.h"
#include "pcg_kernels.cuh"

struct pcg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    int sms = 0;
    int smem_optin = 0;
    uint64_t launches = 0;
    unsigned* status = nullptr;   // device status word (PCG_DEV_* bits)
    // copy streams of the whole-batch transfers (made on first use): host
    // copies run there, beside the kernels on 'stream'
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t copy_ev[2] = {};
    // side streams for the independent launches of one phase (made on first
    // use): they fork from 'stream' at an event and 'stream' waits for each
    // of them before the phase's next launch, so captured graphs hold them
    // as parallel branches
    static constexpr int kForks = 8;
    cudaStream_t fork_st[kForks] = {};
    cudaEvent_t fork_ev[kForks + 1] = {};   // [0] fork, [1 + q] join of side stream q
    // the owner's reference (dropped by pcg_destroy) plus one per live object
    // made on this context: the context, its streams and its status word are
    // freed with the last reference, so objects may be destroyed after it
    std::atomic<int> refs{1};
};

namespace pcg {

int fail(pcg_ctx* ctx, int code, const std::string& msg);
void ctx_retain(pcg_ctx* ctx);    // an object made on ctx holds it
void ctx_release(pcg_ctx* ctx);   // ... and lets it go after its own teardown
int cuda_fail(pcg_ctx* ctx, cudaError_t e, const char* what);

#define PCG_CU(ctx, call)                                                   \
    do {                                                                    \
        cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess) return ::pcg::cuda_fail((ctx), e_, #call);   \
    } while (0)
#define PCG_TRY(x)                    \
    do {                              \
        int r_ = (x);                 \
        if (r_ != PCG_OK) return r_;  \
    } while (0)

// Allocations made while an AllocStream is alive (on this thread) come
// from the stream-ordered device pool and go back to it on release, tied to
// that stream; without one, DevBuf uses cudaMalloc / cudaFree.
class AllocStream {
public:
    explicit AllocStream(cudaStream_t s);
    ~AllocStream();
    AllocStream(const AllocStream&) = delete;
    AllocStream& operator=(const AllocStream&) = delete;
private:
    cudaStream_t prev_;
};

// Device allocation owned by the library.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes), cap_(o.cap_), stream_(o.stream_), dev_(o.dev_)
    {
        o.p = nullptr;
        o.bytes = 0;
        o.cap_ = 0;
        o.stream_ = nullptr;
    }
    DevBuf& operator=(DevBuf&& o) noexcept
    {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            cap_ = o.cap_;
            stream_ = o.stream_;
            dev_ = o.dev_;
            o.p = nullptr;
            o.bytes = 0;
            o.cap_ = 0;
            o.stream_ = nullptr;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    cudaError_t alloc(size_t b);
    void release();
    template <class T>
    T* as() const { return static_cast<T*>(p); }
private:
    size_t cap_ = 0;                   // pool block size (0: cudaMalloc)
    cudaStream_t stream_ = nullptr;    // stream the pool block is ordered on
    int dev_ = 0;                      // device of the pool block
};

// Device allocations the library has made with cudaMalloc, and pool blocks
// it has handed out again, since the process started.
void alloc_stats(uint64_t* mallocs, uint64_t* reuses);
// Failure injection on the host: the nth DevBuf allocation from now fails
// with cudaErrorMemoryAllocation without touching the device (0 = off).
void fail_alloc_after(uint64_t nth);

// Page-locked host allocation (staging for end-to-end copies).
struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
    HostBuf() = default;
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
    ~HostBuf() { release(); }
    cudaError_t alloc(size_t b);
    void release();
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// ------------------------------------------------------------------ tuning

// Launch-shape choices, cached by shape bucket (process-wide, optionally
// persisted as JSON).
class Tuner {
public:
    static Tuner& get();
    bool lookup(const std::string& key, int* value);
    void store(const std::string& key, int value);
    void load(const std::string& path);
    void save(const std::string& path);
private:
    std::map<std::string, int> table_;
};

// ------------------------------------------------------------------ diffusion

struct DiffInstance {
    pcg_grid_params g{};
    std::vector<pcg_substrate_params> subs;
    uint64_t dens_off = 0;
    uint64_t pitch = 0;       // elements between substrates (multiple of 32)
    uint32_t px = 0;          // row pitch: nx rounded up to 4 floats (16-byte rows)
    uint32_t vox_base = 0;
    uint64_t nvox() const { return static_cast<uint64_t>(g.nx) * g.ny * g.nz; }
    uint64_t rows() const { return static_cast<uint64_t>(g.ny) * g.nz; }
    int ndim() const { return g.nz > 1 ? 3 : 2; }
};

// Plane jobs launched together: the planes whose shared memory allows the
// same number of CTAs per SM, launched with the largest one's size.
struct PlaneList {
    DevBuf jobs;
    uint32_t n = 0;
    uint32_t floats = 0;       // largest plane_floats of the jobs
    uint64_t units = 0;        // voxel-substrates covered
};

struct SweepList {
    int kind = 0;              // 0 row tiles (TMA), 1 column tiles (TMA), 2 any length (global)
    int nmax = 0;
    uint32_t n = 0;
    DevBuf tiles;
    TmaCfg tc{4, 3, 0, 1};
    int ggrid = 1;
    uint64_t lines = 0;        // lines covered (for tuning keys)
    uint64_t units = 0;        // voxel-substrates covered
};

class Diffusion {
public:
    pcg_ctx* ctx = nullptr;
    std::vector<DiffInstance> inst;
    uint64_t dens_elems = 0;
    uint64_t total_vox = 0;        // sum nx*ny*nz
    uint64_t total_vox_sub = 0;    // sum nx*ny*nz*S
    DevBuf dens, rules, tab, faces, grad_jobs, tmaps;
    uint32_t n_faces = 0;
    std::vector<SweepList> lists[3];
    // Instances whose x-y planes fit shared memory run their x and y sweeps
    // as one plane pass (planes); rest[0] / rest[1] hold the x / y tiles of
    // the others.  sweep(0) then launches planes + rest[0], sweep(1) rest[1].
    std::vector<PlaneList> planes;
    // 3-D instances whose x-z planes fit run their z sweep as one pass per
    // x-z plane (zplanes); rest[2] holds the z tiles of the others.
    std::vector<PlaneList> zplanes;
    std::vector<SweepList> rest[3];
    bool use_planes = true;            // set before build()
    std::string shapes;

    // Lays out the density arena, builds the Thomas tables and the tile
    // lists; 'tune' measures launch shapes on the data (density must be
    // initialised first when tuning, see tune()).
    int build(pcg_ctx* c, std::vector<DiffInstance> instances);
    int tune();                                    // restore-safe: density is saved and put back
    int pin(int kind, int param);                  // one shape for every TMA list of a kind (0 x, 1 columns)
    int sweep(int axis, bool fuse_faces, const uint8_t* mask);
    int sweeps(bool fuse_faces, const uint8_t* mask);
    int dirichlet();
    int gradients(float* gx, float* gy, float* gz);   // device arrays of total_vox_sub floats, dense per instance
    int upload(uint32_t i, const float* host, bool async_pinned = false);
    int download(uint32_t i, float* host, bool async_pinned = false);
    int fill(uint32_t i, const float* values);
    int launches_per_step(bool three_d_only = false) const;
    // Plane launches: runs of 'merge' consecutive occupancy classes share
    // one launch (at the largest plane's shared memory); 1 = one launch per
    // class, 0 = one launch per pass.  Chosen by tune() unless pinned.
    int plane_merge = 1;
    int regroup_planes(int merge);
    // Voxel-substrates the sweep launches of one sub-step cover, summed over
    // launches (each moves 8 bytes per unit: one read, one write).
    uint64_t sweep_units_per_step() const;
    uint64_t device_bytes() const;
    std::string describe() const;

private:
    int build_axis(int axis, const std::vector<uint8_t>* skip, std::vector<SweepList>& ls);
    int build_planes();
    // plane jobs per occupancy class (class kPlaneClasses - k: k CTAs per
    // SM), their largest plane and the voxel-substrates they cover
    static constexpr int kPlaneClasses = 32;
    std::vector<PlaneJob> cls_jobs_[2][kPlaneClasses];
    uint32_t cls_floats_[2][kPlaneClasses] = {};
    uint64_t cls_units_[2][kPlaneClasses] = {};
    std::vector<uint8_t> plane_inst_;    // instance's x + y sweeps run as planes
    std::vector<uint8_t> zplane_inst_;   // instance's z sweep runs as x-z planes
    int launch_planes(const std::vector<PlaneList>& pls, bool fuse_faces, const uint8_t* mask);
    int prepare_forks();   // the side streams launch_planes forks to
    bool planes_for(int axis) const { return axis < 2 ? !planes.empty() : !zplanes.empty(); }
    int default_configs(int axis);
    int config_list(SweepList& l, int param);
    int launch_list(const SweepList& l, bool fuse_faces, const uint8_t* mask);
    std::vector<LineRule> h_rules_;
    std::vector<float> h_tab_;
    std::vector<uint32_t> rule_index_;   // (inst, s, axis) -> rule
    std::vector<uint8_t> tensor_ok_;     // rule has a 3-D tensor map (column tiles)
    uint32_t rule_of(size_t i, uint32_t s, int axis) const;
};

// ------------------------------------------------------------------ cells

class Cells {
public:
    pcg_ctx* ctx = nullptr;
    uint32_t max_cells = 0;
    uint32_t n = 0;
    uint32_t n_rate = 0;          // sum over instances of n_cells * S
    std::vector<CellInst> h_inst;
    DevBuf inst, soa, cell_inst, rates, coef, coef_cells, coef_flags, active;
    // FP64 master positions, three arrays of max_cells (x, y, z); the SoA's
    // FP32 positions are their rounding.  The AB2 update starts from a
    // master only while it rounds to the SoA's value, so a position written
    // through the SoA (uploads, host edits) replaces the master.  All-ones
    // (NaN) = no master.
    DevBuf pos64;
    int sec_block = 256;   // threads per block of the secretion kernel
    bool has_active = false;
    bool inst_dirty = true, coef_dirty = true, order_dirty = true;
    double coef_dt = -1.0;
    // secretion ordering (launch_sec_order): keys the first pass's keys in
    // cell order, (skeys, sorder) the order, ktmp / vtmp the passes' work
    // arrays; after the sort ktmp[n] holds the run count and vals the run
    // starts; coef the
    // constants in sorted order (c0, c1, c2 arrays), coef_cells the same
    // constants in cell order (coef_dirty: stale) and coef_flags which of
    // c0 / c1 each instance has.  tiles: the instances' 2048-cell tiles
    // (rebuilt with the instance table), so_passes x so_bits the digits.
    DevBuf keys, vals, skeys, sorder, ktmp, vtmp, sort_scr, run_scr, tiles, inst_tile;
    DevBuf run_word;   // per run: instance and density element of its voxel (make_run_word)
    uint32_t invalid_key = 0;
    uint32_t ntiles = 0, max_tiles = 0, n_inst_tiled = 0;
    int so_passes = 1, so_bits = 0;
    // kernel launches of one build_order (constants already in cell order)
    int order_launches() const;
    // the constants in cell order, when stale (cap: rate capacity)
    int cell_constants(uint32_t cap);

    int create(pcg_ctx* c, uint32_t max_cells, uint32_t rate_capacity, uint32_t n_instances);
    int sync_inst();
    int upload_soa(uint32_t cell_off, uint32_t count, const float* soa, uint32_t soa_max, uint32_t first_field,
                   uint32_t n_fields);
    int download_soa(uint32_t cell_off, uint32_t count, float* soa, uint32_t soa_max, uint32_t first_field,
                     uint32_t n_fields);
    int set_rates(uint32_t rate_off, uint32_t count, const double* sec, const double* upt, const double* sat,
                  const double* ne);
    int set_active(uint32_t cell_off, uint32_t count, const uint8_t* act);
    int set_cell_instances(const std::vector<uint32_t>& per_instance_counts);
    // Drop the masters of cells [off, off + count) (their FP32 positions count).
    int clear_masters(uint32_t off, uint32_t count);
    // Positions of cells [off, off + count) as the AB2 update would start
    // from them (the master where it rounds to the FP32 value, else the FP32
    // value): three host arrays of count doubles at xyz.
    int download_positions(uint32_t off, uint32_t count, double* xyz);
    // Recompute secretion constants / ordering when stale.
    int prepare_secretion(double dt, uint64_t total_vox);
    int build_order(uint64_t total_vox);   // order, runs and (once a dt is known) the constants
    int sorted_constants();   // cell-order constants when stale, then their permutation
    int secrete(Diffusion& d, const uint8_t* mask);
    uint64_t device_bytes() const;
};

// ------------------------------------------------------------------ mechanics

class Mechanics {
public:
    pcg_ctx* ctx = nullptr;
    uint32_t total_mvox = 0;
    uint32_t cap = 0;
    ForceShape fshape;     // launch shape of the force pass
    int bin_block = 256;   // threads per block of the binning kernels
    int int_block = 256;   // threads per block of the AB2 kernel
    bool diag = false;
    // lazy_sorder: binning leaves the stable order out (a batch's steps never
    // read it); stable_order() makes it from the same binning on request.
    // sorder_valid: it matches the last binning.
    bool lazy_sorder = false, sorder_valid = false;
    // binning: keys / slots (voxel key and arrival slot per cell), counts
    // (per voxel, + 1), start (the cell-start table), placed ((x key, cell)
    // in arrival order per voxel), sorder (the stable order: by voxel, then
    // index), spos / sprm (positions and strengths in the force order: by
    // voxel, then x; the cell's index in sprm's third component)
    DevBuf keys, slots, placed, sorder, counts, start, scan_scr, spos, sprm, dcnt, dhash;

    int create(pcg_ctx* c, uint32_t total_mvox, uint32_t max_cells);
    int forces(Cells& c, const uint8_t* mask);       // binsort + force_pass
    int binsort(Cells& c, const uint8_t* mask);      // bin, counting sort, cell-start table, sorted SoA
    int stable_order(uint32_t n);                    // sorder from the last binning, when not yet made
    int force_pass(Cells& c, const uint8_t* mask);
    int integrate(Cells& c, float dt_override, const uint8_t* mask);
    int launches_forces(uint32_t n) const;
    uint64_t device_bytes() const;
};

// Mechanics grid of the reference (cell_mechanics.mm:26-41).
void fill_mech_inst(CellInst& ci, const pcg_mechanics_params& m, float x_min, float y_min, float z_min);
void fill_diff_inst(CellInst& ci, const DiffInstance& d);

int key_bits_for(uint64_t n_keys);

// The moves of CellData::removeCell (cell_data.cpp:408-498: the last cell
// takes the freed place) called for each of 'indices' in descending order,
// skipping indices at or past the current count, as phase 3 of
// updatePhenotypes does (cell_phenotype.cpp:838-844).  Each move (x, y):
// the cell that started at place y ends at place x; every other place below
// the returned count keeps its cell.  Moves are sorted by destination.
uint32_t removal_plan(uint32_t n_cells, const uint32_t* indices, uint32_t count, std::vector<uint2>* moves);

}  // namespace pcg
