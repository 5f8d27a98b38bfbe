// runtime.cu — engines behind the C ABI (see runtime.h).
#include "runtime.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <unordered_map>

namespace pcg {

int fail(pcg_ctx* ctx, int code, const std::string& msg)
{
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(pcg_ctx* ctx, cudaError_t e, const char* what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (ctx) ctx->err = m;
    return e == cudaErrorMemoryAllocation ? PCG_ERR_OOM : PCG_ERR_CUDA;
}

// ------------------------------------------------------------------ device pool
//
// Stream-ordered caching of device blocks.  A block released by a DevBuf
// that was allocated under an AllocStream goes back to the pool with an
// event recorded on that stream; it is handed out again only once the event
// has completed, so no kernel still using it can see it reused, and nothing
// synchronises the device (cudaFree would).  Requests are rounded up to a
// size class (512-byte steps below 4 KiB, above it four classes per power of
// two) and a free block of exactly that class is reused.  On an allocation
// failure the idle blocks are returned to the driver and the allocation is
// retried.  The pool lives until process exit (never destroyed, so no CUDA
// call runs during static destruction).

namespace {

thread_local cudaStream_t tl_alloc_stream = nullptr;

// Library-wide allocation counters and the host-side failure injector
// (pcg_debug_alloc_stats / pcg_debug_fail_alloc).
std::atomic<uint64_t> g_mallocs{0}, g_reuses{0}, g_fail_in{0};

// True when the injector says this allocation is to fail.
bool injected_failure()
{
    uint64_t v = g_fail_in.load();
    while (v > 0) {
        if (g_fail_in.compare_exchange_weak(v, v - 1)) return v == 1;
    }
    return false;
}

struct PoolBlock {
    void* p;
    int device;
    cudaEvent_t ev;
};

class DevicePool {
public:
    static DevicePool& get()
    {
        static DevicePool* pool = new DevicePool();
        return *pool;
    }
    cudaError_t take(size_t want, void** out, size_t* got, int* device)
    {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        *device = dev;
        const size_t b = round_up(want);
        {
            std::lock_guard<std::mutex> lk(mu_);
            const auto range = free_.equal_range(b);
            for (auto it = range.first; it != range.second; ++it) {
                if (it->second.device != dev) continue;
                const cudaError_t q = cudaEventQuery(it->second.ev);
                if (q == cudaErrorNotReady) continue;
                if (q != cudaSuccess) cudaGetLastError();
                *out = it->second.p;
                *got = it->first;
                cudaEventDestroy(it->second.ev);
                free_.erase(it);
                g_reuses++;
                return cudaSuccess;
            }
        }
        e = cudaMalloc(out, b);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            trim(dev);
            e = cudaMalloc(out, b);
        }
        if (e != cudaSuccess) {
            *out = nullptr;
            return e;
        }
        g_mallocs++;
        *got = b;
        return cudaSuccess;
    }
    // false: the caller frees the block itself (no event could be recorded)
    bool give(void* p, size_t bytes, cudaStream_t st, int dev)
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
            cudaGetLastError();
            return false;
        }
        cudaEvent_t ev = nullptr;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (cudaEventRecord(ev, st) != cudaSuccess) {
            cudaGetLastError();
            cudaEventDestroy(ev);
            return false;
        }
        std::lock_guard<std::mutex> lk(mu_);
        free_.emplace(bytes, PoolBlock{p, dev, ev});
        return true;
    }
    void trim(int dev)
    {
        std::lock_guard<std::mutex> lk(mu_);
        for (auto it = free_.begin(); it != free_.end();) {
            if (it->second.device == dev && cudaEventQuery(it->second.ev) == cudaSuccess) {
                cudaEventDestroy(it->second.ev);
                cudaFree(it->second.p);
                it = free_.erase(it);
            } else {
                cudaGetLastError();
                ++it;
            }
        }
    }

private:
    // Block sizes: 512-byte steps below 4 KiB, above it four classes per
    // power of two (2^e x {1, 1.25, 1.5, 1.75}, at most 25% over), so a
    // rebuild whose buffers differ a little in size from the last one's
    // finds the freed blocks again instead of allocating anew.
    static size_t round_up(size_t b)
    {
        if (b < 4096) return (b + 511) / 512 * 512;
        const int e = 63 - __builtin_clzll(static_cast<unsigned long long>(b));
        const size_t step = static_cast<size_t>(1) << (e - 2);
        return (b + step - 1) / step * step;
    }
    std::mutex mu_;
    std::multimap<size_t, PoolBlock> free_;
};

}  // namespace

AllocStream::AllocStream(cudaStream_t s) : prev_(tl_alloc_stream) { tl_alloc_stream = s; }
AllocStream::~AllocStream() { tl_alloc_stream = prev_; }

cudaError_t DevBuf::alloc(size_t b)
{
    release();
    if (b == 0) return cudaSuccess;
    if (injected_failure()) return cudaErrorMemoryAllocation;
    if (tl_alloc_stream) {
        size_t got = 0;
        const cudaError_t e = DevicePool::get().take(b, &p, &got, &dev_);
        if (e != cudaSuccess) {
            p = nullptr;
            return e;
        }
        bytes = b;
        cap_ = got;
        stream_ = tl_alloc_stream;
        return cudaSuccess;
    }
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) {
        p = nullptr;
        return e;
    }
    g_mallocs++;
    bytes = b;
    cap_ = 0;
    stream_ = nullptr;
    return cudaSuccess;
}

void alloc_stats(uint64_t* mallocs, uint64_t* reuses)
{
    if (mallocs) *mallocs = g_mallocs.load();
    if (reuses) *reuses = g_reuses.load();
}

void fail_alloc_after(uint64_t nth) { g_fail_in.store(nth); }

void DevBuf::release()
{
    if (p) {
        if (!(stream_ && cap_ && DevicePool::get().give(p, cap_, stream_, dev_))) cudaFree(p);
    }
    p = nullptr;
    bytes = 0;
    cap_ = 0;
    stream_ = nullptr;
}

cudaError_t HostBuf::alloc(size_t b)
{
    release();
    if (b == 0) return cudaSuccess;
    cudaError_t e = cudaMallocHost(&p, b);
    if (e != cudaSuccess) {
        p = nullptr;
        return e;
    }
    bytes = b;
    return cudaSuccess;
}

void HostBuf::release()
{
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
}

uint32_t removal_plan(uint32_t n_cells, const uint32_t* indices, uint32_t count, std::vector<uint2>* moves)
{
    std::vector<uint32_t> r(indices, indices + count);
    std::sort(r.begin(), r.end(), std::greater<uint32_t>());
    std::unordered_map<uint32_t, uint32_t> at;   // place -> starting place of the cell there (absent: its own)
    auto cell_at = [&](uint32_t p) {
        const auto it = at.find(p);
        return it == at.end() ? p : it->second;
    };
    uint32_t num = n_cells;
    for (const uint32_t idx : r) {
        if (idx >= num) continue;
        const uint32_t last = num - 1;
        if (idx != last) at[idx] = cell_at(last);
        at.erase(last);
        --num;
    }
    moves->clear();
    for (const auto& kv : at)
        if (kv.first < num && kv.second != kv.first) moves->push_back(make_uint2(kv.first, kv.second));
    std::sort(moves->begin(), moves->end(), [](const uint2& a, const uint2& b) { return a.x < b.x; });
    return num;
}

int key_bits_for(uint64_t n_keys)
{
    int b = 0;
    while ((1ull << b) < n_keys) ++b;
    return b;
}

// ------------------------------------------------------------------ tuner

static std::mutex g_tune_mu;

Tuner& Tuner::get()
{
    static Tuner t;
    return t;
}

bool Tuner::lookup(const std::string& key, int* value)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = table_.find(key);
    if (it == table_.end()) return false;
    *value = it->second;
    return true;
}

void Tuner::store(const std::string& key, int value)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    table_[key] = value;
}

// Flat JSON object of "key": int pairs.
void Tuner::load(const std::string& path)
{
    std::ifstream f(path);
    if (!f) return;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string s = ss.str();
    size_t i = 0;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    while ((i = s.find('"', i)) != std::string::npos) {
        const size_t j = s.find('"', i + 1);
        if (j == std::string::npos) break;
        const std::string key = s.substr(i + 1, j - i - 1);
        const size_t c = s.find(':', j);
        if (c == std::string::npos) break;
        table_[key] = std::atoi(s.c_str() + c + 1);
        i = s.find_first_of(",}", c);
        if (i == std::string::npos) break;
    }
}

void Tuner::save(const std::string& path)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::ofstream f(path);
    if (!f) return;
    f << "{\n";
    size_t k = 0;
    for (auto& kv : table_) f << "  \"" << kv.first << "\": " << kv.second << (++k < table_.size() ? ",\n" : "\n");
    f << "}\n";
}

// ------------------------------------------------------------------ diffusion

// Largest plane (with its tables) the fused x + y kernel takes: two CTAs
// per SM fit the 227 KB of shared memory.
static constexpr size_t kPlaneMaxSmem = 112 * 1024;


static uint32_t axis_n(const pcg_grid_params& g, int a) { return a == 0 ? g.nx : (a == 1 ? g.ny : g.nz); }
static float axis_h(const pcg_grid_params& g, int a) { return a == 0 ? g.dx : (a == 1 ? g.dy : g.dz); }

uint32_t Diffusion::rule_of(size_t i, uint32_t s, int axis) const
{
    size_t k = 0;
    for (size_t q = 0; q < i; ++q) k += inst[q].subs.size() * 3;
    return rule_index_[k + s * 3 + axis];
}

int Diffusion::build(pcg_ctx* c, std::vector<DiffInstance> instances)
{
    ctx = c;
    inst = std::move(instances);
    dens_elems = 0;
    total_vox = total_vox_sub = 0;
    h_rules_.clear();
    h_tab_.clear();
    rule_index_.clear();
    std::vector<FaceJob> fj;
    for (size_t i = 0; i < inst.size(); ++i) {
        DiffInstance& d = inst[i];
        const pcg_grid_params& g = d.g;
        if (g.nx == 0 || g.ny == 0 || g.nz == 0) return fail(ctx, PCG_ERR_INVALID, "grid with a zero dimension");
        if (d.subs.size() != g.n_substrates) return fail(ctx, PCG_ERR_INVALID, "substrate count mismatch");
        const uint64_t nv = d.nvox();
        if (nv > 0xFFFFFFFFull) return fail(ctx, PCG_ERR_INVALID, "grid larger than 2^32 voxels");
        d.px = (g.nx + 3u) & ~3u;
        d.pitch = (d.rows() * d.px + 31) / 32 * 32;
        d.dens_off = dens_elems;
        d.vox_base = static_cast<uint32_t>(total_vox);
        dens_elems += d.pitch * g.n_substrates;
        total_vox += nv;
        total_vox_sub += nv * g.n_substrates;
        if (total_vox > 0xFFFFFFF0ull) return fail(ctx, PCG_ERR_INVALID, "more than 2^32 voxels in one batch");
        const int nd = d.ndim();
        for (uint32_t s = 0; s < g.n_substrates; ++s) {
            const pcg_substrate_params& sp = d.subs[s];
            for (int a = 0; a < 3; ++a) {
                if (a == 2 && nd < 3) {
                    rule_index_.push_back(0xFFFFFFFFu);
                    continue;
                }
                const uint32_t n = axis_n(g, a);
                const double h = axis_h(g, a);
                // D dt / h^2 and the split decay, in FP64 from the FP32 parameters
                // (microenvironment.mm:86-92; decay lambda dt / d per sweep)
                const double cc = static_cast<double>(sp.diffusion_coefficient) * static_cast<double>(g.dt) / (h * h);
                const double hd = static_cast<double>(sp.decay_rate) * static_cast<double>(g.dt) / nd;
                const bool dir = sp.dirichlet_enabled != 0;
                const double T = sp.target_value;
                LineRule r{};
                r.tab = static_cast<uint32_t>(h_tab_.size());
                r.n = n;
                r.c = static_cast<float>(cc);
                r.T = sp.target_value;
                r.dir = dir ? 1u : 0u;
                r.inst = static_cast<uint32_t>(i);
                h_tab_.resize(h_tab_.size() + tab_floats(std::max<uint32_t>(n, 1)), 0.f);
                float* tb = h_tab_.data() + r.tab;
                // position i: g_i = c / den_i = -c'_i and 1 / den_i (chunked layout)
                auto put = [tb](uint32_t i, double g, double inv) {
                    tb[(i / 4) * 8 + i % 4] = static_cast<float>(g);
                    tb[(i / 4) * 8 + 4 + i % 4] = static_cast<float>(inv);
                };
                // the end interior nodes' diagonal: the reference's 1 + c + hd
                // (diffusion_2d.metal:48), or with the consistent Dirichlet
                // option the interior one on Dirichlet lines
                const double b_int = 1.0 + 2.0 * cc + hd;
                const double b_bnd = (dir && sp.dirichlet_consistent) ? b_int : 1.0 + cc + hd;
                if (n == 3) {
                    put(1, 0.0, 1.0 / b_int);
                    r.fold = dir ? static_cast<float>(2.0 * cc * T) : 0.f;
                } else if (n >= 4) {
                    double cp = -cc / b_bnd;
                    put(1, -cp, 1.0 / b_bnd);
                    for (uint32_t m = 2; m + 2 < n; ++m) {
                        const double den = b_int + cc * cp;
                        cp = -cc / den;
                        put(m, -cp, 1.0 / den);
                    }
                    const double den = b_bnd + cc * cp;
                    put(n - 2, cc / den, 1.0 / den);
                    r.fold = dir ? static_cast<float>(cc * T) : 0.f;
                }
                rule_index_.push_back(static_cast<uint32_t>(h_rules_.size()));
                h_rules_.push_back(r);
            }
            if (sp.dirichlet_enabled) {
                FaceJob f{};
                f.base = d.dens_off + s * d.pitch;
                f.nx = g.nx;
                f.ny = g.ny;
                f.nz = g.nz;
                f.px = d.px;
                f.T = sp.target_value;
                fj.push_back(f);
            }
        }
    }
    PCG_CU(ctx, dens.alloc(std::max<uint64_t>(dens_elems, 32) * sizeof(float)));
    PCG_CU(ctx, cudaMemsetAsync(dens.p, 0, dens.bytes, ctx->stream));
    PCG_CU(ctx, rules.alloc(std::max<size_t>(h_rules_.size(), 1) * sizeof(LineRule)));
    PCG_CU(ctx, tab.alloc(std::max<size_t>(h_tab_.size(), 8) * sizeof(float)));
    if (!h_rules_.empty())
        PCG_CU(ctx, cudaMemcpyAsync(rules.p, h_rules_.data(), h_rules_.size() * sizeof(LineRule), cudaMemcpyHostToDevice, ctx->stream));
    if (!h_tab_.empty())
        PCG_CU(ctx, cudaMemcpyAsync(tab.p, h_tab_.data(), h_tab_.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    // tensor maps, four 128-byte slots per rule (kMapsPerRule): x rules use
    // slot 0 (2-D row map) and slot 1 (x-y plane map); y / z rules one 3-D
    // column map per tile width in slots 0-2 (32, 16, 8 columns), z rules
    // the x-z plane map in slot 3.  tensor_ok_ bit w: the slot-w column map
    // exists.
    tensor_ok_.assign(h_rules_.size(), 0);
    {
        std::vector<unsigned char> maps(std::max<size_t>(h_rules_.size(), 1) * kMapsPerRule * 128, 0);
        for (size_t i = 0; i < inst.size(); ++i) {
            const DiffInstance& d = inst[i];
            for (uint32_t s = 0; s < d.g.n_substrates; ++s) {
                float* block = dens.as<float>() + d.dens_off + s * d.pitch;
                for (int a = 0; a < 3; ++a) {
                    if (a == 2 && d.ndim() < 3) continue;
                    const uint32_t rule = rule_of(i, s, a);
                    const uint32_t n = axis_n(d.g, a);
                    unsigned char* m = maps.data() + static_cast<size_t>(rule) * kMapsPerRule * 128;
                    if (a == 0) {
                        if (n <= kRowTensorMaxN && encode_row_map(m, block, d.g.nx, d.rows(), d.px)) tensor_ok_[rule] = 1;
                        continue;
                    }
                    if (n > kTensorMaxN) continue;
                    for (int w = 0; w < 3; ++w)
                        if (encode_column_map(m + w * 128, block, d.g.nx, d.g.ny, d.g.nz, d.px, a, n, 32u >> w))
                            tensor_ok_[rule] |= static_cast<uint8_t>(1u << w);
                }
            }
        }
        // plane maps (slot 1 of each x rule) for the instances whose x-y
        // planes fit the plane kernel's shared memory
        plane_inst_.assign(inst.size(), 0);
        for (size_t i = 0; use_planes && i < inst.size(); ++i) {
            const DiffInstance& d = inst[i];
            const uint32_t nx = d.g.nx, ny = d.g.ny;
            if (d.g.n_substrates == 0 || nx > kRowTensorMaxN || ny > 256 ||
                sweep_planes_smem(plane_floats(nx, ny)) > kPlaneMaxSmem)
                continue;
            bool ok = true;
            for (uint32_t s = 0; s < d.g.n_substrates && ok; ++s) {
                const uint32_t rule = rule_of(i, s, 0);
                unsigned char* m = maps.data() + static_cast<size_t>(rule) * kMapsPerRule * 128;
                ok = (tensor_ok_[rule] & 1u) &&
                     encode_plane_map(m + 128, dens.as<float>() + d.dens_off + s * d.pitch, nx, ny, d.rows(), d.px);
            }
            plane_inst_[i] = ok ? 1 : 0;
        }
        // x-z plane maps (slot 3 of each z rule) for the z sweep
        zplane_inst_.assign(inst.size(), 0);
        for (size_t i = 0; use_planes && i < inst.size(); ++i) {
            const DiffInstance& d = inst[i];
            const uint32_t nx = d.g.nx, nz = d.g.nz;
            if (d.ndim() < 3 || d.g.n_substrates == 0 || ((nx + 3u) & ~3u) > 256 || nz > 256 ||
                sweep_planes_smem(plane_floats(nx, nz, true)) > kPlaneMaxSmem)
                continue;
            bool ok = true;
            for (uint32_t s = 0; s < d.g.n_substrates && ok; ++s) {
                const uint32_t rule = rule_of(i, s, 2);
                unsigned char* m = maps.data() + static_cast<size_t>(rule) * kMapsPerRule * 128;
                ok = encode_xz_plane_map(m + 3 * 128, dens.as<float>() + d.dens_off + s * d.pitch, nx, d.g.ny, nz,
                                         d.px);
            }
            zplane_inst_[i] = ok ? 1 : 0;
        }
        PCG_CU(ctx, tmaps.alloc(maps.size()));
        PCG_CU(ctx, cudaMemcpyAsync(tmaps.p, maps.data(), maps.size(), cudaMemcpyHostToDevice, ctx->stream));
    }
    n_faces = static_cast<uint32_t>(fj.size());
    PCG_CU(ctx, faces.alloc(std::max<size_t>(fj.size(), 1) * sizeof(FaceJob)));
    if (!fj.empty()) PCG_CU(ctx, cudaMemcpyAsync(faces.p, fj.data(), fj.size() * sizeof(FaceJob), cudaMemcpyHostToDevice, ctx->stream));
    for (int a = 0; a < 3; ++a) {
        PCG_TRY(build_axis(a, nullptr, lists[a]));
        PCG_TRY(default_configs(a));
    }
    return build_planes();
}

// Plane jobs grouped by shared-memory size, so small planes are not charged
// the largest plane's footprint; largest planes first.
// Plane lists from per-class jobs: runs of 'merge' consecutive non-empty
// classes (0: all of them) become one list, launched with the largest
// plane's shared memory.
static int plane_lists(pcg_ctx* ctx, const std::vector<PlaneJob>* jobs, const uint32_t* fl, const uint64_t* un,
                       int classes, int merge, std::vector<PlaneList>& out)
{
    std::vector<int> used;
    for (int c = classes - 1; c >= 0; --c)
        if (!jobs[c].empty()) used.push_back(c);
    const size_t per = merge <= 0 ? std::max<size_t>(used.size(), 1) : static_cast<size_t>(merge);
    out.clear();
    out.resize((used.size() + per - 1) / per);
    for (size_t q = 0; q < out.size(); ++q) {
        PlaneList& pl = out[q];
        std::vector<PlaneJob> all;
        for (size_t k = q * per; k < std::min(used.size(), (q + 1) * per); ++k) {
            const int c = used[k];
            all.insert(all.end(), jobs[c].begin(), jobs[c].end());
            pl.floats = std::max(pl.floats, fl[c]);
            pl.units += un[c];
        }
        pl.n = static_cast<uint32_t>(all.size());
        PCG_CU(ctx, pl.jobs.alloc(all.size() * sizeof(PlaneJob)));
        PCG_CU(ctx, cudaMemcpyAsync(pl.jobs.p, all.data(), all.size() * sizeof(PlaneJob), cudaMemcpyHostToDevice,
                                    ctx->stream));
    }
    if (!out.empty()) PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));   // the host vectors go
    return PCG_OK;
}

int Diffusion::regroup_planes(int merge)
{
    plane_merge = merge;
    PCG_TRY(plane_lists(ctx, cls_jobs_[0], cls_floats_[0], cls_units_[0], kPlaneClasses, merge, planes));
    PCG_TRY(plane_lists(ctx, cls_jobs_[1], cls_floats_[1], cls_units_[1], kPlaneClasses, merge, zplanes));
    return PCG_OK;
}

// x-y plane jobs (one per z slab of each substrate of each plane instance),
// x-z plane jobs (one per y of each substrate of each z-plane instance), and
// the tiles of the instances without planes.
int Diffusion::build_planes()
{
    planes.clear();
    zplanes.clear();
    for (auto& r : rest) r.clear();
    bool any = false;
    for (size_t i = 0; i < inst.size(); ++i) any = any || plane_inst_[i] || zplane_inst_[i];
    if (any) PCG_CU(ctx, sweep_planes_prepare());   // before the occupancy queries
    // Classes by the plane CTAs an SM holds for the plane's shared memory
    // (class kMaxCtas - k for k CTAs), so each plane runs at the occupancy
    // its own size allows; a class launches with its largest plane's size,
    // which by construction allows the same k.
    constexpr int kMaxCtas = kPlaneClasses;
    auto cls = [&](uint32_t pf) { return kMaxCtas - std::min(std::max(sweep_planes_ctas(pf), 1), kMaxCtas); };
    std::vector<PlaneJob>* jobs = cls_jobs_[0];
    std::vector<PlaneJob>* zjobs = cls_jobs_[1];
    uint32_t* fl = cls_floats_[0];
    uint32_t* zfl = cls_floats_[1];
    uint64_t* un = cls_units_[0];
    uint64_t* zun = cls_units_[1];
    for (int c = 0; c < kPlaneClasses; ++c) {
        jobs[c].clear();
        zjobs[c].clear();
        fl[c] = zfl[c] = 0;
        un[c] = zun[c] = 0;
    }
    for (size_t i = 0; i < inst.size(); ++i) {
        const DiffInstance& d = inst[i];
        const uint32_t nx = d.g.nx, ny = d.g.ny, nz = d.g.nz;
        if (plane_inst_[i]) {
            const uint32_t pf = plane_floats(nx, ny);
            const int c = cls(pf);
            for (uint32_t s = 0; s < d.g.n_substrates; ++s) {
                const uint32_t rx_i = rule_of(i, s, 0);
                const LineRule& rx = h_rules_[rx_i];
                const LineRule& ry = h_rules_[rule_of(i, s, 1)];
                for (uint32_t k = 0; k < nz; ++k) {
                    PlaneJob j{};
                    j.map = rx_i * kMapsPerRule + 1;
                    j.row0 = k * ny;
                    j.nx = nx;
                    j.ny = ny;
                    j.tab_x = rx.tab;
                    j.tab_y = ry.tab;
                    j.fold_x = rx.fold;
                    j.T_x = rx.T;
                    j.fold_y = ry.fold;
                    j.T_y = ry.T;
                    j.inst = static_cast<uint32_t>(i) | (rx.dir ? kPlaneDirX : 0u) | (ry.dir ? kPlaneDirY : 0u) |
                             ((d.ndim() == 2 && ry.dir) ? kPlaneFaces : 0u);
                    jobs[c].push_back(j);
                }
            }
            fl[c] = std::max(fl[c], pf);
            un[c] += d.nvox() * d.g.n_substrates;
        }
        if (zplane_inst_[i]) {
            const uint32_t pf = plane_floats(nx, nz, true);
            const int c = cls(pf);
            for (uint32_t s = 0; s < d.g.n_substrates; ++s) {
                const uint32_t rz_i = rule_of(i, s, 2);
                const LineRule& rz = h_rules_[rz_i];
                for (uint32_t y = 0; y < ny; ++y) {
                    PlaneJob j{};
                    j.map = rz_i * kMapsPerRule + 3;
                    j.row0 = y;
                    j.nx = nx;
                    j.ny = nz;
                    j.tab_y = rz.tab;
                    j.fold_y = rz.fold;
                    j.T_y = rz.T;
                    j.inst = static_cast<uint32_t>(i) | kPlaneZ | (rz.dir ? (kPlaneDirY | kPlaneFaces) : 0u) |
                             ((y == 0 || y + 1 == ny) ? kPlaneSlabFace : 0u);
                    zjobs[c].push_back(j);
                }
            }
            zfl[c] = std::max(zfl[c], pf);
            zun[c] += d.nvox() * d.g.n_substrates;
        }
    }
    PCG_TRY(regroup_planes(plane_merge));
    for (int a = 0; a < 3; ++a) {
        if (!planes_for(a)) continue;
        PCG_TRY(build_axis(a, a < 2 ? &plane_inst_ : &zplane_inst_, rest[a]));
        for (auto& l : rest[a]) PCG_TRY(config_list(l, 0));
    }
    return prepare_forks();
}

// Copy a line rule into a tile descriptor.
static void fill_rule(SweepTile& t, const LineRule& r)
{
    t.n = r.n;
    t.tab = r.tab;
    t.fold = r.fold;
    t.T = r.T;
    t.inst = r.inst | (r.dir ? 0x80000000u : 0u);
}

// Tile lists of one axis: lines up to kTmaMaxN go to the pipelined TMA
// kernels (x: 32 lines per tile; y/z: 32 columns per tile), longer lines to
// the one-thread-per-line kernel.
int Diffusion::build_axis(int axis, const std::vector<uint8_t>* skip, std::vector<SweepList>& ls)
{
    std::vector<SweepTile> fast_t, glob_t;
    int fast_nmax = 0, glob_nmax = 0;
    uint64_t fast_lines = 0, glob_lines = 0, fast_units = 0, glob_units = 0;
    const int kind_fast = axis == 0 ? 0 : 1;
    for (size_t i = 0; i < inst.size(); ++i) {
        if (skip && (*skip)[i]) continue;
        const DiffInstance& d = inst[i];
        const pcg_grid_params& g = d.g;
        const int nd = d.ndim();
        if (axis == 2 && nd < 3) continue;
        const uint32_t n = axis_n(g, axis);
        const bool fast = n <= kTmaMaxN;
        auto& out = fast ? fast_t : glob_t;
        int& nmax = fast ? fast_nmax : glob_nmax;
        uint64_t& nl = fast ? fast_lines : glob_lines;
        (fast ? fast_units : glob_units) += d.nvox() * g.n_substrates;
        nmax = std::max<int>(nmax, static_cast<int>(n));
        const bool final_axis = axis == nd - 1;
        for (uint32_t s = 0; s < g.n_substrates; ++s) {
            const uint32_t rule = rule_of(i, s, axis);
            const bool dir = d.subs[s].dirichlet_enabled != 0;
            const uint64_t sbase = d.dens_off + s * d.pitch;
            if (axis == 0) {
                const uint64_t lines = d.rows();
                for (uint64_t l0 = 0; l0 < lines; l0 += 32) {
                    SweepTile t{};
                    t.base = sbase + l0 * d.px;
                    fill_rule(t, h_rules_[rule]);
                    t.count = static_cast<uint32_t>(std::min<uint64_t>(32, lines - l0));
                    t.rs = d.px;
                    t.nx = g.nx;
                    t.outer = static_cast<uint32_t>(l0);
                    t.map = rule * kMapsPerRule;
                    t.width = 32;
                    t.nslab = 1;
                    t.face = TILE_ROWS | ((fast && tensor_ok_[rule]) ? TILE_TENSOR : 0u);
                    out.push_back(t);
                }
                nl += lines;
            } else {
                // y: families over (i, k), stride px; z: families over (i, j), stride ny*px.
                // With tensor maps, the last (narrow) tile of each slab takes
                // 16 or 8 columns from 2 or 4 adjacent slabs, so its lanes are
                // not left idle.
                const uint32_t outer = axis == 1 ? g.nz : g.ny;
                const uint64_t ostride = axis == 1 ? static_cast<uint64_t>(d.px) * g.ny : d.px;
                const uint32_t rs = axis == 1 ? d.px : d.px * g.ny;
                for (uint32_t i0 = 0; i0 < g.nx; i0 += 32) {
                    const uint32_t cnt = std::min<uint32_t>(32, g.nx - i0);
                    int w = 0;
                    if (fast && tensor_ok_[rule]) {
                        if (cnt <= 8 && (tensor_ok_[rule] & 4u)) w = 2;
                        else if (cnt <= 16 && (tensor_ok_[rule] & 2u)) w = 1;
                        if (!(tensor_ok_[rule] & (1u << w))) w = -1;
                    } else {
                        w = -1;
                    }
                    const uint32_t width = w < 0 ? 32u : (32u >> w);
                    const uint32_t group = 32u / width;
                    for (uint32_t o = 0; o < outer; o += group) {
                        SweepTile t{};
                        t.base = sbase + o * ostride + i0;
                        fill_rule(t, h_rules_[rule]);
                        t.count = cnt;
                        t.rs = rs;
                        t.i0 = i0;
                        t.nx = g.nx;
                        t.outer = o;
                        t.outer_n = outer;
                        t.width = static_cast<uint16_t>(width);
                        t.nslab = static_cast<uint16_t>(std::min(group, outer - o));
                        t.map = rule * kMapsPerRule + static_cast<uint32_t>(w < 0 ? 0 : w);
                        if (w >= 0) t.face |= TILE_TENSOR;
                        if (axis == 2) t.face |= TILE_AXIS_Z;
                        if (final_axis && dir) t.face |= TILE_FACE;
                        out.push_back(t);
                    }
                }
                nl += static_cast<uint64_t>(g.nx) * outer;
            }
        }
    }
    // larger lines first so the persistent loop ends evenly
    auto by_n = [](const SweepTile& a, const SweepTile& b) { return a.n > b.n; };
    std::stable_sort(fast_t.begin(), fast_t.end(), by_n);
    std::stable_sort(glob_t.begin(), glob_t.end(), by_n);
    ls.clear();
    ls.resize(2);
    ls[0].kind = kind_fast;
    ls[0].nmax = fast_nmax;
    ls[0].n = static_cast<uint32_t>(fast_t.size());
    ls[0].lines = fast_lines;
    ls[0].units = fast_units;
    ls[1].kind = 2;
    ls[1].nmax = glob_nmax;
    ls[1].n = static_cast<uint32_t>(glob_t.size());
    ls[1].lines = glob_lines;
    ls[1].units = glob_units;
    for (int q = 0; q < 2; ++q) {
        const auto& v = q == 0 ? fast_t : glob_t;
        PCG_CU(ctx, ls[q].tiles.alloc(std::max<size_t>(v.size(), 1) * sizeof(SweepTile)));
        if (!v.empty())
            PCG_CU(ctx, cudaMemcpyAsync(ls[q].tiles.p, v.data(), v.size() * sizeof(SweepTile), cudaMemcpyHostToDevice, ctx->stream));
    }
    return PCG_OK;
}

// Launch shape of one TMA list.  'param' = warps * 16 + stages picks one
// shape; 0 takes the shape that keeps the most bytes in flight per SM.
// Stage size: x tiles need 32 rows of the longest line's pitch (tensor
// box or bulk copy); column tiles 32 x n rounded up to whole chunks of 4
// rows, which the solve may read past the last row; then the longest
// line's coefficient table.
static int tma_tab_floats(const SweepList& l) { return static_cast<int>(tab_floats(static_cast<uint32_t>(l.nmax))); }
static int tma_stage_floats(const SweepList& l)
{
    const uint32_t n = static_cast<uint32_t>(l.nmax);
    const uint32_t r4 = (n + 3u) & ~3u;
    const uint32_t span = l.kind == 0 ? std::max(row_smem_pitch(std::min(n, kRowTensorMaxN)), r4) : r4;
    // whole 128-byte units, so every stage starts 128-byte aligned (tensor
    // copies need it); the table area then starts on 32 bytes
    return static_cast<int>((32u * span + static_cast<uint32_t>(tma_tab_floats(l)) + 31u) / 32u * 32u);
}

int Diffusion::config_list(SweepList& l, int param)
{
    if (l.n == 0) return PCG_OK;
    if (l.kind == 2) {
        const uint64_t ctas = (static_cast<uint64_t>(l.n) * 32 + 127) / 128;
        l.ggrid = static_cast<int>(std::min<uint64_t>(std::max<uint64_t>(ctas, 1), static_cast<uint64_t>(ctx->sms) * 16));
        return PCG_OK;
    }
    const bool rows = l.kind == 0;
    const int sf = tma_stage_floats(l);
    int best_w = 0, best_s = 0, best_occ = 0;
    double best_flight = -1.0;
    for (int w : {1, 2, 3, 4, 6, 8}) {
        for (int st : {2, 3, 4}) {
            if (param && param != w * 16 + st) continue;
            const int occ = sweep_tma_occupancy(rows, w, st, sf);
            if (occ <= 0) continue;
            // warps computing per SM x tiles in flight per warp
            const double flight = static_cast<double>(occ) * w * (st - 1) * sf + 0.5 * occ * w;
            if (flight > best_flight) {
                best_flight = flight;
                best_w = w;
                best_s = st;
                best_occ = occ;
            }
        }
    }
    if (best_w == 0) return fail(ctx, PCG_ERR_INVALID, "sweep tile does not fit shared memory");
    l.tc.warps = best_w;
    l.tc.stages = best_s;
    l.tc.stage_floats = sf;
    l.tc.tab_floats = tma_tab_floats(l);
    const uint64_t ctas = (l.n + best_w - 1) / best_w;
    l.tc.grid = static_cast<int>(std::min<uint64_t>(ctas, static_cast<uint64_t>(best_occ) * ctx->sms));
    return PCG_OK;
}

int Diffusion::pin(int kind, int param)
{
    if (!param) return PCG_OK;
    if ((param & 15) < 2 || (param & 15) > 4 || (param >> 4) < 1 || (param >> 4) > 8)
        return fail(ctx, PCG_ERR_INVALID, "bad pinned launch shape");
    for (int a = 0; a < 3; ++a)
        for (auto& l : lists[a])
            if (l.kind == kind && l.n) PCG_TRY(config_list(l, param));
    for (int a = 0; a < 3; ++a)
        for (auto& l : rest[a])
            if (l.kind == kind && l.n) PCG_TRY(config_list(l, param));
    return PCG_OK;
}

int Diffusion::default_configs(int axis)
{
    for (auto& l : lists[axis]) PCG_TRY(config_list(l, 0));
    return PCG_OK;
}

int Diffusion::launch_list(const SweepList& l, bool fuse, const uint8_t* mask)
{
    if (l.n == 0) return PCG_OK;
    float* d = dens.as<float>();
    const SweepTile* t = l.tiles.as<SweepTile>();
    const float* tb = tab.as<float>();
    cudaError_t e;
    if (l.kind == 2) e = launch_sweep_global(ctx->stream, d, t, l.n, tb, fuse ? 1 : 0, mask, l.ggrid);
    else
        e = launch_sweep_tma(ctx->stream, l.kind == 0, d, t, l.n, tb, tmaps.p, fuse ? 1 : 0, mask, ctx->status, l.tc);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "sweep launch");
    ctx->launches++;
    return PCG_OK;
}

// Side streams and their events (made on first use, outside capture).
static int ensure_forks(pcg_ctx* ctx, int n)
{
    for (int q = 0; q < n; ++q)
        if (!ctx->fork_st[q]) PCG_CU(ctx, cudaStreamCreateWithFlags(&ctx->fork_st[q], cudaStreamNonBlocking));
    for (int q = 0; q <= n; ++q)
        if (!ctx->fork_ev[q]) PCG_CU(ctx, cudaEventCreateWithFlags(&ctx->fork_ev[q], cudaEventDisableTiming));
    return PCG_OK;
}

int Diffusion::prepare_forks()
{
    const size_t n = std::max(planes.size(), zplanes.size());
    return n > 1 ? ensure_forks(ctx, std::min<int>(static_cast<int>(n) - 1, pcg_ctx::kForks)) : PCG_OK;
}

// The plane lists of a pass hold disjoint planes: the first list runs on the
// context stream, the others on side streams forked from it, and the context
// stream waits for all of them.  One list's last CTAs then overlap the next
// list's first, where launches in sequence would drain the GPU between them.
int Diffusion::launch_planes(const std::vector<PlaneList>& pls, bool fuse, const uint8_t* mask)
{
    const int side = std::min<int>(static_cast<int>(pls.size()) - 1, pcg_ctx::kForks);
    if (side > 0) {
        for (int q = 0; q <= side; ++q)
            if (!ctx->fork_ev[q] || (q < side && !ctx->fork_st[q]))
                return fail(ctx, PCG_ERR_INVALID, "plane side streams were not made");
        PCG_CU(ctx, cudaEventRecord(ctx->fork_ev[0], ctx->stream));
        for (int q = 0; q < side; ++q) PCG_CU(ctx, cudaStreamWaitEvent(ctx->fork_st[q], ctx->fork_ev[0], 0));
    }
    for (size_t k = 0; k < pls.size(); ++k) {
        const PlaneList& pl = pls[k];
        const cudaStream_t st = k == 0 ? ctx->stream : ctx->fork_st[(k - 1) % side];
        cudaError_t e = launch_sweep_planes(st, pl.jobs.as<PlaneJob>(), pl.n, tab.as<float>(), tmaps.p, pl.floats,
                                            fuse ? 1 : 0, mask, ctx->status);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "plane sweep launch");
        ctx->launches++;
    }
    for (int q = 0; q < side; ++q) {
        PCG_CU(ctx, cudaEventRecord(ctx->fork_ev[1 + q], ctx->fork_st[q]));
        PCG_CU(ctx, cudaStreamWaitEvent(ctx->stream, ctx->fork_ev[1 + q], 0));
    }
    return PCG_OK;
}

int Diffusion::sweep(int axis, bool fuse, const uint8_t* mask)
{
    if (planes_for(axis)) {
        if (axis == 0) PCG_TRY(launch_planes(planes, fuse, mask));
        if (axis == 2) PCG_TRY(launch_planes(zplanes, fuse, mask));
        for (const auto& l : rest[axis]) PCG_TRY(launch_list(l, fuse, mask));
        return PCG_OK;
    }
    for (const auto& l : lists[axis]) PCG_TRY(launch_list(l, fuse, mask));
    return PCG_OK;
}

uint64_t Diffusion::sweep_units_per_step() const
{
    uint64_t u = 0;
    for (int a = 0; a < 3; ++a) {
        if (planes_for(a)) {
            if (a == 0)
                for (const auto& pl : planes) u += pl.units;
            if (a == 2)
                for (const auto& pl : zplanes) u += pl.units;
            for (const auto& l : rest[a]) u += l.units;
        } else {
            for (const auto& l : lists[a]) u += l.units;
        }
    }
    return u;
}

int Diffusion::sweeps(bool fuse, const uint8_t* mask)
{
    for (int a = 0; a < 3; ++a) PCG_TRY(sweep(a, fuse, mask));
    return PCG_OK;
}

int Diffusion::launches_per_step(bool) const
{
    int k = 0;
    for (int a = 0; a < 3; ++a) {
        if (planes_for(a)) {
            if (a == 0) k += static_cast<int>(planes.size());
            if (a == 2) k += static_cast<int>(zplanes.size());
            for (const auto& l : rest[a]) k += l.n > 0 ? 1 : 0;
        } else {
            for (const auto& l : lists[a]) k += l.n > 0 ? 1 : 0;
        }
    }
    return k;
}

int Diffusion::dirichlet()
{
    if (n_faces == 0) return PCG_OK;
    cudaError_t e = launch_dirichlet(ctx->stream, dens.as<float>(), faces.as<FaceJob>(), n_faces);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "dirichlet launch");
    ctx->launches++;
    return PCG_OK;
}

int Diffusion::gradients(float* gx, float* gy, float* gz)
{
    std::vector<GradJob> jobs;
    uint64_t out = 0, maxv = 0;
    for (const auto& d : inst) {
        for (uint32_t s = 0; s < d.g.n_substrates; ++s) {
            GradJob j{};
            j.base = d.dens_off + s * d.pitch;
            j.out_base = out;
            j.nx = d.g.nx;
            j.ny = d.g.ny;
            j.nz = d.g.nz;
            j.px = d.px;
            j.inv_dx = 1.0f / d.g.dx;
            j.inv_dy = 1.0f / d.g.dy;
            j.inv_dz = 1.0f / d.g.dz;
            jobs.push_back(j);
            out += d.nvox();
            maxv = std::max<uint64_t>(maxv, d.nvox());
        }
    }
    if (jobs.empty()) return PCG_OK;
    PCG_CU(ctx, grad_jobs.alloc(jobs.size() * sizeof(GradJob)));
    PCG_CU(ctx, cudaMemcpyAsync(grad_jobs.p, jobs.data(), jobs.size() * sizeof(GradJob), cudaMemcpyHostToDevice,
                                ctx->stream));
    cudaError_t e = launch_gradients(ctx->stream, dens.as<float>(), gx, gy, gz, grad_jobs.as<GradJob>(),
                                     static_cast<uint32_t>(jobs.size()), maxv);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "gradients launch");
    ctx->launches++;
    // the job table must outlive the kernel
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return PCG_OK;
}

// Host arrays are dense [s][k][j][i]; device rows are px floats apart.
int Diffusion::upload(uint32_t i, const float* host, bool async_pinned)
{
    const DiffInstance& d = inst[i];
    const size_t nv = d.nvox();
    for (uint32_t s = 0; s < d.g.n_substrates; ++s) {
        float* dst = dens.as<float>() + d.dens_off + s * d.pitch;
        PCG_CU(ctx, cudaMemcpy2DAsync(dst, d.px * sizeof(float), host + s * nv, d.g.nx * sizeof(float),
                                      d.g.nx * sizeof(float), d.rows(), cudaMemcpyHostToDevice, ctx->stream));
    }
    if (!async_pinned) PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return PCG_OK;
}

int Diffusion::download(uint32_t i, float* host, bool async_pinned)
{
    const DiffInstance& d = inst[i];
    const size_t nv = d.nvox();
    for (uint32_t s = 0; s < d.g.n_substrates; ++s) {
        const float* src = dens.as<float>() + d.dens_off + s * d.pitch;
        PCG_CU(ctx, cudaMemcpy2DAsync(host + s * nv, d.g.nx * sizeof(float), src, d.px * sizeof(float),
                                      d.g.nx * sizeof(float), d.rows(), cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (!async_pinned) PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return PCG_OK;
}

int Diffusion::fill(uint32_t i, const float* values)
{
    const DiffInstance& d = inst[i];
    std::vector<float> tmp(d.rows() * d.px);
    for (uint32_t s = 0; s < d.g.n_substrates; ++s) {
        std::fill(tmp.begin(), tmp.end(), values[s]);
        float* dst = dens.as<float>() + d.dens_off + s * d.pitch;
        PCG_CU(ctx, cudaMemcpyAsync(dst, tmp.data(), tmp.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    }
    return PCG_OK;
}

uint64_t Diffusion::device_bytes() const
{
    uint64_t b = dens.bytes + rules.bytes + tab.bytes + faces.bytes;
    for (int a = 0; a < 3; ++a)
        for (const auto& l : lists[a]) b += l.tiles.bytes;
    for (int a = 0; a < 3; ++a)
        for (const auto& l : rest[a]) b += l.tiles.bytes;
    for (const auto& pl : planes) b += pl.jobs.bytes;
    for (const auto& pl : zplanes) b += pl.jobs.bytes;
    return b;
}

std::string Diffusion::describe() const
{
    std::ostringstream o;
    const char* ax = "xyz";
    if (!planes.empty() || !zplanes.empty()) o << "plane-classes-per-launch=" << (plane_merge == 0 ? std::string("all") : std::to_string(plane_merge)) << " ";
    for (const auto& pl : planes) o << "xy:planes(jobs=" << pl.n << ",smem=" << sweep_planes_smem(pl.floats) << ") ";
    for (const auto& pl : zplanes) o << "z:xz-planes(jobs=" << pl.n << ",smem=" << sweep_planes_smem(pl.floats) << ") ";
    for (int a = 0; a < 3; ++a)
        for (const auto& l : planes_for(a) ? rest[a] : lists[a]) {
            if (l.n == 0) continue;
            o << ax[a] << ":";
            if (l.kind != 2)
                o << (l.kind == 0 ? "x-tma(" : "cols-tma(") << "warps=" << l.tc.warps << ",stages=" << l.tc.stages
                  << ",grid=" << l.tc.grid;
            else o << "global(grid=" << l.ggrid;
            o << ",tiles=" << l.n << ",nmax=" << l.nmax << ") ";
        }
    return o.str();
}

// Measure candidate launch shapes on the real data; the density is saved
// before and restored after, so tuning leaves the state untouched.
int Diffusion::tune()
{
    if (dens_elems == 0) return PCG_OK;
    DevBuf backup;
    if (backup.alloc(dens.bytes) != cudaSuccess) {
        cudaGetLastError();
        return PCG_OK;   // not enough memory to tune safely: keep the defaults
    }
    PCG_CU(ctx, cudaMemcpyAsync(backup.p, dens.p, dens.bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    cudaEvent_t e0, e1;
    PCG_CU(ctx, cudaEventCreate(&e0));
    PCG_CU(ctx, cudaEventCreate(&e1));
    auto time_list = [&](SweepList& l, float* ms) -> int {
        PCG_TRY(launch_list(l, false, nullptr));   // warm
        PCG_CU(ctx, cudaEventRecord(e0, ctx->stream));
        for (int r = 0; r < 3; ++r) PCG_TRY(launch_list(l, false, nullptr));
        PCG_CU(ctx, cudaEventRecord(e1, ctx->stream));
        PCG_CU(ctx, cudaEventSynchronize(e1));
        PCG_CU(ctx, cudaEventElapsedTime(ms, e0, e1));
        return PCG_OK;
    };
    auto bucket = [](uint64_t v) {
        int b = 0;
        while ((1ull << (b + 1)) <= v) ++b;
        return b;
    };
    int rc = PCG_OK;
    for (int a = 0; a < 3 && rc == PCG_OK; ++a) {
        // the lists a sub-step launches
        std::vector<SweepList>& la = planes_for(a) ? rest[a] : lists[a];
        if (la.empty()) continue;
        SweepList& l = la[0];
        if (l.n == 0) continue;
        const std::string key = std::string(l.kind == 0 ? "x" : "cols") + ":n" + std::to_string(l.nmax) + ":l" +
                                std::to_string(bucket(l.lines));
        int best = 0;
        if (!Tuner::get().lookup(key, &best)) {
            float best_ms = 1e30f;
            std::vector<int> cands;
            for (int w : {1, 2, 3, 4, 6, 8})
                for (int st : {2, 3, 4})
                    if (sweep_tma_occupancy(l.kind == 0, w, st, tma_stage_floats(l)) > 0) cands.push_back(w * 16 + st);
            for (int c : cands) {
                rc = config_list(l, c);
                if (rc != PCG_OK) break;
                float ms = 0;
                rc = time_list(l, &ms);
                if (rc != PCG_OK) break;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = c;
                }
            }
            if (rc != PCG_OK) break;
            Tuner::get().store(key, best);
        }
        rc = config_list(l, best);
    }
    // plane launches: one per occupancy class (parallel graph branches) or
    // runs of classes merged into fewer, larger launches
    if (rc == PCG_OK && (!planes.empty() || !zplanes.empty())) {
        int ncls[2] = {0, 0};
        uint64_t njobs = 0;
        for (int p = 0; p < 2; ++p)
            for (int c = 0; c < kPlaneClasses; ++c) {
                ncls[p] += cls_jobs_[p][c].empty() ? 0 : 1;
                njobs += cls_jobs_[p][c].size();
            }
        const std::string key = "planes:x" + std::to_string(ncls[0]) + ":z" + std::to_string(ncls[1]) + ":j" +
                                std::to_string(bucket(njobs));
        int best = 1;
        if (!Tuner::get().lookup(key, &best)) {
            float best_ms = 1e30f;
            auto passes = [&]() -> int {
                PCG_TRY(launch_planes(planes, false, nullptr));
                return launch_planes(zplanes, false, nullptr);
            };
            for (int m : {1, 2, 3, 0}) {
                rc = regroup_planes(m);
                if (rc != PCG_OK) break;
                rc = passes();   // warm
                if (rc != PCG_OK) break;
                cudaError_t ce = cudaEventRecord(e0, ctx->stream);
                for (int r = 0; r < 3 && rc == PCG_OK && ce == cudaSuccess; ++r) rc = passes();
                if (ce == cudaSuccess) ce = cudaEventRecord(e1, ctx->stream);
                if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
                float ms = 0;
                if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
                if (ce != cudaSuccess) rc = cuda_fail(ctx, ce, "plane grouping timing");
                if (rc != PCG_OK) break;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = m;
                }
            }
            if (rc == PCG_OK) Tuner::get().store(key, best);
        }
        if (rc == PCG_OK) rc = regroup_planes(best);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaError_t ce = cudaMemcpyAsync(dens.p, backup.p, dens.bytes, cudaMemcpyDeviceToDevice, ctx->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
    if (rc != PCG_OK) return rc;
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "tune restore");
    return PCG_OK;
}

// ------------------------------------------------------------------ cells

void fill_diff_inst(CellInst& ci, const DiffInstance& d)
{
    ci.nx = d.g.nx;
    ci.ny = d.g.ny;
    ci.nz = d.g.nz;
    ci.S = d.g.n_substrates;
    ci.dx = d.g.dx;
    ci.dy = d.g.dy;
    ci.dz = d.g.dz;
    ci.x_min = d.g.x_min;
    ci.y_min = d.g.y_min;
    ci.z_min = d.g.z_min;
    ci.dens_off = d.dens_off;
    ci.sub_pitch = d.pitch;
    ci.px = d.px;
    ci.vox_base = d.vox_base;
}

void fill_mech_inst(CellInst& ci, const pcg_mechanics_params& m, float x_min, float y_min, float z_min)
{
    ci.mnx = m.mech_grid_nx;
    ci.mny = m.mech_grid_ny;
    ci.mnz = m.mech_grid_nz;
    ci.vs = m.mechanics_voxel_size;
    ci.maxd = m.max_interaction_distance;
    ci.mx_min = x_min;
    ci.my_min = y_min;
    ci.mz_min = z_min;
    // integrate.metal:63-65 with the mechanics GridParams (cell_mechanics.mm:57-67), FP32
    ci.box_hi_x = x_min + static_cast<float>(m.mech_grid_nx) * m.mechanics_voxel_size;
    ci.box_hi_y = y_min + static_cast<float>(m.mech_grid_ny) * m.mechanics_voxel_size;
    ci.box_hi_z = z_min + static_cast<float>(m.mech_grid_nz) * m.mechanics_voxel_size;
    ci.dt_mech = m.dt;
}

int Cells::create(pcg_ctx* c, uint32_t maxc, uint32_t rate_capacity, uint32_t n_instances)
{
    ctx = c;
    // a secretion run names its instance in 24 bits (make_run_word)
    if (n_instances >= kRunNone) return fail(ctx, PCG_ERR_INVALID, "more instances than a batch can hold");
    max_cells = std::max<uint32_t>(maxc, 1);
    n = 0;
    n_rate = 0;
    h_inst.assign(std::max<uint32_t>(n_instances, 1), CellInst{});
    PCG_CU(ctx, inst.alloc(h_inst.size() * sizeof(CellInst)));
    PCG_CU(ctx, soa.alloc(static_cast<size_t>(NUM_FIELDS) * max_cells * sizeof(float)));
    PCG_CU(ctx, cudaMemsetAsync(soa.p, 0, soa.bytes, ctx->stream));
    PCG_CU(ctx, cell_inst.alloc(static_cast<size_t>(max_cells) * sizeof(uint32_t)));
    PCG_CU(ctx, cudaMemsetAsync(cell_inst.p, 0, cell_inst.bytes, ctx->stream));
    const size_t rc = std::max<uint32_t>(rate_capacity, 1);
    PCG_CU(ctx, rates.alloc(4 * rc * sizeof(double)));
    PCG_CU(ctx, cudaMemsetAsync(rates.p, 0, rates.bytes, ctx->stream));
    PCG_CU(ctx, coef.alloc(3 * rc * sizeof(double)));
    PCG_CU(ctx, coef_cells.alloc(3 * rc * sizeof(double)));
    PCG_CU(ctx, coef_flags.alloc(h_inst.size() * sizeof(uint32_t)));
    PCG_CU(ctx, cudaMemsetAsync(coef_flags.p, 0xFF, coef_flags.bytes, ctx->stream));   // all terms until prepared
    PCG_CU(ctx, active.alloc(max_cells));
    PCG_CU(ctx, pos64.alloc(3ull * max_cells * sizeof(double)));
    PCG_CU(ctx, cudaMemsetAsync(pos64.p, 0xFF, pos64.bytes, ctx->stream));   // no masters yet
    for (DevBuf* b : {&keys, &vals, &skeys, &sorder, &ktmp, &vtmp})
        PCG_CU(ctx, b->alloc((static_cast<size_t>(max_cells) + 1) * sizeof(uint32_t)));
    PCG_CU(ctx, run_word.alloc((static_cast<size_t>(max_cells) + 1) * sizeof(uint64_t)));
    max_tiles = so_max_tiles(max_cells, static_cast<uint32_t>(h_inst.size()));
    PCG_CU(ctx, tiles.alloc(static_cast<size_t>(max_tiles) * sizeof(SegTile)));
    PCG_CU(ctx, inst_tile.alloc(h_inst.size() * sizeof(uint32_t)));
    PCG_CU(ctx, sort_scr.alloc(so_scratch_bytes(max_tiles)));
    PCG_CU(ctx, run_scr.alloc(so_run_scratch_bytes(max_cells)));
    PCG_CU(ctx, cudaMemsetAsync(ktmp.p, 0, ktmp.bytes, ctx->stream));   // run count 0 until the first order
    inst_dirty = coef_dirty = order_dirty = true;
    return PCG_OK;
}

int Cells::sync_inst()
{
    if (!inst_dirty) return PCG_OK;
    PCG_CU(ctx, cudaMemcpyAsync(inst.p, h_inst.data(), h_inst.size() * sizeof(CellInst), cudaMemcpyHostToDevice,
                                ctx->stream));
    // the secretion order's tiles and digits follow the instances' cell
    // ranges and grids
    std::vector<SegTile> ht;
    std::vector<uint32_t> hit;
    so_tiles(h_inst.data(), static_cast<uint32_t>(h_inst.size()), ht, hit);
    if (ht.size() > max_tiles) return fail(ctx, PCG_ERR_INVALID, "cell ranges need more sort tiles than allocated");
    ntiles = static_cast<uint32_t>(ht.size());
    n_inst_tiled = static_cast<uint32_t>(hit.size());
    if (n_inst_tiled) PCG_CU(ctx, cudaMemcpyAsync(inst_tile.p, hit.data(), hit.size() * sizeof(uint32_t),
                                                  cudaMemcpyHostToDevice, ctx->stream));
    uint32_t max_vox = 1;
    for (const CellInst& ci : h_inst) max_vox = std::max(max_vox, ci.nx * ci.ny * ci.nz);
    so_plan(max_vox, &so_passes, &so_bits);
    if (ntiles) PCG_CU(ctx, cudaMemcpyAsync(tiles.p, ht.data(), ht.size() * sizeof(SegTile), cudaMemcpyHostToDevice,
                                            ctx->stream));
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    inst_dirty = false;
    return PCG_OK;
}

int Cells::upload_soa(uint32_t off, uint32_t count, const float* host, uint32_t soa_max, uint32_t first,
                      uint32_t nf)
{
    if (count == 0 || nf == 0) return PCG_OK;
    float* dst = soa.as<float>() + static_cast<size_t>(first) * max_cells + off;
    PCG_CU(ctx, cudaMemcpy2DAsync(dst, static_cast<size_t>(max_cells) * sizeof(float),
                                  host + static_cast<size_t>(first) * soa_max, static_cast<size_t>(soa_max) * sizeof(float),
                                  static_cast<size_t>(count) * sizeof(float), nf, cudaMemcpyHostToDevice, ctx->stream));
    const uint32_t last = first + nf;
    if (first <= F_TOTAL_VOL && F_TOTAL_VOL < last) coef_dirty = true;
    if (first <= F_VOXEL_IDX && F_VOXEL_IDX < last) order_dirty = true;
    return PCG_OK;
}

int Cells::download_soa(uint32_t off, uint32_t count, float* host, uint32_t soa_max, uint32_t first, uint32_t nf)
{
    if (count == 0 || nf == 0) return PCG_OK;
    const float* src = soa.as<float>() + static_cast<size_t>(first) * max_cells + off;
    PCG_CU(ctx, cudaMemcpy2DAsync(host + static_cast<size_t>(first) * soa_max, static_cast<size_t>(soa_max) * sizeof(float),
                                  src, static_cast<size_t>(max_cells) * sizeof(float),
                                  static_cast<size_t>(count) * sizeof(float), nf, cudaMemcpyDeviceToHost, ctx->stream));
    return PCG_OK;
}

int Cells::set_rates(uint32_t off, uint32_t count, const double* sec, const double* upt, const double* sat,
                     const double* ne)
{
    const size_t cap = rates.bytes / (4 * sizeof(double));
    if (static_cast<size_t>(off) + count > cap) return fail(ctx, PCG_ERR_INVALID, "rate arrays exceed capacity");
    const double* src[4] = {sec, upt, sat, ne};
    for (int q = 0; q < 4; ++q) {
        double* dst = rates.as<double>() + q * cap + off;
        if (src[q])
            PCG_CU(ctx, cudaMemcpyAsync(dst, src[q], static_cast<size_t>(count) * sizeof(double), cudaMemcpyHostToDevice,
                                        ctx->stream));
        else
            PCG_CU(ctx, cudaMemsetAsync(dst, 0, static_cast<size_t>(count) * sizeof(double), ctx->stream));
    }
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    coef_dirty = true;
    return PCG_OK;
}

int Cells::set_active(uint32_t off, uint32_t count, const uint8_t* act)
{
    if (act) {
        PCG_CU(ctx, cudaMemcpyAsync(active.as<uint8_t>() + off, act, count, cudaMemcpyHostToDevice, ctx->stream));
        PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));   // the caller may reuse 'act' on return
        has_active = true;
    } else {
        PCG_CU(ctx, cudaMemsetAsync(active.as<uint8_t>() + off, 1, count, ctx->stream));
    }
    order_dirty = true;
    return PCG_OK;
}

int Cells::set_cell_instances(const std::vector<uint32_t>& counts)
{
    std::vector<uint32_t> ci;
    for (size_t i = 0; i < counts.size(); ++i) ci.insert(ci.end(), counts[i], static_cast<uint32_t>(i));
    if (ci.size() > max_cells) return fail(ctx, PCG_ERR_INVALID, "more cells than capacity");
    if (!ci.empty()) PCG_CU(ctx, cudaMemcpyAsync(cell_inst.p, ci.data(), ci.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
    return PCG_OK;
}

int Cells::clear_masters(uint32_t off, uint32_t count)
{
    if (count == 0) return PCG_OK;
    for (int a = 0; a < 3; ++a)
        PCG_CU(ctx, cudaMemsetAsync(pos64.as<double>() + static_cast<size_t>(a) * max_cells + off, 0xFF,
                                    static_cast<size_t>(count) * sizeof(double), ctx->stream));
    return PCG_OK;
}

int Cells::download_positions(uint32_t off, uint32_t count, double* xyz)
{
    if (count == 0) return PCG_OK;
    std::vector<float> p32(3ull * count);
    PCG_CU(ctx, cudaMemcpy2DAsync(xyz, static_cast<size_t>(count) * sizeof(double), pos64.as<double>() + off,
                                  static_cast<size_t>(max_cells) * sizeof(double),
                                  static_cast<size_t>(count) * sizeof(double), 3, cudaMemcpyDeviceToHost, ctx->stream));
    PCG_TRY(download_soa(off, count, p32.data(), count, F_POS_X, 3));
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    for (size_t q = 0; q < 3ull * count; ++q)
        if (static_cast<float>(xyz[q]) != p32[q]) xyz[q] = p32[q];
    return PCG_OK;
}

int Cells::build_order(uint64_t total_vox)
{
    PCG_TRY(sync_inst());
    invalid_key = static_cast<uint32_t>(total_vox);
    // with the constants known, the sort's last pass moves them into the order
    const bool consts = coef_dt >= 0.0;
    const uint32_t cap = static_cast<uint32_t>(rates.bytes / (4 * sizeof(double)));
    if (consts) PCG_TRY(cell_constants(cap));
    cudaError_t e = launch_sec_order(ctx->stream, tiles.as<SegTile>(), ntiles, inst_tile.as<uint32_t>(), n_inst_tiled,
                                     n, so_passes, so_bits, soa.as<float>(),
                                     max_cells, inst.as<CellInst>(), has_active ? active.as<uint8_t>() : nullptr,
                                     cell_inst.as<uint32_t>(), invalid_key, keys.as<uint32_t>(), ktmp.as<uint32_t>(),
                                     vtmp.as<uint32_t>(), skeys.as<uint32_t>(), sorder.as<uint32_t>(), sort_scr.p,
                                     ktmp.as<uint32_t>() + n, vals.as<uint32_t>(), run_word.as<uint64_t>(), run_scr.p,
                                     consts ? coef_cells.as<double>() : nullptr, coef.as<double>(), cap,
                                     coef_flags.as<uint32_t>());
    if (e != cudaSuccess) return cuda_fail(ctx, e, "secretion order");
    ctx->launches += so_launches(ntiles, so_passes, n);
    order_dirty = false;
    return PCG_OK;
}

int Cells::cell_constants(uint32_t cap)
{
    if (!coef_dirty) return PCG_OK;
    cudaError_t e = launch_sec_cell_consts(ctx->stream, soa.as<float>(), max_cells, n, cell_inst.as<uint32_t>(),
                                           inst.as<CellInst>(), rates.as<double>(), cap, coef_dt, coef_cells.as<double>(),
                                           coef_flags.as<uint32_t>(), static_cast<uint32_t>(h_inst.size()));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "secretion constants");
    if (n) ctx->launches++;
    coef_dirty = false;
    return PCG_OK;
}

int Cells::order_launches() const
{
    return so_launches(ntiles, so_passes, n);
}

int Cells::sorted_constants()
{
    const uint32_t cap = static_cast<uint32_t>(rates.bytes / (4 * sizeof(double)));
    PCG_TRY(cell_constants(cap));
    cudaError_t e = launch_sec_permute(ctx->stream, skeys.as<uint32_t>(), sorder.as<uint32_t>(), n,
                                       cell_inst.as<uint32_t>(), inst.as<CellInst>(), invalid_key,
                                       coef_flags.as<uint32_t>(), coef_cells.as<double>(), cap, coef.as<double>());
    if (e != cudaSuccess) return cuda_fail(ctx, e, "secretion permute");
    if (n) ctx->launches++;
    return PCG_OK;
}

int Cells::prepare_secretion(double dt, uint64_t total_vox)
{
    PCG_TRY(sync_inst());
    if (coef_dt != dt) coef_dirty = true;
    const bool stale = coef_dirty;
    coef_dt = dt;
    if (order_dirty || invalid_key != static_cast<uint32_t>(total_vox)) return build_order(total_vox);
    if (stale) return sorted_constants();
    return PCG_OK;
}

int Cells::secrete(Diffusion& d, const uint8_t* mask)
{
    uint32_t max_s = 0;
    for (const CellInst& ci : h_inst) max_s = std::max(max_s, ci.S);
    cudaError_t e = launch_secrete(ctx->stream, d.dens.as<float>(), vals.as<uint32_t>(), run_word.as<uint64_t>(),
                                   ktmp.as<uint32_t>() + n, n, max_s,
                                   inst.as<CellInst>(), coef.as<double>(),
                                   static_cast<uint32_t>(rates.bytes / (4 * sizeof(double))),
                                   coef_flags.as<uint32_t>(), mask, sec_block);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "secretion launch");
    if (n && max_s) ctx->launches++;
    return PCG_OK;
}

uint64_t Cells::device_bytes() const
{
    return inst.bytes + soa.bytes + pos64.bytes + cell_inst.bytes + rates.bytes + coef.bytes + coef_cells.bytes + coef_flags.bytes + active.bytes +
           keys.bytes + vals.bytes +
           skeys.bytes + sorder.bytes + ktmp.bytes + vtmp.bytes + sort_scr.bytes + tiles.bytes + inst_tile.bytes +
           run_scr.bytes +
           run_word.bytes;
}

// ------------------------------------------------------------------ mechanics

int Mechanics::create(pcg_ctx* c, uint32_t tmv, uint32_t maxc)
{
    ctx = c;
    total_mvox = tmv;
    cap = std::max<uint32_t>(maxc, 1);
    PCG_CU(ctx, mech_forces_prepare());
    for (DevBuf* b : {&keys, &slots, &sorder, &dcnt, &dhash})
        PCG_CU(ctx, b->alloc(static_cast<size_t>(cap) * sizeof(uint32_t)));
    PCG_CU(ctx, placed.alloc(static_cast<size_t>(cap) * sizeof(uint2)));
    PCG_CU(ctx, counts.alloc((static_cast<size_t>(tmv) + 1) * sizeof(uint32_t)));
    PCG_CU(ctx, start.alloc((static_cast<size_t>(tmv) + 1) * sizeof(uint32_t)));
    PCG_CU(ctx, cudaMemsetAsync(start.p, 0, start.bytes, ctx->stream));
    PCG_CU(ctx, scan_scr.alloc(scan_scratch_bytes(static_cast<uint64_t>(tmv) + 1)));
    // one spare element: the force loop loads the next candidate without a bounds test
    PCG_CU(ctx, spos.alloc((static_cast<size_t>(cap) + 1) * sizeof(float4)));
    PCG_CU(ctx, sprm.alloc((static_cast<size_t>(cap) + 1) * sizeof(float4)));
    return PCG_OK;
}

int Mechanics::launches_forces(uint32_t n) const
{
    (void)n;
    return 1 /*memset*/ + 1 /*bin*/ + scan_launches(total_mvox + 1ull) + 2 /*place, order*/ + 1 /*forces*/;
}

// computeForces: bin -> counting sort (start table, stable order, sorted SoA) -> forces
int Mechanics::forces(Cells& c, const uint8_t* mask)
{
    PCG_TRY(binsort(c, mask));
    return force_pass(c, mask);
}

int Mechanics::binsort(Cells& c, const uint8_t* mask)
{
    if (c.n == 0) return PCG_OK;
    if (c.n > cap) return fail(ctx, PCG_ERR_INVALID, "more cells than the mechanics capacity");
    PCG_TRY(c.sync_inst());
    cudaStream_t st = ctx->stream;
    PCG_CU(ctx, cudaMemsetAsync(counts.p, 0, counts.bytes, st));
    cudaError_t e = launch_mech_bin(st, c.soa.as<float>(), c.max_cells, c.n, c.cell_inst.as<uint32_t>(),
                                    c.inst.as<CellInst>(), keys.as<uint32_t>(), slots.as<uint32_t>(),
                                    counts.as<uint32_t>(), mask, bin_block);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "bin launch");
    e = scan_exclusive(st, counts.as<uint32_t>(), start.as<uint32_t>(), static_cast<uint64_t>(total_mvox) + 1, scan_scr.p);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "start-table scan");
    e = launch_mech_order(st, c.soa.as<float>(), c.max_cells, keys.as<uint32_t>(), slots.as<uint32_t>(),
                          start.as<uint32_t>(), c.n, placed.as<uint2>(), lazy_sorder ? nullptr : sorder.as<uint32_t>(),
                          spos.as<float4>(), sprm.as<float4>(), bin_block);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "bin order launch");
    ctx->launches += launches_forces(c.n) - 2;   // the memset is not a kernel; forces counted below
    sorder_valid = !lazy_sorder;
    return PCG_OK;
}

int Mechanics::stable_order(uint32_t n)
{
    if (sorder_valid || n == 0) return PCG_OK;
    cudaError_t e = launch_mech_stable_order(ctx->stream, keys.as<uint32_t>(), start.as<uint32_t>(), placed.as<uint2>(),
                                             n, sorder.as<uint32_t>());
    if (e != cudaSuccess) return cuda_fail(ctx, e, "stable order launch");
    ctx->launches++;
    sorder_valid = true;
    return PCG_OK;
}

int Mechanics::force_pass(Cells& c, const uint8_t* mask)
{
    if (c.n == 0) return PCG_OK;
    cudaStream_t st = ctx->stream;
    cudaError_t e = launch_mech_forces(st, spos.as<float4>(), sprm.as<float4>(), start.as<uint32_t>(), c.n,
                           c.cell_inst.as<uint32_t>(), c.inst.as<CellInst>(), c.soa.as<float>(), c.max_cells, diag ? dcnt.as<uint32_t>() : nullptr, diag ? dhash.as<uint32_t>() : nullptr,
                           mask, fshape);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "forces launch");
    ctx->launches++;
    return PCG_OK;
}

int Mechanics::integrate(Cells& c, float dt_override, const uint8_t* mask)
{
    if (c.n == 0) return PCG_OK;
    PCG_TRY(c.sync_inst());
    cudaError_t e = launch_mech_integrate(ctx->stream, c.soa.as<float>(), c.pos64.as<double>(), c.max_cells, c.n,
                                          c.cell_inst.as<uint32_t>(), c.inst.as<CellInst>(), dt_override, mask,
                                          int_block);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "integrate launch");
    ctx->launches++;
    bool refresh = false;
    for (const auto& ci : c.h_inst) refresh = refresh || (ci.flags & INST_REFRESH_VOXELS);
    if (refresh) c.order_dirty = true;
    return PCG_OK;
}

uint64_t Mechanics::device_bytes() const
{
    return keys.bytes + slots.bytes + placed.bytes + sorder.bytes + counts.bytes +
           start.bytes + scan_scr.bytes + spos.bytes + sprm.bytes + dcnt.bytes + dhash.bytes;
}

}  // namespace pcg
