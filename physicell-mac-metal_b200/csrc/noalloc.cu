// noalloc.cu — pcg_sort_pairs_static: a stable radix sort of (key, value)
// pairs (mechanics-voxel keys with cell indices give the mechanics
// binning's cell order), run on caller-owned device buffers with every piece of
// scratch taken from one fixed file-scope device array, so that the call
// makes no device allocation of any kind (no cudaMalloc / cudaFree, no
// allocating library).
//
// It is meant for callers that cannot allocate device memory at the point
// of the call: a serving process that has partitioned the whole device
// up front and must not have a request fail with out-of-memory half way,
// or host code that must not make allocation calls, which can synchronise
// the device and stall work on other streams.
#include <mutex>

#include "runtime.h"

namespace pcg {

namespace {

constexpr uint32_t kStaticMaxPairs = PCG_SORT_STATIC_MAX_PAIRS;
constexpr size_t kTmpBytes = static_cast<size_t>(kStaticMaxPairs) * sizeof(uint32_t);   // one ping-pong array
// Per-tile digit histograms and the scan's tile sums for kStaticMaxPairs
// keys take about 129 KiB; the reservation leaves room and is checked against the
// sort's own requirement before the first use.
constexpr size_t kHistBytes = 512u << 10;
constexpr size_t kScratchBytes = 2 * kTmpBytes + kHistBytes;

// The only scratch of pcg_sort_pairs_static (2.5 MiB per device).  Nothing
// in it has to start at zero: every pass writes the histograms, tile sums
// and ping-pong keys it later reads.
static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {};

// Makes ctx's device current for the life of the guard and puts the
// caller's device back afterwards.
class DeviceGuard {
public:
    cudaError_t enter(int device)
    {
        cudaError_t e = cudaGetDevice(&prev_);
        if (e != cudaSuccess) return e;
        if (prev_ == device) return cudaSuccess;
        e = cudaSetDevice(device);
        if (e == cudaSuccess) switched_ = true;
        return e;
    }
    ~DeviceGuard()
    {
        if (switched_) cudaSetDevice(prev_);
    }
private:
    int prev_ = -1;
    bool switched_ = false;
};

// Device address of g_sort_scratch on ctx's device (the current device),
// looked up once per device; the same set-up loads the sort's kernels, so
// that no later call loads a module (which can allocate device memory).
int scratch_for(pcg_ctx* ctx, unsigned char** out)
{
    if (ctx->device < 0 || ctx->device >= kMaxDevices) return fail(ctx, PCG_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[ctx->device]) {
        if (radix_sort_scratch_bytes(kStaticMaxPairs, 32) > kHistBytes)
            return fail(ctx, PCG_ERR_INVALID, "static sort scratch reservation is smaller than the sort needs");
        void* p = nullptr;
        PCG_CU(ctx, cudaGetSymbolAddress(&p, g_sort_scratch));
        PCG_CU(ctx, sort_kernels_load());
        g_addr[ctx->device] = static_cast<unsigned char*>(p);
    }
    *out = g_addr[ctx->device];
    return PCG_OK;
}

bool overlap(const void* a, const void* b, size_t bytes)
{
    const auto x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return x < y + bytes && y < x + bytes;
}

}  // namespace

}  // namespace pcg

using namespace pcg;

extern "C" pcg_status pcg_sort_pairs_static(pcg_ctx* ctx, const uint32_t* keys_in, const uint32_t* vals_in,
                                            uint32_t* keys_out, uint32_t* vals_out, uint32_t n, int key_bits)
{
    if (!ctx) return PCG_ERR_INVALID;
    if (key_bits < 1 || key_bits > 32) return fail(ctx, PCG_ERR_INVALID, "key_bits must be in 1..32");
    if (n > kStaticMaxPairs)
        return fail(ctx, PCG_ERR_INVALID, "pcg_sort_pairs_static: n = " + std::to_string(n) + " exceeds the static limit of " +
                                              std::to_string(kStaticMaxPairs) + " pairs");
    DeviceGuard guard;   // the context's device stays current for the whole call
    PCG_CU(ctx, guard.enter(ctx->device));
    unsigned char* scr = nullptr;
    PCG_TRY(scratch_for(ctx, &scr));
    if (n == 0) return PCG_OK;
    if (!keys_in || !vals_in || !keys_out || !vals_out) return fail(ctx, PCG_ERR_INVALID, "null buffer");
    const size_t b = static_cast<size_t>(n) * sizeof(uint32_t);
    const void* ins[2] = {keys_in, vals_in};
    const void* outs[2] = {keys_out, vals_out};
    for (const void* o : outs)
        for (const void* i : ins)
            if (overlap(o, i, b)) return fail(ctx, PCG_ERR_INVALID, "output overlaps an input");
    if (overlap(keys_out, vals_out, b)) return fail(ctx, PCG_ERR_INVALID, "keys_out overlaps vals_out");
    uint32_t* k_tmp = reinterpret_cast<uint32_t*>(scr);
    uint32_t* v_tmp = reinterpret_cast<uint32_t*>(scr + kTmpBytes);
    void* hist = scr + 2 * kTmpBytes;
    PCG_CU(ctx, radix_sort_pairs(ctx->stream, keys_in, vals_in, keys_out, vals_out, k_tmp, v_tmp, n, key_bits, hist));
    ctx->launches += static_cast<uint64_t>(radix_sort_launches(n, key_bits));
    return PCG_OK;
}
