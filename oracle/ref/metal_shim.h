/*
 * metal_shim.h — lets the reference's Metal compute shaders
 * (shaders/diffusion_2d.metal, mechanics.metal, integrate.metal) compile as
 * plain C++ on the CPU, so the reference's own kernel bodies can be run as
 * the checker for the oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * A Metal kernel becomes an ordinary function taking the thread id as its
 * last argument; ref_wrap.cpp calls it once per thread id.  Address-space
 * qualifiers vanish, `constant` references become const references, and the
 * few Metal builtins the shaders use are given their documented meanings
 * (as_type = bit cast, clamp = min(max(x, lo), hi), relaxed atomics).
 * Arithmetic is IEEE FP32 (the reference compiles with fast math on the
 * GPU; on the CPU the plain IEEE meaning of the written formulas is used).
 */
#ifndef PCG_METAL_SHIM_H
#define PCG_METAL_SHIM_H
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>

typedef uint32_t uint;
#define kernel
#define device
#define constant const

typedef std::atomic<uint32_t> atomic_uint;
using std::atomic_fetch_add_explicit;
using std::atomic_load_explicit;
using std::atomic_store_explicit;
using std::memory_order_relaxed;
using std::sqrt;

template <class T, class U>
static inline T as_type(U u)
{
    static_assert(sizeof(T) == sizeof(U), "as_type size");
    T t;
    std::memcpy(&t, &u, sizeof t);
    return t;
}
static inline int clamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline float clamp(float v, float lo, float hi) { return std::fmin(std::fmax(v, lo), hi); }
static inline uint min(uint a, uint b) { return a < b ? a : b; }
#endif
