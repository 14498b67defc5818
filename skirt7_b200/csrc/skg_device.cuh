// skg_device.cuh -- device-side building blocks shared by every kernel of the library:
// counter-based Philox4x32-10 random numbers, small vector helpers and the error word.
#pragma once
#include <cstdint>
#include <cfloat>
#include <cuda_runtime.h>

#define SKG_HD __host__ __device__ __forceinline__
#define SKG_D __device__ __forceinline__

namespace skg {

// ------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11): a bijection of a 128-bit counter under a 64-bit key, ten rounds of two 32x32->64
// multiplies with a Weyl-sequence key schedule.  Every packet owns a disjoint counter range
// (packet id in the upper words), so results do not depend on scheduling.
struct Philox {
    uint32_t key0, key1;      // seed
    uint32_t c1, c2, c3;      // packet id / stream words
    uint32_t c0;              // draw block counter
    uint32_t b0, b1, b2, b3;  // the current block (named, not an array: stays in registers)
    int      left;            // unread words of the block

    SKG_D void init(uint64_t seed, uint64_t packet, uint32_t stream) {
        key0 = (uint32_t)seed; key1 = (uint32_t)(seed >> 32);
        c1 = (uint32_t)packet; c2 = (uint32_t)(packet >> 32); c3 = stream;
        c0 = 0; left = 0;
    }
    SKG_D void refill() {
        uint32_t x0 = c0, x1 = c1, x2 = c2, x3 = c3;
        uint32_t k0 = key0, k1 = key1;
#pragma unroll
        for (int r = 0; r < 10; r++) {
            uint32_t hi0 = __umulhi(0xD2511F53u, x0), lo0 = 0xD2511F53u * x0;
            uint32_t hi1 = __umulhi(0xCD9E8D57u, x2), lo1 = 0xCD9E8D57u * x2;
            uint32_t y0 = hi1 ^ x1 ^ k0, y1 = lo1, y2 = hi0 ^ x3 ^ k1, y3 = lo0;
            x0 = y0; x1 = y1; x2 = y2; x3 = y3;
            k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
        }
        b0 = x0; b1 = x1; b2 = x2; b3 = x3;
        left = 4;
        c0++;
    }
    SKG_D uint32_t next32() {
        if (left == 0) refill();
        const int i = 4 - (left--);
        return (i == 0) ? b0 : (i == 1) ? b1 : (i == 2) ? b2 : b3;
    }
    // uniform deviate in the open interval (0,1) with 2^-32 resolution (the reference's MT19937
    // deviates also exclude 0 and 1, Random.cpp:125)
    SKG_D double uniform() { return ((double)next32() + 0.5) * 2.3283064365386963e-10; }
    SKG_D float uniformf() {
        // 24 significant bits, strictly inside (0,1)
        return ((float)(next32() >> 8) + 0.5f) * 5.9604644775390625e-08f;
    }
};

// ------------------------------------------------------------------------------------------
template<typename R> struct V3 { R x, y, z; };
template<typename R> SKG_HD V3<R> mk3(R a, R b, R c) { V3<R> v; v.x = a; v.y = b; v.z = c; return v; }

// error word bits (OR-ed into a device status word; read back by the host)
enum : uint32_t {
    ERR_STEP_BUDGET = 1u << 0,
    ERR_NAN_TAU     = 1u << 1,
    ERR_BAD_CELL    = 1u << 2,
    ERR_SCATT_BUDGET= 1u << 3,
    ERR_CAPACITY    = 1u << 4,
};

SKG_D void atomic_add_f64(double* p, double v) { atomicAdd(p, v); }

}  // namespace skg
