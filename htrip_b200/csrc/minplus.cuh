// Packed u16 tropical (min, +) arithmetic for sm_100a.
//
// Distances are uint16 with INF = 60000, the reference's dist_t / INF
// (include/htrip/types.hpp:34,45).  The reference's product is the clamped
// sum add_dist(a, b) = min(a + b, INF) (types.hpp:66-70); its AVX2 loops use
// _mm256_adds_epu16 followed by _mm256_min_epu16 against a value <= INF,
// which is the same function.  Every update here computes exactly
//     c' = min(c, min(a + b, INF))      with a, b, c in [0, INF]
// on two lanes packed in one 32-bit register, using the sm_90+ PTX packed
// integer instructions add.u16x2 (wrapping, no saturation) and min.u16x2:
//
//  * fast form, valid when a <= INF_HEADROOM (a + b <= 65535 for every
//    b <= INF, so add.u16x2 cannot wrap, and a sum >= INF loses to c <= INF):
//        c' = min.u16x2(add.u16x2(b, aa), c)
//  * clamped form, valid for every a <= INF: with t = INF - a,
//        c' = min.u16x2(add.u16x2(min.u16x2(b, tt), aa), c)
//    because min(b, INF - a) + a = min(a + b, INF) never exceeds INF.
//  * a == INF: the update is a no-op (min(a + b, INF) = INF >= c) and is
//    skipped.
// aa / tt are a / t replicated into both halves.
#pragma once
#include <cstdint>

namespace hb {

typedef uint16_t u16;
typedef uint32_t u32;

constexpr u16 INF = 60000;
constexpr u32 INF2 = 0xEA60EA60u;          // INF in both halves
constexpr u32 INF_HEADROOM = 65535u - INF; // 5535

// Traversal weight of the edge between two adjacent cells of weights wu, wv
// (GridMap::edgeWeight, grid_map.hpp:327-334): INF if either is INF or more,
// else max(1, (wu + wv) / 2).
__host__ __device__ __forceinline__ u16 edge_weight(u16 wu, u16 wv) {
    if (wu >= INF || wv >= INF) return INF;
    const u16 avg = (u16)(((u32)wu + (u32)wv) / 2);
    return avg == 0 ? (u16)1 : avg;
}

__device__ __forceinline__ u32 add2(u32 a, u32 b) {
    u32 r;
    asm("add.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ u32 min2(u32 a, u32 b) {
    u32 r;
    asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ u32 max2(u32 a, u32 b) {
    u32 r;
    asm("max.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
// a (low 16 bits) replicated into both halves.
__device__ __forceinline__ u32 splat(u32 a) { return __byte_perm(a, 0, 0x1010); }

// c' = min(c, min(b + a, INF)) lane-wise, a <= INF_HEADROOM.
__device__ __forceinline__ u32 acc_fast(u32 c, u32 b, u32 aa) { return min2(add2(b, aa), c); }
// c' = min(c, min(b + a, INF)) lane-wise, any a <= INF (tt = splat(INF - a)).
__device__ __forceinline__ u32 acc_clamp(u32 c, u32 b, u32 aa, u32 tt) {
    return min2(add2(min2(b, tt), aa), c);
}

// Scalar clamped tropical product (add_dist, types.hpp:66).
__host__ __device__ __forceinline__ u32 sat_add(u32 a, u32 b) {
    u32 s = a + b;
    return s < INF ? s : INF;
}

}  // namespace hb
