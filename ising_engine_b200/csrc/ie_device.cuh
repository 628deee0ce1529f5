// Device primitives of the B200 Metropolis engine: the master ChaCha8 stream
// (random access by draw index), the per-cell Xoshiro256++ x8 lanes seeded by
// SplitMix64, the reference's fast_exp in uncontracted f64, and the 8x8 bit
// transpose between the reference spin-word layout and the lane-major layout.
#pragma once
#include <cstdint>

namespace ie {

// ---------------------------------------------------------------------------
// Master stream: rand_chacha 0.3.1 ChaCha8Rng (8 rounds, 64-bit block counter
// in words 12-13, stream id 0 in 14-15). rand_core's BlockRng hands out u64
// draws as two consecutive u32 words, low first, so draw k is words
// (2(k%8), 2(k%8)+1) of block k/8. Every draw on this path is 64-bit
// (gen::<u64> at ultimate.rs:272 / engine.rs:596, gen::<f64> at engine.rs:727).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t rotl32(uint32_t x, int k) { return __funnelshift_l(x, x, k); }

#define IE_QR(a, b, c, d)                              \
    a += b; d ^= a; d = rotl32(d, 16);                 \
    c += d; b ^= c; b = rotl32(b, 12);                 \
    a += b; d ^= a; d = rotl32(d, 8);                  \
    c += d; b ^= c; b = rotl32(b, 7);

__device__ __forceinline__ uint64_t chacha8_draw(const uint32_t key[8], uint64_t k) {
    const uint64_t blk = k >> 3;
    const int w = (int)(k & 7);
    uint32_t x0 = 0x61707865u, x1 = 0x3320646eu, x2 = 0x79622d32u, x3 = 0x6b206574u;
    uint32_t x4 = key[0], x5 = key[1], x6 = key[2], x7 = key[3];
    uint32_t x8 = key[4], x9 = key[5], x10 = key[6], x11 = key[7];
    uint32_t x12 = (uint32_t)blk, x13 = (uint32_t)(blk >> 32), x14 = 0u, x15 = 0u;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        IE_QR(x0, x4, x8, x12) IE_QR(x1, x5, x9, x13) IE_QR(x2, x6, x10, x14) IE_QR(x3, x7, x11, x15)
        IE_QR(x0, x5, x10, x15) IE_QR(x1, x6, x11, x12) IE_QR(x2, x7, x8, x13) IE_QR(x3, x4, x9, x14)
    }
    x0 += 0x61707865u; x1 += 0x3320646eu; x2 += 0x79622d32u; x3 += 0x6b206574u;
    x4 += key[0]; x5 += key[1]; x6 += key[2]; x7 += key[3];
    x8 += key[4]; x9 += key[5]; x10 += key[6]; x11 += key[7];
    x12 += (uint32_t)blk; x13 += (uint32_t)(blk >> 32);
    uint32_t lo = x0, hi = x1;
    if (w == 1) { lo = x2; hi = x3; }
    if (w == 2) { lo = x4; hi = x5; }
    if (w == 3) { lo = x6; hi = x7; }
    if (w == 4) { lo = x8; hi = x9; }
    if (w == 5) { lo = x10; hi = x11; }
    if (w == 6) { lo = x12; hi = x13; }
    if (w == 7) { lo = x14; hi = x15; }
    return (uint64_t)lo | ((uint64_t)hi << 32);
}
#undef IE_QR

// ---------------------------------------------------------------------------
// Xoshiro256PlusPlusX8 (engine.rs:81-172). Lane l of a cell's generator is
// seeded with SplitMix64 outputs 4l..4l+3 of seed = base_seed + cell
// (lane-major fill, engine.rs:96-101); output i of SplitMix64 is
// mix(seed + (i+1) * golden_gamma).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t splitmix_at(uint64_t seed, uint64_t i) {
    uint64_t z = seed + (i + 1) * 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

// Xoshiro256++ on 32-bit halves (lo, hi) of s0..s3. One step of the state
// (engine.rs:113-121) is s1' = s1^s2^s0, s0' = s0^s3^s1, s2' = s2^s0^(s1<<17),
// s3' = rotl(s3^s1, 45): one 3-input XOR per half for s0, s1, s2 and a funnel
// shift pair for s3, so the step's dependency depth is two instructions.
struct Xoshiro {
    uint32_t a0, a1, b0, b1, c0, c1, d0, d1;  // s0, s1, s2, s3 as (lo, hi)
    __device__ __forceinline__ static uint32_t xor3(uint32_t x, uint32_t y, uint32_t z) {
        uint32_t r;
        asm("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(r) : "r"(x), "r"(y), "r"(z));
        return r;
    }
    __device__ __forceinline__ void set(int i, uint64_t v) {
        const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
        if (i == 0) { a0 = lo; a1 = hi; }
        else if (i == 1) { b0 = lo; b1 = hi; }
        else if (i == 2) { c0 = lo; c1 = hi; }
        else { d0 = lo; d1 = hi; }
    }
    __device__ __forceinline__ void seed_lane(uint64_t cell_seed, int lane) {
#pragma unroll
        for (int i = 0; i < 4; i++) set(i, splitmix_at(cell_seed, 4 * lane + i));
    }
    __device__ __forceinline__ void advance() {
        const uint32_t t0 = b0 << 17, t1 = __funnelshift_l(b0, b1, 17);
        const uint32_t x0 = d0 ^ b0, x1 = d1 ^ b1;
        const uint32_t nb0 = xor3(b0, c0, a0), nb1 = xor3(b1, c1, a1);
        const uint32_t na0 = xor3(a0, d0, b0), na1 = xor3(a1, d1, b1);
        const uint32_t nc0 = xor3(c0, a0, t0), nc1 = xor3(c1, a1, t1);
        d1 = __funnelshift_l(x1, x0, 13);  // rotl by 45 = halves swapped, then rotl by 13
        d0 = __funnelshift_l(x0, x1, 13);
        a0 = na0;
        a1 = na1;
        b0 = nb0;
        b1 = nb1;
        c0 = nc0;
        c1 = nc1;
    }
    // Raw 64-bit output of engine.rs:110-112; the reference's uniform is
    // (result >> 12) * 2^-52 exactly.
    __device__ __forceinline__ uint64_t next() {
        const uint64_t s0 = ((uint64_t)a1 << 32) | a0, s3 = ((uint64_t)d1 << 32) | d0;
        const uint64_t result = rotl64(s0 + s3, 23) + s0;
        advance();
        return result;
    }
    // Top 32 bits of the next output (the output's uniform is determined to
    // within 2^-32 by them).
    __device__ __forceinline__ uint32_t next_hi() {
        const uint64_t s0 = ((uint64_t)a1 << 32) | a0, s3 = ((uint64_t)d1 << 32) | d0;
        const uint64_t result = rotl64(s0 + s3, 23) + s0;
        advance();
        return (uint32_t)(result >> 32);
    }
    // Jump: the state after D more steps, given the coefficients (bit i of
    // poly[i / 64] = coefficient of x^i) of x^D mod P(x), P the characteristic
    // polynomial of the state transition M: M^D s = sum of r_i M^i s over the
    // set coefficients r_i (Cayley-Hamilton), accumulated over 256 steps.
    __device__ __forceinline__ void jump(const uint64_t* __restrict__ poly) {
        uint32_t j[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
        for (int w = 0; w < 8; w++) {
            const uint32_t p = (uint32_t)(__ldg(poly + (w >> 1)) >> (32 * (w & 1)));
#pragma unroll 4
            for (int b = 0; b < 32; b++) {
                const uint32_t m = 0u - ((p >> b) & 1u);
                j[0] ^= a0 & m;
                j[1] ^= a1 & m;
                j[2] ^= b0 & m;
                j[3] ^= b1 & m;
                j[4] ^= c0 & m;
                j[5] ^= c1 & m;
                j[6] ^= d0 & m;
                j[7] ^= d1 & m;
                advance();
            }
        }
        a0 = j[0];
        a1 = j[1];
        b0 = j[2];
        b1 = j[3];
        c0 = j[4];
        c1 = j[5];
        d0 = j[6];
        d1 = j[7];
    }
};

// ---------------------------------------------------------------------------
// fast_exp (engine.rs:181-205) in f64 with every operation explicitly rounded,
// in the reference's evaluation order, so no multiply-add is ever fused: the
// result is bit-identical to the uncontracted host evaluation.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double fast_exp_rn(double x) {
    if (x < -20.0) x = -20.0;
    if (x > 0.0) x = 0.0;
    const double r = __dmul_rn(x, 0.0625);
    const double r2 = __dmul_rn(r, r);
    const double r3 = __dmul_rn(r2, r);
    double p = __dadd_rn(1.0, r);
    p = __dadd_rn(p, __dmul_rn(0.5, r2));
    p = __dadd_rn(p, __dmul_rn(1.0 / 6.0, r3));
    p = __dadd_rn(p, __dmul_rn(__dmul_rn(1.0 / 24.0, r2), r2));
    p = __dadd_rn(p, __dmul_rn(__dmul_rn(1.0 / 120.0, r2), r3));
    p = __dadd_rn(p, __dmul_rn(__dmul_rn(1.0 / 720.0, r3), r3));
    const double p2 = __dmul_rn(p, p);
    const double p4 = __dmul_rn(p2, p2);
    const double p8 = __dmul_rn(p4, p4);
    return __dmul_rn(p8, p8);
}

// Metropolis threshold for an integer dE > 0 at inverse temperature beta:
// the reference accepts iff (res >> 12) * 2^-52 < fast_exp(-dE * beta), i.e.
// iff res <= (ceil(fast_exp(-dE*beta) * 2^52) << 12) - 1. dE <= 0 always
// accepts (all-ones threshold).
__device__ __forceinline__ uint64_t metropolis_threshold(int de, double beta) {
    if (de <= 0) return ~0ULL;
    const double f = fast_exp_rn(__dmul_rn(-(double)de, beta));
    const double scaled = __dmul_rn(f, 4503599627370496.0);  // 2^52, exact
    const uint64_t t = (uint64_t)ceil(scaled);
    return t >= (1ULL << 52) ? ~0ULL : ((t << 12) - 1ULL);
}

// 8x8 bit transpose of a u64 (byte i, bit j) -> (byte j, bit i). Maps the
// reference word layout (bit r = replica r, r = 8*call + lane) to the
// lane-major layout (byte lane, bit call) and back (it is an involution).
__host__ __device__ __forceinline__ uint64_t transpose8x8(uint64_t x) {
    uint64_t t;
    t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAULL;
    x ^= t ^ (t << 7);
    t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCULL;
    x ^= t ^ (t << 14);
    t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ULL;
    x ^= t ^ (t << 28);
    return x;
}

// Spreads the 4 low bits of b to bit 0 of 4 bytes (bit k -> byte k).
__device__ __forceinline__ uint32_t spread4(uint32_t b) { return ((b & 0xFu) * 0x00204081u) & 0x01010101u; }

}  // namespace ie
