// qc_codec.cuh -- QC int4 byte -> FP8 E4M3 conversion shared by the
// promotion kernels.
#pragma once
#include <cstdint>

namespace ftdx {

// Four QC bytes -> E4M3 bytes of the four Re parts and of the four Im parts.
// Sign-magnitude nibble: bit 3 sign, bits 2:0 magnitude (0..7).  E4M3 codes of
// the integers 0..7 are 00 38 40 44 48 4A 4C 4E.  The magnitude nibbles of two
// bytes (Im0, Re0, Im1, Re1, low to high) are the four selectors of one byte
// permute over that table, giving the codes of two samples interleaved; two
// more permutes split them into the Re and the Im word, and each sign goes to
// bit 7 (Re: bit 7 of the byte already; Im: bit 3, shifted up by 4).
__device__ __forceinline__ void qc4_to_e4m3(uint32_t w, uint32_t& re, uint32_t& im) {
  constexpr uint32_t kLo = 0x44403800u, kHi = 0x4E4C4A48u;
  const uint32_t m = w & 0x77777777u;
  // a byte permute reads only the low 16 bits (four selectors) of its selector
  const uint32_t c01 = __byte_perm(kLo, kHi, m);        // Im0 Re0 Im1 Re1
  const uint32_t c23 = __byte_perm(kLo, kHi, m >> 16);  // Im2 Re2 Im3 Re3
  re = __byte_perm(c01, c23, 0x7531u) | (w & 0x80808080u);
  im = __byte_perm(c01, c23, 0x6420u) | ((w << 4) & 0x80808080u);
}

// Four QC bytes -> FP6 E3M2 codes (one per byte, bits 5:0) of the four Re
// and the four Im parts.  E3M2 (bias 3, two mantissa bits) holds the integers
// 0..7 exactly: codes 00 0C 10 12 14 15 16 17; the sign is bit 5.
__device__ __forceinline__ void qc4_to_e3m2(uint32_t w, uint32_t& re, uint32_t& im) {
  constexpr uint32_t kLo = 0x12100C00u, kHi = 0x17161514u;
  const uint32_t mr = (w >> 4) & 0x07070707u;
  const uint32_t mi = w & 0x07070707u;
  uint32_t sr = mr | (mr >> 4);
  sr = (sr & 0xFFu) | ((sr >> 8) & 0xFF00u);
  uint32_t si = mi | (mi >> 4);
  si = (si & 0xFFu) | ((si >> 8) & 0xFF00u);
  re = __byte_perm(kLo, kHi, sr) | ((w >> 2) & 0x20202020u);
  im = __byte_perm(kLo, kHi, si) | ((w << 2) & 0x20202020u);
}

// Four QC bytes -> signed 8-bit integers (two's complement, one per byte) of
// the four Re and the four Im parts; sign-magnitude -0 becomes 0.
__device__ __forceinline__ void qc4_to_s8(uint32_t w, uint32_t& re, uint32_t& im) {
  const uint32_t mr = (w >> 4) & 0x07070707u, mi = w & 0x07070707u;
  const uint32_t sr = ((w >> 7) & 0x01010101u) * 0xFFu, si = ((w >> 3) & 0x01010101u) * 0xFFu;
  re = __vsub4(mr ^ sr, sr);  // per byte: sign ? -m : m
  im = __vsub4(mi ^ si, si);
}

// Sixteen 6-bit codes (one per byte of c[0..3], byte b of c[q] = element
// 4q + b) -> the 12-byte packed group of the TMA's 16 x U6 type: element e at
// bits [6e, 6e + 6) of the little-endian 96-bit group.
__device__ __forceinline__ void pack16_u6(const uint32_t (&c)[4], uint32_t (&p)[3]) {
  uint32_t t[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t w = c[q];
    t[q] = (w & 0x3Fu) | (((w >> 8) & 0x3Fu) << 6) | (((w >> 16) & 0x3Fu) << 12) |
           (((w >> 24) & 0x3Fu) << 18);
  }
  p[0] = t[0] | (t[1] << 24);
  p[1] = (t[1] >> 8) | (t[2] << 16);
  p[2] = (t[2] >> 16) | (t[3] << 8);
}

// Four (4,4)b two's-complement bytes (low nibble Re, high nibble Im, each in
// [-8, 7]: the XEngine's packet format, promote_data.cuh:66-67) -> E4M3 bytes
// of the Re and of the Im parts.  Nibbles 0..7 are 0..7 (E4M3 codes 00 38 40
// 44 48 4A 4C 4E); 8..15 are -8..-1 (D0 CE CC CA C8 C4 C0 B8).  For two bytes
// at a time the low three bits of the nibbles (Re0, Im0, Re1, Im1) select from
// the positive and from the negative table, and a third permute over 00 / FF
// turns each nibble's bit 3 into a byte mask that picks between them; two more
// permutes split the interleaved codes into the Re and the Im word.
__device__ __forceinline__ uint32_t tc_pick(uint32_t m, uint32_t signsel) {
  constexpr uint32_t kP0 = 0x44403800u, kP1 = 0x4E4C4A48u;
  constexpr uint32_t kN0 = 0xCACCCED0u, kN1 = 0xB8C0C4C8u;
  const uint32_t pos = __byte_perm(kP0, kP1, m), neg = __byte_perm(kN0, kN1, m);
  const uint32_t mask = __byte_perm(0u, 0xFFFFFFFFu, signsel);  // selector 4: FF, 0: 00
  return (pos & ~mask) | (neg & mask);
}
__device__ __forceinline__ void tc4_to_e4m3(uint32_t w, uint32_t& re, uint32_t& im) {
  const uint32_t m = w & 0x77777777u;
  const uint32_t c01 = tc_pick(m, (w >> 1) & 0x4444u);         // Re0 Im0 Re1 Im1
  const uint32_t c23 = tc_pick(m >> 16, (w >> 17) & 0x4444u);  // Re2 Im2 Re3 Im3
  re = __byte_perm(c01, c23, 0x6420u);
  im = __byte_perm(c01, c23, 0x7531u);
}

}  // namespace ftdx
