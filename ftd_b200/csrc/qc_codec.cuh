// qc_codec.cuh -- QC int4 byte -> FP8 E4M3 conversion shared by the
// promotion kernels.
#pragma once
#include <cstdint>

namespace ftdx {

// Four QC bytes -> E4M3 bytes of the four Re parts and of the four Im parts.
// Sign-magnitude nibble: bit 3 sign, bits 2:0 magnitude (0..7).  E4M3 codes of
// the integers 0..7 are 00 38 40 44 48 4A 4C 4E; a byte permute indexed by the
// magnitude looks them up, the sign goes to bit 7.
__device__ __forceinline__ void qc4_to_e4m3(uint32_t w, uint32_t& re, uint32_t& im) {
  constexpr uint32_t kLo = 0x44403800u, kHi = 0x4E4C4A48u;
  const uint32_t mr = (w >> 4) & 0x07070707u;
  const uint32_t mi = w & 0x07070707u;
  uint32_t sr = mr | (mr >> 4);
  sr = (sr & 0xFFu) | ((sr >> 8) & 0xFF00u);
  uint32_t si = mi | (mi >> 4);
  si = (si & 0xFFu) | ((si >> 8) & 0xFF00u);
  re = __byte_perm(kLo, kHi, sr) | (w & 0x80808080u);
  im = __byte_perm(kLo, kHi, si) | ((w << 4) & 0x80808080u);
}

}  // namespace ftdx
