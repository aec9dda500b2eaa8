// develop.h — argent-post's `develop` (crates/argent-post/src/tonemap.rs:
// 216-391): exposure -> tone map -> saturation -> sRGB OETF -> TPDF dither
// -> 8 bits.  The host builds argent's per-grade tables exactly as
// `Prepared::new` does (tonemap.rs:285-309); the device evaluates the fast
// path per pixel from them (develop.cuh, k_develop).
#pragma once
#include <cstdint>
#include <vector>

namespace argent {

enum { TM_AGX = 0, TM_ACES = 1, TM_KHRONOS = 2, TM_REINHARD = 3, TM_CLAMP = 4 };
enum { AGX_BASE = 0, AGX_PUNCHY = 1, AGX_GOLDEN = 2 };

// BitCurve (tonemap.rs:233-258): a table over the f32 bit pattern.
constexpr uint32_t CURVE_MANT_BITS = 9;
constexpr uint32_t CURVE_SHIFT = 23 - CURVE_MANT_BITS;
constexpr int LUT_SEGMENTS = 4096;

struct DevelopTables {
  float k;                    // exposure scale
  int op;                     // TM_*
  float sat;                  // AgX: look saturation x grade saturation; others: grade saturation
  int ncurves;                // AgX: 1 (shared CDL) or 3
  int pick[3];
  uint32_t curve_base;
  uint32_t curve_len;         // entries per curve
  std::vector<float> curves;  // ncurves * curve_len
  float enc_lo, enc_scale;    // Lut1 (color.rs:37-64)
  uint32_t enc_last;          // segments
  std::vector<float> enc;     // enc_last + 1 entries
};

// tonemap.rs:285-309 for a grade (exposure_ev, op, look, saturation).
DevelopTables develop_tables(float exposure_ev, int op, int look, float saturation);

}  // namespace argent
