// scene_prep.h — host-side tables a scene needs before it can render:
// light-selection CDF (scene.rs:88-110), equirect environment weights and
// sampling CDFs (envmap.rs:141-177), the LinearRgb basis (envmap.rs:178-257),
// the GGX energy-compensation table (microfacet.rs:112-140) and the camera
// white-balance matrix (color.rs:48-55).  Compiled with -ffp-contract=off so
// each table matches argent's f32 arithmetic.
#pragma once
#include <cstdint>
#include <vector>

#include "../../../include/argent_gpu.h"

namespace argent {

struct LightTable {
  std::vector<int> lights;     // emitting panel indices
  std::vector<float> cdf;      // normalised by total power
  float env_pick = 0.0f;
};

// `Scene::rebuild_lights` for the panels of `desc`.
LightTable build_lights(const ArgentSceneDesc& desc);

// Derived panel geometry (`Panel::new`, light.rs:30-33).
void panel_frame(const ArgentPanel& p, float n[3], float* area, float* hu_l2, float* hv_l2);

struct EnvTables {
  int width = 0, height = 0;
  std::vector<float> weights;      // 3 per texel (LinearRgb basis weights)
  std::vector<float> conditional;  // (width+1) per row
  std::vector<float> marginal;     // height+1
  float total = 0.0f;
};
EnvTables build_env(const float* rgb, int width, int height);

// LinearRgb: basis[3][471] and the 3x3 inverse.
void linear_rgb(float basis[3][471], float inv[3][3]);

// E(mu, sqrt(alpha)) on a 32x32 grid.
void ggx_energy_table(float out[32 * 32]);

// XYZ -> camera RGB (row-major 3x3).
void camera_matrix(bool has_white, const float white[3], float out[9]);

// Sobol direction numbers for the sampler's four dimensions, [dim][bit].
void sobol_directions(uint32_t out[4][32]);

// CIE luminance of a 1 nm table (spectrum.rs:413-420).
float luminance_y_table(const float* t);

}  // namespace argent
