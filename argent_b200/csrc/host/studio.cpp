// studio.cpp — host restatement of argent-core's studio rigs, camera and
// framing (argent_host.h):
//   Studio::build, emitter, floor_at   core/src/studio.rs:15-200
//   Panel::facing                      core/src/light.rs:37-47
//   Camera::look_at, Camera::project   core/src/camera.rs:38-80
//   View::named, views::frame          core/src/views.rs:17-83
// plus the seeded synthetic HDRI that stands in for a photographed one.
#include <cctype>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/argent_host.h"

extern "C" {
void argent_bake_emitter(float kelvin, float intensity, float* out);
void argent_bake_rgb_illuminant(const float* rgb, float* out);
void argent_material_plastic(const float* rgb, float eta, float roughness, ArgentMaterial* m);
void argent_material_diffuse(const float* rgb, ArgentMaterial* m);
void argent_blackbody_white(float kelvin, float* xyz);
}

namespace {

struct V {
  float x, y, z;
};
V vadd(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }
V vsub(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }
V vmul(V a, float s) { return V{a.x * s, a.y * s, a.z * s}; }
float vdot(V a, V b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
V vcross(V a, V b) { return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V vnorm(V a) { return vmul(a, 1.0f / std::sqrt(vdot(a, a))); }
float vlen(V a) { return std::sqrt(vdot(a, a)); }
void st(float* o, V v) {
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
}
V ld(const float* p) { return V{p[0], p[1], p[2]}; }

// light.rs:37-47
void panel_facing(ArgentPanel* p, V pos, V target, float w, float h, V up_hint, int emits, float kelvin,
                  float intensity) {
  std::memset(p, 0, sizeof(*p));
  V n = vnorm(vsub(target, pos));
  V right = vcross(up_hint, n);
  if (vdot(right, right) < 1e-6f) right = vcross(V{1, 0, 0}, n);
  right = vnorm(right);
  V up = vcross(n, right);
  st(p->center, pos);
  st(p->hu, vmul(right, 0.5f * w));
  st(p->hv, vmul(up, 0.5f * h));
  p->emits = emits;
  p->camera_visible = 0;
  p->feather = 0.35f;
  if (emits) argent_bake_emitter(kelvin, intensity, p->emission);
}

std::string lower(const char* s) {
  std::string r(s ? s : "");
  size_t a = r.find_first_not_of(" \t\n"), b = r.find_last_not_of(" \t\n");
  r = a == std::string::npos ? std::string() : r.substr(a, b - a + 1);
  for (auto& c : r) c = (char)std::tolower((unsigned char)c);
  return r;
}

}  // namespace

extern "C" {

// studio.rs:252-355 + floor_at (studio.rs:359-362).  Fills up to 16 panels,
// the gradient env, the floor material and the floor's fade radii (already
// scaled by the rig factor), and the white point.  floor_y is the piece's
// lowest point; the floor sits 0.005 mm below it (shot.rs:227-230).
int argent_studio_build(const char* name, float radius, float floor_y, ArgentPanel* panels, int32_t* num_panels,
                        ArgentEnv* env, ArgentMaterial* floor_material, ArgentFloor* floor, int32_t* has_white,
                        float* white_xyz) {
  std::string s = lower(name);
  int id = -1;
  if (s == "noir" || s == "brand" || s == "dark" || s == "black") id = 0;
  if (s == "white" || s == "listing" || s == "etsy" || s == "seamless") id = 1;
  if (s == "velvet" || s == "box") id = 2;
  if (s == "ember" || s == "underworld" || s == "forge" || s == "fire") id = 3;
  if (s == "window" || s == "daylight" || s == "natural") id = 4;
  if (id < 0 || !panels || !num_panels || !env || !floor_material || !floor || !has_white || !white_xyz)
    return ARGENT_E_INVALID;
  float k = std::fmax(radius / 15.0f, 0.2f);
  auto at = [&](float x, float y, float z) { return vmul(V{x, y, z}, k); };
  V o{0, 0, 0}, up{0, 1, 0};
  int n = 0;
  auto box_ = [&](V pos, float w, float h, float kelvin, float i) {
    panel_facing(&panels[n++], pos, o, w * k, h * k, up, 1, kelvin, i);
  };
  auto flag = [&](V pos, float w, float h) { panel_facing(&panels[n++], pos, o, w * k, h * k, up, 0, 0, 0); };
  std::memset(env, 0, sizeof(*env));
  env->kind = ARGENT_ENV_GRADIENT;
  auto grad = [&](const float t[3], const float hz[3], const float b[3], float power) {
    argent_bake_rgb_illuminant(t, env->top);
    argent_bake_rgb_illuminant(hz, env->horizon);
    argent_bake_rgb_illuminant(b, env->bottom);
    env->power = power;
  };
  float fa = 0, fb = 0, kelvin_white = -1;
  if (id == 0) {  // Noir
    box_(at(0, 270, 110), 340, 240, 5600, 3.2f);
    box_(at(-230, 70, -50), 70, 540, 5600, 7.5f);
    box_(at(230, 70, -50), 70, 540, 5600, 7.5f);
    box_(at(30, 90, 330), 520, 300, 5400, 0.9f);
    box_(at(0, 260, -230), 300, 90, 6000, 1.4f);
    const float t[3] = {0.010f, 0.010f, 0.011f}, hz[3] = {0.006f, 0.006f, 0.0065f}, b[3] = {0.002f, 0.002f, 0.002f};
    grad(t, hz, b, 0.6f);
    const float fl[3] = {0.003f, 0.003f, 0.0032f};
    argent_material_plastic(fl, 1.49f, 0.09f, floor_material);
    fa = 40;
    fb = 130;
    kelvin_white = 5600;
  } else if (id == 1) {  // White
    box_(at(0, 300, 60), 460, 420, 5800, 2.6f);
    box_(at(-270, 110, 90), 260, 380, 5800, 1.7f);
    box_(at(270, 110, 90), 260, 380, 5800, 1.7f);
    box_(at(0, 70, 340), 460, 220, 5800, 1.2f);
    flag(at(-170, 60, -170), 170, 420);
    flag(at(170, 60, -170), 170, 420);
    flag(at(0, 120, -260), 300, 160);
    flag(at(0, 10, 260), 420, 60);
    const float t[3] = {1.8f, 1.8f, 1.8f}, hz[3] = {0.55f, 0.55f, 0.56f}, b[3] = {0.9f, 0.9f, 0.9f};
    grad(t, hz, b, 0.45f);
    const float fl[3] = {0.86f, 0.86f, 0.86f};
    argent_material_diffuse(fl, floor_material);
    fa = 80;
    fb = 260;
    kelvin_white = 5800;
  } else if (id == 2) {  // Velvet
    box_(at(-160, 220, 160), 220, 220, 3400, 3.2f);
    box_(at(240, 70, -40), 70, 460, 4200, 4.0f);
    box_(at(-60, 120, -280), 260, 80, 3800, 2.0f);
    const float t[3] = {0.006f, 0.004f, 0.004f}, hz[3] = {0.012f, 0.005f, 0.005f}, b[3] = {0.004f, 0.001f, 0.001f};
    grad(t, hz, b, 0.7f);
    const float fl[3] = {0.10f, 0.012f, 0.02f};
    argent_material_diffuse(fl, floor_material);
    fa = 60;
    fb = 200;
    kelvin_white = 4300;
  } else if (id == 3) {  // Ember
    box_(at(-210, 40, -150), 80, 420, 1900, 9.0f);
    box_(at(210, 40, -150), 80, 420, 2100, 9.0f);
    box_(at(60, 220, 220), 220, 180, 9000, 1.4f);
    box_(at(0, -5, -220), 260, 60, 1700, 2.5f);
    const float t[3] = {0.002f, 0.002f, 0.003f}, hz[3] = {0.010f, 0.004f, 0.002f}, b[3] = {0.001f, 0.0005f, 0.0003f};
    grad(t, hz, b, 0.8f);
    const float fl[3] = {0.004f, 0.003f, 0.003f};
    argent_material_plastic(fl, 1.5f, 0.12f, floor_material);
    fa = 40;
    fb = 150;
  } else {  // Window
    box_(at(-300, 160, 80), 300, 380, 6500, 3.0f);
    box_(at(260, 80, 120), 300, 300, 5800, 0.35f);
    flag(at(160, 60, -220), 160, 300);
    const float t[3] = {0.30f, 0.32f, 0.36f}, hz[3] = {0.20f, 0.20f, 0.21f}, b[3] = {0.08f, 0.08f, 0.08f};
    grad(t, hz, b, 0.8f);
    const float fl[3] = {0.30f, 0.29f, 0.28f};
    argent_material_plastic(fl, 1.5f, 0.35f, floor_material);
    fa = 70;
    fb = 220;
    kelvin_white = 6500;
  }
  *num_panels = n;
  floor->enabled = 1;
  floor->y = floor_y - 0.005f;
  floor->material = -1;  // the caller places the floor material in its list
  floor->fade_start = fa * k;
  floor->fade_end = fb * k;
  if (kelvin_white > 0) {
    *has_white = 1;
    argent_blackbody_white(kelvin_white, white_xyz);
  } else {
    *has_white = 0;
    white_xyz[0] = white_xyz[1] = white_xyz[2] = 0.0f;
  }
  return ARGENT_OK;
}

// camera.rs:38-54
void argent_camera_look_at(const float* pos, const float* target, const float* up_hint, float focal_mm, float f_stop,
                           float aspect, ArgentCamera* c) {
  std::memset(c, 0, sizeof(*c));
  V p = ld(pos), t = ld(target), uh = ld(up_hint);
  V forward = vnorm(vsub(t, p));
  V right = vcross(forward, uh);
  if (vdot(right, right) < 1e-8f) right = vcross(forward, V{0, 0, 1});
  right = vnorm(right);
  V up = vcross(right, forward);
  float long_half = 18.0f / focal_mm;
  float hw, hh;
  if (aspect >= 1.0f) {
    hw = long_half;
    hh = long_half / aspect;
  } else {
    hw = long_half * aspect;
    hh = long_half;
  }
  st(c->pos, p);
  st(c->forward, forward);
  st(c->right, right);
  st(c->up, up);
  c->half_w = hw;
  c->half_h = hh;
  c->focus_dist = vlen(vsub(t, p));
  c->lens_radius = f_stop > 0.0f ? 0.5f * focal_mm / f_stop : 0.0f;
}

// views.rs:17-30
int argent_view_named(const char* name, float* az, float* el, float* fill) {
  std::string s = lower(name);
  struct {
    const char* n[2];
    float a, e, f;
  } t[] = {{{"hero", ""}, 34, 26, 0.72f},        {{"front", "face"}, 0, 6, 0.70f},
           {{"side", "profile"}, 90, 6, 0.72f},  {{"top", ""}, 0, 62, 0.70f},
           {{"three-quarter", "34"}, 45, 24, 0.72f}, {{"back", ""}, 160, 16, 0.72f},
           {{"low", ""}, 22, 3, 0.72f},          {{"detail", "macro"}, 14, 34, 0.92f}};
  for (auto& e : t)
    for (int i = 0; i < 2; ++i)
      if (e.n[i][0] && s == e.n[i]) {
        *az = e.a;
        *el = e.e;
        *fill = e.f;
        return ARGENT_OK;
      }
  return ARGENT_E_INVALID;
}

// views.rs:45-83: place a camera along (azimuth, elevation) so `points`
// fill `fill` of the frame, centred.
void argent_frame(const float* points, uint32_t n, float azimuth_deg, float elevation_deg, float fill, float focal_mm,
                  float f_stop, float aspect, ArgentCamera* cam) {
  V lo{3.40282347e38f, 3.40282347e38f, 3.40282347e38f}, hi{-3.40282347e38f, -3.40282347e38f, -3.40282347e38f};
  for (uint32_t i = 0; i < n; ++i) {
    V p = ld(points + 3 * i);
    lo = V{std::fmin(lo.x, p.x), std::fmin(lo.y, p.y), std::fmin(lo.z, p.z)};
    hi = V{std::fmax(hi.x, p.x), std::fmax(hi.y, p.y), std::fmax(hi.z, p.z)};
  }
  V center = vmul(vadd(lo, hi), 0.5f);
  float radius = std::fmax(vlen(vmul(vsub(hi, lo), 0.5f)), 1e-3f);
  float ra = azimuth_deg * (3.14159265358979323846f / 180.0f), re = elevation_deg * (3.14159265358979323846f / 180.0f);
  float sa = std::sin(ra), ca = std::cos(ra), se = std::sin(re), ce = std::cos(re);
  V dir{sa * ce, se, ca * ce};
  V up = std::fabs(dir.y) > 0.98f ? V{0, 0, 1} : V{0, 1, 0};
  float half = std::fmin(18.0f / focal_mm, 18.0f / focal_mm * (aspect < 1.0f ? aspect : 1.0f / aspect));
  float fillc = std::fmax(fill, 0.05f);
  float dist = radius / std::sin(std::atan(half)) / fillc;
  V target = center;
  float fu[3] = {up.x, up.y, up.z};
  auto look = [&]() {
    V pos = vadd(target, vmul(dir, dist));
    float fp[3] = {pos.x, pos.y, pos.z}, ft[3] = {target.x, target.y, target.z};
    argent_camera_look_at(fp, ft, fu, focal_mm, f_stop, aspect, cam);
  };
  look();
  for (int it = 0; it < 6; ++it) {
    float mnx = 3.40282347e38f, mxx = -3.40282347e38f, mny = 3.40282347e38f, mxy = -3.40282347e38f;
    V cp = ld(cam->pos), cf = ld(cam->forward), cr = ld(cam->right), cu = ld(cam->up);
    for (uint32_t i = 0; i < n; ++i) {
      V d = vsub(ld(points + 3 * i), cp);
      float z = vdot(d, cf);
      if (z <= 1e-6f) continue;  // camera.rs:73-78
      float x = vdot(d, cr) / z / cam->half_w - cam->shift[0];
      float y = vdot(d, cu) / z / cam->half_h - cam->shift[1];
      mnx = std::fmin(mnx, x);
      mxx = std::fmax(mxx, x);
      mny = std::fmin(mny, y);
      mxy = std::fmax(mxy, y);
    }
    if (mnx > mxx) break;
    float ext = std::fmax((mxx - mnx) * 0.5f, (mxy - mny) * 0.5f);
    float cx = (mxx + mnx) * 0.5f * cam->half_w;
    float cy = (mxy + mny) * 0.5f * cam->half_h;
    float pd = vdot(vsub(center, cp), cf);
    target = vadd(target, vadd(vmul(cr, cx * pd), vmul(cu, cy * pd)));
    dist *= ext / fillc;
    look();
  }
}

// Seeded equirect HDRI standing in for a photographed one: per-texel
// lognormal radiance (sigma given, in texel space) on a dim grey base plus
// three hot Gaussian lobes; linear sRGB, row-major width*height*3.
void argent_synth_hdri(uint32_t width, uint32_t height, float sigma, uint32_t seed, float* rgb) {
  auto hash = [](uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
  };
  uint32_t sh = hash(seed);
  auto unif = [&](uint32_t k) { return ((float)(hash(k ^ sh) >> 8) + 0.5f) * (1.0f / 16777216.0f); };
  // three lobes at seeded (u, v) with seeded colour temperature-like tints
  float lu[3], lv[3], lw[3], lc[3][3];
  for (int i = 0; i < 3; ++i) {
    lu[i] = unif(0x100 + i);
    lv[i] = 0.15f + 0.4f * unif(0x200 + i);
    lw[i] = 0.01f + 0.02f * unif(0x300 + i);
    float t = unif(0x400 + i);
    lc[i][0] = 60.0f * (1.0f + 0.3f * t);
    lc[i][1] = 60.0f;
    lc[i][2] = 60.0f * (1.3f - 0.3f * t);
  }
  for (uint32_t y = 0; y < height; ++y)
    for (uint32_t x = 0; x < width; ++x) {
      uint32_t k = y * width + x;
      // Box-Muller from two hashed uniforms
      float u1 = unif(2 * k + 1), u2 = unif(2 * k + 2);
      float g = std::sqrt(-2.0f * std::log(u1)) * std::cos(6.28318530718f * u2);
      float base = 0.05f * std::exp(sigma * g - 0.5f * sigma * sigma);
      float u = ((float)x + 0.5f) / (float)width, v = ((float)y + 0.5f) / (float)height;
      float sky = v < 0.5f ? 1.0f : 0.35f;  // brighter upper hemisphere
      float c[3] = {base * sky, base * sky, base * sky * 1.05f};
      for (int i = 0; i < 3; ++i) {
        float du = std::fabs(u - lu[i]);
        du = std::fmin(du, 1.0f - du);
        float dv = v - lv[i];
        float e = std::exp(-(du * du + dv * dv) / (2.0f * lw[i] * lw[i]));
        for (int q = 0; q < 3; ++q) c[q] += lc[i][q] * e;
      }
      for (int q = 0; q < 3; ++q) rgb[3 * (size_t)k + q] = c[q];
    }
}

}  // extern "C"
