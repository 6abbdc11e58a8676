// Rendering and images in the Lua front-end: dort.render (lua_render.cpp:
// make / render_sync / get_image over the C ABI's wavefront and per-pixel
// renderers; the adjoint pair, which the reference does not have, beside
// them), dort.image (lua_image.cpp: Radiance HDR read / write, PNG
// write, the tone maps, bias_variance and the reference's image test
// test_convergence), and the small modules dort.sampler, dort.filter,
// dort.chrono, dort.stats and dort.env.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>

#include "frontend.h"

namespace dortlua {

bool check_recti(lua_State* l, int idx, int64_t out[4]);   // values.cpp

// ---- images ---------------------------------------------------------------------------

std::shared_ptr<Image> check_image(lua_State* l, int idx) {
  return check_shared<Image>(l, idx, IMAGE_T);
}

void push_image(lua_State* l, std::shared_ptr<Image> img) { push_shared(l, IMAGE_T, std::move(img)); }

static std::shared_ptr<Image> check_image_kind(lua_State* l, int idx, bool hdr) {
  auto img = check_image(l, idx);
  if(img->hdr != hdr) {
    luaL_argerror(l, idx, hdr ? "expected an HDR (float) image" : "expected an 8-bit image");
  }
  return img;
}

// Radiance RGBE: per pixel the largest channel's exponent, 8-bit mantissas
// truncated (the encoder of the reference's stb_image_write); flat scanlines.
static bool write_rgbe_file(const char* path, const Image& img) {
  std::FILE* f = std::fopen(path, "wb");
  if(!f) { return false; }
  std::fprintf(f, "#?RADIANCE\n# Written by dort_b200\nFORMAT=32-bit_rle_rgbe\n\n-Y %u +X %u\n",
               img.h, img.w);
  std::vector<unsigned char> row(size_t(img.w) * 4);
  for(uint32_t y = 0; y < img.h; ++y) {
    for(uint32_t x = 0; x < img.w; ++x) {
      const float* p = &img.px[3 * (size_t(y) * img.w + x)];
      float mx = std::max(p[0], std::max(p[1], p[2]));
      unsigned char* o = &row[4 * size_t(x)];
      if(mx < 1e-32f) {
        o[0] = o[1] = o[2] = o[3] = 0;
      } else {
        int e;
        float norm = float(std::frexp(mx, &e)) * 256.f / mx;
        for(int c = 0; c < 3; ++c) {
          float v = p[c] * norm;
          o[c] = (unsigned char)(v < 0.f ? 0.f : (v > 255.f ? 255.f : v));
        }
        o[3] = (unsigned char)(e + 128);
      }
    }
    std::fwrite(row.data(), 1, row.size(), f);
  }
  std::fclose(f);
  return true;
}

static bool read_rgbe_file(const char* path, Image& img, std::string& err) {
  std::ifstream f(path, std::ios::binary);
  if(!f) { err = std::string("Could not open image file for reading: ") + path; return false; }
  std::string line;
  uint32_t w = 0, h = 0;
  while(std::getline(f, line)) {
    if(line.rfind("-Y ", 0) == 0) {
      if(std::sscanf(line.c_str(), "-Y %u +X %u", &h, &w) != 2) { err = "bad HDR resolution line"; return false; }
      break;
    }
  }
  if(w == 0 || h == 0) { err = "not a Radiance HDR file"; return false; }
  img.w = w; img.h = h; img.hdr = true;
  img.px.assign(size_t(w) * h * 3, 0.f);
  std::vector<unsigned char> rgbe(size_t(w) * 4);
  for(uint32_t y = 0; y < h; ++y) {
    unsigned char hd[4];
    if(!f.read(reinterpret_cast<char*>(hd), 4)) { err = "truncated HDR file"; return false; }
    bool rle = w >= 8 && w < 32768 && hd[0] == 2 && hd[1] == 2 && !(hd[2] & 0x80);
    if(rle) {
      if(uint32_t(hd[2] << 8 | hd[3]) != w) { err = "bad HDR scanline"; return false; }
      for(int c = 0; c < 4; ++c) {
        uint32_t x = 0;
        while(x < w) {
          int n = f.get();
          if(n == EOF) { err = "truncated HDR file"; return false; }
          if(n > 128) {
            n -= 128;
            int v = f.get();
            if(v == EOF || x + uint32_t(n) > w) { err = "bad HDR run"; return false; }
            for(int k = 0; k < n; ++k) { rgbe[4 * size_t(x++) + c] = (unsigned char)v; }
          } else {
            if(n == 0 || x + uint32_t(n) > w) { err = "bad HDR run"; return false; }
            for(int k = 0; k < n; ++k) {
              int v = f.get();
              if(v == EOF) { err = "truncated HDR file"; return false; }
              rgbe[4 * size_t(x++) + c] = (unsigned char)v;
            }
          }
        }
      }
    } else {
      std::memcpy(rgbe.data(), hd, 4);
      if(!f.read(reinterpret_cast<char*>(rgbe.data() + 4), std::streamsize(4 * size_t(w) - 4))) {
        err = "truncated HDR file";
        return false;
      }
    }
    for(uint32_t x = 0; x < w; ++x) {
      const unsigned char* q = &rgbe[4 * size_t(x)];
      float s = q[3] ? std::ldexp(1.f, int(q[3]) - 136) : 0.f;
      float* o = &img.px[3 * (size_t(y) * w + x)];
      o[0] = q[0] * s; o[1] = q[1] * s; o[2] = q[2] * s;
    }
  }
  return true;
}

// PNG (8-bit RGB) with stored (uncompressed) deflate blocks: no external
// compression library needed.
static uint32_t crc32_of(const unsigned char* p, size_t n, uint32_t crc = 0) {
  static uint32_t table[256];
  static bool init = false;
  if(!init) {
    for(uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for(int k = 0; k < 8; ++k) { c = (c & 1) ? 0xedb88320u ^ (c >> 1) : c >> 1; }
      table[i] = c;
    }
    init = true;
  }
  crc = ~crc;
  for(size_t i = 0; i < n; ++i) { crc = table[(crc ^ p[i]) & 0xff] ^ (crc >> 8); }
  return ~crc;
}

static bool write_png_file(const char* path, const Image& img) {
  std::vector<unsigned char> raw;
  raw.reserve((size_t(img.w) * 3 + 1) * img.h);
  for(uint32_t y = 0; y < img.h; ++y) {
    raw.push_back(0);
    for(uint32_t x = 0; x < img.w * 3; ++x) {
      raw.push_back((unsigned char)img.px[size_t(y) * img.w * 3 + x]);
    }
  }
  std::vector<unsigned char> z = {0x78, 0x01};
  size_t pos = 0;
  do {
    size_t n = std::min<size_t>(65535, raw.size() - pos);
    bool last = pos + n == raw.size();
    z.push_back(last ? 1 : 0);
    z.push_back((unsigned char)(n & 0xff));
    z.push_back((unsigned char)(n >> 8));
    z.push_back((unsigned char)(~n & 0xff));
    z.push_back((unsigned char)((~n >> 8) & 0xff));
    z.insert(z.end(), raw.begin() + long(pos), raw.begin() + long(pos + n));
    pos += n;
  } while(pos < raw.size());
  uint32_t a = 1, b = 0;
  for(unsigned char c : raw) { a = (a + c) % 65521; b = (b + a) % 65521; }
  uint32_t adler = (b << 16) | a;
  for(int k = 3; k >= 0; --k) { z.push_back((unsigned char)(adler >> (8 * k))); }

  std::FILE* f = std::fopen(path, "wb");
  if(!f) { return false; }
  auto be32 = [&](uint32_t v) {
    unsigned char b4[4] = {(unsigned char)(v >> 24), (unsigned char)(v >> 16),
                           (unsigned char)(v >> 8), (unsigned char)v};
    std::fwrite(b4, 1, 4, f);
  };
  auto chunk = [&](const char* tag, const std::vector<unsigned char>& data) {
    be32(uint32_t(data.size()));
    std::vector<unsigned char> td(tag, tag + 4);
    td.insert(td.end(), data.begin(), data.end());
    std::fwrite(td.data(), 1, td.size(), f);
    be32(crc32_of(td.data(), td.size()));
  };
  const unsigned char sig[8] = {0x89, 'P', 'N', 'G', 0x0d, 0x0a, 0x1a, 0x0a};
  std::fwrite(sig, 1, 8, f);
  std::vector<unsigned char> ihdr = {(unsigned char)(img.w >> 24), (unsigned char)(img.w >> 16),
                                     (unsigned char)(img.w >> 8), (unsigned char)img.w,
                                     (unsigned char)(img.h >> 24), (unsigned char)(img.h >> 16),
                                     (unsigned char)(img.h >> 8), (unsigned char)img.h,
                                     8, 2, 0, 0, 0};
  chunk("IHDR", ihdr);
  chunk("IDAT", z);
  chunk("IEND", {});
  std::fclose(f);
  return true;
}

static int image_read(lua_State* l) {
  const char* path = luaL_checkstring(l, 1);
  int p = params_index(l, 2);
  bool hdr = param_bool_opt(l, p, "hdr", false);
  params_check_unused(l, p);
  if(!hdr) { return luaL_error(l, "only Radiance HDR images can be read ({hdr = true})"); }
  auto img = std::make_shared<Image>();
  std::string err;
  if(!read_rgbe_file(path, *img, err)) { return luaL_error(l, "%s", err.c_str()); }
  push_image(l, img);
  return 1;
}

static int image_write_png(lua_State* l) {
  const char* path = luaL_checkstring(l, 1);
  auto img = check_image_kind(l, 2, false);
  if(!write_png_file(path, *img)) { return luaL_error(l, "Could not open file for writing: %s", path); }
  return 0;
}

static int image_write_rgbe(lua_State* l) {
  const char* path = luaL_checkstring(l, 1);
  auto img = check_image_kind(l, 2, true);
  if(!write_rgbe_file(path, *img)) { return luaL_error(l, "Could not open file for writing: %s", path); }
  return 0;
}

// Portable float map (PF, little-endian, bottom row first): signed floats,
// for images that are gradients rather than radiance (the adjoint's).
static bool write_pfm_file(const char* path, const Image& img) {
  std::FILE* f = std::fopen(path, "wb");
  if(!f) { return false; }
  std::fprintf(f, "PF\n%u %u\n-1.0\n", img.w, img.h);
  for(uint32_t y = img.h; y-- > 0;) {
    std::fwrite(&img.px[3 * size_t(y) * img.w], sizeof(float), 3 * size_t(img.w), f);
  }
  return std::fclose(f) == 0;
}

static int image_write_pfm(lua_State* l) {
  const char* path = luaL_checkstring(l, 1);
  auto img = check_image_kind(l, 2, true);
  if(!write_pfm_file(path, *img)) { return luaL_error(l, "Could not open file for writing: %s", path); }
  return 0;
}

static std::shared_ptr<Image> new_hdr_image(uint32_t w, uint32_t h) {
  auto img = std::make_shared<Image>();
  img->w = w;
  img->h = h;
  img->hdr = true;
  img->px.assign(size_t(w) * h * 3, 0.f);
  return img;
}

// a * x + y over two HDR images of one size (a gradient step)
static int image_axpy(lua_State* l) {
  float a = float(luaL_checknumber(l, 1));
  auto x = check_image_kind(l, 2, true);
  auto y = check_image_kind(l, 3, true);
  if(x->w != y->w || x->h != y->h) { return luaL_error(l, "axpy: images of different sizes"); }
  auto out = new_hdr_image(x->w, x->h);
  for(size_t i = 0; i < out->px.size(); ++i) { out->px[i] = a * x->px[i] + y->px[i]; }
  push_image(l, out);
  return 1;
}

// every channel clamped to [lo, hi]
static int image_clamp(lua_State* l) {
  auto x = check_image_kind(l, 1, true);
  float lo = float(luaL_checknumber(l, 2)), hi = float(luaL_checknumber(l, 3));
  auto out = new_hdr_image(x->w, x->h);
  for(size_t i = 0; i < out->px.size(); ++i) {
    float v = x->px[i];
    out->px[i] = v < lo ? lo : (v > hi ? hi : v);
  }
  push_image(l, out);
  return 1;
}

template<class F>
static std::shared_ptr<Image> map_channels(const Image& in, F f) {
  auto out = std::make_shared<Image>();
  out->w = in.w; out->h = in.h; out->hdr = false;
  out->px.resize(in.px.size());
  for(size_t i = 0; i < in.px.size(); ++i) { out->px[i] = float(f(in.px[i])); }
  return out;
}

// tonemap.cpp:6-14: sRGB curve, quantized as (int)(v * 256) clamped to 0..255
static int image_tonemap_srgb(lua_State* l) {
  auto img = check_image_kind(l, 1, true);
  float scale = lua_gettop(l) >= 2 ? float(luaL_checknumber(l, 2)) : 1.f;
  push_image(l, map_channels(*img, [&](float lin) {
    lin *= scale;
    float g = lin >= 0.0031308f ? 1.055f * std::pow(lin, 1.f / 2.4f) - 0.055f : lin * 12.92f;
    int v = int(g * 256.f);
    return v < 0 ? 0 : (v > 255 ? 255 : v);
  }));
  return 1;
}

// tonemap.cpp:16-22, as the reference computes it: the value pow(x * scale,
// 1 / gamma) is clamped to [0, 1] and truncated, without a 255 scale, so
// channels come out 0 or 1
static int image_tonemap_gamma(lua_State* l) {
  auto img = check_image_kind(l, 1, true);
  float gamma = lua_gettop(l) >= 2 ? float(luaL_checknumber(l, 2)) : 1.f;
  float scale = lua_gettop(l) >= 3 ? float(luaL_checknumber(l, 3)) : 1.f;
  push_image(l, map_channels(*img, [&](float lin) {
    float v = float(int32_t(std::pow(lin * scale, 1.f / gamma)));
    v = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
    return int(uint8_t(v));
  }));
  return 1;
}

static int image_get_res(lua_State* l) {
  auto img = check_image(l, 1);
  lua_pushinteger(l, img->w);
  lua_pushinteger(l, img->h);
  return 2;
}

// lua_image.cpp:179-222: sums of |ref - tested| and (ref - tested)^2 over a
// rectangle, all channels
static int image_bias_variance(lua_State* l) {
  auto ref = check_image_kind(l, 1, true), test = check_image_kind(l, 2, true);
  int64_t r[4];
  check_recti(l, 3, r);
  if(r[2] > int64_t(ref->w) || r[3] > int64_t(ref->h)) { return luaL_error(l, "Rect is out of the ref_image"); }
  if(r[2] > int64_t(test->w) || r[3] > int64_t(test->h)) { return luaL_error(l, "Rect is out of the tested_image"); }
  float bias = 0.f, var = 0.f;
  for(int64_t y = r[1]; y < r[3]; ++y) {
    for(int64_t x = r[0]; x < r[2]; ++x) {
      for(int c = 0; c < 3; ++c) {
        float d = ref->px[3 * (size_t(y) * ref->w + size_t(x)) + c] -
                  test->px[3 * (size_t(y) * test->w + size_t(x)) + c];
        bias += std::fabs(d);
        var += d * d;
      }
    }
  }
  lua_pushnumber(l, bias);
  lua_pushnumber(l, var);
  return 2;
}

// Abramowitz & Stegun 26.2.23 (the approximation the reference uses for
// the inverse normal CDF, math.cpp:4-19)
static float normal_cdf_inverse(float p) {
  auto approx = [](float t) {
    const float c0 = 2.515517f, c1 = 0.802853f, c2 = 0.010328f;
    const float d0 = 1.432788f, d1 = 0.189269f, d2 = 0.001308f;
    return t - ((c2 * t + c1) * t + c0) / (((d2 * t + d1) * t + d0) * t + 1.f);
  };
  if(p <= 0.f || p >= 1.f) { return NAN; }
  return p < 0.5f ? -approx(std::sqrt(-2.f * std::log(p))) : approx(std::sqrt(-2.f * std::log(1.f - p)));
}

// The reference's image test (convergence_test.cpp:10-101): tiles from the
// whole image down to min_tile_size; a tile fails when the largest channel
// difference of its means exceeds stddev / sqrt(pixels) * |Phi^-1(p / 2)| +
// bias, stddev = variation * the larger of the image's and the tile's
// largest mean channel; p is the p-value split over all tiles.  Returns nil
// or the first failing tile, as a message.
static int image_test_convergence(lua_State* l) {
  auto ref = check_image_kind(l, 1, true), test = check_image_kind(l, 2, true);
  int p = params_index(l, 3);
  double min_tile = param_number(l, p, "min_tile_size");
  float variation = float(param_number(l, p, "variation"));
  float bias = float(param_number_opt(l, p, "bias", 0.0));
  float p_value = float(param_number(l, p, "p_value"));
  params_check_unused(l, p);
  if(ref->w != test->w || ref->h != test->h) {
    return luaL_error(l, "Reference and test images have mismatched resolution");
  }
  int32_t w = int32_t(ref->w), h = int32_t(ref->h);
  auto mean = [&](const Image& img, int32_t x0, int32_t y0, int32_t x1, int32_t y1, float out[3]) {
    double s[3] = {0, 0, 0};
    for(int32_t y = y0; y < y1; ++y) {
      for(int32_t x = x0; x < x1; ++x) {
        for(int c = 0; c < 3; ++c) { s[c] += img.px[3 * (size_t(y) * img.w + size_t(x)) + c]; }
      }
    }
    double n = double(x1 - x0) * double(y1 - y0);
    for(int c = 0; c < 3; ++c) { out[c] = float(s[c] / n); }
  };
  uint32_t max_depth = 0;
  while((std::min(w, h) >> (max_depth + 1)) >= int32_t(min_tile)) { ++max_depth; }
  float test_count = float(((1u << (2 * max_depth + 2)) - 1) / 3);
  float test_p = 1.f - std::pow(1.f - p_value, 1.f / test_count);
  float inv_phi = normal_cdf_inverse(test_p * 0.5f);
  float ref_mean[3];
  mean(*ref, 0, 0, w, h, ref_mean);
  for(uint32_t depth = 0; depth <= max_depth; ++depth) {
    int32_t size = std::min(w, h) >> depth;
    for(int32_t ty = 0; ty < (h + size - 1) / size; ++ty) {
      for(int32_t tx = 0; tx < (w + size - 1) / size; ++tx) {
        int32_t x0 = tx * size, y0 = ty * size;
        int32_t x1 = std::min((tx + 1) * size, w), y1 = std::min((ty + 1) * size, h);
        float tr[3], tt[3];
        mean(*ref, x0, y0, x1, y1, tr);
        mean(*test, x0, y0, x1, y1, tt);
        float diff = std::max(tt[0] - tr[0], std::max(tt[1] - tr[1], tt[2] - tr[2]));
        float sg = variation * std::max(ref_mean[0], std::max(ref_mean[1], ref_mean[2]));
        float sl = variation * std::max(tr[0], std::max(tr[1], tr[2]));
        float bg = bias * std::max(ref_mean[0], std::max(ref_mean[1], ref_mean[2]));
        float bl = bias * std::max(tr[0], std::max(tr[1], tr[2]));
        float count = float(x1 - x0) * float(y1 - y0);
        float max_diff = -std::max(sg, sl) / std::sqrt(count) * inv_phi + std::min(bg, bl);
        if(std::fabs(diff) > max_diff) {
          char msg[256];
          std::snprintf(msg, sizeof(msg), "tile (%d,%d):(%d,%d) has diff %f, but threshold is %f",
                        x0, y0, x1, y1, double(diff), double(max_diff));
          lua_pushstring(l, msg);
          return 1;
        }
      }
    }
  }
  lua_pushnil(l);
  return 1;
}

int open_image(lua_State* l) {
  const luaL_Reg methods[] = {{nullptr, nullptr}};
  register_type(l, IMAGE_T, methods, gc_shared<Image>);
  const luaL_Reg funs[] = {
      {"read", image_read}, {"write_png", image_write_png}, {"write_rgbe", image_write_rgbe},
      {"tonemap_srgb", image_tonemap_srgb}, {"tonemap_gamma", image_tonemap_gamma},
      {"get_res", image_get_res}, {"bias_variance", image_bias_variance},
      {"test_convergence", image_test_convergence}, {"write_pfm", image_write_pfm},
      {"axpy", image_axpy}, {"clamp", image_clamp}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

// ---- samplers and filters --------------------------------------------------------------

struct Sampler { uint32_t seed = 1; };
struct Filter { bool box = true; double rx = 0.5, ry = 0.5; };

static int sampler_random(lua_State* l) {
  int p = params_index(l, 1);
  param_uint_opt(l, p, "samples_per_pixel", 1);
  auto s = std::make_shared<Sampler>();
  s->seed = param_uint_opt(l, p, "seed", 1);
  params_check_unused(l, p);
  push_shared(l, SAMPLER_T, s);
  return 1;
}

static int sampler_stratified(lua_State* l) {
  int p = params_index(l, 1);
  param_uint_opt(l, p, "samples_per_x", 1);
  param_uint_opt(l, p, "samples_per_y", 1);
  auto s = std::make_shared<Sampler>();
  s->seed = param_uint_opt(l, p, "seed", 1);
  params_check_unused(l, p);
  push_shared(l, SAMPLER_T, s);
  return 1;
}

int open_sampler(lua_State* l) {
  const luaL_Reg methods[] = {{nullptr, nullptr}};
  register_type(l, SAMPLER_T, methods, gc_shared<Sampler>);
  const luaL_Reg funs[] = {{"make_random", sampler_random}, {"make_stratified", sampler_stratified},
                           {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

static void filter_radius(lua_State* l, int p, Filter& f) {
  double r = param_number_opt(l, p, "radius", 0.5);
  f.rx = param_number_opt(l, p, "radius_x", r);
  f.ry = param_number_opt(l, p, "radius_y", r);
}

static int filter_box(lua_State* l) {
  int p = params_index(l, 1);
  auto f = std::make_shared<Filter>();
  filter_radius(l, p, *f);
  params_check_unused(l, p);
  push_shared(l, FILTER_T, f);
  return 1;
}

static int filter_other(lua_State* l) {
  int p = params_index(l, 1);
  auto f = std::make_shared<Filter>();
  f->box = false;
  filter_radius(l, p, *f);
  param_take(l, p, "alpha") && (lua_pop(l, 1), true);
  param_take(l, p, "b") && (lua_pop(l, 1), true);
  param_take(l, p, "c") && (lua_pop(l, 1), true);
  param_take(l, p, "tau") && (lua_pop(l, 1), true);
  params_check_unused(l, p);
  push_shared(l, FILTER_T, f);
  return 1;
}

int open_filter(lua_State* l) {
  const luaL_Reg methods[] = {{nullptr, nullptr}};
  register_type(l, FILTER_T, methods, gc_shared<Filter>);
  const luaL_Reg funs[] = {{"make_box", filter_box}, {"make_triangle", filter_other},
                           {"make_gaussian", filter_other}, {"make_mitchell", filter_other},
                           {"make_lanczos_sinc", filter_other}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

// ---- dort.render (lua_render.cpp:102-401) -------------------------------------------

static int render_make(lua_State* l) {
  auto scene = check_shared<Scene>(l, 1, SCENE_T);
  int p = params_index(l, 2);
  auto job = std::make_shared<RenderJob>();
  job->scene = scene;
  dort_render_params& rp = job->params;
  rp.struct_size = sizeof(rp);
  rp.width = param_uint_opt(l, p, "x_res", 800);
  rp.height = param_uint_opt(l, p, "y_res", 600);
  if(param_take(l, p, "filter")) {
    auto f = check_shared<Filter>(l, -1, FILTER_T);
    lua_pop(l, 1);
    if(!f->box || f->rx != 0.5 || f->ry != 0.5) {
      return luaL_error(l, "only the box filter of radius 0.5 is supported by this renderer");
    }
  }
  rp.seed = 42;   // the reference's default sampler: RandomSampler(1, 42)
  if(param_take(l, p, "sampler")) {
    rp.seed = check_shared<Sampler>(l, -1, SAMPLER_T)->seed;
    lua_pop(l, 1);
  }
  std::string method = param_string_opt(l, p, "renderer", "pt");
  rp.iterations = param_uint_opt(l, p, "iterations", 1);
  std::shared_ptr<Camera> cam = scene->camera;
  if(param_take(l, p, "camera")) {
    cam = check_shared<Camera>(l, -1, CAM_T);
    lua_pop(l, 1);
  }
  if(!cam) { return luaL_error(l, "No camera is set in the scene and no camera was given."); }
  rp.camera = cam->c;
  if(method == "pt" || method == "path") {
    rp.min_depth = param_uint_opt(l, p, "min_depth", 0);
    rp.max_depth = param_uint_opt(l, p, "max_depth", 5);
    rp.only_direct = param_bool_opt(l, p, "only_direct", false);
    rp.sample_all_lights = param_bool_opt(l, p, "sample_all_lights", false);
    std::string st = param_string_opt(l, p, "direct_strategy", "mis");
    if(st == "mis") { rp.direct_strategy = DORT_DIRECT_MIS; }
    else if(st == "bsdf") { rp.direct_strategy = DORT_DIRECT_BSDF; }
    else if(st == "light") { rp.direct_strategy = DORT_DIRECT_LIGHT; }
    else { return luaL_error(l, "Unknown direct strategy '%s'", st.c_str()); }
    // not reference parameters: roulette off for derivative checks
    // (DORT_PT_NO_ROULETTE); autotune = true times the wavefront's candidate
    // tunings on this frame before rendering it (dort_gpu_autotune_wavefront)
    if(!param_bool_opt(l, p, "roulette", true)) { rp.renderer_flags |= DORT_PT_NO_ROULETTE; }
    job->autotune = param_bool_opt(l, p, "autotune", false);
  } else if(method == "lt" || method == "light") {
    // lua_render.cpp:146-150: path lengths min_depth + 2 .. max_depth + 2
    rp.renderer = DORT_RENDERER_LT;
    rp.min_depth = param_uint_opt(l, p, "min_depth", 0);
    rp.max_depth = param_uint_opt(l, p, "max_depth", 5);
  } else if(method == "bdpt") {
    // lua_render.cpp:151-159; the per-(s, t) debug films are not kept
    rp.renderer = DORT_RENDERER_BDPT;
    rp.min_depth = param_uint_opt(l, p, "min_depth", 0);
    rp.max_depth = param_uint_opt(l, p, "max_depth", 5);
    if(!param_bool_opt(l, p, "use_t1_paths", true)) {
      rp.renderer_flags |= DORT_BDPT_NO_T1_PATHS;
    }
    if(!param_string_opt(l, p, "debug_image_dir", "").empty()) {
      return luaL_error(l, "debug_image_dir is not supported by this build's bdpt renderer");
    }
  } else if(method == "dot" || method == "vcm" || method == "sppm") {
    return luaL_error(l, "renderer '%s' is not available in this build "
                      "(\"pt\", \"lt\" and \"bdpt\")", method.c_str());
  } else {
    return luaL_error(l, "Unrecognized rendering method: %s", method.c_str());
  }
  params_check_unused(l, p);
  push_shared(l, JOB_T, job);
  return 1;
}

static std::shared_ptr<RenderJob> check_job(lua_State* l, int idx) {
  return check_shared<RenderJob>(l, idx, JOB_T);
}

static int render_sync(lua_State* l) {
  auto job = check_job(l, 1);
  if(job->started) { return luaL_error(l, "This render job has already started"); }
  job->started = true;
  auto img = std::make_shared<Image>();
  img->w = job->params.width;
  img->h = job->params.height;
  img->hdr = true;
  img->px.assign(size_t(img->w) * img->h * 3, 0.f);
  if(job->scene->handle) {
    // the wavefront for "pt", the light or bidirectional tracer when asked for
    const bool wavefront = job->params.renderer == DORT_RENDERER_PT;
    dort_wavefront_tuning tuning{};
    const dort_wavefront_tuning* tp = nullptr;
    if(wavefront && job->autotune) {
      if(dort_gpu_autotune_wavefront(job->scene->handle, &job->params, 0.0, &tuning, nullptr) !=
         DORT_OK) {
        return luaL_error(l, "%s", dort_gpu_last_error());
      }
      tp = &tuning;
    }
    int rc = wavefront
        ? dort_gpu_render_wavefront(job->scene->handle, &job->params, tp, img->px.data(), nullptr)
        : dort_gpu_render(job->scene->handle, &job->params, img->px.data(), nullptr);
    if(rc != DORT_OK) { return luaL_error(l, "%s", dort_gpu_last_error()); }
  }
  job->image = img;
  job->finished = true;
  return 0;
}

// film->to_image<PixelRgb8> (image.hpp:60-64): floor(256 x) clamped to 0..255
static int render_get_image(lua_State* l) {
  auto job = check_job(l, 1);
  if(!job->finished) {
    return luaL_error(l, job->started ? "Render has not finished yet" : "Render has not been started");
  }
  int p = params_index(l, 2);
  bool hdr = param_bool_opt(l, p, "hdr", false);
  params_check_unused(l, p);
  if(hdr) {
    auto img = std::make_shared<Image>(*job->image);
    push_image(l, img);
  } else {
    push_image(l, map_channels(*job->image, [](float v) {
      int q = int(std::floor(256.f * v));
      return q < 0 ? 0 : (q > 255 ? 255 : q);
    }));
  }
  return 1;
}

// ---- the adjoint (no reference counterpart) ----------------------------------------------
//
// Gradients of an image loss with respect to per-triangle Lambert albedo and
// emitted radiance (dort_gpu_adjoint_forward / _backward).  Per-triangle
// values travel as HDR images of tri_count x 1 pixels, in the order the scene
// flattened its triangles.
//   dort.render.triangle_params(scene)          -> albedo, emission
//   dort.render.adjoint_forward(job, {albedo =, emission =})   -> image
//   dort.render.adjoint_backward(job, {dl_dimage =, albedo =, emission =})
//                                                -> d_albedo, d_emission
//   dort.render.loss_l2(image, target)          -> loss, dloss_dimage
// Without `emission`, the backward pass differentiates at the emission the
// scene was built with.

static uint32_t scene_tri_count(const Scene& sc) { return uint32_t(sc.flat.tris.size() / 3); }

static bool scene_has_emitters(const Scene& sc) {
  for(float v : sc.flat.tri_emission) {
    if(v != 0.f) { return true; }
  }
  return false;
}

static const float* tri_image(lua_State* l, int p, const char* key, const Scene& sc,
                              std::shared_ptr<Image>& keep) {
  if(!param_take(l, p, key)) { return nullptr; }
  keep = check_image_kind(l, -1, true);
  lua_pop(l, 1);
  if(keep->w != scene_tri_count(sc) || keep->h != 1) {
    luaL_error(l, "%s must be a %u x 1 image (one pixel per triangle)", key, scene_tri_count(sc));
  }
  return keep->px.data();
}

static int render_triangle_params(lua_State* l) {
  auto scene = check_shared<Scene>(l, 1, SCENE_T);
  const FlatScene& f = scene->flat;
  uint32_t n = scene_tri_count(*scene);
  auto alb = new_hdr_image(n, 1), em = new_hdr_image(n, 1);
  for(uint32_t t = 0; t < n && !f.materials.empty(); ++t) {
    const dort_material& m = f.materials[f.tri_material.empty() ? 0 : f.tri_material[t]];
    if(m.kind == DORT_MAT_LAMBERT) {
      for(int c = 0; c < 3; ++c) { alb->px[3 * size_t(t) + c] = m.color[c]; }
    }
  }
  for(size_t i = 0; i < f.tri_emission.size() && i < em->px.size(); ++i) {
    em->px[i] = f.tri_emission[i];
  }
  push_image(l, alb);
  push_image(l, em);
  return 2;
}

static std::shared_ptr<RenderJob> check_adjoint_job(lua_State* l, int idx) {
  auto job = check_shared<RenderJob>(l, idx, JOB_T);
  if(job->params.renderer != DORT_RENDERER_PT) {
    luaL_error(l, "the adjoint differentiates the \"pt\" renderer only");
  }
  if(!job->scene->handle) { luaL_error(l, "the adjoint needs a GPU (record mode has none)"); }
  return job;
}

static int render_adjoint_forward(lua_State* l) {
  auto job = check_adjoint_job(l, 1);
  int p = params_index(l, 2);
  std::shared_ptr<Image> ka, ke;
  const float* alb = tri_image(l, p, "albedo", *job->scene, ka);
  const float* em = tri_image(l, p, "emission", *job->scene, ke);
  params_check_unused(l, p);
  auto img = new_hdr_image(job->params.width, job->params.height);
  if(dort_gpu_adjoint_forward(job->scene->handle, &job->params, alb, em, img->px.data()) !=
     DORT_OK) {
    return luaL_error(l, "%s", dort_gpu_last_error());
  }
  push_image(l, img);
  return 1;
}

static int render_adjoint_backward(lua_State* l) {
  auto job = check_adjoint_job(l, 1);
  int p = params_index(l, 2);
  if(!param_take(l, p, "dl_dimage")) { return luaL_error(l, "dl_dimage is required"); }
  auto g = check_image_kind(l, -1, true);
  lua_pop(l, 1);
  if(g->w != job->params.width || g->h != job->params.height) {
    return luaL_error(l, "dl_dimage must have the render's size");
  }
  std::shared_ptr<Image> ka, ke;
  const float* alb = tri_image(l, p, "albedo", *job->scene, ka);
  const float* em = tri_image(l, p, "emission", *job->scene, ke);
  params_check_unused(l, p);
  const bool lights = scene_has_emitters(*job->scene);
  if(!em && lights) { em = job->scene->flat.tri_emission.data(); }
  uint32_t n = scene_tri_count(*job->scene);
  auto da = new_hdr_image(n, 1), de = new_hdr_image(n, 1);
  if(dort_gpu_adjoint_backward(job->scene->handle, &job->params, alb, em, g->px.data(),
                               da->px.data(), lights ? de->px.data() : nullptr) != DORT_OK) {
    return luaL_error(l, "%s", dort_gpu_last_error());
  }
  push_image(l, da);
  push_image(l, de);
  return 2;
}

static int render_loss_l2(lua_State* l) {
  auto a = check_image_kind(l, 1, true);
  auto b = check_image_kind(l, 2, true);
  if(a->w != b->w || a->h != b->h) { return luaL_error(l, "loss_l2: images of different sizes"); }
  auto g = new_hdr_image(a->w, a->h);
  double loss = 0.0;
  if(dort_gpu_loss_l2(a->px.data(), b->px.data(), a->px.size(), &loss, g->px.data()) != DORT_OK) {
    return luaL_error(l, "%s", dort_gpu_last_error());
  }
  lua_pushnumber(l, loss);
  push_image(l, g);
  return 2;
}

static int render_unsupported(lua_State* l) {
  return luaL_error(l, "asynchronous rendering and previews need a GUI and are not supported");
}

int open_render(lua_State* l) {
  const luaL_Reg methods[] = {{nullptr, nullptr}};
  register_type(l, JOB_T, methods, gc_shared<RenderJob>);
  const luaL_Reg funs[] = {
      {"make", render_make}, {"render_sync", render_sync}, {"get_image", render_get_image},
      {"render_async", render_unsupported}, {"image_to_pixbuf", render_unsupported},
      {"cancel", render_unsupported}, {"get_preview", render_unsupported},
      {"get_progress", render_unsupported}, {"triangle_params", render_triangle_params},
      {"adjoint_forward", render_adjoint_forward}, {"adjoint_backward", render_adjoint_backward},
      {"loss_l2", render_loss_l2}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

// ---- dort.chrono, dort.stats, dort.env ---------------------------------------------------

constexpr const char* TIME_T = "dort.Time";
using Clock = std::chrono::steady_clock;

static int chrono_now(lua_State* l) {
  push_value(l, TIME_T, Clock::now());
  return 1;
}
static double chrono_diff_s(lua_State* l) {
  auto a = *static_cast<Clock::time_point*>(luaL_checkudata(l, 1, TIME_T));
  auto b = *static_cast<Clock::time_point*>(luaL_checkudata(l, 2, TIME_T));
  return std::chrono::duration<double>(b - a).count();
}
static int chrono_difference_s(lua_State* l) { lua_pushnumber(l, chrono_diff_s(l)); return 1; }
static int chrono_difference_ns(lua_State* l) { lua_pushnumber(l, chrono_diff_s(l) * 1e9); return 1; }

int open_chrono(lua_State* l) {
  const luaL_Reg methods[] = {{nullptr, nullptr}};
  register_type(l, TIME_T, methods, nullptr);
  const luaL_Reg funs[] = {{"now", chrono_now}, {"difference_s", chrono_difference_s},
                           {"difference_ns", chrono_difference_ns}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

static int stats_noop(lua_State*) { return 0; }

int open_stats(lua_State* l) {
  const luaL_Reg funs[] = {{"reset", stats_noop}, {"write_and_reset", stats_noop},
                           {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

static std::vector<std::string>& argv_store() {
  static std::vector<std::string> v;
  return v;
}

void set_argv(std::vector<std::string> argv) { argv_store() = std::move(argv); }

static int env_get_argv(lua_State* l) {
  const auto& v = argv_store();
  lua_createtable(l, int(v.size()), 0);
  for(size_t i = 0; i < v.size(); ++i) {
    lua_pushlstring(l, v[i].data(), v[i].size());
    lua_rawseti(l, -2, lua_Integer(i + 1));
  }
  return 1;
}

int open_env(lua_State* l) {
  const luaL_Reg funs[] = {{"get_argv", env_get_argv}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

}  // namespace dortlua
