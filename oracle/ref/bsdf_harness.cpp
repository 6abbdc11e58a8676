// Microfacet harness around the reference renderer's own GGX distribution.
//
// TEST INFRASTRUCTURE ONLY: compiled with the reference's sources by
// oracle/Makefile into oracle/_ref/.  Exposes MicrofacetDistrib
// (src/dort/microfacet.cpp:7-86) of type GGX over flat arrays so that the
// oracle's float64 restatement of D, G1 and the half-vector sampler can be
// pinned against the reference's float code.  Nothing in the product links
// it.
#include <cstddef>

#include "dort/geometry.hpp"
#include "dort/microfacet.hpp"
#include "dort/vec_2.hpp"

using namespace dort;

extern "C" {

// out[i] = D(m_i) for the GGX distribution of roughness alpha
// (microfacet.cpp:19-36).
void dref_ggx_d(float alpha, size_t n, const float* m, float* out) {
  MicrofacetDistrib d(MicrofacetType::GGX, alpha);
  for(size_t i = 0; i < n; ++i) {
    out[i] = d.d(Vector(m[3 * i], m[3 * i + 1], m[3 * i + 2]));
  }
}

// out[i] = G1(v_i, m_i) (microfacet.cpp:38-58).
void dref_ggx_g1(float alpha, size_t n, const float* v, const float* m, float* out) {
  MicrofacetDistrib d(MicrofacetType::GGX, alpha);
  for(size_t i = 0; i < n; ++i) {
    out[i] = d.g1(Vector(v[3 * i], v[3 * i + 1], v[3 * i + 2]),
                  Vector(m[3 * i], m[3 * i + 1], m[3 * i + 2]));
  }
}

// Half vectors sampled from the uniforms uv[2i], uv[2i+1] with their pdfs
// (microfacet.cpp:64-86).
void dref_ggx_sample_m(float alpha, size_t n, const float* uv, float* out_m, float* out_pdf) {
  MicrofacetDistrib d(MicrofacetType::GGX, alpha);
  for(size_t i = 0; i < n; ++i) {
    float pdf = 0.f;
    Vector m = d.sample_m(Vec2(uv[2 * i], uv[2 * i + 1]), pdf);
    out_m[3 * i] = m.v.x;
    out_m[3 * i + 1] = m.v.y;
    out_m[3 * i + 2] = m.v.z;
    out_pdf[i] = pdf;
  }
}

}  // extern "C"
