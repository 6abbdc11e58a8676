// dort_gpu_bsdf_probe: one material's BxDF code (pt.cuh) evaluated and
// sampled for caller-given directions in the local shading frame, on the GPU
// or compiled for the host.  A diagnostic for checking the BxDF formulas and
// samplers against a float64 restatement (value, pdf, sampled direction, and
// the distribution of many samples); the renderers never call it.
#include <string>

#include "common.h"
#include "pt.cuh"
#include "scene_build.h"

namespace dort_gpu {
namespace {

struct ProbeArgs {
  DevMaterial m;
  size_t n;
  const float* wo;    // 3n: the fixed direction (towards the viewer)
  const float* wi;    // 3n: the direction evaluated (towards the light), or null
  const float* u;     // 3n: uniforms of the sampler, or null
  float* f;           // 3n: f(wi, wo)
  float* pdf;         // n:  pdf of sampling wi given wo
  float* swi;         // 3n: sampled direction
  float* sf;          // 3n: its f
  float* spdf;        // n:  its pdf (0: no sample)
};

DG_HD void probe_one(const ProbeArgs& a, size_t i) {
  V3 wo = v3(a.wo[3 * i], a.wo[3 * i + 1], a.wo[3 * i + 2]);
  if(a.wi) {
    V3 wi = v3(a.wi[3 * i], a.wi[3 * i + 1], a.wi[3 * i + 2]);
    V3 f = bxdf_eval<true>(a.m, wi, wo, F_ALL);
    a.f[3 * i] = f.x;
    a.f[3 * i + 1] = f.y;
    a.f[3 * i + 2] = f.z;
    a.pdf[i] = bxdf_pdf<true>(a.m, wi, wo, F_ALL);
  }
  if(a.u) {
    V3 wg = v3(0.f, 0.f, 0.f);
    float pdf = 0.f;
    uint32_t flags = 0;
    V3 f = bxdf_sample<true>(a.m, wo, F_ALL, a.u[3 * i], a.u[3 * i + 1], a.u[3 * i + 2], wg,
                             pdf, flags);
    a.swi[3 * i] = wg.x;
    a.swi[3 * i + 1] = wg.y;
    a.swi[3 * i + 2] = wg.z;
    a.sf[3 * i] = f.x;
    a.sf[3 * i + 1] = f.y;
    a.sf[3 * i + 2] = f.z;
    a.spdf[i] = pdf;
  }
}

__global__ void bsdf_probe_kernel(ProbeArgs a) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n;
      i += size_t(gridDim.x) * blockDim.x) {
    probe_one(a, i);
  }
}

}  // namespace
}  // namespace dort_gpu

using namespace dort_gpu;

extern "C" int dort_gpu_bsdf_probe(const dort_material* material, size_t n, const float* wo,
                                   const float* wi, const float* u, float* out_f,
                                   float* out_pdf, float* out_wi, float* out_sf,
                                   float* out_spdf, int on_device) try {
  clear_error();
  if(!material || (n && !wo) || (wi && (!out_f || !out_pdf)) ||
     (u && (!out_wi || !out_sf || !out_spdf))) {
    return fail(DORT_ERR_INVALID, "null argument");
  }
  ProbeArgs a{};
  std::string err;
  if(!material_to_device(*material, a.m, err)) { return fail(DORT_ERR_INVALID, err); }
  a.n = n;
  if(n == 0) { return DORT_OK; }
  if(!on_device) {
    a.wo = wo; a.wi = wi; a.u = u;
    a.f = out_f; a.pdf = out_pdf; a.swi = out_wi; a.sf = out_sf; a.spdf = out_spdf;
    for(size_t i = 0; i < n; ++i) { probe_one(a, i); }
    return DORT_OK;
  }
  // device: one buffer for the inputs and outputs, copied in and out
  const size_t v3b = 3 * n * sizeof(float), v1b = n * sizeof(float);
  size_t bytes = v3b + (wi ? v3b + v3b + v1b : 0) + (u ? v3b + v3b + v3b + v1b : 0);
  char* d = nullptr;
  if(dev_alloc(&d, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(DORT_ERR_OOM, "cudaMalloc for the BSDF probe failed");
  }
  char* p = d;
  auto take = [&](size_t b) { char* r = p; p += b; return reinterpret_cast<float*>(r); };
  float* d_wo = take(v3b);
  float *d_wi = nullptr, *d_f = nullptr, *d_pdf = nullptr;
  float *d_u = nullptr, *d_swi = nullptr, *d_sf = nullptr, *d_spdf = nullptr;
  if(wi) { d_wi = take(v3b); d_f = take(v3b); d_pdf = take(v1b); }
  if(u) { d_u = take(v3b); d_swi = take(v3b); d_sf = take(v3b); d_spdf = take(v1b); }
  cudaStream_t st = 0;
  bool ok = cudaMemcpyAsync(d_wo, wo, v3b, cudaMemcpyHostToDevice, st) == cudaSuccess;
  if(ok && wi) { ok = cudaMemcpyAsync(d_wi, wi, v3b, cudaMemcpyHostToDevice, st) == cudaSuccess; }
  if(ok && u) { ok = cudaMemcpyAsync(d_u, u, v3b, cudaMemcpyHostToDevice, st) == cudaSuccess; }
  if(ok) {
    a.wo = d_wo; a.wi = d_wi; a.u = d_u;
    a.f = d_f; a.pdf = d_pdf; a.swi = d_swi; a.sf = d_sf; a.spdf = d_spdf;
    unsigned blocks = unsigned(std::min<size_t>((n + 255) / 256, 148 * 8));
    bsdf_probe_kernel<<<blocks, 256, 0, st>>>(a);
    ok = cudaGetLastError() == cudaSuccess;
  }
  if(ok && wi) {
    ok = cudaMemcpyAsync(out_f, d_f, v3b, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaMemcpyAsync(out_pdf, d_pdf, v1b, cudaMemcpyDeviceToHost, st) == cudaSuccess;
  }
  if(ok && u) {
    ok = cudaMemcpyAsync(out_wi, d_swi, v3b, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaMemcpyAsync(out_sf, d_sf, v3b, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaMemcpyAsync(out_spdf, d_spdf, v1b, cudaMemcpyDeviceToHost, st) == cudaSuccess;
  }
  ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
  cudaFree(d);
  if(!ok) {
    return fail(DORT_ERR_CUDA, std::string("BSDF probe failed: ") +
                               cudaGetErrorString(cudaGetLastError()));
  }
  return DORT_OK;
} DORT_ABI_CATCH
