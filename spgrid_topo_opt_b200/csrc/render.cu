// Headless density renderer: the reference's CUDA visualiser
// (misc/volume_rendering_kernel.cu, misc/volume_renderer.cpp) without its window,
// OpenGL pixel buffer and texture unit.  The density blocks become an 8-bit
// volume in global memory (volume_renderer.cpp:410-480), a thread per pixel
// traces the camera ray and the frames accumulate into a float buffer; the
// packed RGBA image comes back to the host.
//
// Two modes, as the reference's:
//  * surface (render_surface, volume_rendering_kernel.cu:340-385): voxel DDA to
//    the first voxel above the threshold (get_next_hit, :214-270), three
//    ambient-occlusion rays towards random directions lit by a two-colour sky
//    (trace, :272-318), a grey background when the ray misses;
//  * volume (render_volume, :387-437): 1025 jittered steps of 0.01 through the
//    volume, exp(-extinction * max(0.01 * sum - threshold, 0)).
// Deliberate differences: the random numbers come from a counter-based hash
// (PCG hash, Jarzynski & Olano, "Hash Functions for GPU Rendering", JCGT 2020)
// keyed by pixel, frame and draw instead of per-thread cuRAND states, so that a
// CPU restatement draws the same numbers; the primary direction is normalised
// by a division by its length (the reference multiplies by an approximate
// reciprocal square root); a point sample reads voxel clamp(floor(t * res)) of
// the texture coordinate t.  Mirroring (the viewer's box_scale) doubles the box
// on the chosen axes and reflects coordinates past the volume's far face.
// This file is compiled without fused multiply-adds.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "band.hpp"

namespace sgs {
namespace {

constexpr int RENDER_MAX_STEPS = 1025;  // maxSteps (:129)
constexpr float RENDER_TSTEP = 0.01f;   // tstep (:131)

struct Camera {
  float m[12];  // rows of the 3x4 camera matrix (c_invViewMatrix)
};

struct VolumeView {
  const uint8_t* vox;  // x fastest: x + y*W + z*W*H
  int res[3];
  float3 scale;     // 2 on mirrored axes, else 1 (box_scale)
  float3 box_size;  // half extents: res / max(res), times scale
  float3 box_res;   // res times scale
  float slice;
};

__host__ __device__ inline uint32_t pcg_hash(uint32_t v) {
  const uint32_t state = v * 747796405u + 2891336453u;
  const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}

// a float in (0, 1] (like curand_uniform) from 24 bits of the hash
struct Rng {
  uint32_t key, n;
  __device__ float next() { return float((pcg_hash(key + n++) >> 8) + 1u) * (1.0f / 16777216.0f); }
};

__device__ inline float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ inline float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ inline float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ inline float3 mul(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ inline float3 scale(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ inline float3 addc(float3 a, float s) { return f3(a.x + s, a.y + s, a.z + s); }
__device__ inline float3 divv(float3 a, float3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ inline float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ inline float sgnf(float x) { return x > 0 ? 1.0f : (x < 0 ? -1.0f : 0.0f); }

__device__ inline bool inside_unit_cube(float3 p) {
  return -1.0f < p.x && p.x < 1.0f && -1.0f < p.y && p.y < 1.0f && -1.0f < p.z && p.z < 1.0f;
}

// tex3D with normalised coordinates, point filtering, clamped addressing, 8-bit
// values read as v / 255; the coordinate p in [-1, 1] goes through the
// reference's wrap_coord (mirroring off) first (:133-158).
__device__ inline float point_sample(const VolumeView& V, float3 p) {
  p = mul(addc(scale(p, 0.5f), 0.5f), V.scale);
  if (p.x > 1) p.x = 2 - p.x;
  if (p.y > 1) p.y = 2 - p.y;
  if (p.z > 1) p.z = 2 - p.z;
  p = addc(scale(p, 2.0f), -1.0f);
  const float3 t = addc(scale(p, 0.5f), 0.5f);
  const float tc[3] = {t.x, t.y, t.z};
  int i[3];
  for (int a = 0; a < 3; ++a) i[a] = min(max(int(floorf(tc[a] * float(V.res[a]))), 0), V.res[a] - 1);
  return float(__ldg(V.vox + (size_t(i[2]) * V.res[1] + i[1]) * V.res[0] + i[0])) / 255.0f;
}

// sample_tex (:145-152): a world position inside the box
__device__ inline float sample_world(const VolumeView& V, float3 pos) {
  const float3 p = divv(pos, V.box_size);
  if (!inside_unit_cube(p) || p.z > 2 * V.slice - 1) return 0;
  return point_sample(V, p);
}

// sample_tex_int (:155-164): the voxel at integer position ipos
__device__ inline float sample_voxel(const VolumeView& V, float3 ipos) {
  const float3 p = addc(scale(divv(addc(ipos, 0.5f), V.box_res), 2.0f), -1.0f);
  if (!inside_unit_cube(p) || p.z > 2 * V.slice - 1) return 0;
  return point_sample(V, p);
}

// intersectBox (:55-76)
__device__ inline bool intersect_box(float3 o, float3 d, float3 bmin, float3 bmax, float* tnear, float* tfar) {
  const float3 inv = divv(f3(1.0f, 1.0f, 1.0f), d);
  const float3 tbot = mul(inv, sub(bmin, o)), ttop = mul(inv, sub(bmax, o));
  const float3 tmin = f3(fminf(ttop.x, tbot.x), fminf(ttop.y, tbot.y), fminf(ttop.z, tbot.z));
  const float3 tmax = f3(fmaxf(ttop.x, tbot.x), fmaxf(ttop.y, tbot.y), fmaxf(ttop.z, tbot.z));
  *tnear = fmaxf(fmaxf(tmin.x, tmin.y), fmaxf(tmin.x, tmin.z));
  *tfar = fminf(fminf(tmax.x, tmax.y), fminf(tmax.x, tmax.z));
  return *tfar > *tnear;
}

// get_next_hit, DDA variant (:214-270): the first voxel above the threshold
// along the ray and the entry point into it.
__device__ bool next_hit(const VolumeView& V, float3 o, float3 d, float threshold, float3* hit_pos) {
  const float len = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
  d = f3(d.x / len, d.y / len, d.z / len);
  float tnear, tfar;
  if (!intersect_box(o, d, scale(V.box_size, -1.0f), V.box_size, &tnear, &tfar)) return false;
  if (tnear < 0.0f) tnear = 0.0f;
  const float3 pos = add(o, scale(d, tnear + 1e-4f));
  const float3 ri = divv(f3(1.0f, 1.0f, 1.0f), d);
  const float3 rs = f3(sgnf(d.x), sgnf(d.y), sgnf(d.z));
  const float3 org = scale(scale(add(pos, V.box_size), 0.5f), V.box_res.x / V.box_size.x);
  float3 ipos = f3(floorf(org.x), floorf(org.y), floorf(org.z));
  float3 dis = mul(add(addc(sub(ipos, org), 0.5f), scale(rs, 0.5f)), ri);
  for (int i = 0; i < RENDER_MAX_STEPS; ++i) {
    if (sample_voxel(V, ipos) > threshold) {
      const float3 mini = mul(sub(addc(sub(ipos, org), 0.5f), scale(rs, 0.5f)), ri);
      const float t = fmaxf(mini.x, fmaxf(mini.y, mini.z)) * (V.box_size.x / V.box_res.x) * 2.0f;
      *hit_pos = add(pos, scale(d, t));
      return true;
    }
    // the step as the reference writes it, dis += mm * rs * ri on all three
    // components (an axis-parallel ray turns the others into NaN there too)
    float3 mm;
    if (dis.x <= dis.y && dis.x < dis.z) mm = f3(1, 0, 0);
    else if (dis.y <= dis.x && dis.y <= dis.z) mm = f3(0, 1, 0);
    else mm = f3(0, 0, 1);
    dis = add(dis, mul(mul(mm, rs), ri));
    ipos = add(ipos, mul(mm, rs));
  }
  return false;
}

// The camera ray of pixel (x, y) with jitter (r0, r1) (:349-360): u, v in
// [-1, 1] scaled by the image width, direction (u, v, -2) normalised and
// rotated, origin the camera position.
__device__ inline void camera_ray(const Camera& C, unsigned x, unsigned y, unsigned W, float r0, float r1, float* u,
                                  float* v, float3* o, float3* d) {
  *u = ((float(x) + r0) / float(W)) * 2.0f - 1.0f;
  *v = ((float(y) + r1) / float(W)) * 2.0f - 1.0f;
  *o = f3(C.m[3], C.m[7], C.m[11]);
  float3 dir = f3(*u, *v, -2.0f);
  const float len = sqrtf(dot3(dir, dir));
  dir = f3(dir.x / len, dir.y / len, dir.z / len);
  *d = f3(dot3(dir, f3(C.m[0], C.m[1], C.m[2])), dot3(dir, f3(C.m[4], C.m[5], C.m[6])),
          dot3(dir, f3(C.m[8], C.m[9], C.m[10])));
}

__device__ inline uint32_t pack_rgba(float r, float g, float b, float a) {
  r = __saturatef(r);
  g = __saturatef(g);
  b = __saturatef(b);
  a = __saturatef(a);
  return (uint32_t(a * 255) << 24) | (uint32_t(b * 255) << 16) | (uint32_t(g * 255) << 8) | uint32_t(r * 255);
}

__device__ inline uint32_t pixel_key(uint32_t pixel, uint32_t frame, uint32_t seed) {
  return pcg_hash(pixel + pcg_hash(seed + frame * 0x9E3779B9u));
}

// Accumulate this frame's colour and, on the last frame, write the vignetted
// average (:362-384).
__device__ inline void finish_pixel(float* buf, uint32_t* out, size_t idx, float3 c, float u, float v, int frame,
                                    bool last) {
  buf[idx * 3 + 0] += c.x;
  buf[idx * 3 + 1] += c.y;
  buf[idx * 3 + 2] += c.z;
  if (!last) return;
  const float scale_ = 1.0f - 0.15f * (u * u + v * v);
  const float n = float(frame);
  out[idx] = pack_rgba(scale_ * (buf[idx * 3 + 0] / n), scale_ * (buf[idx * 3 + 1] / n),
                       scale_ * (buf[idx * 3 + 2] / n), scale_ * 1.0f);
}

__global__ void render_surface_kernel(VolumeView V, Camera C, unsigned W, unsigned H, float threshold, uint32_t seed,
                                      int frame, bool last, float* __restrict__ buf, uint32_t* __restrict__ out) {
  const unsigned x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  const size_t idx = size_t(y) * W + x;
  Rng rng{pixel_key(uint32_t(idx), uint32_t(frame), seed), 0};
  float u, v;
  float3 o, d;
  const float r0 = rng.next(), r1 = rng.next();
  camera_ray(C, x, y, W, r0, r1, &u, &v, &o, &d);
  // trace (:272-318)
  float3 sum = f3(0.86f, 0.85f, 0.9f), pos;
  if (next_hit(V, o, d, threshold, &pos)) {
    sum = f3(0.0f, 0.0f, 0.0f);
    const int samples = 3;
    for (int j = 0; j < samples; ++j) {
      const float a = rng.next(), b = rng.next();
      // sample_sphere (:166-171)
      const float sx = a * 2 - 1, phi = b * 2 * 3.14159265358979f, yz = sqrtf(1 - sx * sx);
      const float3 dir = f3(sx, yz * cosf(phi), yz * sinf(phi));
      float3 unused;
      const bool blocked = next_hit(V, pos, dir, threshold, &unused);
      const float c1 = fmaxf(0.0f, fminf(dot3(dir, f3(0.6f, 0.75f, 0.15f)) * 0.5f + 0.5f, 1.0f));
      const float3 light = add(scale(f3(0.9f, 0.7f, 0.3f), c1), scale(f3(0.4f, 0.5f, 0.9f), 1 - c1));
      if (!blocked) sum = add(sum, scale(light, 2.0f / samples));
    }
  }
  finish_pixel(buf, out, idx, sum, u, v, frame, last);
}

__global__ void render_volume_kernel(VolumeView V, Camera C, unsigned W, unsigned H, float threshold,
                                     float extinction, uint32_t seed, int frame, bool last, float* __restrict__ buf,
                                     uint32_t* __restrict__ out) {
  const unsigned x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  const size_t idx = size_t(y) * W + x;
  Rng rng{pixel_key(uint32_t(idx), uint32_t(frame), seed), 0};
  float u, v;
  float3 o, d;
  const float r0 = rng.next(), r1 = rng.next();
  camera_ray(C, x, y, W, r0, r1, &u, &v, &o, &d);
  float sum = 0, tnear, tfar;
  if (intersect_box(o, d, scale(V.box_size, -1.0f), V.box_size, &tnear, &tfar)) {
    if (tnear < 0.0f) tnear = 0.0f;
    float3 pos = add(o, scale(d, tnear + 1e-4f));
    const float3 step = scale(d, RENDER_TSTEP);
    for (int i = 0; i < RENDER_MAX_STEPS; ++i) {
      sum += sample_world(V, add(pos, scale(step, rng.next())));
      pos = add(pos, step);
    }
  }
  sum = float(double(sum) * 1e-2);
  sum = fmaxf(sum - threshold * 1, 0.0f);
  const float e = 1 - expf(-extinction * sum);
  const float g = 1 - e;
  finish_pixel(buf, out, idx, f3(g, g, g), u, v, frame, last);
}

// ---- the volume from density blocks (volume_renderer.cpp:410-480) ----
// bounding box of the cells with positive density, per axis
__global__ void density_bbox_kernel(long ncells, const int* __restrict__ base, const double* __restrict__ rho,
                                    int* __restrict__ box) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= ncells || !(rho[t] > 0)) return;
  const long b = t >> 6;
  const int e = int(t & 63);
  const int c[3] = {base[3 * b] + (e >> 4), base[3 * b + 1] + ((e >> 2) & 3), base[3 * b + 2] + (e & 3)};
  for (int a = 0; a < 3; ++a) {
    atomicMin(box + a, c[a]);
    atomicMax(box + 3 + a, c[a] + 1);
  }
}

// voxel = 0 for density 0, else uchar(d * 254) + 1 (d first mapped back from a
// SIMP stiffness when reverse_mapping); cells outside the box are dropped
__global__ void density_voxels_kernel(long ncells, const int* __restrict__ base, const double* __restrict__ rho,
                                      int x0, int y0, int z0, int W, int H, int D, int reverse_mapping,
                                      uint8_t* __restrict__ vox) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= ncells) return;
  const long b = t >> 6;
  const int e = int(t & 63);
  const int x = base[3 * b] + (e >> 4) - x0, y = base[3 * b + 1] + ((e >> 2) & 3) - y0,
            z = base[3 * b + 2] + (e & 3) - z0;
  if (x < 0 || y < 0 || z < 0 || x >= W || y >= H || z >= D) return;
  double d = rho[t];
  if (reverse_mapping && d > 0) d = pow(d - 1e-6, 0.33333333) * (1 - 1e-6);
  uint8_t v = 0;
  if (d != 0) v = uint8_t(min(max(int(d * 254), 0), 254) + 1);
  vox[(size_t(z) * H + y) * W + x] = v;
}

// Render blocks that live on the device.  box_out receives the volume's
// resolution.
void render_device(const int* base_d, const double* rho_d, long nblocks, const sgs_render_params& p, uint32_t* rgba,
                   int32_t* res_out, cudaStream_t stream) {
  if (p.width <= 0 || p.height <= 0 || p.frames <= 0 || (p.mode != 0 && p.mode != 1))
    throw CudaError("render: invalid image size, frame count or mode", SGS_ERR_INPUT);
  const long ncells = nblocks * 64;
  DevBuf<int> box;
  box.alloc(6);
  const int init[6] = {1 << 30, 1 << 30, 1 << 30, 0, 0, 0};
  SGS_CUDA(cudaMemcpyAsync(box.p, init, sizeof(init), cudaMemcpyHostToDevice, stream));
  if (ncells)
    density_bbox_kernel<<<blocks_for(ncells, 256), 256, 0, stream>>>(ncells, base_d, rho_d, box.p);
  SGS_CUDA(cudaGetLastError());
  int bb[6];
  SGS_CUDA(cudaMemcpyAsync(bb, box.p, sizeof(bb), cudaMemcpyDeviceToHost, stream));
  SGS_CUDA(cudaStreamSynchronize(stream));
  int res[3];
  for (int a = 0; a < 3; ++a) res[a] = bb[3 + a] - bb[a];
  if (res[0] <= 0 || res[1] <= 0 || res[2] <= 0) throw CudaError("render: no cell with positive density", SGS_ERR_INPUT);
  if (res_out)
    for (int a = 0; a < 3; ++a) res_out[a] = res[a];
  DevBuf<uint8_t> vox;
  vox.alloc(size_t(res[0]) * res[1] * res[2]);
  vox.zero(stream);
  density_voxels_kernel<<<blocks_for(ncells, 256), 256, 0, stream>>>(ncells, base_d, rho_d, bb[0], bb[1], bb[2],
                                                                     res[0], res[1], res[2], p.reverse_mapping, vox.p);
  SGS_CUDA(cudaGetLastError());
  VolumeView V;
  V.vox = vox.p;
  const int rmax = std::max(res[0], std::max(res[1], res[2]));
  for (int a = 0; a < 3; ++a) V.res[a] = res[a];
  const float sc[3] = {(p.mirror & 1) ? 2.0f : 1.0f, (p.mirror & 2) ? 2.0f : 1.0f, (p.mirror & 4) ? 2.0f : 1.0f};
  V.scale = make_float3(sc[0], sc[1], sc[2]);
  V.box_size = make_float3(float(res[0]) / float(rmax) * sc[0], float(res[1]) / float(rmax) * sc[1],
                           float(res[2]) / float(rmax) * sc[2]);
  V.box_res = make_float3(float(res[0]) * sc[0], float(res[1]) * sc[1], float(res[2]) * sc[2]);
  V.slice = p.slice;
  Camera C;
  for (int k = 0; k < 12; ++k) C.m[k] = p.camera[k];
  const size_t npix = size_t(p.width) * p.height;
  DevBuf<float> buf;
  DevBuf<uint32_t> out;
  buf.alloc(npix * 3);
  buf.zero(stream);
  out.alloc(npix);
  const dim3 blk(16, 16), grd((p.width + 15) / 16, (p.height + 15) / 16);
  for (int f = 1; f <= p.frames; ++f) {
    const bool last = f == p.frames;
    if (p.mode == 0)
      render_surface_kernel<<<grd, blk, 0, stream>>>(V, C, unsigned(p.width), unsigned(p.height), p.threshold, p.seed,
                                                     f, last, buf.p, out.p);
    else
      render_volume_kernel<<<grd, blk, 0, stream>>>(V, C, unsigned(p.width), unsigned(p.height), p.threshold,
                                                    p.extinction, p.seed, f, last, buf.p, out.p);
    SGS_CUDA(cudaGetLastError());
  }
  SGS_CUDA(cudaMemcpyAsync(rgba, out.p, npix * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
  g_d2h_bytes += npix * sizeof(uint32_t);
  SGS_CUDA(cudaStreamSynchronize(stream));
}

}  // namespace
}  // namespace sgs

using namespace sgs;

SGS_API int sgs_render(const int32_t* block_base, int64_t nblocks, const double* density, const sgs_render_params* p,
                       uint32_t* rgba, int32_t* volume_res) {
  if (!block_base || !density || !p || !rgba || nblocks <= 0) return SGS_ERR_INPUT;
  try {
    cudaStream_t s;
    SGS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::unique_ptr<CUstream_st, void (*)(cudaStream_t)> guard(s, [](cudaStream_t q) { cudaStreamDestroy(q); });
    DevBuf<int> base;
    DevBuf<double> rho;
    base.upload(block_base, size_t(nblocks) * 3, s);
    rho.upload(density, size_t(nblocks) * 64, s);
    render_device(base.p, rho.p, long(nblocks), *p, rgba, volume_res, s);
  } catch (const CudaError& e) {
    return e.code;
  } catch (const std::exception&) {
    return SGS_ERR_INTERNAL;
  }
  return 0;
}

SGS_API int sgs_band_render(sgs_band* b, const sgs_render_params* p, uint32_t* rgba, int32_t* volume_res) {
  if (!b || !b->band || !p || !rgba) return SGS_ERR_INPUT;
  try {
    Band& B = *b->band;
    render_device(B.base.p, B.rho.p, B.n, *p, rgba, volume_res, B.stream);
  } catch (const CudaError& e) {
    b->error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    b->error = e.what();
    return SGS_ERR_INTERNAL;
  }
  return 0;
}
