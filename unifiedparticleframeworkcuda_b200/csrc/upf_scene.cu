// upf_scene.cu — scene construction on the device.
//
// Particles that fill a closed triangle mesh: the reference's
// ObjectLoader::LoadParticles (src/cpu/ObjectLoader.cpp:8-97), which places a
// staggered lattice over the mesh's bounding box and keeps every lattice
// point whose segment from a fixed outside point crosses the mesh an odd
// number of times, or that lies on a face (Polygon::DoesLineIntersect /
// DoesPointTouch, src/cpu/Polygon.cpp). The reference tests every point
// against every face on one CPU thread; here one thread tests one point,
// the faces stream through shared memory in tiles shared by the CTA, and an
// order-keeping compaction writes the kept points in the reference's
// x-major, then y, then z order. Every float expression is the reference's,
// with its operation order and roundings (-fmad=false; the face data and
// the lattice coordinates, which the reference accumulates by repeated
// addition, are computed on the host in the same order), so the positions
// are bit-identical.
//
// The OBJ reader follows ObjLoader::Load (src/cpu/ObjLoader.cpp:58-233).
#include <cuda_runtime.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/upf.h"
#include "upf_internal.h"

namespace upf {
namespace {

// Polygon's tolerance for parallel lines and touching points
// (static const float kAlmostZero, Polygon.cpp:3)
constexpr float kAlmostZero = 0.000001f;

// One triangle as the reference's Polygon holds it after three AddVertex
// calls (Polygon.cpp:20-35): the vertices, the unit normal, the plane
// offset d = -v0.n, the projection axes of the 2D edge tests, and the point
// outside the polygon used by IsPointInPlaneInside (its bounding box's
// minimum minus 1; the box starts at the origin, as Polygon's constructor
// sets it).
// The edge tests work on two coordinates (fi, si) picked by the normal;
// the vertices and the outside point are stored already projected (p2: 3
// corners x 2, o2), which selects values and changes none. q = -(d +
// outside.n) is DoesLineIntersect's numerator for segments that start at
// the lattice's outside point, the same for every lattice point.
struct __align__(16) FaceData {
  float p2[6];
  float o2[2];
  float n[3];
  float d;
  float q;
  int fi, si;
  int unused;  // 64 bytes: whole 16-byte words for the tile loads
};
static_assert(sizeof(FaceData) == 64, "face record");

// --------------------------------------------------------------- host side
float host_min(float a, float b) { return (b < a) ? b : a; }  // std::min(a, b)
float host_max(float a, float b) { return (a < b) ? b : a; }  // std::max(a, b)

FaceData make_face(const float* t9, float bmin[3], float bmax[3]) {
  FaceData f{};
  for (int a = 0; a < 3; ++a) bmin[a] = bmax[a] = 0.0f;
  for (int j = 0; j < 3; ++j)
    for (int a = 0; a < 3; ++a) {
      bmin[a] = host_min(t9[3 * j + a], bmin[a]);
      bmax[a] = host_max(t9[3 * j + a], bmax[a]);
    }
  // normal_ = (v0 - v1).cross(v2 - v1), then Vector3::normalize
  // (vmmlib/vector3.h: length = sqrtf(x*x + y*y + z*z); ll = 1.0 / l in
  // double, stored as float; each component *= ll)
  const float a0 = t9[0] - t9[3], a1 = t9[1] - t9[4], a2 = t9[2] - t9[5];
  const float b0 = t9[6] - t9[3], b1 = t9[7] - t9[4], b2 = t9[8] - t9[5];
  float n0 = a1 * b2 - a2 * b1, n1 = a2 * b0 - a0 * b2, n2 = a0 * b1 - a1 * b0;
  const float l = sqrtf(n0 * n0 + n1 * n1 + n2 * n2);
  if (l != 0.0f) {
    const float ll = (float)(1.0 / (double)l);
    n0 *= ll;
    n1 *= ll;
    n2 *= ll;
  }
  f.n[0] = n0;
  f.n[1] = n1;
  f.n[2] = n2;
  f.d = -(t9[0] * n0 + t9[1] * n1 + t9[2] * n2);
  // ArePointsOnBothSidesOfTheLine's projection (Polygon.cpp:74-92)
  if (n0 == 0.0f) {
    f.fi = 0;
    f.si = (n1 == 0.0f) ? 1 : 2;
  } else {
    f.fi = 1;
    f.si = 2;
  }
  for (int j = 0; j < 3; ++j) {
    f.p2[2 * j] = t9[3 * j + f.fi];
    f.p2[2 * j + 1] = t9[3 * j + f.si];
  }
  // IsPointInPlaneInside's outside point, boundary_min_ - 1 (Polygon.cpp:124)
  f.o2[0] = bmin[f.fi] - 1.0f;
  f.o2[1] = bmin[f.si] - 1.0f;
  return f;
}

// ------------------------------------------------------------- device side
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float dot3(const float* a, const float* b) {
  return fa(fa(fm(a[0], b[0]), fm(a[1], b[1])), fm(a[2], b[2]));
}

// Polygon::ArePointsOnBothSidesOfTheLine (Polygon.cpp:70-104) on projected
// points (x = coordinate fi, y = coordinate si)
__device__ __forceinline__ bool both_sides(float2 ls, float2 le, float2 p1, float2 p2) {
  const float dxES = fs(le.x, ls.x);
  const float dx1E = fs(p1.x, le.x);
  const float dySE = fs(ls.y, le.y);
  const float dyE1 = fs(le.y, p1.y);
  const bool c1 = fm(dySE, dx1E) > fm(dyE1, dxES);
  const float dx2E = fs(p2.x, le.x);
  const float dyE2 = fs(le.y, p2.y);
  const bool c2 = fm(dySE, dx2E) > fm(dyE2, dxES);
  return c1 != c2;
}

// Polygon::IsPointInPlaneInside (Polygon.cpp:120-141)
__device__ __forceinline__ bool inside_polygon(const FaceData& f, const float* pt) {
  const float2 p = make_float2(f.fi == 0 ? pt[0] : pt[1], f.si == 1 ? pt[1] : pt[2]);
  const float2 o = make_float2(f.o2[0], f.o2[1]);
  const float2 v[3] = {make_float2(f.p2[0], f.p2[1]), make_float2(f.p2[2], f.p2[3]), make_float2(f.p2[4], f.p2[5])};
  bool inside = false;
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const float2 s = v[e], t = v[(e + 1) % 3];
    if (both_sides(o, p, s, t) && both_sides(s, t, o, p)) inside = !inside;
  }
  return inside;
}

// Polygon::DoesLineIntersect (Polygon.cpp:45-68) for the segment from the
// lattice's outside point st to a lattice point, dv = point - st. The
// numerator f.q was computed on the host with the same operations. The
// quotient t = q / den is rounded as the reference rounds it; it is only
// skipped where its rounded value certainly lies outside [0, 1]: q and den
// of opposite signs (t < 0; |q| >= 2^-100 and |den| <= 2^20 keep the
// quotient clear of underflow to -0), or |q| > 2 |den| (t >= 2).
__device__ __forceinline__ bool line_intersects(const FaceData& f, const float* st, const float* dv) {
  const float den = dot3(dv, f.n);
  if (fabsf(den) < kAlmostZero) return false;
  const float q = f.q, aq = fabsf(q), ad = fabsf(den);
  if (aq > 2.0f * ad) return false;
  if ((q < 0.0f) != (den < 0.0f) && aq >= 7.8886091e-31f && ad <= 1048576.0f) return false;
  const float t = __fdiv_rn(q, den);
  if (t < 0.0f || t > 1.0f) return false;
  const float hit[3] = {fa(st[0], fm(dv[0], t)), fa(st[1], fm(dv[1], t)), fa(st[2], fm(dv[2], t))};
  return inside_polygon(f, hit);
}

// Polygon::DoesPointTouch (Polygon.cpp:107-117)
__device__ __forceinline__ bool point_touches(const FaceData& f, const float* pt) {
  const float eq = fa(dot3(pt, f.n), f.d);
  if (fabsf(eq) > kAlmostZero) return false;
  return inside_polygon(f, pt);
}

constexpr int kVoxelThreads = 256;
constexpr int kFaceTile = 256;  // faces per shared-memory tile (16 KB)

struct Lattice {
  const float* xs;      // [nx]
  const float* ys;      // [2][ny] (by x parity)
  const float* zs;      // [2][nz]
  uint32_t nx, ny, nz;
  float outside[3];     // mesh box minimum - spacing
};

// The inside test of ObjectLoader::LoadParticles' innermost loop
// (ObjectLoader.cpp:57-76) for lattice point `idx` (x-major, then y, then
// z); `keep[idx]` = 1 if the point becomes a particle. Every thread of the
// CTA walks the faces in the same order, tile by tile.
__global__ void __launch_bounds__(kVoxelThreads) k_voxel_flags(const FaceData* __restrict__ faces, uint32_t nf,
                                                               const Lattice L, uint64_t npts,
                                                               uint8_t* __restrict__ keep) {
  __shared__ FaceData tile[kFaceTile];
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = idx < npts;
  float pt[3] = {0.0f, 0.0f, 0.0f};
  if (live) {
    const uint32_t z = (uint32_t)(idx % L.nz);
    const uint64_t xy = idx / L.nz;
    const uint32_t y = (uint32_t)(xy % L.ny);
    const uint32_t x = (uint32_t)(xy / L.ny);
    const uint32_t par = x & 1u;
    pt[0] = L.xs[x];
    pt[1] = L.ys[par * L.ny + y];
    pt[2] = L.zs[par * L.nz + z];
  }
  const float dv[3] = {fs(pt[0], L.outside[0]), fs(pt[1], L.outside[1]), fs(pt[2], L.outside[2])};
  bool add = false, done = !live;
  for (uint32_t base = 0; base < nf; base += kFaceTile) {
    const uint32_t cnt = nf - base < (uint32_t)kFaceTile ? nf - base : (uint32_t)kFaceTile;
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) tile[k] = faces[base + k];
    __syncthreads();
    if (done) continue;
    for (uint32_t k = 0; k < cnt; ++k) {
      const FaceData& f = tile[k];
      if (line_intersects(f, L.outside, dv)) {
        add = !add;
      } else if (point_touches(f, pt)) {
        add = true;
        done = true;
        break;
      }
    }
  }
  if (live) keep[idx] = add ? 1 : 0;
}

constexpr int kScanThreads = 1024;

// Kept points per block of kScanThreads lattice points.
__global__ void __launch_bounds__(kScanThreads) k_voxel_block_counts(const uint8_t* __restrict__ keep, uint64_t n,
                                                                     uint32_t* __restrict__ counts) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = __syncthreads_count(i < n && keep[i]);
  if (threadIdx.x == 0) counts[blockIdx.x] = (uint32_t)c;
}

// Exclusive prefix of the block counts, one CTA walking them in chunks;
// the total goes to offs[nblocks].
__global__ void __launch_bounds__(kScanThreads) k_voxel_scan(const uint32_t* __restrict__ counts, uint32_t nblocks,
                                                             uint32_t* __restrict__ offs) {
  __shared__ uint32_t warp_sums[kScanThreads / 32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t base = 0; base < nblocks; base += kScanThreads) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < nblocks ? counts[i] : 0u;
    uint32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = warp_sums[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += u;
      }
      warp_sums[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const uint32_t before = carry + (warp ? warp_sums[warp - 1] : 0u) + incl - v;
    if (i < nblocks) offs[i] = before;
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) carry = before + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) offs[nblocks] = carry;
}

// Writes each kept point's particle position at its rank among the kept
// points: ((x - min) * scale) per axis (ObjectLoader.cpp:79-80).
__global__ void __launch_bounds__(kScanThreads) k_voxel_scatter(const uint8_t* __restrict__ keep, uint64_t n,
                                                                const uint32_t* __restrict__ offs, const Lattice L,
                                                                float3 mn, float3 scale, float4* __restrict__ out) {
  __shared__ uint32_t warp_cnt[kScanThreads / 32];
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool k = i < n && keep[i];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t ball = __ballot_sync(0xffffffffu, k);
  if (lane == 0) warp_cnt[warp] = __popc(ball);
  __syncthreads();
  uint32_t before = offs[blockIdx.x];
  for (int w = 0; w < warp; ++w) before += warp_cnt[w];
  before += __popc(ball & ((1u << lane) - 1u));
  if (!k) return;
  const uint32_t z = (uint32_t)(i % L.nz);
  const uint64_t xy = i / L.nz;
  const uint32_t y = (uint32_t)(xy % L.ny);
  const uint32_t x = (uint32_t)(xy / L.ny);
  const uint32_t par = x & 1u;
  out[before] = make_float4(fm(fs(L.xs[x], mn.x), scale.x), fm(fs(L.ys[par * L.ny + y], mn.y), scale.y),
                            fm(fs(L.zs[par * L.nz + z], mn.z), scale.z), 0.0f);
}

// Lattice coordinates along one axis as the reference accumulates them:
// start, then += step once per point (ObjectLoader.cpp:52-84).
void accumulate(std::vector<float>& out, float start, float step, uint32_t count) {
  out.resize(count);
  float c = start;
  for (uint32_t k = 0; k < count; ++k) {
    out[k] = c;
    c += step;
  }
}

// Number of loop iterations of `for (int i = 0; i <= steps; ++i)`.
uint64_t loop_count(float steps) {
  if (!(steps >= 0.0f)) return 0;
  uint64_t c = (uint64_t)steps + 1;
  while (c > 0 && (float)(c - 1) > steps) --c;  // the comparison is done in float
  while ((float)c <= steps) ++c;
  return c;
}

template <class T>
cudaError_t dmalloc(T** p, size_t count) {
  if (inject_alloc_failure()) {
    set_error("cudaMalloc of %zu bytes failed: injected by upf_test_fail_allocation", count * sizeof(T));
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc((void**)p, count * sizeof(T) + 16);
}

}  // namespace
}  // namespace upf

using namespace upf;

upf_status upf_mesh_particles(int device, const float* tri9, uint32_t n_tri, float scale_x, float scale_y,
                              float scale_z, float spacing, float* pos4, uint32_t capacity, uint32_t* n_out) {
  const char* who = "upf_mesh_particles";
  if (!n_out || (n_tri > 0 && !tri9) || !(spacing > 0.0f) || !(scale_x > 0.0f) || !(scale_y > 0.0f) ||
      !(scale_z > 0.0f) || (capacity > 0 && !pos4)) {
    set_error("%s: bad arguments", who);
    return UPF_ERR_INVALID_ARG;
  }
  *n_out = 0;
  if (n_tri == 0) return UPF_OK;  // the reference returns no particles for a mesh without faces
  // faces and the mesh's bounding box (ObjectLoader.cpp:31-44)
  std::vector<FaceData> faces(n_tri);
  float mn[3], mx[3];
  for (uint32_t t = 0; t < n_tri; ++t) {
    float bmin[3], bmax[3];
    faces[t] = make_face(tri9 + 9 * (size_t)t, bmin, bmax);  // q is set below, once the box is known
    for (int a = 0; a < 3; ++a) {
      if (t == 0) {
        mn[a] = bmin[a];
        mx[a] = bmax[a];
      } else {
        mn[a] = host_min(mn[a], bmin[a]);
        mx[a] = host_max(mx[a], bmax[a]);
      }
    }
  }
  // the segments' common start, outside = min_vec - spacing (ObjectLoader.cpp:50)
  const float outside[3] = {mn[0] - spacing, mn[1] - spacing, mn[2] - spacing};
  for (uint32_t t = 0; t < n_tri; ++t) {
    const FaceData& f = faces[t];
    faces[t].q = -(f.d + (outside[0] * f.n[0] + outside[1] * f.n[1] + outside[2] * f.n[2]));
  }
  // the lattice (ObjectLoader.cpp:46-86)
  const float x_steps = (mx[0] - mn[0]) * scale_x / spacing;
  const float y_steps = (mx[1] - mn[1]) * scale_y / spacing;
  const float z_steps = (mx[2] - mn[2]) * scale_z / spacing;
  const uint64_t nx = loop_count(x_steps), ny = loop_count(y_steps), nz = loop_count(z_steps);
  const uint64_t npts = nx * ny * nz;
  if (npts == 0) return UPF_OK;
  if (nx > (1u << 30) || ny > (1u << 30) || nz > (1u << 30) || npts > ((uint64_t)1 << 31)) {
    set_error("%s: a lattice of %llu x %llu x %llu points is beyond the 2^31-point limit (spacing %g for a "
              "box of %g x %g x %g after scaling)",
              who, (unsigned long long)nx, (unsigned long long)ny, (unsigned long long)nz, spacing,
              (mx[0] - mn[0]) * scale_x, (mx[1] - mn[1]) * scale_y, (mx[2] - mn[2]) * scale_z);
    return UPF_ERR_INVALID_ARG;
  }
  std::vector<float> xs, ys, zs, tmp;
  accumulate(xs, mn[0], spacing / scale_x, (uint32_t)nx);
  ys.reserve(2 * ny);
  zs.reserve(2 * nz);
  for (int par = 0; par < 2; ++par) {  // current_pos[1], [2] restart at each x (y) with x's parity
    accumulate(tmp, mn[1] + par * spacing / (2 * scale_y), spacing / scale_y, (uint32_t)ny);
    ys.insert(ys.end(), tmp.begin(), tmp.end());
    accumulate(tmp, mn[2] + par * spacing / (2 * scale_z), spacing / scale_z, (uint32_t)nz);
    zs.insert(zs.end(), tmp.begin(), tmp.end());
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("%s: no CUDA device", who);
    return UPF_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    set_error("%s: bad device %d", who, device);
    return UPF_ERR_INVALID_ARG;
  }
  NvtxRange nv(who);
  cudaError_t e = cudaSetDevice(device);
  const uint32_t nblk = (uint32_t)((npts + kScanThreads - 1) / kScanThreads);
  FaceData* d_faces = nullptr;
  float *d_xs = nullptr, *d_ys = nullptr, *d_zs = nullptr;
  uint8_t* d_keep = nullptr;
  uint32_t *d_counts = nullptr, *d_offs = nullptr;
  float4* d_out = nullptr;
  cudaStream_t st = nullptr;
  uint32_t total = 0;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = dmalloc(&d_faces, n_tri);
  if (e == cudaSuccess) e = dmalloc(&d_xs, xs.size());
  if (e == cudaSuccess) e = dmalloc(&d_ys, ys.size());
  if (e == cudaSuccess) e = dmalloc(&d_zs, zs.size());
  if (e == cudaSuccess) e = dmalloc(&d_keep, npts);
  if (e == cudaSuccess) e = dmalloc(&d_counts, nblk);
  if (e == cudaSuccess) e = dmalloc(&d_offs, (size_t)nblk + 1);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_faces, faces.data(), sizeof(FaceData) * n_tri, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_xs, xs.data(), sizeof(float) * xs.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_ys, ys.data(), sizeof(float) * ys.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_zs, zs.data(), sizeof(float) * zs.size(), cudaMemcpyHostToDevice, st);
  Lattice L{d_xs, d_ys, d_zs, (uint32_t)nx, (uint32_t)ny, (uint32_t)nz, {outside[0], outside[1], outside[2]}};
  if (e == cudaSuccess) {
    k_voxel_flags<<<(uint32_t)((npts + kVoxelThreads - 1) / kVoxelThreads), kVoxelThreads, 0, st>>>(d_faces, n_tri, L,
                                                                                                  npts, d_keep);
    k_voxel_block_counts<<<nblk, kScanThreads, 0, st>>>(d_keep, npts, d_counts);
    k_voxel_scan<<<1, kScanThreads, 0, st>>>(d_counts, nblk, d_offs);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&total, d_offs + nblk, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  upf_status status = UPF_OK;
  if (e == cudaSuccess) {
    *n_out = total;
    if (pos4 && total > capacity) {
      set_error("%s: the mesh gives %u particles, capacity is %u", who, total, capacity);
      status = UPF_ERR_INVALID_ARG;
    } else if (pos4 && total > 0) {
      e = dmalloc(&d_out, total);
      if (e == cudaSuccess) {
        k_voxel_scatter<<<nblk, kScanThreads, 0, st>>>(d_keep, npts, d_offs, L, make_float3(mn[0], mn[1], mn[2]),
                                                       make_float3(scale_x, scale_y, scale_z), d_out);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaMemcpyAsync(pos4, d_out, sizeof(float4) * total, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
  }
  if (st) cudaStreamSynchronize(st);
  cudaFree(d_faces);
  cudaFree(d_xs);
  cudaFree(d_ys);
  cudaFree(d_zs);
  cudaFree(d_keep);
  cudaFree(d_counts);
  cudaFree(d_offs);
  cudaFree(d_out);
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    if (e != cudaErrorMemoryAllocation || !std::strstr(upf_last_error(), "injected"))
      set_error("%s: %s", who, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? UPF_ERR_ALLOC : UPF_ERR_CUDA;
  }
  return status;
}

// ObjLoader::Load + LoadFaces (src/cpu/ObjLoader.cpp:17-233): "v x y z" lines
// are vertices, "f" lines triangles (the first three corners of the line),
// everything else (comments, groups, vt, vn, materials) is skipped. Numbers
// are read with the reference's own sscanf conversions ("%f%f%f" after
// "v ", "%d/%d/%d ..." after "f "). The reference reads only v/vt/vn corners
// (any other spelling leaves its indices undefined); here "a", "a/b" and
// "a//c" corners are read too. Corner indices are 1-based into all of the
// file's vertices; an index outside them is an error (the reference reads
// out of bounds). The reference's read loop (while (!feof) { fgets; ... })
// handles a newline-terminated last line twice: when the file ends with an
// "f" line, its triangle is listed twice, and the inside test then toggles
// twice for every segment that crosses it, so that face no longer counts.
// Filling is bit-identical only with the same face list, so the last line
// is read twice here too (lines are read whole; the reference splits lines
// longer than 255 characters).
upf_status upf_obj_read_triangles(const char* path, float* tri9, uint32_t capacity, uint32_t* n_out) {
  const char* who = "upf_obj_read_triangles";
  if (!path || !n_out || (capacity > 0 && !tri9)) {
    set_error("%s: bad arguments", who);
    return UPF_ERR_INVALID_ARG;
  }
  *n_out = 0;
  FILE* fp = std::fopen(path, "r");
  if (!fp) {
    set_error("%s: cannot open %s: %s", who, path, std::strerror(errno));
    return UPF_ERR_IO;
  }
  std::vector<float> verts;
  std::vector<int> corners;
  std::string line;
  char chunk[4096];
  long lineno = 0;
  bool bad = false, again = false;
  std::string why;
  for (;;) {
    if (bad) break;
    if (std::fgets(chunk, sizeof chunk, fp)) {
      line.assign(chunk);
      while (!line.empty() && line.back() != '\n' && std::fgets(chunk, sizeof chunk, fp)) line.append(chunk);
      ++lineno;
    } else if (!again && !line.empty() && line.back() == '\n') {
      again = true;  // the reference's loop reads the last line once more
    } else {
      break;
    }
    const char* b = line.c_str();
    if (std::strncmp("v ", b, 2) == 0) {
      float x = 0, y = 0, z = 0;
      if (std::sscanf(b + 2, "%f%f%f", &x, &y, &z) != 3) {
        bad = true;
        why = "a vertex line without three numbers";
      }
      verts.push_back(x);
      verts.push_back(y);
      verts.push_back(z);
    } else if (std::strncmp("f ", b, 2) == 0) {
      int c[9];
      int got = std::sscanf(b + 2, "%d/%d/%d %d/%d/%d %d/%d/%d", &c[0], &c[1], &c[2], &c[3], &c[4], &c[5], &c[6],
                            &c[7], &c[8]);
      int v0, v1, v2;
      if (got == 9) {
        v0 = c[0], v1 = c[3], v2 = c[6];
      } else if (std::sscanf(b + 2, "%d//%d %d//%d %d//%d", &c[0], &c[1], &c[2], &c[3], &c[4], &c[5]) == 6 ||
                 std::sscanf(b + 2, "%d/%d %d/%d %d/%d", &c[0], &c[1], &c[2], &c[3], &c[4], &c[5]) == 6) {
        v0 = c[0], v1 = c[2], v2 = c[4];
      } else if (std::sscanf(b + 2, "%d %d %d", &c[0], &c[1], &c[2]) == 3) {
        v0 = c[0], v1 = c[1], v2 = c[2];
      } else {
        bad = true;
        why = "a face line without three corners";
        break;
      }
      corners.push_back(v0);
      corners.push_back(v1);
      corners.push_back(v2);
    }
  }
  std::fclose(fp);
  if (bad) {
    set_error("%s: %s line %ld: %s", who, path, lineno, why.c_str());
    return UPF_ERR_IO;
  }
  const size_t nv = verts.size() / 3, nt = corners.size() / 3;
  if (nt > 0xffffffffu) {
    set_error("%s: %s has too many faces", who, path);
    return UPF_ERR_INVALID_ARG;
  }
  for (size_t k = 0; k < corners.size(); ++k) {
    if (corners[k] < 1 || (size_t)corners[k] > nv) {
      set_error("%s: %s face %zu refers to vertex %d of %zu", who, path, k / 3 + 1, corners[k], nv);
      return UPF_ERR_IO;
    }
  }
  *n_out = (uint32_t)nt;
  if (!tri9) return UPF_OK;
  if (nt > capacity) {
    set_error("%s: %s holds %zu faces, capacity is %u", who, path, nt, capacity);
    return UPF_ERR_INVALID_ARG;
  }
  for (size_t k = 0; k < corners.size(); ++k)
    for (int a = 0; a < 3; ++a) tri9[3 * k + a] = verts[3 * (size_t)(corners[k] - 1) + a];
  return UPF_OK;
}

// ---------------------------------------------------------------- lattice fluid and box walls
namespace upf {
namespace {

struct FluidBlock {
  int nx, ny, nz;
  float spacing, jitter;
  double off[3];
};

// A rigid body's surface particles (the procedural shapes of the coupling
// workload, in place of voxelising an OBJ model): point k in the body frame,
// then rotated and moved, x = R p + c, in double and stored as float.
//   sphere (shape 0): a Fibonacci lattice of n points on radius r;
//   cube (1): a k x k grid of cell centres on each face of half-edge r, faces
//     in the order -x, +x, -y, +y, -z, +z (the grid's first index runs along
//     the next axis after the face's normal);
//   torus (2): an nu x nv grid of (u, v) cell centres, major radius r, minor
//     radius r / 3.
struct RigidSurface {
  int shape;
  double r;
  uint32_t n, k, nu, nv;
  double R[9], c[3];
};

__global__ void k_rigid_surface(const RigidSurface S, float4* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n) return;
  const double pi = 3.141592653589793;
  double p[3];
  if (S.shape == 0) {
    const double t = (double)i + 0.5;
    const double phi = acos(1.0 - 2.0 * t / (double)S.n);
    const double theta = pi * (1.0 + sqrt(5.0)) * t;
    p[0] = S.r * (cos(theta) * sin(phi));
    p[1] = S.r * (sin(theta) * sin(phi));
    p[2] = S.r * cos(phi);
  } else if (S.shape == 1) {
    const uint32_t kk = S.k * S.k, face = i / kk, j = i % kk;
    const uint32_t ia = j / S.k, ib = j % S.k;
    const double a = ((double)ia + 0.5) / (double)S.k * 2.0 * S.r - S.r;
    const double b = ((double)ib + 0.5) / (double)S.k * 2.0 * S.r - S.r;
    const int axis = (int)(face / 2);
    p[axis] = (face & 1) ? S.r : -S.r;
    p[(axis + 1) % 3] = a;
    p[(axis + 2) % 3] = b;
  } else {
    const uint32_t iu = i / S.nv, iv = i % S.nv;
    const double u = ((double)iu + 0.5) / (double)S.nu * 2.0 * pi;
    const double v = ((double)iv + 0.5) / (double)S.nv * 2.0 * pi;
    const double a = S.r / 3.0;
    p[0] = (S.r + a * cos(v)) * cos(u);
    p[1] = (S.r + a * cos(v)) * sin(u);
    p[2] = a * sin(v);
  }
  double x[3];
  for (int r = 0; r < 3; ++r) x[r] = S.R[3 * r] * p[0] + S.R[3 * r + 1] * p[1] + S.R[3 * r + 2] * p[2] + S.c[r];
  out[i] = make_float4((float)x[0], (float)x[1], (float)x[2], 0.0f);
}

// Scene::createFluidObject (Scene.cpp:597-646), particle k of the iy, ix, iz
// loops: x = jitter + ix * spacing in float, then x + (drand48() - 0.5) *
// jitter + offset in double, stored as float; the reference's drand48() is
// the macro rand() / RAND_MAX (global.h:12), integer division: 0.
__global__ void k_fluid_block(const FluidBlock B, uint64_t n, float4* __restrict__ out) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int iz = (int)(k % (uint64_t)B.nz);
  const uint64_t q = k / (uint64_t)B.nz;
  const int ix = (int)(q % (uint64_t)B.nx);
  const int iy = (int)(q / (uint64_t)B.nx);
  const double shift = __dmul_rn(-0.5, (double)B.jitter);
  const float f[3] = {fa(B.jitter, fm((float)ix, B.spacing)), fa(B.jitter, fm((float)iy, B.spacing)),
                      fa(B.jitter, fm((float)iz, B.spacing))};
  float p[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) p[a] = __double2float_rn(__dadd_rn(__dadd_rn((double)f[a], shift), B.off[a]));
  out[k] = make_float4(p[0], p[1], p[2], 0.0f);
}

struct BoxWalls {
  int nx, ny, nz, layers;
  float spacing, distance;
  float delta[3];
  float start[3];
  uint64_t s1, s2, s3;  // particles of the xz, xy and yz plane pairs
};

// Scene::createBoxBoundaryFrozenParticlesMultiLayers (Scene.cpp:1045-1212;
// one layer: createBoxBoundaryFrozenParticles, 890-1043): particle k of the
// reference's three loop nests, ground/ceiling, back/front, left/right,
// each nest emitting the pair's two particles in turn. A particle not
// strictly above the z-index origin in every coordinate sets *bad (where
// the reference aborts).
__global__ void k_box_walls(const BoxWalls W, float4* __restrict__ pos, float4* __restrict__ nrm,
                            int* __restrict__ bad) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= W.s1 + W.s2 + W.s3) return;
  const int g = (int)(k & 1u);  // first or second wall of the pair
  const uint64_t t = k >> 1;
  const int L = W.layers;
  const float sp = W.spacing;
  const float bx = fa(W.start[0], W.distance), by = fa(W.start[1], W.distance), bz = fa(W.start[2], W.distance);
  float p[3], n[3] = {0.0f, 0.0f, 0.0f};
  if (k < W.s1) {
    const int y = (int)(t % L);
    const uint64_t r = t / L;
    const int z = (int)(r % (uint64_t)(W.nz + 2));
    const int x = (int)(r / (uint64_t)(W.nz + 2));
    p[0] = fa(bx, fm((float)x, sp));
    p[1] = g == 0 ? fs(by, fm((float)y, sp)) : fa(fa(by, W.delta[1]), fm((float)y, sp));
    p[2] = fa(bz, fm((float)z, sp));
    n[1] = g == 0 ? 1.0f : -1.0f;
  } else if (k < W.s1 + W.s2) {
    const uint64_t u = t - (W.s1 >> 1);
    const int zl = (int)(u % L);
    const uint64_t r = u / L;
    const int y = 1 + (int)(r % (uint64_t)W.ny);
    const int x = (int)(r / (uint64_t)W.ny);
    p[0] = fa(bx, fm((float)x, sp));
    p[1] = fa(by, fm((float)y, sp));
    p[2] = g == 0 ? fs(bz, fm((float)zl, sp)) : fa(fa(bz, W.delta[2]), fm((float)zl, sp));
    n[2] = g == 0 ? 1.0f : -1.0f;
  } else {
    const uint64_t u = t - ((W.s1 + W.s2) >> 1);
    const int xl = (int)(u % L);
    const uint64_t r = u / L;
    const int z = 1 + (int)(r % (uint64_t)W.nz);
    const int y = 1 + (int)(r / (uint64_t)W.nz);
    p[0] = g == 0 ? fs(bx, fm((float)xl, sp)) : fa(fa(bx, W.delta[0]), fm((float)xl, sp));
    p[1] = fa(by, fm((float)y, sp));
    p[2] = fa(bz, fm((float)z, sp));
    n[0] = g == 0 ? 1.0f : -1.0f;
  }
  pos[k] = make_float4(p[0], p[1], p[2], 0.0f);
  nrm[k] = make_float4(n[0], n[1], n[2], 0.0f);
  if (!(fs(p[0], W.start[0]) > 0.0f && fs(p[1], W.start[1]) > 0.0f && fs(p[2], W.start[2]) > 0.0f)) *bad = 1;
}

// runs `launch` on a fresh stream of `device`, with its outputs in device
// buffers copied to the host arrays
upf_status generate(const char* who, int device, uint64_t n, float* pos4, float* nrm4,
                    cudaError_t (*launch)(const void* args, uint64_t n, float4* pos, float4* nrm, int* bad,
                                          cudaStream_t st),
                    const void* args, bool* bad_out) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("%s: no CUDA device", who);
    return UPF_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    set_error("%s: bad device %d", who, device);
    return UPF_ERR_INVALID_ARG;
  }
  cudaError_t e = cudaSetDevice(device);
  cudaStream_t st = nullptr;
  float4 *d_pos = nullptr, *d_nrm = nullptr;
  int* d_bad = nullptr;
  int bad = 0;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = dmalloc(&d_pos, n);
  if (e == cudaSuccess && nrm4) e = dmalloc(&d_nrm, n);
  if (e == cudaSuccess) e = dmalloc(&d_bad, 1);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0, sizeof(int), st);
  if (e == cudaSuccess) e = launch(args, n, d_pos, d_nrm, d_bad, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(pos4, d_pos, sizeof(float4) * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && nrm4) e = cudaMemcpyAsync(nrm4, d_nrm, sizeof(float4) * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (st) cudaStreamSynchronize(st);
  cudaFree(d_pos);
  cudaFree(d_nrm);
  cudaFree(d_bad);
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    if (e != cudaErrorMemoryAllocation || !std::strstr(upf_last_error(), "injected"))
      set_error("%s: %s", who, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? UPF_ERR_ALLOC : UPF_ERR_CUDA;
  }
  if (bad_out) *bad_out = bad != 0;
  return UPF_OK;
}

}  // namespace
}  // namespace upf

upf_status upf_scene_fluid_block(int device, const float box_min[3], const float box_max[3], float spacing,
                                 float jitter, const float offset[3], float* pos4, uint32_t capacity,
                                 uint32_t* n_out) {
  const char* who = "upf_scene_fluid_block";
  if (!box_min || !box_max || !offset || !n_out || !(spacing > 0.0f) || (capacity > 0 && !pos4)) {
    set_error("%s: bad arguments", who);
    return UPF_ERR_INVALID_ARG;
  }
  FluidBlock B{};
  int64_t num[3];
  for (int a = 0; a < 3; ++a) {
    const float q = (box_max[a] - box_min[a]) / spacing;
    if (!(q < 2147483647.0f)) {
      set_error("%s: box / spacing too large", who);
      return UPF_ERR_INVALID_ARG;
    }
    num[a] = q > 0.0f ? (int64_t)(int)q : 0;  // Vector3i(delta / Vector3f(spacing)); no particles below 1
    B.off[a] = (double)offset[a];
  }
  B.nx = (int)num[0], B.ny = (int)num[1], B.nz = (int)num[2];
  B.spacing = spacing;
  B.jitter = jitter;
  const uint64_t n = (uint64_t)num[0] * (uint64_t)num[1] * (uint64_t)num[2];
  if (n > 0xffffffffu) {
    set_error("%s: %llu particles exceed 2^32 - 1", who, (unsigned long long)n);
    return UPF_ERR_INVALID_ARG;
  }
  *n_out = (uint32_t)n;
  if (!pos4 || n == 0) return UPF_OK;
  if (n > capacity) {
    set_error("%s: the block holds %llu particles, capacity is %u", who, (unsigned long long)n, capacity);
    return UPF_ERR_INVALID_ARG;
  }
  auto launch = [](const void* a, uint64_t n, float4* pos, float4*, int*, cudaStream_t st) {
    k_fluid_block<<<(uint32_t)((n + 255) / 256), 256, 0, st>>>(*static_cast<const FluidBlock*>(a), n, pos);
    return cudaGetLastError();
  };
  return generate(who, device, n, pos4, nullptr, launch, &B, nullptr);
}

upf_status upf_scene_box_boundary(int device, const float container_min[3], const float container_max[3],
                                  const float zindex_start[3], float spacing, float support_radius,
                                  float distance_frozen_to_boundary, int32_t layers, float* pos4, float* normal4,
                                  uint32_t capacity, uint32_t* n_out) {
  const char* who = "upf_scene_box_boundary";
  if (!container_min || !container_max || !zindex_start || !n_out || !(spacing > 0.0f) || layers < 1 ||
      layers > 8 || (capacity > 0 && (!pos4 || !normal4))) {
    set_error("%s: bad arguments (layers 1..8)", who);
    return UPF_ERR_INVALID_ARG;
  }
  BoxWalls W{};
  int64_t num[3];
  for (int a = 0; a < 3; ++a) {
    const float mn = container_min[a] - distance_frozen_to_boundary;
    const float mx = container_max[a] + distance_frozen_to_boundary;
    W.delta[a] = mx - mn;
    const float q = W.delta[a] / spacing;
    if (!(q < 2147483647.0f) || !(q >= 0.0f)) {
      set_error("%s: container / spacing out of range", who);
      return UPF_ERR_INVALID_ARG;
    }
    num[a] = (int64_t)(int)q;
    W.start[a] = zindex_start[a];
  }
  W.nx = (int)num[0], W.ny = (int)num[1], W.nz = (int)num[2], W.layers = layers;
  W.spacing = spacing;
  W.distance = support_radius - distance_frozen_to_boundary;
  const uint64_t L2 = 2 * (uint64_t)layers;
  W.s1 = L2 * (uint64_t)(num[0] + 2) * (uint64_t)(num[2] + 2);
  W.s2 = L2 * (uint64_t)(num[0] + 2) * (uint64_t)num[1];
  W.s3 = L2 * (uint64_t)num[1] * (uint64_t)num[2];
  const uint64_t n = W.s1 + W.s2 + W.s3;
  if (n > 0xffffffffu) {
    set_error("%s: %llu particles exceed 2^32 - 1", who, (unsigned long long)n);
    return UPF_ERR_INVALID_ARG;
  }
  *n_out = (uint32_t)n;
  if (!pos4 || n == 0) return UPF_OK;
  if (n > capacity) {
    set_error("%s: the walls hold %llu particles, capacity is %u", who, (unsigned long long)n, capacity);
    return UPF_ERR_INVALID_ARG;
  }
  auto launch = [](const void* a, uint64_t n, float4* pos, float4* nrm, int* bad, cudaStream_t st) {
    k_box_walls<<<(uint32_t)((n + 255) / 256), 256, 0, st>>>(*static_cast<const BoxWalls*>(a), pos, nrm, bad);
    return cudaGetLastError();
  };
  bool bad = false;
  upf_status s = generate(who, device, n, pos4, normal4, launch, &W, &bad);
  if (s == UPF_OK && bad) {
    set_error("%s: a wall particle lies at or below the z-index origin (the reference aborts here); move "
              "zindex_start below the container by more than support_radius", who);
    return UPF_ERR_INVALID_ARG;
  }
  return s;
}

upf_status upf_scene_rigid_surface(int device, int32_t shape, float radius, uint32_t n_target, const float rot9[9],
                                   const float center[3], float* pos4, uint32_t capacity, uint32_t* n_out) {
  const char* who = "upf_scene_rigid_surface";
  if (shape < 0 || shape > 2 || !(radius > 0.0f) || n_target == 0 || !rot9 || !center || !n_out ||
      (capacity > 0 && !pos4)) {
    set_error("%s: bad arguments (shape 0 sphere, 1 cube, 2 torus; radius > 0; n_target > 0)", who);
    return UPF_ERR_INVALID_ARG;
  }
  RigidSurface S{};
  S.shape = shape;
  S.r = (double)radius;
  uint64_t n = n_target;
  if (shape == 1) {
    S.k = (uint32_t)std::max(2.0, std::nearbyint(std::sqrt((double)n_target / 6.0)));
    n = 6ull * S.k * S.k;
  } else if (shape == 2) {
    // nu around the major circle, nv around the minor one, near-square cells
    S.nu = (uint32_t)std::max(8.0, std::nearbyint(std::sqrt((double)n_target * 3.0)));
    S.nv = (uint32_t)std::max(4.0, std::nearbyint((double)n_target / (double)S.nu));
    n = (uint64_t)S.nu * S.nv;
  }
  if (n > 0xffffffffu) {
    set_error("%s: too many points", who);
    return UPF_ERR_INVALID_ARG;
  }
  S.n = (uint32_t)n;
  for (int k = 0; k < 9; ++k) S.R[k] = (double)rot9[k];
  for (int a = 0; a < 3; ++a) S.c[a] = (double)center[a];
  *n_out = S.n;
  if (!pos4) return UPF_OK;
  if (n > capacity) {
    set_error("%s: the surface holds %llu particles, capacity is %u", who, (unsigned long long)n, capacity);
    return UPF_ERR_INVALID_ARG;
  }
  auto launch = [](const void* a, uint64_t n, float4* pos, float4*, int*, cudaStream_t st) {
    k_rigid_surface<<<(uint32_t)((n + 255) / 256), 256, 0, st>>>(*static_cast<const RigidSurface*>(a), pos);
    return cudaGetLastError();
  };
  return generate(who, device, n, pos4, nullptr, launch, &S, nullptr);
}
