// kernels.cu -- device kernels of the tracer and their launchers.
#include <atomic>

#include "kernels.h"

namespace pt {

__global__ void k_gather_tri_bvh(const float4* __restrict__ primitives, const uint32_t* __restrict__ tri_idx,
                                 float4* __restrict__ tri_bvh, uint32_t triangle_offset, uint32_t index_offset,
                                 uint32_t count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t slot = index_offset + i;
  const uint32_t tri = tri_idx[slot];
  const float4* p = primitives + (size_t)(triangle_offset + tri) * 3;
  const float4 a = p[0], b = p[1], c = p[2];
  float4* o = tri_bvh + (size_t)slot * 3;
  o[0] = make_float4(a.x, a.y, a.z, __uint_as_float(tri));
  o[1] = make_float4(b.x - a.x, b.y - a.y, b.z - a.z, 0.0f);
  o[2] = make_float4(c.x - a.x, c.y - a.y, c.z - a.z, 0.0f);
}

cudaError_t launch_gather_tri_bvh(const float4* primitives, const uint32_t* triangle_indices, float4* tri_bvh,
                                  uint32_t triangle_offset, uint32_t index_offset, uint32_t count,
                                  cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  k_gather_tri_bvh<<<(count + 255) / 256, 256, 0, st>>>(primitives, triangle_indices, tri_bvh, triangle_offset,
                                                         index_offset, count);
  return cudaGetLastError();
}

constexpr int kMegaBlock = 128;

// Sum of WorkCount over a warp, added to the global tallies by lane 0.
__device__ __forceinline__ void flush_counts(const WorkCount& w, unsigned long long* g) {
  // Every lane of the warp reaches this point; reconverge before the shuffles.
  __syncwarp();
  unsigned long long v[8] = {w.rays, w.tlas_interior, w.blas_entries, w.blas_interior, w.tri_tests, w.hits, w.nee,
                             w.cdf_reads};
  for (int i = 0; i < 8; ++i) {
    unsigned long long x = v[i];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    v[i] = x;
  }
  if ((threadIdx.x & 31) == 0)
    for (int i = 0; i < 8; ++i) atomicAdd(g + i, v[i]);
}

template <bool COUNT, int MINB, int MODE>
__global__ void __launch_bounds__(kMegaBlock, MINB) k_render_mega(DevScene S, TraceCfg tc, PathCfg pc, FrameCfg fc,
                                                                  float4* __restrict__ image, Counters* ctr,
                                                                  unsigned long long* work) {
  extern __shared__ uint32_t smem[];
  const uint32_t tid = threadIdx.x;
  uint32_t* stk = smem + tid;
  const uint32_t stride = blockDim.x;
  const uint32_t tiles_x = (fc.W + 15u) / 16u;
  const uint32_t tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
  const uint32_t x = tx * 16u + (tid & 15u), y = ty * 8u + (tid >> 4);
  WorkCount wc{};
  if (x < fc.W && y < fc.H) {
    const uint32_t pix = y * fc.W + x;
    float4 px = fc.acc * pc.spp > 0 ? image[pix] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (uint32_t s = 0; s < pc.spp; ++s) {
      const uint32_t acc = fc.acc * pc.spp + s;
      PathState ps;
      path_begin(ps, pc, fc.ivp, fc.eye, x, y, fc.W, fc.H, acc);
      ShadowReq rq;
      rq.active = false;
      bool shadow = false;
      // One trace call site for path segments and shadow rays alike.
      while ((ps.flags & kAlive) || shadow) {
        Hit h;
        trace_closest<COUNT>(S, shadow ? rq.o : ps.o, shadow ? rq.d : ps.d, h, stk, stride, tc, ctr, &wc,
                             shadow ? rq.limit : 3.0e38f);
        if (shadow) {
          path_on_shadow<MODE>(ps, rq, h.t);
          shadow = false;
          continue;
        }
        if (COUNT && h.t < 1e30f) wc.hits++;
        path_on_hit<MODE>(S, pc, ps, h, rq);
        if (rq.active) {
          shadow = true;
          if (COUNT) wc.nee++;
        }
      }
      px = accumulate(px, ps.color, acc);
    }
    image[pix] = px;
  }
  if (COUNT) flush_counts(wc, work);
}

static size_t stack_smem_bytes(const TraceCfg& tc, int block) {
  return (size_t)trace_smem_words(tc) * block * 4;
}

// Raises the dynamic shared memory limit of a traversal kernel once per device:
// stacks of at most 2 x 64 entries plus the cold words, 128 threads.
constexpr int kTraceSmemLimit = (2 * 64 + kColdWords) * 128 * 4;  // 128-thread blocks

template <typename K>
static cudaError_t stack_limit(K kernel, std::atomic<uint64_t>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = dev < 64 ? (uint64_t)1 << dev : 0;
  if (bit && (done.load() & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTraceSmemLimit);
  if (e == cudaSuccess && bit) done.fetch_or(bit);
  return e;
}

template <bool COUNT, int MINB, int MODE>
static cudaError_t launch_mega_variant(const DevScene& S, const TraceCfg& tc, const PathCfg& pc, const FrameCfg& fc,
                                       float4* image, Counters* ctr, unsigned long long* work, cudaStream_t st) {
  static std::atomic<uint64_t> done{0};
  if (cudaError_t e = stack_limit(k_render_mega<COUNT, MINB, MODE>, done)) return e;
  const uint32_t tiles = ((fc.W + 15u) / 16u) * ((fc.H + 7u) / 8u);
  if (tiles == 0) return cudaSuccess;
  k_render_mega<COUNT, MINB, MODE><<<tiles, kMegaBlock, stack_smem_bytes(tc, kMegaBlock), st>>>(S, tc, pc, fc, image,
                                                                                               ctr, work);
  return cudaGetLastError();
}

template <int MODE>
static cudaError_t launch_mega_mode(const DevScene& S, const TraceCfg& tc, const PathCfg& pc, const FrameCfg& fc,
                                    float4* image, Counters* ctr, unsigned long long* work, uint32_t min_blocks,
                                    cudaStream_t st) {
  if (work) return launch_mega_variant<true, 1, MODE>(S, tc, pc, fc, image, ctr, work, st);
  switch (min_blocks) {
    case 4: return launch_mega_variant<false, 4, MODE>(S, tc, pc, fc, image, ctr, nullptr, st);
    case 8: return launch_mega_variant<false, 8, MODE>(S, tc, pc, fc, image, ctr, nullptr, st);
    default: return launch_mega_variant<false, 6, MODE>(S, tc, pc, fc, image, ctr, nullptr, st);
  }
}

cudaError_t launch_render_mega(const DevScene& S, const TraceCfg& tc, const PathCfg& pc, const FrameCfg& fc,
                               float4* image, Counters* ctr, unsigned long long* work, uint32_t min_blocks,
                               cudaStream_t st) {
  switch (pc.nee_mode) {
    case 0: return launch_mega_mode<0>(S, tc, pc, fc, image, ctr, work, min_blocks, st);
    case 1: return launch_mega_mode<1>(S, tc, pc, fc, image, ctr, work, min_blocks, st);
    default: return launch_mega_mode<2>(S, tc, pc, fc, image, ctr, work, min_blocks, st);
  }
}

constexpr int kTraceBlock = 128;

__global__ void __launch_bounds__(kTraceBlock) k_trace_rays(DevScene S, TraceCfg tc, const float* __restrict__ rays,
                                                            uint32_t n, Hit* __restrict__ out, Counters* ctr) {
  extern __shared__ uint32_t smem[];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* r = rays + (size_t)i * 6;
  Hit h;
  trace_closest(S, v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5]), h, smem + threadIdx.x, blockDim.x, tc, ctr);
  out[i] = h;
}

cudaError_t launch_trace_rays(const DevScene& S, const TraceCfg& tc, const float* rays, uint32_t n, Hit* out,
                              Counters* ctr, cudaStream_t st) {
  static std::atomic<uint64_t> done{0};
  if (cudaError_t e = stack_limit(k_trace_rays, done)) return e;
  if (n == 0) return cudaSuccess;
  k_trace_rays<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, stack_smem_bytes(tc, kTraceBlock), st>>>(
      S, tc, rays, n, out, ctr);
  return cudaGetLastError();
}

}  // namespace pt
