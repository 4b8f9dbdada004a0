// prep.cu -- row preparation kernels (HBM-bound, one pass over the input).
//
// Replaces computeL2Norm / kernelL2Norm (cuRPLSH src/internal/norm.cu:15-202)
// and adds the quantised operand copies the tensor-core pass reads:
//   * squared L2 norm in FP32 (fixed reduction order: per-lane sequential over
//     128-bit loads, then a butterfly), cached at add() time for the database;
//   * BF16 hi = bf16(x), lo = bf16(x - hi) (the 3 x BF16 exact form);
//   * FP8-E4M3 x / s with a per-row FP32 scale s = max|x| / 448.
// One warp per row; 128-bit vector loads when the row allows them.  Unlike the
// reference kernel there is no shape specialisation, so any d and any row count
// is handled without partial-warp shuffles or out-of-bounds rows.
#include <cuda_fp8.h>

#include <cstring>

#include "common.cuh"
#include "fused_knn.h"

namespace curplsh_b200 {

namespace {

constexpr int kPrepWarps = 8;
constexpr float kE4M3Max = 448.f;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ uint8_t to_e4m3(float v) {
  return (uint8_t)__nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
}

// Value of augmented column c (0..kAugCols-1) of a row with squared norm s:
// database rows [n1 n2 n3 1 1 1], query rows [1 1 1 m1 m2 m3], where the three
// BF16 terms sum to s (successive rounding of the remainders).
__device__ __forceinline__ float aug_value(int aug, int c, float s) {
  const float t1 = __bfloat162float(__float2bfloat16_rn(s));
  const float r1 = s - t1;
  const float t2 = __bfloat162float(__float2bfloat16_rn(r1));
  const float t3 = r1 - t2;
  const float terms[3] = {t1, t2, t3};
  if (aug == kAugDatabase) return c < 3 ? terms[c] : 1.f;
  return c < 3 ? 1.f : terms[c - 3];
}

// One warp prepares row r (< the padded row count) of one matrix.
__device__ __forceinline__ void prep_row(const float* __restrict__ x, long long ldx, long long r, int nrows, int d,
                                         float* __restrict__ norms, float pad_norm, __nv_bfloat16* __restrict__ hi,
                                         __nv_bfloat16* __restrict__ lo, long long ld16, uint8_t* __restrict__ f8,
                                         float* __restrict__ scale, long long ld8, int vec4, int aug,
                                         uint32_t* __restrict__ lo_nonzero = nullptr, float fixed_scale = 0.f) {
  const int lane = threadIdx.x & 31;
  if (r >= nrows) {
    if (norms && lane == 0) norms[r] = pad_norm;
    if (scale && lane == 0) scale[r] = 0.f;
    if (hi)
      for (long long i = lane; i < ld16; i += 32) hi[r * ld16 + i] = __float2bfloat16_rn(0.f);
    if (lo)
      for (long long i = lane; i < ld16; i += 32) lo[r * ld16 + i] = __float2bfloat16_rn(0.f);
    if (f8)
      for (long long i = lane; i < ld8; i += 32) f8[r * ld8 + i] = 0;
    return;
  }
  const float* row = x + r * ldx;
  float s = 0.f, m = 0.f;
  if (vec4) {
    const float4* row4 = reinterpret_cast<const float4*>(row);
    for (int i = lane; i < d / 4; i += 32) {
      const float4 v = __ldg(row4 + i);
      s = fmaf(v.x, v.x, s);
      s = fmaf(v.y, v.y, s);
      s = fmaf(v.z, v.z, s);
      s = fmaf(v.w, v.w, s);
      m = fmaxf(m, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
    }
  } else {
    for (int i = lane; i < d; i += 32) {
      const float v = __ldg(row + i);
      s = fmaf(v, v, s);
      m = fmaxf(m, fabsf(v));
    }
  }
  s = warp_sum(s);
  if (norms && lane == 0) norms[r] = s;
  if (!hi && !lo && !f8) return;
  // query rows of the augmented forms are stored as -2q (exact in BF16)
  const float hsc = aug == kAugQuery ? -2.f : 1.f;
  bool lo_any = false;  // some element is not exactly a BF16 value
  float inv = 1.f;
  if (f8) {
    m = warp_max(m);
    // an all-zero row gets scale 0 (its codes are 0 whatever the scale); a
    // zero query row with a norm tail gets 1, so its tail 1/s_q is finite
    float sc = fixed_scale > 0.f ? fixed_scale : m / kE4M3Max;
    const bool q_tail = aug == kAugF8Query;
    if (q_tail && !(sc > 0.f)) sc = 1.f;
    inv = sc > 0.f ? 1.f / sc : 0.f;
    if (scale && lane == 0) scale[r] = (m > 0.f || q_tail) ? sc : 0.f;
  }
  if (vec4) {
    const float4* row4 = reinterpret_cast<const float4*>(row);
    for (int i = lane; i < d / 4; i += 32) {
      const float4 v = __ldg(row4 + i);
      if (hi) {
        const __nv_bfloat16 h0 = __float2bfloat16_rn(v.x), h1 = __float2bfloat16_rn(v.y);
        const __nv_bfloat16 h2 = __float2bfloat16_rn(v.z), h3 = __float2bfloat16_rn(v.w);
        __nv_bfloat162 a, b;
        a.x = __float2bfloat16_rn(hsc * __bfloat162float(h0));
        a.y = __float2bfloat16_rn(hsc * __bfloat162float(h1));
        b.x = __float2bfloat16_rn(hsc * __bfloat162float(h2));
        b.y = __float2bfloat16_rn(hsc * __bfloat162float(h3));
        uint2 pk;
        pk.x = *reinterpret_cast<uint32_t*>(&a);
        pk.y = *reinterpret_cast<uint32_t*>(&b);
        *reinterpret_cast<uint2*>(hi + r * ld16 + 4 * i) = pk;
        if (lo) {
          __nv_bfloat162 c, e;
          c.x = __float2bfloat16_rn(hsc * (v.x - __bfloat162float(h0)));
          c.y = __float2bfloat16_rn(hsc * (v.y - __bfloat162float(h1)));
          e.x = __float2bfloat16_rn(hsc * (v.z - __bfloat162float(h2)));
          e.y = __float2bfloat16_rn(hsc * (v.w - __bfloat162float(h3)));
          uint2 pl;
          pl.x = *reinterpret_cast<uint32_t*>(&c);
          pl.y = *reinterpret_cast<uint32_t*>(&e);
          *reinterpret_cast<uint2*>(lo + r * ld16 + 4 * i) = pl;
          lo_any |= ((pl.x | pl.y) & 0x7FFF7FFFu) != 0u;  // ignore -0
        }
      }
      if (f8) {
        const uint32_t q = (uint32_t)to_e4m3(v.x * inv) | ((uint32_t)to_e4m3(v.y * inv) << 8) |
                           ((uint32_t)to_e4m3(v.z * inv) << 16) | ((uint32_t)to_e4m3(v.w * inv) << 24);
        *reinterpret_cast<uint32_t*>(f8 + r * ld8 + 4 * i) = q;
      }
    }
    if (hi)
      for (long long i = d + lane; i < ld16; i += 32) {
        const int c = (int)(i - d);
        hi[r * ld16 + i] = __float2bfloat16_rn(aug && c < kAugCols ? aug_value(aug, c, s) : 0.f);
        if (lo) lo[r * ld16 + i] = __float2bfloat16_rn(0.f);
      }
    if (f8)
      for (long long i = d + lane; i < ld8; i += 32) f8[r * ld8 + i] = 0;
  } else {
    if (hi)
      for (long long i = lane; i < ld16; i += 32) {
        if (i < d) {
          const float v = row[i];
          const __nv_bfloat16 h = __float2bfloat16_rn(v);
          hi[r * ld16 + i] = __float2bfloat16_rn(hsc * __bfloat162float(h));
          if (lo) {
            lo[r * ld16 + i] = __float2bfloat16_rn(hsc * (v - __bfloat162float(h)));
            lo_any |= v != __bfloat162float(h);
          }
        } else {
          const int c = (int)(i - d);
          hi[r * ld16 + i] = __float2bfloat16_rn(aug && c < kAugCols ? aug_value(aug, c, s) : 0.f);
          if (lo) lo[r * ld16 + i] = __float2bfloat16_rn(0.f);
        }
      }
    if (f8)
      for (long long i = lane; i < ld8; i += 32) {
        const float v = i < d ? row[i] : 0.f;
        f8[r * ld8 + i] = to_e4m3(v * inv);
      }
  }
  if (f8 && (aug == kAugF8Query || aug == kAugF8Database)) {
    // the BF16 norm tail at byte t8 (a 32-byte K step of the last 128-byte
    // chunk): a_h b_h + a_h b_l + a_l b_h = a b to ~2^-16 relative
    const long long t8 = fp8_tail_offset(d, ld8);
    if (t8 > 0) {
      __syncwarp();  // after the zero fill above, which covers these bytes
      float v = 0.f;
      if (aug == kAugF8Query)
        v = inv;  // 1 / s_q
      else if (fixed_scale > 0.f)
        v = -0.5f * s / fixed_scale;  // -||x||^2 / (2 s)
      const float vh = __bfloat162float(__float2bfloat16_rn(v));
      const float vl = v - vh;  // exact
      float e = 0.f;
      if (aug == kAugF8Query)
        e = lane < 2 ? vh : (lane == 2 ? vl : 0.f);
      else
        e = lane == 1 ? vl : (lane == 0 || lane == 2 ? vh : 0.f);
      if (lane < 16) reinterpret_cast<__nv_bfloat16*>(f8 + r * ld8 + t8)[lane] = __float2bfloat16_rn(e);
    }
  }
  if (lo_nonzero && __any_sync(0xffffffffu, lo_any) && lane == 0) atomicOr(lo_nonzero, 1u);
}

__global__ void __launch_bounds__(kPrepWarps * 32) prep_rows_kernel(
    const float* __restrict__ x, long long ldx, int nrows, long long nrows_pad, int d, float* __restrict__ norms,
    float pad_norm, __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, long long ld16,
    uint8_t* __restrict__ f8, float* __restrict__ scale, long long ld8, int vec4, int aug,
    uint32_t* __restrict__ lo_nonzero, float fixed_scale) {
  const long long r = (long long)blockIdx.x * kPrepWarps + (threadIdx.x >> 5);
  if (r >= nrows_pad) return;
  prep_row(x, ldx, r, nrows, d, norms, pad_norm, hi, lo, ld16, f8, scale, ld8, vec4, aug, lo_nonzero, fixed_scale);
}

// Smallest and largest positive value of s[0, n) as order bits (positive
// floats order as unsigned integers): out[0] = min (start 0xFFFFFFFF),
// out[1] = max (start 0).
__global__ void positive_range_kernel(const float* __restrict__ s, long long n, uint32_t* __restrict__ out) {
  uint32_t lo = 0xFFFFFFFFu, hi = 0u;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float v = s[i];
    if (v > 0.f) {
      lo = min(lo, __float_as_uint(v));
      hi = max(hi, __float_as_uint(v));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&out[0], lo);
    atomicMax(&out[1], hi);
  }
}

struct PrepSegmentArgs {
  PrepSegment seg[kPrepMaxSegments];
  int vec4[kPrepMaxSegments];
  int num, d, aug;
  float pad_norm;
  long long ld16, ld8;
};

// Several matrices (segments) of one dimension in one launch; each CTA
// prepares kPrepWarps consecutive rows of one segment.
__global__ void __launch_bounds__(kPrepWarps * 32) prep_segments_kernel(const __grid_constant__ PrepSegmentArgs a) {
  int lo_i = 0, hi_i = a.num - 1;  // last segment with block_begin <= blockIdx.x
  while (lo_i < hi_i) {
    const int mid = (lo_i + hi_i + 1) >> 1;
    if (a.seg[mid].block_begin <= (long long)blockIdx.x)
      lo_i = mid;
    else
      hi_i = mid - 1;
  }
  const PrepSegment& g = a.seg[lo_i];
  const long long r = ((long long)blockIdx.x - g.block_begin) * kPrepWarps + (threadIdx.x >> 5);
  if (r >= g.rows) return;
  prep_row(g.x, a.d, r, g.nrows, a.d, g.norms, a.pad_norm, g.hi, g.lo, a.ld16, g.f8, g.scale, a.ld8, a.vec4[lo_i],
           a.aug);
}

__global__ void __launch_bounds__(kPrepWarps * 32)
    l2_norms_kernel(const float* __restrict__ x, long long n, int d, float* __restrict__ norms, int squared,
                    int vec4) {
  const long long r = (long long)blockIdx.x * kPrepWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const float* row = x + r * (long long)d;
  float s = 0.f;
  if (vec4) {
    const float4* row4 = reinterpret_cast<const float4*>(row);
    for (int i = lane; i < d / 4; i += 32) {
      const float4 v = __ldg(row4 + i);
      s = fmaf(v.x, v.x, s);
      s = fmaf(v.y, v.y, s);
      s = fmaf(v.z, v.z, s);
      s = fmaf(v.w, v.w, s);
    }
  } else {
    for (int i = lane; i < d; i += 32) {
      const float v = __ldg(row + i);
      s = fmaf(v, v, s);
    }
  }
  s = warp_sum(s);
  if (lane == 0) norms[r] = squared ? s : sqrtf(s);
}

__global__ void fill_results_kernel(int* idx, float* dist, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (idx) idx[i] = -1;
    if (dist) dist[i] = 3.402823466e38f;
  }
}

__global__ void add_count_kernel(unsigned long long* acc, const int* cnt) {
  if (*cnt) *acc += (unsigned long long)*cnt;
}

__global__ void fill_u32_if_kernel(uint32_t* p, long long n, uint32_t v, const int* cond) {
  if (*cond == 0) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

// One warp per query: the j-th smallest (1-based) of `count` floats, by a
// most-significant-digit radix select on their order bits (4 passes of 8
// bits, a 256-bin warp histogram in shared memory).
constexpr int kSelectWarps = 8;
__global__ void __launch_bounds__(kSelectWarps * 32)
    estimate_select_kernel(const float* __restrict__ minima, int count, int nq, int j, uint32_t* __restrict__ out) {
  __shared__ uint32_t hist_all[kSelectWarps][256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = blockIdx.x * kSelectWarps + warp;
  if (q >= nq) return;
  if (count < j || j < 1) {
    if (lane == 0) out[q] = kOrdInf;
    return;
  }
  uint32_t* hist = hist_all[warp];
  const float* v = minima + (size_t)q * count;
  uint32_t prefix = 0, mask = 0, rank = (uint32_t)j;
  for (int shift = 24; shift >= 0; shift -= 8) {
#pragma unroll
    for (int b = 0; b < 8; ++b) hist[lane * 8 + b] = 0u;
    __syncwarp();
    for (int i = lane; i < count; i += 32) {
      const uint32_t o = f2ord(v[i]);
      if ((o & mask) == prefix) atomicAdd(&hist[(o >> shift) & 255u], 1u);
    }
    __syncwarp();
    // the digit whose bucket holds the rank-th key: lane l sums bins 8l..8l+7
    uint32_t c[8], s = 0;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      c[b] = hist[lane * 8 + b];
      s += c[b];
    }
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const uint32_t excl = incl - s;
    const bool mine = excl < rank && rank <= incl;
    uint32_t digit = 0, before = 0;
    if (mine) {
      uint32_t acc = excl;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        if (acc < rank && rank <= acc + c[b]) {
          digit = (uint32_t)(lane * 8 + b);
          before = acc;
        }
        acc += c[b];
      }
    }
    const int src = __ffs(__ballot_sync(0xffffffffu, mine)) - 1;
    digit = __shfl_sync(0xffffffffu, digit, src);
    before = __shfl_sync(0xffffffffu, before, src);
    prefix |= digit << shift;
    mask |= 255u << shift;
    rank -= before;
    __syncwarp();
  }
  if (lane == 0) out[q] = prefix;
}

// One block per listed row: dst row i <- src row rows[i].
__global__ void gather_rows_kernel(const float* __restrict__ src, int d, const int* __restrict__ rows,
                                   float* __restrict__ dst) {
  const int i = blockIdx.x;
  const float* s = src + (size_t)rows[i] * d;
  float* t = dst + (size_t)i * d;
  for (int c = threadIdx.x; c < d; c += blockDim.x) t[c] = s[c];
}

// One block per listed row: result row rows[i] <- row i.
__global__ void scatter_results_kernel(const int* __restrict__ in_idx, const float* __restrict__ in_dist,
                                       const int* __restrict__ rows, int k, int* __restrict__ out_idx,
                                       float* __restrict__ out_dist) {
  const int i = blockIdx.x;
  const size_t o = (size_t)rows[i] * k, s = (size_t)i * k;
  for (int c = threadIdx.x; c < k; c += blockDim.x) {
    out_idx[o + c] = in_idx[s + c];
    out_dist[o + c] = in_dist[s + c];
  }
}

}  // namespace

cudaError_t launch_prep_rows(const float* x, long long ldx, int nrows, long long nrows_pad, int d, float* norms,
                             float pad_norm, __nv_bfloat16* hi, __nv_bfloat16* lo, long long ld16, uint8_t* f8,
                             float* scale, long long ld8, cudaStream_t st, int aug, uint32_t* lo_nonzero,
                             float fixed_scale) {
  if (nrows_pad <= 0) return cudaSuccess;
  const int vec4 = (d % 4 == 0) && (ldx % 4 == 0) && ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
  const long long blocks = (nrows_pad + kPrepWarps - 1) / kPrepWarps;
  prep_rows_kernel<<<(unsigned)blocks, kPrepWarps * 32, 0, st>>>(x, ldx, nrows, nrows_pad, d, norms, pad_norm, hi,
                                                                 lo, ld16, f8, scale, ld8, vec4, aug, lo_nonzero,
                                                                 fixed_scale);
  return cudaGetLastError();
}

cudaError_t launch_positive_range(const float* s, long long n, uint32_t* out, cudaStream_t st) {
  const uint32_t init[2] = {0xFFFFFFFFu, 0u};
  cudaError_t e = cudaMemcpyAsync(out, init, sizeof(init), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess || n <= 0) return e;
  long long blocks = (n + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  positive_range_kernel<<<(unsigned)blocks, 256, 0, st>>>(s, n, out);
  return cudaGetLastError();
}

cudaError_t launch_prep_segments(PrepSegment* segs, int n, int d, long long ld16, long long ld8, float pad_norm,
                                 int aug, cudaStream_t st) {
  if (n < 1 || n > kPrepMaxSegments) return cudaErrorInvalidValue;
  PrepSegmentArgs a;
  memset(&a, 0, sizeof(a));
  long long blocks = 0;
  for (int i = 0; i < n; ++i) {
    segs[i].block_begin = blocks;
    blocks += (segs[i].rows + kPrepWarps - 1) / kPrepWarps;
    a.seg[i] = segs[i];
    a.vec4[i] = (d % 4 == 0) && ((reinterpret_cast<uintptr_t>(segs[i].x) & 15) == 0);
  }
  if (blocks == 0) return cudaSuccess;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
  a.num = n;
  a.d = d;
  a.aug = aug;
  a.pad_norm = pad_norm;
  a.ld16 = ld16;
  a.ld8 = ld8;
  prep_segments_kernel<<<(unsigned)blocks, kPrepWarps * 32, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_l2_norms(const float* x, long long n, int d, float* norms, int squared, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int vec4 = (d % 4 == 0) && ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
  const long long blocks = (n + kPrepWarps - 1) / kPrepWarps;
  l2_norms_kernel<<<(unsigned)blocks, kPrepWarps * 32, 0, st>>>(x, n, d, norms, squared, vec4);
  return cudaGetLastError();
}

cudaError_t launch_fill_u32_if(uint32_t* p, long long n, uint32_t v, const int* cond, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  long long blocks = (n + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  fill_u32_if_kernel<<<(unsigned)blocks, 256, 0, st>>>(p, n, v, cond);
  return cudaGetLastError();
}

cudaError_t launch_add_count(unsigned long long* acc, const int* cnt, cudaStream_t st) {
  add_count_kernel<<<1, 1, 0, st>>>(acc, cnt);
  return cudaGetLastError();
}

cudaError_t launch_fill_results(int* idx, float* dist, long long n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  long long blocks = (n + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  fill_results_kernel<<<(unsigned)blocks, 256, 0, st>>>(idx, dist, n);
  return cudaGetLastError();
}

cudaError_t launch_gather_rows(const float* src, int d, const int* rows, int n, float* dst, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  gather_rows_kernel<<<(unsigned)n, 128, 0, st>>>(src, d, rows, dst);
  return cudaGetLastError();
}

cudaError_t launch_scatter_results(const int* in_idx, const float* in_dist, const int* rows, int n, int k,
                                   int* out_idx, float* out_dist, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  scatter_results_kernel<<<(unsigned)n, 128, 0, st>>>(in_idx, in_dist, rows, k, out_idx, out_dist);
  return cudaGetLastError();
}

cudaError_t launch_estimate_select(const float* minima, int count, int nq, int j, uint32_t* out, cudaStream_t st) {
  if (nq <= 0) return cudaSuccess;
  estimate_select_kernel<<<(unsigned)((nq + kSelectWarps - 1) / kSelectWarps), kSelectWarps * 32, 0, st>>>(
      minima, count, nq, j, out);
  return cudaGetLastError();
}

}  // namespace curplsh_b200
