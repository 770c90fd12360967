// Learned pool sizing: per-tile projection features, and a 16 -> 64 -> 64 -> 3
// multilayer perceptron (BF16 weights, FP32 accumulation) with hand-written
// inference, training and Adam kernels.
//
// The peeler's pools (fragments, ray hits, boundary vertices, triangles) are
// sized before a workspace exists.  The reference sizes them at worst case
// from the face count (warp_peel/events.py:19-33: 8N regions, 32N hits,
// vertices and triangles).  Here a cheap pass projects the mesh into a 16 x 16
// grid of screen tiles and accumulates sixteen features per tile; the
// network predicts each tile's output fragments, triangles and depth layers
// (as log(1 + count)), and the host turns the sums into capacities.  An
// extraction that overflows them reruns with the conservative sizing, so
// outputs never depend on the prediction.
//
// Parameter layout (float, `kParams` values): W1[64][16], b1[64], W2[64][64],
// b2[64], W3[3][64], b3[3].  Weights are applied as BF16 (the rounding of
// the float master copy the optimiser updates); biases and all sums are FP32.
#include <cuda_bf16.h>

#include "../../include/edp.h"
#include "edp_internal.h"

namespace edp {
namespace {

constexpr int kTileAxis = EDP_TILE_AXIS;
constexpr int kTiles = kTileAxis * kTileAxis;
constexpr int kIn = EDP_MLP_INPUTS, kHidden = EDP_MLP_HIDDEN, kOut = EDP_MLP_OUTPUTS;
constexpr int kW1 = 0, kB1 = kW1 + kHidden * kIn, kW2 = kB1 + kHidden,
              kB2 = kW2 + kHidden * kHidden, kW3 = kB2 + kHidden, kB3 = kW3 + kOut * kHidden,
              kParams = kB3 + kOut;
static_assert(kParams == EDP_MLP_PARAMS, "parameter count");
constexpr int kRaw = 12;  // raw accumulators per tile

__device__ inline float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Ordered integer image of a float (for atomic min / max of depths).
__device__ inline int float_order(float x) {
  const int i = __float_as_int(x);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ inline float order_float(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__device__ inline int tile_of(double v) {
  const double c = floor(v * kTileAxis);
  return c < 0.0 ? 0 : c > kTileAxis - 1 ? kTileAxis - 1 : int(c);
}

// raw[tile][k]: 0 triangles by centroid, 1 projected area by centroid,
// 2 box coverage (area spread over the tiles the box meets, by overlap),
// 3 front-facing, 4 back-facing, 5 perimeter, 6 tiny triangles,
// 7 triangles whose box spans tiles, 8 min depth (ordered int), 9 max depth
// (ordered int), 10 depth sum, 11 triangles reaching the near plane.
// totals[0..3]: area sum (float bits), min depth, max depth (ordered ints),
// near-plane count.
__global__ void k_tile_raw(const double *vertices, const int *faces, int nf, const double *camera,
                           const double *settings, float *raw, int *totals) {
  const double xmin = settings[0], ymin = settings[1], xmax = settings[2], ymax = settings[3];
  const bool persp = settings[4] != 0.0;
  const double near = settings[5];
  const double sx = 1.0 / (xmax - xmin), sy = 1.0 / (ymax - ymin);
  for (int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; f < nf;
       f += int64_t(gridDim.x) * blockDim.x) {
    double u[3], v[3], z[3];
    bool clipped = false;
    for (int k = 0; k < 3; ++k) {
      const double *p = vertices + 3 * int64_t(faces[3 * f + k]);
      const double cx = camera[0] * p[0] + camera[1] * p[1] + camera[2] * p[2] + camera[3];
      const double cy = camera[4] * p[0] + camera[5] * p[1] + camera[6] * p[2] + camera[7];
      const double cz = camera[8] * p[0] + camera[9] * p[1] + camera[10] * p[2] + camera[11];
      clipped |= persp && cz < near;
      const double w = persp ? 1.0 / fmax(cz, near) : 1.0;
      u[k] = (cx * w - xmin) * sx;
      v[k] = (cy * w - ymin) * sy;
      z[k] = cz;
    }
    const double cu = (u[0] + u[1] + u[2]) / 3.0, cv = (v[0] + v[1] + v[2]) / 3.0;
    const int t = tile_of(cv) * kTileAxis + tile_of(cu);
    float *r = raw + int64_t(kRaw) * t;
    if (clipped) {
      atomicAdd(&r[11], 1.0f);
      atomicAdd(&totals[3], 1);
      continue;
    }
    const double area2 = (u[1] - u[0]) * (v[2] - v[0]) - (u[2] - u[0]) * (v[1] - v[0]);
    const double area = 0.5 * fabs(area2);
    const double per = hypot(u[1] - u[0], v[1] - v[0]) + hypot(u[2] - u[1], v[2] - v[1]) +
                       hypot(u[0] - u[2], v[0] - v[2]);
    const float zmin = float(fmin(z[0], fmin(z[1], z[2])));
    const float zmax = float(fmax(z[0], fmax(z[1], z[2])));
    atomicAdd(&r[0], 1.0f);
    atomicAdd(&r[1], float(area));
    atomicAdd(&r[area2 >= 0.0 ? 3 : 4], 1.0f);
    atomicAdd(&r[5], float(per));
    if (area < 1e-4 / kTiles) atomicAdd(&r[6], 1.0f);
    atomicMin(reinterpret_cast<int *>(&r[8]), float_order(zmin));
    atomicMax(reinterpret_cast<int *>(&r[9]), float_order(zmax));
    atomicAdd(&r[10], float((z[0] + z[1] + z[2]) / 3.0));
    atomicAdd(reinterpret_cast<float *>(&totals[0]), float(area));
    atomicMin(&totals[1], float_order(zmin));
    atomicMax(&totals[2], float_order(zmax));
    // Box coverage: the area spread over the tiles the box meets, in
    // proportion to the overlap (at most 64 tiles visited per triangle; a
    // larger box adds to its centroid tile).
    const double lu = fmin(u[0], fmin(u[1], u[2])), hu = fmax(u[0], fmax(u[1], u[2]));
    const double lv = fmin(v[0], fmin(v[1], v[2])), hv = fmax(v[0], fmax(v[1], v[2]));
    const int t0 = tile_of(lu), t1 = tile_of(hu), s0 = tile_of(lv), s1 = tile_of(hv);
    const double box = fmax((hu - lu) * (hv - lv), 1e-300);
    if (t0 != t1 || s0 != s1) atomicAdd(&r[7], 1.0f);
    if ((t1 - t0 + 1) * (s1 - s0 + 1) > 64) {
      atomicAdd(&r[2], float(area));
      continue;
    }
    for (int b = s0; b <= s1; ++b)
      for (int a = t0; a <= t1; ++a) {
        const double ou = fmin(hu, double(a + 1) / kTileAxis) - fmax(lu, double(a) / kTileAxis);
        const double ov = fmin(hv, double(b + 1) / kTileAxis) - fmax(lv, double(b) / kTileAxis);
        if (ou > 0.0 && ov > 0.0)
          atomicAdd(&raw[int64_t(kRaw) * (b * kTileAxis + a) + 2], float(area * ou * ov / box));
      }
  }
}

__global__ void k_tile_raw_clear(float *raw, int *totals) {
  for (int i = threadIdx.x; i < kTiles * kRaw; i += blockDim.x) {
    const int k = i % kRaw;
    raw[i] = 0.0f;
    if (k == 8) reinterpret_cast<int *>(raw)[i] = float_order(3.0e38f);
    if (k == 9) reinterpret_cast<int *>(raw)[i] = float_order(-3.0e38f);
  }
  if (threadIdx.x == 0) {
    totals[0] = 0;
    totals[1] = float_order(3.0e38f);
    totals[2] = float_order(-3.0e38f);
    totals[3] = 0;
  }
}

// The sixteen features of each tile (one thread per tile).  Counts are taken
// per 4,096 faces of the mesh and lengths per sqrt(faces / 4,096), so that a
// mesh ten times finer over the same shapes gives about the same features
// (the network trained on 4K-64K faces then sizes larger meshes too).
__global__ void k_tile_finish(const float *raw, const int *totals, int nf, float *features) {
  const int t = threadIdx.x + blockIdx.x * blockDim.x;
  if (t >= kTiles) return;
  const float *r = raw + int64_t(kRaw) * t;
  const float tile_area = 1.0f / kTiles, tile_side = 1.0f / kTileAxis;
  const float gmin = order_float(totals[1]), gmax = order_float(totals[2]);
  const float span = gmax > gmin ? gmax - gmin : 1.0f;
  const float count = r[0];
  const float per = 4096.0f / float(nf > 0 ? nf : 1);  // counts per 4,096 faces
  const float len = sqrtf(per);
  const float zlo = count > 0.0f ? (order_float(__float_as_int(r[8])) - gmin) / span : 1.0f;
  const float zhi = count > 0.0f ? (order_float(__float_as_int(r[9])) - gmin) / span : 0.0f;
  const float zmean = count > 0.0f ? (r[10] / count - gmin) / span : 0.5f;
  float *out = features + int64_t(kIn) * t;
  out[0] = log1pf(count * per);
  out[1] = log1pf(r[1] / tile_area);
  out[2] = log1pf(r[2] / tile_area);
  out[3] = log1pf(r[3] * per);
  out[4] = log1pf(r[4] * per);
  out[5] = log1pf(r[5] / tile_side * len);
  out[6] = log1pf(r[6] * per);
  out[7] = log1pf(r[7] * per);
  out[8] = zlo;
  out[9] = zhi;
  out[10] = zmean;
  out[11] = log1pf(r[11] * per);
  out[12] = count > 0.0f ? r[3] / count : 0.5f;  // front-facing share
  out[13] = log1pf(__int_as_float(totals[0]));
  out[14] = (float(t % kTileAxis) + 0.5f) * tile_side;
  out[15] = (float(t / kTileAxis) + 0.5f) * tile_side;
}

// ---------------------------------------------------------------- inference
// One warp per 16 rows: layers 1 and 2 on the tensor cores (mma.sync
// m16n8k16, BF16 operands, FP32 accumulators), layer 3 (64 -> 3) on the FP32
// pipe.  The warp's activations stay in shared memory between layers.

__device__ inline uint32_t pack_bf16(float lo, float hi) {
  const uint32_t a = __bfloat16_as_ushort(__float2bfloat16_rn(lo));
  const uint32_t b = __bfloat16_as_ushort(__float2bfloat16_rn(hi));
  return a | (b << 16);
}

__device__ inline void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

constexpr int kInferWarps = 4;

// relu(x W^T + b) for the warp's 16 rows x [16][K] (row stride ldx) and
// W [64][K] (K = 16 or 64), into act [16][64].  Fragment layouts of
// m16n8k16 (PTX ISA): lane = 4 g + t; A holds rows g and g + 8 at columns
// 2t, 2t + 1 and those plus 8; B holds column g at rows 2t, 2t + 1 (+ 8);
// the accumulator holds rows g, g + 8 at columns 2t, 2t + 1.
template <int K>
__device__ inline void dense_relu_mma(const float *x, int ldx, const float *w, const float *b,
                                      float *act) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  uint32_t a[K / 16][4];
  for (int kt = 0; kt < K / 16; ++kt) {
    const int c0 = kt * 16 + 2 * t;
    a[kt][0] = pack_bf16(x[g * ldx + c0], x[g * ldx + c0 + 1]);
    a[kt][1] = pack_bf16(x[(g + 8) * ldx + c0], x[(g + 8) * ldx + c0 + 1]);
    a[kt][2] = pack_bf16(x[g * ldx + c0 + 8], x[g * ldx + c0 + 9]);
    a[kt][3] = pack_bf16(x[(g + 8) * ldx + c0 + 8], x[(g + 8) * ldx + c0 + 9]);
  }
  __syncwarp();
  for (int nt = 0; nt < kHidden / 8; ++nt) {
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    const int n = nt * 8 + g;  // this lane's B column: output unit n
    for (int kt = 0; kt < K / 16; ++kt) {
      const int k0 = kt * 16 + 2 * t;
      const uint32_t b0 = pack_bf16(w[n * K + k0], w[n * K + k0 + 1]);
      const uint32_t b1 = pack_bf16(w[n * K + k0 + 8], w[n * K + k0 + 9]);
      mma_bf16(c, a[kt], b0, b1);
    }
    const int col = nt * 8 + 2 * t;
    act[g * kHidden + col] = fmaxf(c[0] + b[col], 0.f);
    act[g * kHidden + col + 1] = fmaxf(c[1] + b[col + 1], 0.f);
    act[(g + 8) * kHidden + col] = fmaxf(c[2] + b[col], 0.f);
    act[(g + 8) * kHidden + col + 1] = fmaxf(c[3] + b[col + 1], 0.f);
  }
  __syncwarp();
}

__global__ void __launch_bounds__(32 * kInferWarps) k_mlp_infer(const float *params,
                                                                 const float *x, int rows,
                                                                 float *y) {
  __shared__ float s_x[kInferWarps][16][kIn];
  __shared__ float s_h1[kInferWarps][16][kHidden];
  __shared__ float s_h2[kInferWarps][16][kHidden];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tiles = (rows + 15) / 16;
  for (int tile = blockIdx.x * kInferWarps + warp; tile < tiles; tile += gridDim.x * kInferWarps) {
    const int row0 = tile * 16;
    for (int i = lane; i < 16 * kIn; i += 32) {
      const int r = row0 + i / kIn;
      s_x[warp][i / kIn][i % kIn] = r < rows ? x[int64_t(r) * kIn + i % kIn] : 0.f;
    }
    __syncwarp();
    dense_relu_mma<kIn>(&s_x[warp][0][0], kIn, params + kW1, params + kB1, &s_h1[warp][0][0]);
    dense_relu_mma<kHidden>(&s_h1[warp][0][0], kHidden, params + kW2, params + kB2,
                            &s_h2[warp][0][0]);
    // Layer 3: lanes over (row, output) pairs, FP32 sums of BF16 weights.
    for (int i = lane; i < 16 * kOut; i += 32) {
      const int r = i / kOut, o = i % kOut;
      float s = params[kB3 + o];
      for (int k = 0; k < kHidden; ++k)
        s += s_h2[warp][r][k] * bf16_round(params[kW3 + o * kHidden + k]);
      if (row0 + r < rows) y[int64_t(row0 + r) * kOut + o] = s;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- training
// One block per 64-row tile at a time (grid-stride over tiles): forward in
// FP32 with BF16-rounded weights (the same values the tensor cores take),
// squared error on the masked targets, backward, and the block's gradient
// sums added to `grad` once at the end.  loss[0] += sum of squared errors.
constexpr int kTrainRows = 64, kTrainBlock = 256;

__global__ void __launch_bounds__(kTrainBlock) k_mlp_grad(const float *params, const float *x,
                                                          const float *target, const float *mask,
                                                          int rows, float scale, float *grad,
                                                          float *loss) {
  extern __shared__ float smem[];
  float *w = smem;                        // kParams: BF16-rounded weights, FP32 biases
  float *g = w + kParams;                 // kParams gradient sums of this block
  float *sx = g + kParams;                // [64][16]
  float *h1 = sx + kTrainRows * kIn;      // [64][64]
  float *h2 = h1 + kTrainRows * kHidden;  // [64][64]
  float *dh = h2 + kTrainRows * kHidden;  // [64][64] (dH2)
  float *dy = dh + kTrainRows * kHidden;  // [64][3]
  __shared__ float s_loss;
  const int tid = threadIdx.x;
  for (int i = tid; i < kParams; i += kTrainBlock) {
    const bool weight = i < kB1 || (i >= kW2 && i < kB2) || (i >= kW3 && i < kB3);
    w[i] = weight ? bf16_round(params[i]) : params[i];
    g[i] = 0.f;
  }
  if (tid == 0) s_loss = 0.f;
  __syncthreads();
  const int tiles = (rows + kTrainRows - 1) / kTrainRows;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int row0 = tile * kTrainRows;
    const int live = min(kTrainRows, rows - row0);
    for (int i = tid; i < kTrainRows * kIn; i += kTrainBlock)
      sx[i] = i / kIn < live ? x[int64_t(row0) * kIn + i] : 0.f;
    __syncthreads();
    for (int i = tid; i < kTrainRows * kHidden; i += kTrainBlock) {
      const int r = i / kHidden, o = i % kHidden;
      float s = w[kB1 + o];
      for (int k = 0; k < kIn; ++k) s += sx[r * kIn + k] * w[kW1 + o * kIn + k];
      h1[i] = fmaxf(s, 0.f);
    }
    __syncthreads();
    for (int i = tid; i < kTrainRows * kHidden; i += kTrainBlock) {
      const int r = i / kHidden, o = i % kHidden;
      float s = w[kB2 + o];
      for (int k = 0; k < kHidden; ++k) s += h1[r * kHidden + k] * w[kW2 + o * kHidden + k];
      h2[i] = fmaxf(s, 0.f);
    }
    __syncthreads();
    for (int i = tid; i < kTrainRows * kOut; i += kTrainBlock) {
      const int r = i / kOut, o = i % kOut;
      float d = 0.f;
      if (r < live) {
        float s = w[kB3 + o];
        for (int k = 0; k < kHidden; ++k) s += h2[r * kHidden + k] * w[kW3 + o * kHidden + k];
        const int64_t at = int64_t(row0 + r) * kOut + o;
        const float e = (s - target[at]) * mask[at];
        atomicAdd(&s_loss, e * e);
        d = 2.f * e * scale;
      }
      dy[i] = d;
    }
    __syncthreads();
    // Layer 3 gradients and dH2 = (dY W3) * relu'(H2).
    for (int i = tid; i < kOut * kHidden; i += kTrainBlock) {
      const int o = i / kHidden, k = i % kHidden;
      float s = 0.f;
      for (int r = 0; r < kTrainRows; ++r) s += dy[r * kOut + o] * h2[r * kHidden + k];
      g[kW3 + i] += s;
    }
    if (tid < kOut) {
      float s = 0.f;
      for (int r = 0; r < kTrainRows; ++r) s += dy[r * kOut + tid];
      g[kB3 + tid] += s;
    }
    for (int i = tid; i < kTrainRows * kHidden; i += kTrainBlock) {
      const int r = i / kHidden, k = i % kHidden;
      float s = 0.f;
      for (int o = 0; o < kOut; ++o) s += dy[r * kOut + o] * w[kW3 + o * kHidden + k];
      dh[i] = h2[i] > 0.f ? s : 0.f;
    }
    __syncthreads();
    // Layer 2 gradients (dH2^T H1) and dH1 = (dH2 W2) * relu'(H1).
    for (int i = tid; i < kHidden * kHidden; i += kTrainBlock) {
      const int o = i / kHidden, k = i % kHidden;
      float s = 0.f;
      for (int r = 0; r < kTrainRows; ++r) s += dh[r * kHidden + o] * h1[r * kHidden + k];
      g[kW2 + i] += s;
    }
    for (int o = tid; o < kHidden; o += kTrainBlock) {
      float s = 0.f;
      for (int r = 0; r < kTrainRows; ++r) s += dh[r * kHidden + o];
      g[kB2 + o] += s;
    }
    __syncthreads();
    for (int i = tid; i < kTrainRows * kHidden; i += kTrainBlock) {
      const int r = i / kHidden, k = i % kHidden;
      float s = 0.f;
      for (int o = 0; o < kHidden; ++o) s += dh[r * kHidden + o] * w[kW2 + o * kHidden + k];
      h2[i] = h1[i] > 0.f ? s : 0.f;  // dH1, kept in h2's buffer
    }
    __syncthreads();
    // Layer 1 gradients (dH1^T X).
    for (int i = tid; i < kHidden * kIn; i += kTrainBlock) {
      const int o = i / kIn, k = i % kIn;
      float s = 0.f;
      for (int r = 0; r < kTrainRows; ++r) s += h2[r * kHidden + o] * sx[r * kIn + k];
      g[kW1 + i] += s;
    }
    for (int o = tid; o < kHidden; o += kTrainBlock) {
      float s = 0.f;
      for (int r = 0; r < kTrainRows; ++r) s += h2[r * kHidden + o];
      g[kB1 + o] += s;
    }
    __syncthreads();
  }
  for (int i = tid; i < kParams; i += kTrainBlock)
    if (g[i] != 0.f) atomicAdd(&grad[i], g[i]);
  if (tid == 0) atomicAdd(loss, s_loss);
}

// Adam (Kingma and Ba 2015) on the FP32 master parameters; clears the
// gradient for the next step.  step is 1-based.
__global__ void k_adam(float *params, float *grad, float *m, float *v, int count, float lr,
                       float beta1, float beta2, float eps, int step) {
  const float c1 = 1.f - powf(beta1, float(step)), c2 = 1.f - powf(beta2, float(step));
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const float gi = grad[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * gi;
    const float vi = beta2 * v[i] + (1.f - beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    grad[i] = 0.f;
  }
}

constexpr size_t kGradSmem =
    sizeof(float) * (2 * kParams + kTrainRows * (kIn + 3 * kHidden + kOut));

}  // namespace
}  // namespace edp

using namespace edp;

extern "C" {

int edp_tile_features(const double *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                      const double *camera, const double *settings, float *scratch,
                      float *features, void *stream) {
  if (nv < 0 || nf < 0 || nf >= (int64_t(1) << 31) || !camera || !settings || !scratch ||
      !features || (nf > 0 && (!vertices || !faces)))
    return EDP_ERR_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int *totals = reinterpret_cast<int *>(scratch + kTiles * kRaw);
  k_tile_raw_clear<<<1, 256, 0, st>>>(scratch, totals);
  const int64_t blocks = nf > 0 ? (nf + 255) / 256 : 1;
  k_tile_raw<<<unsigned(blocks < 148 * 8 ? blocks : 148 * 8), 256, 0, st>>>(
      vertices, faces, int(nf), camera, settings, scratch, totals);
  k_tile_finish<<<1, kTiles, 0, st>>>(scratch, totals, int(nf), features);
  cudaError_t e = cudaPeekAtLastError();
  return e == cudaSuccess ? EDP_OK : record_cuda_failure(e, "edp_tile_features");
}

int edp_mlp_infer(const float *params, const float *x, int64_t rows, float *y, void *stream) {
  if (rows < 0 || rows >= (int64_t(1) << 31) || !params || (rows > 0 && (!x || !y)))
    return EDP_ERR_ARGUMENT;
  if (rows == 0) return EDP_OK;
  const int64_t tiles = (rows + 15) / 16;
  const int64_t blocks = (tiles + kInferWarps - 1) / kInferWarps;
  k_mlp_infer<<<unsigned(blocks < 148 * 4 ? blocks : 148 * 4), 32 * kInferWarps, 0,
                static_cast<cudaStream_t>(stream)>>>(params, x, int(rows), y);
  cudaError_t e = cudaPeekAtLastError();
  return e == cudaSuccess ? EDP_OK : record_cuda_failure(e, "edp_mlp_infer");
}

int edp_mlp_grad(const float *params, const float *x, const float *target, const float *mask,
                 int64_t rows, float scale, float *grad, float *loss, void *stream) {
  if (rows < 0 || rows >= (int64_t(1) << 31) || !params || !grad || !loss ||
      (rows > 0 && (!x || !target || !mask)))
    return EDP_ERR_ARGUMENT;
  if (rows == 0) return EDP_OK;
  // More than 48 KB of dynamic shared memory needs the kernel's opt-in,
  // once per device.
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return record_cuda_failure(e, "edp_mlp_grad");
  static bool configured[64] = {};
  if (device >= 0 && device < 64 && !configured[device]) {
    e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kGradSmem));
    if (e != cudaSuccess) return record_cuda_failure(e, "edp_mlp_grad");
    configured[device] = true;
  }
  const int64_t tiles = (rows + kTrainRows - 1) / kTrainRows;
  k_mlp_grad<<<unsigned(tiles < 148 * 2 ? tiles : 148 * 2), kTrainBlock, kGradSmem,
               static_cast<cudaStream_t>(stream)>>>(params, x, target, mask, int(rows), scale,
                                                    grad, loss);
  e = cudaPeekAtLastError();
  return e == cudaSuccess ? EDP_OK : record_cuda_failure(e, "edp_mlp_grad");
}

int edp_adam_step(float *params, float *grad, float *m, float *v, int64_t count, float lr,
                  float beta1, float beta2, float eps, int32_t step, void *stream) {
  if (count < 0 || count >= (int64_t(1) << 31) || step < 1 ||
      (count > 0 && (!params || !grad || !m || !v)))
    return EDP_ERR_ARGUMENT;
  if (count == 0) return EDP_OK;
  const int64_t blocks = (count + 255) / 256;
  k_adam<<<unsigned(blocks < 148 * 4 ? blocks : 148 * 4), 256, 0,
           static_cast<cudaStream_t>(stream)>>>(params, grad, m, v, int(count), lr, beta1, beta2,
                                                eps, step);
  cudaError_t e = cudaPeekAtLastError();
  return e == cudaSuccess ? EDP_OK : record_cuda_failure(e, "edp_adam_step");
}

}  // extern "C"
