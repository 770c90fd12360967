// Device-count-aware primitives: exclusive scan, stable LSD radix sort and
// the implicit-tree hierarchy build.  Counts are device scalars so that one
// captured CUDA graph handles any live size up to the allocated capacity
// (the role of the reference's conditional sort buckets, events.py:637-718).
#include <cub/warp/warp_scan.cuh>

#include "../../include/edp.h"
#include "edp_internal.h"

namespace edp {
namespace {

__device__ inline int warp_inclusive(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024).
__device__ inline int block_exclusive(int v, int *smem, int &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  int inc = warp_inclusive(v);
  if (lane == 31) smem[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int s = lane < warps ? smem[lane] : 0;
    int si = warp_inclusive(s);
    if (lane < warps) smem[lane] = si - s;
    if (lane == warps - 1) smem[32] = si;
  }
  __syncthreads();
  int r = smem[warp] + inc - v;
  total = smem[32];
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------- scan
__global__ void k_scan_reduce(const int *__restrict__ in, const int *count, int *partials) {
  __shared__ int smem[33];
  const int n = *count;
  const int64_t base = int64_t(blockIdx.x) * kScanTile;
  if (base >= n) return;
  int sum = 0;
  for (int k = threadIdx.x; k < kScanTile; k += blockDim.x) {
    int64_t i = base + k;
    if (i < n) sum += in[i];
  }
  int total;
  block_exclusive(sum, smem, total);
  if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

__global__ void k_scan_partials(int *partials, const int *count) {
  __shared__ int smem[33];
  const int tiles = int(ceil_div(*count, kScanTile));
  int carry = 0;
  for (int base = 0; base < tiles; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < tiles ? partials[i] : 0;
    int total;
    int e = block_exclusive(v, smem, total);
    if (i < tiles) partials[i] = carry + e;
    carry += total;
  }
}

__global__ void k_scan_apply(const int *__restrict__ in, int *out, const int *count,
                             const int *partials, int *total_out) {
  __shared__ int smem[33];
  const int n = *count;
  const int64_t base = int64_t(blockIdx.x) * kScanTile;
  if (n == 0 && blockIdx.x == 0 && threadIdx.x == 0 && total_out) *total_out = 0;
  if (base >= n) return;
  constexpr int per = kScanTile / 256;  // blockDim.x == 256
  int v[per];
  int sum = 0;
  const int64_t first = base + int64_t(threadIdx.x) * per;
#pragma unroll
  for (int k = 0; k < per; ++k) {
    int64_t i = first + k;
    v[k] = i < n ? in[i] : 0;
    sum += v[k];
  }
  int total;
  int e = block_exclusive(sum, smem, total) + partials[blockIdx.x];
#pragma unroll
  for (int k = 0; k < per; ++k) {
    int64_t i = first + k;
    if (i < n) {
      out[i] = e;
      if (i == n - 1 && total_out) *total_out = e + v[k];
    }
    e += v[k];
  }
}

// ---------------------------------------------------------------- radix sort
template <class K>
__global__ void k_radix_hist(const K *__restrict__ keys, const int *count, int64_t tiles_cap,
                             int shift, int *hist) {
  __shared__ int h[256];
  const int n = *count;
  const int64_t base = int64_t(blockIdx.x) * kSortTile;
  if (base >= n) return;
  h[threadIdx.x] = 0;
  __syncthreads();
  for (int k = threadIdx.x; k < kSortTile; k += blockDim.x) {
    int64_t i = base + k;
    if (i < n) atomicAdd(&h[int((keys[i] >> shift) & 255u)], 1);
  }
  __syncthreads();
  hist[int64_t(threadIdx.x) * tiles_cap + blockIdx.x] = h[threadIdx.x];
}

// One block per digit: exclusive scan of that digit's counts across tiles.
__global__ void k_radix_scan(int *hist, const int *count, int64_t tiles_cap, int *totals) {
  __shared__ int smem[33];
  const int tiles = int(ceil_div(*count, kSortTile));
  int *row = hist + int64_t(blockIdx.x) * tiles_cap;
  int carry = 0;
  for (int base = 0; base < tiles; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < tiles ? row[i] : 0;
    int total;
    int e = block_exclusive(v, smem, total);
    if (i < tiles) row[i] = carry + e;
    carry += total;
  }
  if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// Stable scatter: warp w owns a contiguous run of 256 keys of the tile, in
// eight rounds of 32; peers with equal digits are ranked with match_any.
template <class K>
__global__ void __launch_bounds__(kSortBlock) k_radix_scatter(
    const K *__restrict__ keys, const int *__restrict__ vals, K *keys_out, int *vals_out,
    const int *count, int64_t tiles_cap, int shift, const int *hist, const int *totals) {
  __shared__ int base[256];
  __shared__ int wcount[kSortBlock / 32][256];
  __shared__ int smem[33];
  const int n = *count;
  const int64_t tile0 = int64_t(blockIdx.x) * kSortTile;
  if (tile0 >= n) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  {
    int t = totals[threadIdx.x];
    int total;
    int e = block_exclusive(t, smem, total);
    base[threadIdx.x] = e + hist[int64_t(threadIdx.x) * tiles_cap + blockIdx.x];
  }
  for (int w = 0; w < kSortBlock / 32; ++w) wcount[w][threadIdx.x] = 0;
  __syncthreads();
  K k[kSortItems];
  int d[kSortItems];
  const int64_t run = tile0 + int64_t(warp) * (32 * kSortItems);
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    int64_t i = run + r * 32 + lane;
    if (i < n) {
      k[r] = keys[i];
      d[r] = int((k[r] >> shift) & 255u);
    } else {
      d[r] = 256;
    }
  }
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    unsigned peers = __match_any_sync(0xffffffffu, d[r]);
    if (d[r] < 256 && lane == __ffs(peers) - 1) wcount[warp][d[r]] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    int running = base[threadIdx.x];
    for (int w = 0; w < kSortBlock / 32; ++w) {
      int c = wcount[w][threadIdx.x];
      wcount[w][threadIdx.x] = running;
      running += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    unsigned peers = __match_any_sync(0xffffffffu, d[r]);
    if (d[r] < 256) {
      int pos = wcount[warp][d[r]] + __popc(peers & lt);
      int64_t i = run + r * 32 + lane;
      keys_out[pos] = k[r];
      vals_out[pos] = vals[i];
    }
    __syncwarp();
    if (d[r] < 256 && lane == __ffs(peers) - 1) wcount[warp][d[r]] += __popc(peers);
    __syncwarp();
  }
}

template <class K>
__global__ void k_copy_pairs(const K *keys, const int *vals, K *keys_out, int *vals_out,
                             const int *count) {
  const int n = *count;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    keys_out[i] = keys[i];
    vals_out[i] = vals[i];
  }
}

template <class K>
cudaError_t sort_pairs(K *keys, K *keys_tmp, int *vals, int *vals_tmp, const int *count,
                       int64_t capacity, int bits, SortScratch &s, cudaStream_t st) {
  const int64_t tiles = ceil_div(capacity, kSortTile);
  if (tiles > s.tiles) return cudaErrorInvalidValue;
  const int passes = int(ceil_div(bits, 8));
  K *ka = keys, *kb = keys_tmp;
  int *va = vals, *vb = vals_tmp;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    k_radix_hist<K><<<unsigned(tiles), kSortBlock, 0, st>>>(ka, count, s.tiles, shift, s.hist);
    note_launch();
    k_radix_scan<<<256, 256, 0, st>>>(s.hist, count, s.tiles, s.totals);
    note_launch();
    k_radix_scatter<K><<<unsigned(tiles), kSortBlock, 0, st>>>(ka, va, kb, vb, count, s.tiles, shift, s.hist, s.totals);
    note_launch();
    K *tk = ka; ka = kb; kb = tk;
    int *tv = va; va = vb; vb = tv;
  }
  if (ka != keys)
    k_copy_pairs<K><<<592, 256, 0, st>>>(ka, va, keys, vals, count);
    note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------- hierarchy
__global__ void k_tree_size(const int *count_ptr, int static_count, int *count_out, int *size) {
  int c = count_ptr ? *count_ptr : static_count;
  int p = 1;
  while (p < c) p <<= 1;
  *count_out = c;
  *size = p;
}

__global__ void k_tree_keys(const float4 *lo, const float4 *hi, const int *count, const int *size,
                            uint64_t *keys, int *ids, int layered) {
  const int n = *count, leaves = *size;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < leaves;
       i += int64_t(gridDim.x) * blockDim.x) {
    ids[i] = int(i);
    uint64_t key = ~0ull;
    if (i < n) {
      float4 a = lo[i], b = hi[i];
      if (a.x <= b.x && a.y <= b.y) {
        float cx = fminf(fmaxf((a.x + b.x) * 0.5f, 0.f), 1.f);
        float cy = fminf(fmaxf((a.y + b.y) * 0.5f, 0.f), 1.f);
        uint32_t x = uint32_t(int(cx * 32767.0f)), y = uint32_t(int(cy * 32767.0f));
        key = uint64_t(part1by1(x) | (part1by1(y) << 1));
        if (layered) key |= uint64_t(int(a.z)) << 32;
      }
    }
    keys[i] = key;
  }
}

// Every node of a fresh hierarchy holds the empty box, which overlaps nothing.
__global__ void k_tree_clear(float4 *nodes, int64_t count) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count;
       i += int64_t(gridDim.x) * blockDim.x) {
    nodes[2 * i] = empty_lo();
    nodes[2 * i + 1] = empty_hi();
  }
}

__device__ inline void union_into(float4 *nodes, int node) {
  float4 a = __ldcg(&nodes[4 * node]), c = __ldcg(&nodes[4 * node + 1]);      // child 2 node
  float4 b = __ldcg(&nodes[4 * node + 2]), d = __ldcg(&nodes[4 * node + 3]);  // child 2 node + 1
  __stcg(&nodes[2 * node], make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), 0.f));
  __stcg(&nodes[2 * node + 1], make_float4(fmaxf(c.x, d.x), fmaxf(c.y, d.y), fmaxf(c.z, d.z), 0.f));
}

constexpr int kFitThreads = 256;
constexpr int kFitLeaves = 2 * kFitThreads;  // leaves of one block's subtree

// Leaves and every internal box in one launch.  Leaf i holds the box of item
// ids[i] (the empty box past the item count).  Each block reduces whole
// subtrees of up to kFitLeaves leaves level by level in shared memory; the
// last block to finish then reduces the levels above the subtree roots.
// Unions of binary32 boxes are exact, so the boxes do not depend on the order.
__global__ void __launch_bounds__(kFitThreads)
k_tree_fit(float4 *nodes, const int *ids, const float4 *lo, const float4 *hi, const int *count,
           const int *size, int *done) {
  __shared__ float4 s_lo[kFitThreads], s_hi[kFitThreads];
  __shared__ int s_last;
  const int n = *count, leaves = *size, t = threadIdx.x;
  const int span = leaves < kFitLeaves ? leaves : kFitLeaves;
  const int subtrees = leaves / span;
  auto leaf = [&](int i, float4 &a, float4 &b) {
    const int j = ids[i];
    a = empty_lo();
    b = empty_hi();
    if (j < n) {
      a = lo[j];
      b = hi[j];
    }
    nodes[2 * (leaves + i)] = a;
    nodes[2 * (leaves + i) + 1] = b;
  };
  for (int sub = blockIdx.x; sub < subtrees; sub += gridDim.x) {
    const int first = sub * span;
    if (span == 1) {
      float4 a, b;
      if (t == 0) leaf(first, a, b);
      continue;
    }
    int width = span >> 1, base = (leaves + first) >> 1;  // node id of slot 0 on this level
    if (t < width) {
      float4 a, b, c, e;
      leaf(first + 2 * t, a, b);
      leaf(first + 2 * t + 1, c, e);
      a = make_float4(fminf(a.x, c.x), fminf(a.y, c.y), fminf(a.z, c.z), 0.f);
      b = make_float4(fmaxf(b.x, e.x), fmaxf(b.y, e.y), fmaxf(b.z, e.z), 0.f);
      s_lo[t] = a;
      s_hi[t] = b;
      nodes[2 * (base + t)] = a;
      nodes[2 * (base + t) + 1] = b;
    }
    __syncthreads();
    for (width >>= 1; width >= 1; width >>= 1) {
      base >>= 1;
      float4 a, b;
      if (t < width) {
        const float4 l0 = s_lo[2 * t], l1 = s_lo[2 * t + 1], h0 = s_hi[2 * t], h1 = s_hi[2 * t + 1];
        a = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.f);
        b = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.f);
      }
      __syncthreads();
      if (t < width) {
        s_lo[t] = a;
        s_hi[t] = b;
        nodes[2 * (base + t)] = a;
        nodes[2 * (base + t) + 1] = b;
      }
      __syncthreads();
    }
  }
  __threadfence();
  __syncthreads();
  if (t == 0) s_last = atomicAdd(done, 1) == int(gridDim.x) - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int width = subtrees >> 1; width >= 1; width >>= 1) {
    for (int k = t; k < width; k += blockDim.x) union_into(nodes, width + k);
    __syncthreads();
  }
  if (t == 0) *done = 0;
}

}  // namespace

cudaError_t scan_exclusive(const int *in, int *out, const int *count, int64_t capacity,
                           int *total, SortScratch &s, cudaStream_t st) {
  const int64_t tiles = ceil_div(capacity > 0 ? capacity : 1, kScanTile);
  if (tiles > s.scan_tiles) return cudaErrorInvalidValue;
  k_scan_reduce<<<unsigned(tiles), 256, 0, st>>>(in, count, s.partials);
  note_launch();
  k_scan_partials<<<1, 1024, 0, st>>>(s.partials, count);
  note_launch();
  k_scan_apply<<<unsigned(tiles), 256, 0, st>>>(in, out, count, s.partials, total);
  note_launch();
  return cudaGetLastError();
}

cudaError_t sort_pairs_u64(uint64_t *keys, uint64_t *keys_tmp, int *vals, int *vals_tmp,
                           const int *count, int64_t capacity, int bits, SortScratch &s,
                           cudaStream_t st) {
  return sort_pairs<uint64_t>(keys, keys_tmp, vals, vals_tmp, count, capacity, bits, s, st);
}
cudaError_t sort_pairs_u32(uint32_t *keys, uint32_t *keys_tmp, int *vals, int *vals_tmp,
                           const int *count, int64_t capacity, int bits, SortScratch &s,
                           cudaStream_t st) {
  return sort_pairs<uint32_t>(keys, keys_tmp, vals, vals_tmp, count, capacity, bits, s, st);
}

cudaError_t tree_refit(TreeBuffers &t, const float4 *lo, const float4 *hi, cudaStream_t st) {
  const int64_t subtrees = ceil_div(t.leaves_cap, int64_t(kFitLeaves));
  const unsigned g = unsigned(subtrees < 148 * 8 ? subtrees : 148 * 8);
  k_tree_fit<<<g, kFitThreads, 0, st>>>(t.nodes, t.ids, lo, hi, t.count, t.size, t.flags);
  note_launch();
  return cudaGetLastError();
}

cudaError_t tree_alloc(TreeBuffers &t, int64_t capacity) {
  t.capacity = capacity > 0 ? capacity : 1;
  t.leaves_cap = pow2_at_least(t.capacity);
  EDP_CHECK(cudaMalloc(&t.nodes, sizeof(float4) * 4 * t.leaves_cap));
  EDP_CHECK(cudaMalloc(&t.ids, sizeof(int) * t.leaves_cap));
  EDP_CHECK(cudaMalloc(&t.ids_tmp, sizeof(int) * t.leaves_cap));
  EDP_CHECK(cudaMalloc(&t.keys, sizeof(uint64_t) * t.leaves_cap));
  EDP_CHECK(cudaMalloc(&t.keys_tmp, sizeof(uint64_t) * t.leaves_cap));
  EDP_CHECK(cudaMalloc(&t.flags, sizeof(int)));
  EDP_CHECK(cudaMemset(t.flags, 0, sizeof(int)));
  EDP_CHECK(cudaMalloc(&t.size, sizeof(int) * 2));
  t.count = t.size + 1;
  EDP_CHECK(cudaMemset(t.size, 0, sizeof(int) * 2));
  const int64_t count = 2 * t.leaves_cap;
  k_tree_clear<<<grid_for(count, 256) < 4 * 148 ? grid_for(count, 256) : 4 * 148, 256>>>(t.nodes, count);
  note_launch();
  EDP_CHECK(cudaGetLastError());
  EDP_CHECK(cudaStreamSynchronize(0));
  return cudaSuccess;
}

void tree_free(TreeBuffers &t) {
  cudaFree(t.nodes); cudaFree(t.ids); cudaFree(t.ids_tmp);
  cudaFree(t.keys); cudaFree(t.keys_tmp); cudaFree(t.flags); cudaFree(t.size);
  t = TreeBuffers{};
}

cudaError_t tree_build(TreeBuffers &t, const float4 *lo, const float4 *hi, const int *count_ptr,
                       int static_count, bool layered, SortScratch &s, cudaStream_t st) {
  k_tree_size<<<1, 1, 0, st>>>(count_ptr, static_count, t.count, t.size);
  note_launch();
  const unsigned g = grid_for(t.leaves_cap, 256) < 4 * 148 ? grid_for(t.leaves_cap, 256) : 4 * 148;
  k_tree_keys<<<g, 256, 0, st>>>(lo, hi, t.count, t.size, t.keys, t.ids, layered ? 1 : 0);
  note_launch();
  // Layered keys hold the layer above 30 Morton bits; 48 key bits order them
  // for up to 65536 layers.  Deeper scenes leave higher layer bits unordered,
  // which only loosens the hierarchy: any leaf order gives the same queries.
  int bits = layered ? 48 : 30;
  EDP_CHECK(sort_pairs_u64(t.keys, t.keys_tmp, t.ids, t.ids_tmp, t.count, t.leaves_cap, bits, s, st));
  return tree_refit(t, lo, hi, st);
}

}  // namespace edp

namespace edp {
namespace {
thread_local int64_t g_launches = 0;
thread_local cudaEvent_t *g_marks = nullptr;
thread_local int g_next_mark = 0;  // stages marked so far in this capture
}
void note_launch() { ++g_launches; }
void forget_launches(int64_t n) { g_launches -= n; }
int64_t launch_count() { return g_launches; }

void set_stage_marks(cudaEvent_t *events) {
  g_marks = events;
  g_next_mark = 0;
}

cudaError_t stage_mark(int stage, cudaStream_t st) {
  if (!g_marks) return cudaSuccess;
  if (stage < 0) {  // the start
    g_next_mark = 0;
    return cudaEventRecordWithFlags(g_marks[0], st, cudaEventRecordExternal);
  }
  for (; g_next_mark <= stage && g_next_mark < EDP_STAGE_COUNT; ++g_next_mark) {
    cudaError_t e = cudaEventRecordWithFlags(g_marks[g_next_mark + 1], st, cudaEventRecordExternal);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
}  // namespace edp
