// CSR patterns of the operators built on the device from the element map
// (the host build is build_patterns in host/mesh.cpp; both give sorted rows
// of distinct columns, so the patterns are identical):
//   K  (NN x NN):   row r = the 27 nodes of every element around node r;
//   G  (NN x NNp):  row r = the 8 corner (pressure) nodes of those elements;
//   G^T (NNp x NN): row p = K's row p (the 27 nodes of the elements around
//                   corner p), so it is K's first NNp rows;
//   Z  (NNp x NNp): row p = the corners of every element that shares a node
//                   with an element around p (Z = G^T diag G).
// One block per row gathers the candidates into shared memory, sorts them
// (bitonic) and keeps the first of each run; a first pass counts, the host
// turns the counts into row pointers, a second pass writes the columns.  A
// row with more candidates than a block holds raises a flag, and the caller
// falls back to the host build.
#include <climits>

#include "common.cuh"
#include "kernels.h"

namespace cfd {

namespace {

constexpr int kPatThreads = 256;
constexpr int kPatCap = 2048;  // candidates a block sorts (8 per thread)

__global__ void k_inc_count(long long nent, const int* __restrict__ ltog, int* __restrict__ cnt) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nent; i += (long long)gridDim.x * blockDim.x)
    atomicAdd(cnt + ltog[i], 1);
}

__global__ void k_inc_fill(long long nent, const int* __restrict__ ltog, int* __restrict__ pos, int* __restrict__ inc_el) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nent; i += (long long)gridDim.x * blockDim.x) {
    const int slot = atomicAdd(pos + ltog[i], 1);
    inc_el[slot] = (int)(i / 27);
  }
}

// In-place ascending bitonic sort of s[0, n), n a power of two <= kPatCap.
__device__ void block_sort(int* s, int n) {
  for (int k = 2; k <= n; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const int a = s[i], b = s[l];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            s[i] = b;
            s[l] = a;
          }
        }
      }
      __syncthreads();
    }
}

// After block_sort: the number of distinct values below INT_MAX in s[0, n);
// with out, also writes them in order (out[0 .. count)).  Uses sflag (n ints)
// and swarp (kPatThreads / 32 ints) as scratch.
__device__ int block_unique(const int* s, int n, int* sflag, int* swarp, int* out) {
  // each thread owns a contiguous run of n / blockDim.x (at least 1) slots
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per, e = min(n, b + per);
  int c = 0;
  for (int i = b; i < e; i++) {
    const int f = s[i] != INT_MAX && (i == 0 || s[i] != s[i - 1]);
    sflag[i] = f;
    c += f;
  }
  // exclusive prefix of c over the block
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) swarp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < (int)(blockDim.x >> 5) ? swarp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < (int)(blockDim.x >> 5)) swarp[lane] = w;  // inclusive per warp
  }
  __syncthreads();
  const int total = swarp[(blockDim.x >> 5) - 1];
  int pos = x - c + (warp > 0 ? swarp[warp - 1] : 0);
  if (out)
    for (int i = b; i < e; i++)
      if (sflag[i]) out[pos++] = s[i];
  __syncthreads();
  return total;
}

__device__ __forceinline__ int pow2_at_least(int n) {
  int p = 32;
  while (p < n) p <<= 1;
  return p;
}

// mode 0: K rows (27 nodes of the elements around node r); 1: G rows (8
// corners); 2: element adjacency (elements around the 27 nodes of element r).
// pass 0 writes len[r]; pass 1 writes the columns at rp[r].
__global__ void __launch_bounds__(kPatThreads) k_rows(PatArgs a, int mode, int nrows, int pass) {
  __shared__ int s[kPatCap];
  __shared__ int sflag[kPatCap];
  __shared__ int swarp[kPatThreads / 32];
  __shared__ int soff[28];
  for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
    int count;
    if (mode < 2) {
      const int nj = mode == 0 ? 27 : 8;
      const int t0 = a.inc_rp[r], deg = a.inc_rp[r + 1] - t0;
      count = deg * nj;
      if (count > kPatCap) {
        if (threadIdx.x == 0) {
          atomicExch(a.overflow, 1);
          if (pass == 0) a.len[r] = 0;
        }
        continue;
      }
      for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const int e = a.inc_el[t0 + i / nj];
        s[i] = a.ltog[(size_t)e * 27 + i % nj];
      }
    } else {
      // offsets of the 27 incidence lists
      if (threadIdx.x == 0) {
        int o = 0;
        for (int j = 0; j < 27; j++) {
          soff[j] = o;
          const int v = a.ltog[(size_t)r * 27 + j];
          o += a.inc_rp[v + 1] - a.inc_rp[v];
        }
        soff[27] = o;
      }
      __syncthreads();
      count = soff[27];
      if (count > kPatCap) {
        if (threadIdx.x == 0) {
          atomicExch(a.overflow, 1);
          if (pass == 0) a.len[r] = 0;
        }
        __syncthreads();
        continue;
      }
      for (int i = threadIdx.x; i < count; i += blockDim.x) {
        int j = 0;
        while (soff[j + 1] <= i) j++;
        const int v = a.ltog[(size_t)r * 27 + j];
        s[i] = a.inc_el[a.inc_rp[v] + (i - soff[j])];
      }
    }
    const int n = pow2_at_least(count);
    for (int i = count + threadIdx.x; i < n; i += blockDim.x) s[i] = INT_MAX;
    __syncthreads();
    block_sort(s, n);
    const int u = block_unique(s, n, sflag, swarp, pass == 1 ? a.col + a.rp[r] : nullptr);
    if (pass == 0 && threadIdx.x == 0) a.len[r] = u;
  }
}

// Z rows p < NNp: the elements adjacent to the elements around p (sorted,
// distinct), then their corners (sorted, distinct).
__global__ void __launch_bounds__(kPatThreads) k_zrows(PatArgs a, int nrows, int pass) {
  __shared__ int s[kPatCap];
  __shared__ int sflag[kPatCap];
  __shared__ int sel[kPatCap / 8];
  __shared__ int swarp[kPatThreads / 32];
  __shared__ int soff[65];
  __shared__ int sbad;
  for (int p = blockIdx.x; p < nrows; p += gridDim.x) {
    const int t0 = a.inc_rp[p], deg = a.inc_rp[p + 1] - t0;
    if (threadIdx.x == 0) {
      sbad = deg > 64;
      int o = 0;
      for (int q = 0; q < deg && q < 64; q++) {
        soff[q] = o;
        const int e = a.inc_el[t0 + q];
        o += a.adj_rp[e + 1] - a.adj_rp[e];
      }
      soff[deg < 64 ? deg : 64] = o;
      if (o > kPatCap) sbad = 1;
    }
    __syncthreads();
    if (sbad) {
      if (threadIdx.x == 0) {
        atomicExch(a.overflow, 1);
        if (pass == 0) a.len[p] = 0;
      }
      __syncthreads();
      continue;
    }
    int count = soff[deg];
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
      int q = 0;
      while (soff[q + 1] <= i) q++;
      const int e = a.inc_el[t0 + q];
      s[i] = a.adj_col[a.adj_rp[e] + (i - soff[q])];
    }
    int n = pow2_at_least(count);
    for (int i = count + threadIdx.x; i < n; i += blockDim.x) s[i] = INT_MAX;
    __syncthreads();
    block_sort(s, n);
    // the distinct elements (count first: the list must fit sel)
    const int ne = block_unique(s, n, sflag, swarp, nullptr);
    if (ne > kPatCap / 8) {
      if (threadIdx.x == 0) {
        atomicExch(a.overflow, 1);
        if (pass == 0) a.len[p] = 0;
      }
      __syncthreads();
      continue;
    }
    block_unique(s, n, sflag, swarp, sel);
    // their corners
    for (int i = threadIdx.x; i < ne; i += blockDim.x) {
      const int e = sel[i];
      for (int m = 0; m < 8; m++) s[8 * i + m] = a.ltog[(size_t)e * 27 + m];
    }
    count = ne * 8;
    n = pow2_at_least(count);
    for (int i = count + threadIdx.x; i < n; i += blockDim.x) s[i] = INT_MAX;
    __syncthreads();
    block_sort(s, n);
    const int u = block_unique(s, n, sflag, swarp, pass == 1 ? a.col + a.rp[p] : nullptr);
    if (pass == 0 && threadIdx.x == 0) a.len[p] = u;
  }
}

// gt_pos[t] = index in G's columns of (v, p) for the G^T entry t = (p, v).
__global__ void k_gt_pos(int nnp, const int* __restrict__ gt_rp, const int* __restrict__ gt_col,
                         const int* __restrict__ g_rp, const int* __restrict__ g_col, int* __restrict__ gt_pos,
                         int* __restrict__ bad) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnp; p += gridDim.x * blockDim.x)
    for (int t = gt_rp[p]; t < gt_rp[p + 1]; t++) {
      const int v = gt_col[t];
      int lo = g_rp[v], hi = g_rp[v + 1] - 1, at = -1;
      while (lo <= hi) {
        const int mid = (lo + hi) >> 1, c = g_col[mid];
        if (c == p) {
          at = mid;
          break;
        }
        if (c < p)
          lo = mid + 1;
        else
          hi = mid - 1;
      }
      if (at < 0) atomicExch(bad, 1);
      gt_pos[t] = at < 0 ? 0 : at;
    }
}

// first and last column of every row (rows sorted ascending; 0, -1 when empty)
__global__ void k_row_ends(int n, const int* __restrict__ rp, const int* __restrict__ col, int* __restrict__ first,
                           int* __restrict__ last) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int b = rp[r], e = rp[r + 1];
    first[r] = b < e ? col[b] : 0;
    last[r] = b < e ? col[e - 1] : -1;
  }
}

int grid_for(long long n, int threads) {
  const long long g = (n + threads - 1) / threads;
  return (int)(g < 1 ? 1 : (g > 148 * 32 ? 148 * 32 : g));
}

}  // namespace

cudaError_t launch_incidence_count(long long nent, const int* ltog, int* cnt, cudaStream_t s) {
  k_inc_count<<<grid_for(nent, 256), 256, 0, s>>>(nent, ltog, cnt);
  return cudaGetLastError();
}
cudaError_t launch_incidence_fill(long long nent, const int* ltog, int* pos, int* inc_el, cudaStream_t s) {
  k_inc_fill<<<grid_for(nent, 256), 256, 0, s>>>(nent, ltog, pos, inc_el);
  return cudaGetLastError();
}
cudaError_t launch_pattern_rows(const PatArgs& a, int mode, int nrows, int pass, int num_sms, cudaStream_t s) {
  if (nrows <= 0) return cudaSuccess;
  const int grid = nrows < num_sms * 8 ? nrows : num_sms * 8;
  if (mode == 3)
    k_zrows<<<grid, kPatThreads, 0, s>>>(a, nrows, pass);
  else
    k_rows<<<grid, kPatThreads, 0, s>>>(a, mode, nrows, pass);
  return cudaGetLastError();
}
cudaError_t launch_gt_pos(int nnp, const int* gt_rp, const int* gt_col, const int* g_rp, const int* g_col, int* gt_pos,
                          int* bad, cudaStream_t s) {
  k_gt_pos<<<grid_for(nnp, 256), 256, 0, s>>>(nnp, gt_rp, gt_col, g_rp, g_col, gt_pos, bad);
  return cudaGetLastError();
}
cudaError_t launch_row_ends(int n, const int* rp, const int* col, int* first, int* last, cudaStream_t s) {
  k_row_ends<<<grid_for(n, 256), 256, 0, s>>>(n, rp, col, first, last);
  return cudaGetLastError();
}

}  // namespace cfd
