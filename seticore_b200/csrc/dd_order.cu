// The noise statistics of a search, bit-identical to the reference's, for the searches whose
// column sums hold repeated values.
//
// The reference copies the column sums to the host and runs (dedoppler.cu:242-262):
//   nth_element(a, a + mid, a + N);  nth_element(a, a + first, a + mid - 1);
//   nth_element(a + mid + 1, a + last, a + N);
//   median = a[mid];  sum = accumulate(a + first, a + last + 1, 0.0)  (double, in order);
//   m = float(sum) / n;  accum (float) += (f - m) * (f - m) over a[first..last] in order;
//   std_dev = sqrt(accum / n),  n = last + 1 - first.
// The float accumulation depends on the order of its terms, which is the permutation that
// std::nth_element leaves; with many equal column sums (integer-valued power) that order
// moves the deviation by a few 1e-4, beyond what the channel-order emulation of dd_stats.cu
// (about 1e-5 on distinct values) can absorb.  For every search whose order statistics sit
// on values held by kExactStatsTies or more column sums, the kernels below reproduce the
// permutation and then both sequential sums exactly, and overwrite the statistics:
//
// * nth_element is libstdc++'s introselect: while the range holds more than 3 values, a
//   median-of-three pivot (__move_median_to_first of positions first+1, mid, last-1) and an
//   unguarded Hoare partition of [first+1, last) against it, then a final insertion sort;
//   at the depth limit 2*floor(log2 n) a heap selection instead (one thread).  The partition swaps the k-th value >= pivot counted from
//   the left with the k-th value <= pivot counted from the right, for as long as the left one
//   lies before the right one.  With cL(x) values >= pivot left of x and cR(x) values <= pivot
//   at or right of x, the number of swapped pairs is K = max_x min(cL(x), cR(x)), and the cut
//   it returns is L[0] for K = 0, else min(L[K], R[K-1]) (L ascending positions of values >=
//   pivot, R descending positions of values <= pivot).  A step is therefore: count both kinds
//   per segment, locate K and the cut, list the K pairs with their values, write them
//   swapped.  Ranges of up to kSmemRange values run in shared memory.
// * A sequential sum: an accumulator A of p significand bits lies on the grid of its binade
//   (multiples of u = ulp(A)).  While the sum stays in that binade, adding a term t moves A by
//   k = q + round(r) grid steps (q + r = |t| / u, sign of t), and only an exact tie (r = 1/2)
//   depends on A itself: round half to even makes the new A even.  So over a chunk of terms
//   the parity of A before each term is a scan of the maps p -> p ^ (k & 1) and p -> 0, and A
//   before each term is a prefix sum of the k.  The first term whose sum would leave the
//   binade is added with a real floating-point add and the scan restarts from the new
//   binade.  The result is the sequential sum, bit for bit.
#include <algorithm>
#include <atomic>
#include <climits>
#include <type_traits>

#include "dd_common.cuh"
#include "dd_internal.h"

namespace scb {

namespace {

constexpr int kOrdThreads = 1024;
constexpr int kOrdWarps = kOrdThreads / 32;
constexpr int kV4 = 8;                   // float4 groups per lane in one warp step
constexpr int kStep = 32 * 4 * kV4;      // positions per warp step
constexpr int kMaxSegs = kOrderMaxSegs;  // counting segments per partition step
constexpr int kSmemRange = 16384;        // ranges of at most this many values run in shared memory
constexpr int kSmemPairs = kSmemRange / 2 + 1;
constexpr int kSeqPrefix = 2048;         // leading terms of a sum added one by one (thread 0)
constexpr int kTermsPerThreadF = 16;     // terms per thread in one scan chunk of a float sum
constexpr int kTermsPerThreadD = 8;      // ... of a double sum (two registers per term)
constexpr int kSumChunk = kOrdThreads * kTermsPerThreadF;
constexpr int kSumBuf = kSumChunk + kSumChunk / 16;  // one pad word per 16 terms: conflict-free

// Shared memory of the kernel beyond the dynamic shared-memory range buffer.
struct OrdShared {
  int seg_ge[kMaxSegs + 1];  // per segment: values >= pivot; then their exclusive prefix
  int seg_le[kMaxSegs + 1];  // per segment: values <= pivot; then their exclusive prefix
  float pivot;
  int total_ge, total_le;
  int cross, K, lk, rk;
  int warp_i[kOrdWarps];
  long long warp_ll[kOrdWarps];
  unsigned warp_map[kOrdWarps];
  long long warp_ll2[kOrdWarps];
  unsigned warp_map2[kOrdWarps];
  // sequential-sum state
  int s_eu;
  long long s_a;
  long long s_cross;
  long long s_a_at_cross;
  int s_slow;
};

// ---------------------------------------------------------------------------------------
// introselect (libstdc++ bits/stl_algo.h), on a range of `a` (global or shared memory)
// ---------------------------------------------------------------------------------------

// __move_median_to_first(result, a, b, c) with comp = operator<.
__device__ void move_median_to_first(float* v, int result, int x, int y, int z) {
  int m;
  if (v[x] < v[y]) {
    if (v[y] < v[z]) m = y;
    else if (v[x] < v[z]) m = z;
    else m = x;
  } else if (v[x] < v[z]) {
    m = x;
  } else if (v[y] < v[z]) {
    m = z;
  } else {
    m = y;
  }
  const float t = v[result];
  v[result] = v[m];
  v[m] = t;
}

// __insertion_sort(first, last): stable, one thread.
__device__ void insertion_sort(float* v, int first, int last) {
  if (first == last) return;
  for (int i = first + 1; i < last; ++i) {
    const float val = v[i];
    if (val < v[first]) {
      for (int j = i; j > first; --j) v[j] = v[j - 1];
      v[first] = val;
    } else {
      int j = i;
      while (val < v[j - 1]) {
        v[j] = v[j - 1];
        --j;
      }
      v[j] = val;
    }
  }
}

// The heap selection libstdc++ falls back to when introselect reaches its depth limit
// (bits/stl_heap.h __push_heap, __adjust_heap, __make_heap; bits/stl_algo.h __heap_select),
// one thread, on f[0..) with comp = operator<.
__device__ void push_heap_(float* f, int hole, int top, float value) {
  int parent = (hole - 1) / 2;
  while (hole > top && f[parent] < value) {
    f[hole] = f[parent];
    hole = parent;
    parent = (hole - 1) / 2;
  }
  f[hole] = value;
}
__device__ void adjust_heap_(float* f, int hole, int len, float value) {
  const int top = hole;
  int second = hole;
  while (second < (len - 1) / 2) {
    second = 2 * (second + 1);
    if (f[second] < f[second - 1]) second--;
    f[hole] = f[second];
    hole = second;
  }
  if ((len & 1) == 0 && second == (len - 2) / 2) {
    second = 2 * (second + 1);
    f[hole] = f[second - 1];
    hole = second - 1;
  }
  push_heap_(f, hole, top, value);
}
__device__ void heap_select_(float* f, int middle, int last) {
  if (middle >= 2) {
    for (int parent = (middle - 2) / 2;; --parent) {
      adjust_heap_(f, parent, middle, f[parent]);
      if (parent == 0) break;
    }
  }
  for (int i = middle; i < last; ++i) {
    if (f[i] < f[0]) {  // __pop_heap(first, middle, i)
      const float value = f[i];
      f[i] = f[0];
      adjust_heap_(f, 0, middle, value);
    }
  }
}

// Exclusive prefix sums of arr[0..n) in place (n <= kMaxSegs), by a block of NT threads;
// arr[n] = the total.  warp_tmp: NT / 32 ints of shared memory.
template <int NT>
__device__ void block_exclusive_scan(int* arr, int n, int* warp_tmp) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int per = (kMaxSegs + NT - 1) / NT;
  constexpr int nw = NT / 32;
  int v[per];
  int tot = 0;
#pragma unroll
  for (int q = 0; q < per; ++q) {
    const int i = tid * per + q;
    v[q] = i < n ? arr[i] : 0;
    tot += v[q];
  }
  int inc = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_tmp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int w = lane < nw ? warp_tmp[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < nw) warp_tmp[lane] = wi - w;
    if (lane == nw - 1) arr[n] = wi;
  }
  __syncthreads();
  int run = warp_tmp[warp] + inc - tot;
#pragma unroll
  for (int q = 0; q < per; ++q) {
    const int i = tid * per + q;
    if (i < n) arr[i] = run;
    run += v[q];
  }
  __syncthreads();
}

__device__ __forceinline__ int warp_incl_scan(int x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// One warp step: the float4 groups at a0 + 128 q + 4 lane (q < kV4, a0 a multiple of 4)
// that overlap [x0, x1), loaded together (an element's position order is (q, lane, c)).
// The buffers are padded so that a group overlapping the end of a range stays inside them.
struct VChunk {
  float4 v[kV4];
  __device__ __forceinline__ void load(const float* __restrict__ a, int a0, int x0, int x1) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < kV4; ++q) {
      const int p = a0 + 128 * q + 4 * lane;
      v[q] = (p + 3 >= x0 && p < x1) ? *reinterpret_cast<const float4*>(a + p) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  __device__ __forceinline__ float at(int q, int c) const {
    return c == 0 ? v[q].x : (c == 1 ? v[q].y : (c == 2 ? v[q].z : v[q].w));
  }
  // 4-bit masks of this lane's group q: values >= p (ge) and <= p (le) inside [x0, x1).
  __device__ __forceinline__ void masks(int q, int a0, int x0, int x1, float p, unsigned& mg, unsigned& ml) const {
    const int base = a0 + 128 * q + 4 * (int)(threadIdx.x & 31);
    mg = ml = 0u;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const bool in = base + c >= x0 && base + c < x1;
      const float f = at(q, c);
      mg |= (in && !(f < p) ? 1u : 0u) << c;
      ml |= (in && !(p < f) ? 1u : 0u) << c;
    }
  }
};

// Segments of a partition step over [s, e): aligned windows of seglen positions from
// A0 = s rounded down to a multiple of 4, clipped to [s, e).
struct Segs {
  int s, e, A0, seglen, nseg;
  __device__ __forceinline__ Segs(int s_, int e_) : s(s_), e(e_), A0(s_ & ~3) {
    const int span = e - A0;
    const int steps = (span + kStep - 1) / kStep;
    seglen = ((steps + kMaxSegs - 1) / kMaxSegs) * kStep;
    nseg = (span + seglen - 1) / seglen;
  }
  __device__ __forceinline__ int start(int g) const { return A0 + g * seglen; }  // aligned
  __device__ __forceinline__ int x0(int g) const { return max(s, start(g)); }
  __device__ __forceinline__ int x1(int g) const { return min(e, start(g) + seglen); }
};

// Position of the value of rank r (0-based, in position order) among the values of one kind
// in segment g; every lane gets it.  The caller guarantees the segment holds it.
__device__ int find_rank(const float* __restrict__ a, const Segs& sg, int g, float p, bool kind_ge, int r) {
  const int lane = threadIdx.x & 31;
  const int x0 = sg.x0(g), x1 = sg.x1(g);
  for (int a0 = sg.start(g); a0 < x1; a0 += kStep) {
    VChunk w;
    w.load(a, a0, x0, x1);
#pragma unroll
    for (int q = 0; q < kV4; ++q) {
      unsigned mg, ml;
      w.masks(q, a0, x0, x1, p, mg, ml);
      const unsigned m = kind_ge ? mg : ml;
      const int cnt = __popc(m);
      const int inc = warp_incl_scan(cnt);
      const int tot = __shfl_sync(0xffffffffu, inc, 31);
      if (r < tot) {
        const int ex = inc - cnt;
        const bool mine = r >= ex && r < inc;
        int pos = 0;
        if (mine) {
          unsigned mm = m;
          for (int t = 0; t < r - ex; ++t) mm &= mm - 1u;
          pos = a0 + 128 * q + 4 * lane + __ffs((int)mm) - 1;
        }
        const int src = __ffs((int)__ballot_sync(0xffffffffu, mine)) - 1;
        return __shfl_sync(0xffffffffu, pos, src);
      }
      r -= tot;
    }
  }
  return INT_MAX;  // not reached when the caller's rank is inside the segment
}

// __unguarded_partition_pivot(first, last) over a[first, last), block-wide: returns the cut.
// lpos/lval/rpos/rval hold at least (last - first) / 2 + 1 entries.
// placed: the median of three is already at `first` (a step prepared by the rounds).
__device__ int partition_step(float* __restrict__ a, int first, int last, int* __restrict__ lpos,
                              float* __restrict__ lval, int* __restrict__ rpos, float* __restrict__ rval,
                              OrdShared& S, bool placed = false) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    if (!placed) move_median_to_first(a, first, first + 1, first + (last - first) / 2, last - 1);
    S.pivot = a[first];
    S.cross = 0;
  }
  __syncthreads();
  const float p = S.pivot;
  const Segs sg(first + 1, last);
  const int nseg = sg.nseg;
  // 1. Counts per segment.
  for (int g = warp; g < nseg; g += kOrdWarps) {
    const int x0 = sg.x0(g), x1 = sg.x1(g);
    int cge = 0, cle = 0;
    for (int a0 = sg.start(g); a0 < x1; a0 += kStep) {
      VChunk w;
      w.load(a, a0, x0, x1);
#pragma unroll
      for (int q = 0; q < kV4; ++q) {
        unsigned mg, ml;
        w.masks(q, a0, x0, x1, p, mg, ml);
        cge += __popc(mg);
        cle += __popc(ml);
      }
    }
    cge = __reduce_add_sync(0xffffffffu, cge);
    cle = __reduce_add_sync(0xffffffffu, cle);
    if (lane == 0) {
      S.seg_ge[g] = cge;
      S.seg_le[g] = cle;
    }
  }
  __syncthreads();
  block_exclusive_scan<kOrdThreads>(S.seg_ge, nseg, S.warp_i);
  block_exclusive_scan<kOrdThreads>(S.seg_le, nseg, S.warp_i);
  const int total_ge = S.seg_ge[nseg], total_le = S.seg_le[nseg];
  // 2. The segment where cL stops being <= cR: the last segment g whose start has
  //    cL = seg_ge[g] <= cR = total_le - seg_le[g] (segment 0 always qualifies).
  for (int g = tid; g < nseg; g += kOrdThreads)
    if (S.seg_ge[g] <= total_le - S.seg_le[g]) atomicMax(&S.cross, g);
  __syncthreads();
  // 3. K = max over positions x of the crossing segment of min(cL(x), cR(x)) (warp 0).
  if (warp == 0) {
    const int g = S.cross;
    const int x0 = sg.x0(g), x1 = sg.x1(g);
    int cl = S.seg_ge[g], cr = total_le - S.seg_le[g];
    int best = 0;
    for (int a0 = sg.start(g); a0 < x1; a0 += kStep) {
      VChunk w;
      w.load(a, a0, x0, x1);
#pragma unroll
      for (int q = 0; q < kV4; ++q) {
        unsigned mg, ml;
        w.masks(q, a0, x0, x1, p, mg, ml);
        const int packed = __popc(mg) | (__popc(ml) << 16);
        const int inc = warp_incl_scan(packed);
        const int ex = inc - packed;
        const int base = a0 + 128 * q + 4 * lane;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const unsigned below = (1u << c) - 1u;
          if (base + c >= x0 && base + c < x1)
            best = max(best, min(cl + (ex & 0xffff) + __popc(mg & below), cr - (ex >> 16) - __popc(ml & below)));
        }
        const int tot = __shfl_sync(0xffffffffu, inc, 31);
        cl += tot & 0xffff;
        cr -= tot >> 16;
      }
    }
    best = max(best, min(cl, cr));  // the position after the segment
    best = __reduce_max_sync(0xffffffffu, best);
    if (lane == 0) S.K = best;
  }
  __syncthreads();
  const int K = S.K;
  // 4. L[K] (warp 0) and R[K-1] (warp 1): the segment holding the rank, then a scan of it.
  if (warp < 2) {
    const bool kind_ge = warp == 0;
    const int* pre = kind_ge ? S.seg_ge : S.seg_le;
    const int rank = kind_ge ? K : total_le - K;  // ascending rank among values of that kind
    const bool exists = kind_ge ? K < total_ge : K >= 1;
    int pos = INT_MAX;
    if (exists) {
      int lo = 0, hi = nseg - 1;  // the last segment g with pre[g] <= rank
      while (lo < hi) {
        const int m = (lo + hi + 1) >> 1;
        if (pre[m] <= rank) lo = m;
        else hi = m - 1;
      }
      pos = find_rank(a, sg, lo, p, kind_ge, rank - pre[lo]);
    }
    if (lane == 0) {
      if (kind_ge) S.lk = pos;
      else S.rk = pos;
    }
  }
  __syncthreads();
  const int cut = K == 0 ? S.lk : min(S.lk, S.rk);
  if (K == 0) return cut;
  // 5. The K pairs: positions and values, listed by rank.
  for (int g = warp; g < nseg; g += kOrdWarps) {
    int rge = S.seg_ge[g], rle = S.seg_le[g];
    if (rge >= K && total_le - S.seg_le[g + 1] >= K) continue;  // no pair has a value in this segment
    const int x0 = sg.x0(g), x1 = sg.x1(g);
    for (int a0 = sg.start(g); a0 < x1; a0 += kStep) {
      VChunk w;
      w.load(a, a0, x0, x1);
#pragma unroll
      for (int q = 0; q < kV4; ++q) {
        unsigned mg, ml;
        w.masks(q, a0, x0, x1, p, mg, ml);
        const int packed = __popc(mg) | (__popc(ml) << 16);
        const int inc = warp_incl_scan(packed);
        const int eg = rge + ((inc - packed) & 0xffff), el = rle + ((inc - packed) >> 16);
        const int base = a0 + 128 * q + 4 * lane;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const unsigned below = (1u << c) - 1u;
          if ((mg >> c) & 1u) {
            const int r = eg + __popc(mg & below);
            if (r < K) {
              lpos[r] = base + c;
              lval[r] = w.at(q, c);
            }
          }
          if ((ml >> c) & 1u) {
            const int rd = total_le - 1 - (el + __popc(ml & below));
            if (rd < K) {
              rpos[rd] = base + c;
              rval[rd] = w.at(q, c);
            }
          }
        }
        const int tot = __shfl_sync(0xffffffffu, inc, 31);
        rge += tot & 0xffff;
        rle += tot >> 16;
      }
    }
  }
  __syncthreads();
  // 6. The swaps: the k-th value >= pivot goes where the k-th value <= pivot was, and back.
  for (int k0 = tid; k0 < K; k0 += 4 * kOrdThreads) {
    int i[4], j[4];
    float vi[4], vj[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = k0 + u * kOrdThreads;
      if (k < K) {
        i[u] = lpos[k];
        j[u] = rpos[k];
        vi[u] = lval[k];
        vj[u] = rval[k];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (k0 + u * kOrdThreads < K) {
        a[i[u]] = vj[u];
        a[j[u]] = vi[u];
      }
    }
  }
  __syncthreads();
  return cut;
}

// The rest of std::nth_element(a + first, a + nth, a + last) as libstdc++ runs it, from a
// range and depth budget reached so far (pending: a step of [first, last) is prepared -- its
// pivot in place, its depth charged -- and runs first): partition steps while the range holds more than 3
// values; at the depth limit a heap selection of [first, nth] and a swap of a[first] with
// a[nth]; else a final insertion sort.  Ranges of up to kSmemRange values are moved to shared
// memory (sdata, slists) for the rest.  lpos..rval: the pair lists, `big` entries each.  A
// cut outside (first, last) -- impossible for a correct partition -- stops the selection and
// sets *bad, so that no later access leaves the range.
__device__ void introselect_from(float* a, int first, int nth, int last, int depth, bool pending, int* lists, int big,
                                 float* sdata, int* slists, OrdShared& S, bool* bad) {
  if (*bad || first == last || nth == last) return;
  if (pending) {
    const int cut = partition_step(a, first, last, lists, reinterpret_cast<float*>(lists + big), lists + 2 * big,
                                   reinterpret_cast<float*>(lists + 3 * big), S, true);
    if (cut <= first || cut >= last) {
      *bad = true;
      return;
    }
    if (cut <= nth) first = cut;
    else last = cut;
  }
  while (last - first > 3 && last - first > kSmemRange) {
    if (depth == 0) {
      if (threadIdx.x == 0) {
        heap_select_(a + first, nth + 1 - first, last - first);
        const float t = a[first];
        a[first] = a[nth];
        a[nth] = t;
      }
      __syncthreads();
      return;
    }
    --depth;
    const int cut = partition_step(a, first, last, lists, reinterpret_cast<float*>(lists + big), lists + 2 * big,
                                   reinterpret_cast<float*>(lists + 3 * big), S);
    if (cut <= first || cut >= last) {
      *bad = true;
      return;
    }
    if (cut <= nth) first = cut;
    else last = cut;
  }
  const int f0 = first, n = last - first;
  if (n > 3) {
    for (int i = threadIdx.x; i < n; i += kOrdThreads) sdata[i] = a[f0 + i];
    __syncthreads();
    int fr = 0, lr = n;
    const int nr = nth - f0;
    bool heap = false;
    while (lr - fr > 3) {
      if (depth == 0) {
        heap = true;
        break;
      }
      --depth;
      const int cut = partition_step(sdata, fr, lr, slists, reinterpret_cast<float*>(slists + kSmemPairs),
                                     slists + 2 * kSmemPairs, reinterpret_cast<float*>(slists + 3 * kSmemPairs), S);
      if (cut <= fr || cut >= lr) {
        *bad = true;
        break;
      }
      if (cut <= nr) fr = cut;
      else lr = cut;
    }
    if (threadIdx.x == 0 && !*bad) {
      if (heap) {
        heap_select_(sdata + fr, nr + 1 - fr, lr - fr);
        const float t = sdata[fr];
        sdata[fr] = sdata[nr];
        sdata[nr] = t;
      } else {
        insertion_sort(sdata, fr, lr);
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += kOrdThreads) a[f0 + i] = sdata[i];
  } else if (threadIdx.x == 0) {
    insertion_sort(a, first, last);
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------------------
// Exact sequential sums
// ---------------------------------------------------------------------------------------

template <typename Acc>
struct AccTraits;
template <>
struct AccTraits<float> {
  static constexpr int P = 24;       // significand bits
  static constexpr int EMIN = -149;  // exponent of the grid of the subnormals
};
template <>
struct AccTraits<double> {
  static constexpr int P = 53;
  static constexpr int EMIN = -1074;
};

// S = A * 2^eu with A on the grid of S's binade (|A| < 2^P).
template <typename Acc>
__device__ void acc_split(Acc S, int* eu, long long* A) {
  using T = AccTraits<Acc>;
  int ex = 0;
  if (S != Acc(0)) frexp(S, &ex);
  int e = ex - T::P;  // floor(log2|S|) - (P - 1)
  if (S == Acc(0) || e < T::EMIN) e = T::EMIN;
  *eu = e;
  *A = (long long)ldexp(S, -e);
}

// A term (a float value, exactly) against the grid 2^eu of an accumulator of P significand
// bits, packed into one word: q (grid steps of |t|, below 2^(P+2)) in the low P + 2 bits,
// then the rounding class of the remainder (0: none or below half, 1: exactly half, 2:
// above half), the sign, "big" (2^(P+1) steps or more, or not finite: the sum always
// leaves the binade) and "nonzero".
template <int P>
struct Packed {
  using W = typename std::conditional<(P <= 24), uint32_t, uint64_t>::type;
  static constexpr int QB = P + 2;
  static constexpr W QMASK = (W(1) << QB) - 1;
  __device__ static __forceinline__ W make(float t, int eu) {
    const uint32_t b = __float_as_uint(t);
    const W neg = (W)(b >> 31) << (QB + 2);
    const int ex = (b >> 23) & 0xff;
    constexpr W kBig = W(1) << (QB + 3), kNz = W(1) << (QB + 4);
    if (ex == 0xff) return neg | kBig | kNz;
    const uint32_t man = b & 0x7fffffu;
    const uint32_t M = ex ? (man | 0x800000u) : man;
    if (M == 0) return neg;
    const int et = ex ? ex - 150 : -149;
    if (et >= eu) {
      const int sh = et - eu;
      if (sh > P - 22) return neg | kBig | kNz;  // M * 2^sh >= 2^(P+1)
      const W q = (W)M << sh;
      return q > (W(1) << (P + 1)) ? (neg | kBig | kNz) : (q | neg | kNz);
    }
    const int s = eu - et;
    if (s > 25) return neg | kNz;  // below a quarter step: rounds to nothing
    const uint32_t rem = M & ((1u << s) - 1u), half = 1u << (s - 1);
    const W cls = rem < half ? 0 : (rem == half ? 1 : 2);
    return (W)(M >> s) | (cls << QB) | neg | kNz;
  }
  __device__ static __forceinline__ long long q(W w) { return (long long)(w & QMASK); }
  __device__ static __forceinline__ int cls(W w) { return (int)((w >> QB) & 3); }
  __device__ static __forceinline__ bool neg(W w) { return (w >> (QB + 2)) & 1; }
  __device__ static __forceinline__ bool big(W w) { return (w >> (QB + 3)) & 1; }
  __device__ static __forceinline__ bool nz(W w) { return (w >> (QB + 4)) & 1; }
  // Grid steps the term adds to an accumulator of parity `par`.
  __device__ static __forceinline__ long long steps(W w, int par) {
    const long long qq = q(w);
    const int c = cls(w);
    const long long k = qq + (c == 2 ? 1 : (c == 1 ? ((par ^ (int)(qq & 1)) & 1) : 0));
    return neg(w) ? -k : k;
  }
  // The parity map of the term: p -> p ^ (k & 1), or p -> 0 for a tie (round half to even).
  __device__ static __forceinline__ unsigned pmap(W w) {
    const int c = cls(w);
    if (c == 1) return 0u;
    return ((c == 2) ^ (int)(q(w) & 1)) ? 1u : 2u;
  }
};

// Parity maps p -> (m >> p) & 1, two bits; composition "first f, then g".
__device__ __forceinline__ unsigned map_then(unsigned f, unsigned g) {
  return ((g >> (f & 1)) & 1) | (((g >> ((f >> 1) & 1)) & 1) << 1);
}

// The terms of v[pos, end) (at most kOrdThreads * TPT of them), staged in shared memory:
// term i - pos at sbuf[r + (r >> 4)], r = i - pos (a pad word per 16 keeps a thread's run of
// consecutive terms free of bank conflicts).  Loads are coalesced and all in flight at once.
template <int TPT, typename TermFn>
__device__ __forceinline__ void stage_terms(const float* __restrict__ v, long long pos, long long end, TermFn term,
                                            float* sbuf) {
  float tv[TPT];
#pragma unroll
  for (int k = 0; k < TPT; ++k) {
    const long long i = pos + threadIdx.x + (long long)k * kOrdThreads;
    tv[k] = i < end ? __ldcg(v + i) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < TPT; ++k) {
    const int r = threadIdx.x + k * kOrdThreads;
    if (pos + r < end) sbuf[r + (r >> 4)] = term(tv[k]);
  }
}

// Sum of term(v[i]) for i in [lo, hi] in index order, rounded after every add as an Acc
// accumulator starting at 0 does.  Block-wide; every thread gets the result.  sbuf: kSumBuf
// floats of shared memory.
template <typename Acc, typename TermFn>
__device__ Acc exact_sequential_sum(const float* __restrict__ v, long long lo, long long hi, TermFn term, float* sbuf,
                                    OrdShared& S) {
  using Tr = AccTraits<Acc>;
  using PK = Packed<Tr::P>;
  using W = typename PK::W;
  constexpr int TPT = sizeof(W) == 4 ? kTermsPerThreadF : kTermsPerThreadD;
  constexpr long long CH = (long long)kOrdThreads * TPT;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr long long kTop = (1ll << Tr::P) - 1;
  constexpr long long kLow = 1ll << (Tr::P - 1);
  __shared__ Acc s_sum;
  const long long pre_end = min(hi + 1, lo + kSeqPrefix);
  stage_terms<TPT>(v, lo, pre_end, term, sbuf);
  __syncthreads();
  if (tid == 0) {
    Acc acc = Acc(0);
    for (int r = 0; r < (int)(pre_end - lo); ++r) acc = acc + (Acc)sbuf[r + (r >> 4)];
    s_sum = acc;
    S.s_slow = 0;
  }
  __syncthreads();
  long long pos = pre_end;
  while (pos <= hi) {
    const long long chunk_end = min(hi + 1, pos + CH);
    stage_terms<TPT>(v, pos, chunk_end, term, sbuf);
    if (tid == 0) {
      const Acc cur = s_sum;
      if (!isfinite(cur)) {
        S.s_slow = 1;
      } else {
        int eu;
        long long A;
        acc_split(cur, &eu, &A);
        S.s_eu = eu;
        S.s_a = A;
      }
      S.s_cross = LLONG_MAX;
    }
    __syncthreads();
    if (S.s_slow) break;
    const int eu = S.s_eu;
    const long long A0 = S.s_a;
    const long long lowb = eu == Tr::EMIN ? 0 : kLow;
    // This thread's run of consecutive terms, classified once.
    const int r0 = tid * TPT;
    W tm[TPT];
    unsigned fmap = 2u;  // identity: 0 -> 0, 1 -> 1
    bool careful = false;
    // The steps of this thread's terms when no tie needs a parity, saturated at kSat (a
    // double grid step count reaches 2^54 per term; the sum only has to tell whether it
    // stays below 2^P).
    constexpr long long kSat = 1ll << 61;
    long long tfast = 0;
#pragma unroll
    for (int j = 0; j < TPT; ++j) {
      const int r = r0 + j;
      tm[j] = pos + r < chunk_end ? PK::make(sbuf[r + (r >> 4)], eu) : W(0);
      fmap = map_then(fmap, PK::pmap(tm[j]));
      careful |= PK::cls(tm[j]) == 1 || PK::neg(tm[j]) || PK::big(tm[j]);
      tfast = min(tfast + PK::steps(tm[j], 0), kSat);
    }
    // The common chunk: no tie (every step count is fixed), no negative term (the sum only
    // grows) and a total that keeps the sum inside its binade: add the total and move on.
    if (!__syncthreads_or(careful)) {
      long long t = tfast;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t = min(t + __shfl_down_sync(0xffffffffu, t, o), kSat);
      if (lane == 0) S.warp_ll[warp] = t;
      __syncthreads();
      long long total = 0;
#pragma unroll 8
      for (int w = 0; w < kOrdWarps; ++w) total = min(total + S.warp_ll[w], kSat);
      if (A0 + total <= kTop) {
        if (tid == 0) s_sum = (Acc)ldexp((Acc)(A0 + total), eu);
        pos = chunk_end;
        __syncthreads();
        continue;
      }
      __syncthreads();  // a crossing inside the chunk: the full scan below finds it
    }
    // Exclusive scan of the parity maps: the parity before this thread's first term.
    unsigned inc = fmap;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc = map_then(y, inc);
    }
    const unsigned yl = __shfl_up_sync(0xffffffffu, inc, 1);
    const unsigned excl_lane = lane ? yl : 2u;
    if (lane == 31) S.warp_map[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      unsigned wi = S.warp_map[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi = map_then(y, wi);
      }
      const unsigned y = __shfl_up_sync(0xffffffffu, wi, 1);
      S.warp_map2[lane] = lane ? y : 2u;
    }
    __syncthreads();
    const unsigned before = map_then(S.warp_map2[warp], excl_lane);
    const int par0 = (int)((before >> (int)(A0 & 1)) & 1);
    // Steps of this thread's terms, then their exclusive prefix over the block.
    long long tsum = 0;
    {
      int pp = par0;
#pragma unroll
      for (int j = 0; j < TPT; ++j) {
        const long long k = PK::steps(tm[j], pp);
        tsum += k;
        pp = PK::cls(tm[j]) == 1 ? 0 : (pp ^ (int)(k & 1));
      }
    }
    long long incs = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, incs, o);
      if (lane >= o) incs += y;
    }
    if (lane == 31) S.warp_ll[warp] = incs;
    __syncthreads();
    if (warp == 0) {
      long long wi = S.warp_ll[lane];
      const long long w0 = wi;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += y;
      }
      S.warp_ll2[lane] = wi - w0;
    }
    __syncthreads();
    long long A = A0 + S.warp_ll2[warp] + incs - tsum;
    // The first term whose sum leaves the binade.  A term toward zero may end below it, on a
    // finer grid: it must keep 2^(P-1) steps with a whole step to spare (unless the grid is
    // already the finest); a term away from zero must stay below 2^P steps.
    long long cross = LLONG_MAX, a_at = 0;
    int par = par0;
#pragma unroll
    for (int j = 0; j < TPT; ++j) {
      const long long i = pos + r0 + j;
      if (i >= chunk_end || cross != LLONG_MAX) continue;
      const W w = tm[j];
      const long long k = PK::steps(w, par);
      const long long nA = A + k;
      const long long mag = nA < 0 ? -nA : nA;
      const long long absA = A < 0 ? -A : A;
      const bool toward = PK::nz(w) && A != 0 && (PK::neg(w) != (A < 0));
      if (PK::big(w) || mag > kTop || (toward && absA - PK::q(w) - 1 < lowb)) {
        cross = i;
        a_at = A;
      } else {
        A = nA;
        par = PK::cls(w) == 1 ? 0 : (par ^ (int)(k & 1));
      }
    }
    if (cross != LLONG_MAX) atomicMin(&S.s_cross, cross);
    __syncthreads();
    const long long c = S.s_cross;
    if (c == LLONG_MAX) {
      // the last thread with terms holds the final accumulator
      if (tid == (int)((chunk_end - 1 - pos) / TPT)) s_sum = (Acc)ldexp((Acc)A, eu);
      pos = chunk_end;
    } else {
      if (cross == c) {
        const int r = (int)(c - pos);
        s_sum = (Acc)ldexp((Acc)a_at, eu) + (Acc)sbuf[r + (r >> 4)];
      }
      pos = c + 1;
    }
    __syncthreads();
  }
  if (S.s_slow && tid == 0) {  // a non-finite accumulator: finish one term at a time
    Acc acc = s_sum;
    for (long long i = pos; i <= hi; ++i) acc = acc + (Acc)term(__ldcg(v + i));
    s_sum = acc;
  }
  __syncthreads();
  const Acc r = s_sum;
  __syncthreads();
  return r;
}

// The double sum of the floats v[lo..hi], in index order.  Every partial sum is a multiple
// of 2^g, g the lowest set bit of any term, and at most sum |v| in magnitude; when that
// bound is below 2^(52+g) every partial sum is a double, so every order of adding gives the
// exact sum, and a parallel reduction equals the sequential one.  Otherwise the sequential
// scan above runs.
__device__ double ordered_double_sum(const float* __restrict__ v, long long lo, long long hi, float* sbuf,
                                     OrdShared& S) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ double s_abs[kOrdWarps], s_sum[kOrdWarps];
  __shared__ int s_g[kOrdWarps];
  double sa = 0.0, ss = 0.0;
  int g = INT_MAX;
  const long long b0 = lo & ~3ll;  // whole float4 groups from an aligned start
  for (long long i0 = b0 + 4ll * tid; i0 <= hi; i0 += 4ll * 4 * kOrdThreads) {
    float4 q[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const long long i = i0 + 4ll * u * kOrdThreads;
      q[u] = i <= hi ? __ldcg(reinterpret_cast<const float4*>(v + i)) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const long long i = i0 + 4ll * u * kOrdThreads;
      const float f4[4] = {q[u].x, q[u].y, q[u].z, q[u].w};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (i + c < lo || i + c > hi) continue;
        const float f = f4[c];
        const uint32_t b = __float_as_uint(f);
        const int ex = (b >> 23) & 0xff;
        const uint32_t man = b & 0x7fffffu;
        const uint32_t M = ex ? (man | 0x800000u) : man;
        if (ex == 0xff) g = INT_MIN;  // not finite: take the sequential path
        else if (M && g != INT_MIN) g = min(g, (ex ? ex - 150 : -149) + __ffs((int)M) - 1);
        sa += fabs((double)f);
        ss += (double)f;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sa += __shfl_down_sync(0xffffffffu, sa, o);
    ss += __shfl_down_sync(0xffffffffu, ss, o);
    g = min(g, __shfl_down_sync(0xffffffffu, g, o));
  }
  if (lane == 0) {
    s_abs[warp] = sa;
    s_sum[warp] = ss;
    s_g[warp] = g;
  }
  __syncthreads();
  double tot_abs = 0.0, tot = 0.0;
  int gmin = INT_MAX;
  for (int w = 0; w < kOrdWarps; ++w) {
    tot_abs += s_abs[w];
    tot += s_sum[w];
    gmin = min(gmin, s_g[w]);
  }
  __syncthreads();
  if (gmin == INT_MAX) return 0.0;  // every term is zero
  if (gmin != INT_MIN && gmin > -1000 && tot_abs < ldexp(1.0, 52 + gmin)) return tot;
  return exact_sequential_sum<double>(v, lo, hi, [](float f) { return f; }, sbuf, S);
}

// ---------------------------------------------------------------------------------------
// The large partition steps as multi-CTA rounds
// ---------------------------------------------------------------------------------------
//
// While the range of an nth_element call is larger than kSmemRange, its partition steps run
// as rounds of three launches over every search of the batch (and both ends' calls at once):
// count (the last CTA of a task scans the counts and finds K and the cut), lists, and swap
// (the last CTA updates the range and moves the next pivot into place).  A task whose range
// fits shared memory, or whose depth budget is spent, goes inactive; its finisher (one CTA)
// carries on from the same state, so any number of rounds gives the same result.

constexpr int kRoundThreads = 256;
constexpr int kRoundWarps = kRoundThreads / 32;

__device__ __forceinline__ OrderTask* order_tasks(const SearchDesc& sd) {
  return reinterpret_cast<OrderTask*>(sd.lists + order_pair_entries(sd.N));
}

// The pair lists of call t (0: the middle, 1 and 2: the ends): four lists of *big entries.
__device__ __forceinline__ int* task_lists(const SearchDesc& sd, int t, int* big) {
  const int N = sd.N;
  if (t == 0) {
    *big = N / 2 + 1;
    return sd.lists;
  }
  *big = N / 4 + 2;
  return sd.lists + (t == 1 ? 0 : 4 * (N / 4 + 2));
}

// The start of call t's first step or the next one (one thread): if its range is still
// larger than kSmemRange and the depth budget allows, the median of three moves to `first`
// as __unguarded_partition_pivot does, and the step's range and segments are recorded.
__device__ void task_next_step(float* a, OrderTask& T) {
  if (T.error || T.last - T.first <= kSmemRange || T.depth == 0) {
    T.active = 0;
    return;
  }
  --T.depth;
  T.sfirst = T.first;
  T.slast = T.last;
  move_median_to_first(a, T.first, T.first + 1, T.first + (T.last - T.first) / 2, T.last - 1);
  T.pivot = a[T.first];
  const Segs sg(T.first + 1, T.last);
  T.nseg = sg.nseg;
  T.seglen = sg.seglen;
  T.active = 1;
}

// Call t of a search starts on [first, last) with target nth (std::nth_element returns at
// once when first == last or nth == last).
__device__ void task_init(float* a, OrderTask& T, int first, int nth, int last) {
  T.first = first;
  T.last = last;
  T.nth = nth;
  T.depth = last > first ? 2 * (31 - __clz(last - first)) : 0;
  T.error = 0;
  T.ticket = 0;
  T.active = 0;
  if (first == last || nth == last) {
    T.first = T.last;  // nothing to do
    return;
  }
  task_next_step(a, T);
}

// Last-CTA election of a round: true in the one CTA that finishes last.
__device__ __forceinline__ bool last_cta(unsigned* ticket, unsigned total) {
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(ticket, 1u) == total - 1;
  __syncthreads();
  if (s_last) __threadfence();
  return s_last;
}

// The column sums copied to the work array; the last CTA of a search starts the middle call.
__global__ void __launch_bounds__(kRoundThreads) order_init_kernel(const __grid_constant__ SearchBatch b,
                                                                   int min_ties) {
  const SearchDesc& sd = b.s[blockIdx.y];
  const int N = sd.N;
  if (N <= 0 || sd.hdr->ties < min_ties) return;
  OrderTask* tasks = order_tasks(sd);
  const int n4 = N / 4;  // both arrays start 256-byte aligned
  const float4* __restrict__ src = reinterpret_cast<const float4*>(sd.colsum);
  float4* dst = reinterpret_cast<float4*>(sd.work);
  for (int i = blockIdx.x * kRoundThreads + threadIdx.x; i < n4; i += gridDim.x * kRoundThreads) dst[i] = __ldcg(src + i);
  if (blockIdx.x == 0)
    for (int i = 4 * n4 + threadIdx.x; i < N; i += kRoundThreads) sd.work[i] = __ldcg(sd.colsum + i);
  if (last_cta(&tasks[0].ticket, gridDim.x) && threadIdx.x == 0) {
    task_init(sd.work, tasks[0], 0, sd.mid, N);
    tasks[1].active = tasks[2].active = 0;
  }
}

// Zeroes the tickets of a search's calls (before the copy launch uses the first).
__global__ void order_reset_kernel(const __grid_constant__ SearchBatch b) {
  OrderTask* tasks = order_tasks(b.s[blockIdx.y]);
  if (threadIdx.x < 3) {
    tasks[threadIdx.x].ticket = 0;
    tasks[threadIdx.x].active = 0;
  }
}

// Round, launch 1: counts per segment; the last CTA of a task scans them and finds K, the
// cut and the next range.
__global__ void __launch_bounds__(kRoundThreads) round_count_kernel(const __grid_constant__ SearchBatch b, int t0,
                                                                    int nt) {
  const int t = t0 + (int)(blockIdx.y % nt);
  const SearchDesc& sd = b.s[blockIdx.y / nt];
  OrderTask& T = order_tasks(sd)[t];
  if (!*(volatile int*)&T.active) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* __restrict__ a = sd.work;
  const float p = T.pivot;
  const Segs sg(T.sfirst + 1, T.slast);
  const int nseg = sg.nseg;
  for (int g = blockIdx.x * kRoundWarps + warp; g < nseg; g += gridDim.x * kRoundWarps) {
    const int x0 = sg.x0(g), x1 = sg.x1(g);
    int cge = 0, cle = 0;
    for (int a0 = sg.start(g); a0 < x1; a0 += kStep) {
      VChunk w;
      w.load(a, a0, x0, x1);
#pragma unroll
      for (int q = 0; q < kV4; ++q) {
        unsigned mg, ml;
        w.masks(q, a0, x0, x1, p, mg, ml);
        cge += __popc(mg);
        cle += __popc(ml);
      }
    }
    cge = __reduce_add_sync(0xffffffffu, cge);
    cle = __reduce_add_sync(0xffffffffu, cle);
    if (lane == 0) {
      T.seg_ge[g] = cge;
      T.seg_le[g] = cle;
    }
  }
  if (!last_cta(&T.ticket, gridDim.x)) return;
  // The scans, in shared memory, written back for the lists launch.
  __shared__ int s_ge[kMaxSegs + 1], s_le[kMaxSegs + 1];
  __shared__ int s_tmp[kRoundWarps];
  __shared__ int s_cross, s_K, s_lk, s_rk;
  for (int g = threadIdx.x; g < nseg; g += kRoundThreads) {
    s_ge[g] = __ldcg(&T.seg_ge[g]);
    s_le[g] = __ldcg(&T.seg_le[g]);
  }
  if (threadIdx.x == 0) s_cross = 0;
  __syncthreads();
  block_exclusive_scan<kRoundThreads>(s_ge, nseg, s_tmp);
  block_exclusive_scan<kRoundThreads>(s_le, nseg, s_tmp);
  const int total_ge = s_ge[nseg], total_le = s_le[nseg];
  for (int g = threadIdx.x; g <= nseg; g += kRoundThreads) {
    T.seg_ge[g] = s_ge[g];
    T.seg_le[g] = s_le[g];
  }
  for (int g = threadIdx.x; g < nseg; g += kRoundThreads)
    if (s_ge[g] <= total_le - s_le[g]) atomicMax(&s_cross, g);
  __syncthreads();
  if (warp == 0) {  // K = max over the crossing segment of min(cL(x), cR(x))
    const int g = s_cross;
    const int x0 = sg.x0(g), x1 = sg.x1(g);
    int cl = s_ge[g], cr = total_le - s_le[g];
    int best = 0;
    for (int a0 = sg.start(g); a0 < x1; a0 += kStep) {
      VChunk w;
      w.load(a, a0, x0, x1);
#pragma unroll
      for (int q = 0; q < kV4; ++q) {
        unsigned mg, ml;
        w.masks(q, a0, x0, x1, p, mg, ml);
        const int packed = __popc(mg) | (__popc(ml) << 16);
        const int inc = warp_incl_scan(packed);
        const int ex = inc - packed;
        const int base = a0 + 128 * q + 4 * lane;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const unsigned below = (1u << c) - 1u;
          if (base + c >= x0 && base + c < x1)
            best = max(best, min(cl + (ex & 0xffff) + __popc(mg & below), cr - (ex >> 16) - __popc(ml & below)));
        }
        const int tot = __shfl_sync(0xffffffffu, inc, 31);
        cl += tot & 0xffff;
        cr -= tot >> 16;
      }
    }
    best = max(best, min(cl, cr));
    best = __reduce_max_sync(0xffffffffu, best);
    if (lane == 0) s_K = best;
  }
  __syncthreads();
  const int K = s_K;
  if (warp < 2) {  // L[K] (warp 0) and R[K-1] (warp 1)
    const bool kind_ge = warp == 0;
    const int* pre = kind_ge ? s_ge : s_le;
    const int rank = kind_ge ? K : total_le - K;
    const bool exists = kind_ge ? K < total_ge : K >= 1;
    int pos = INT_MAX;
    if (exists) {
      int lo = 0, hi = nseg - 1;
      while (lo < hi) {
        const int m = (lo + hi + 1) >> 1;
        if (pre[m] <= rank) lo = m;
        else hi = m - 1;
      }
      pos = find_rank(a, sg, lo, p, kind_ge, rank - pre[lo]);
    }
    if (lane == 0) {
      if (kind_ge) s_lk = pos;
      else s_rk = pos;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int cut = K == 0 ? s_lk : min(s_lk, s_rk);
    T.K = K;
    T.cut = cut;
    if (cut <= T.sfirst || cut >= T.slast) {  // impossible for a correct partition
      T.error = 1;
      T.K = 0;
    } else if (cut <= T.nth) {
      T.first = cut;
    } else {
      T.last = cut;
    }
    T.ticket = 0;
  }
}

// Round, launch 2: the K pairs' positions and values, listed by rank.
__global__ void __launch_bounds__(kRoundThreads) round_lists_kernel(const __grid_constant__ SearchBatch b, int t0,
                                                                    int nt) {
  const int t = t0 + (int)(blockIdx.y % nt);
  const SearchDesc& sd = b.s[blockIdx.y / nt];
  OrderTask& T = order_tasks(sd)[t];
  if (!*(volatile int*)&T.active) return;
  const int K = T.K;
  if (K == 0) return;
  int big;
  int* lists = task_lists(sd, t, &big);
  int* __restrict__ lpos = lists;
  float* __restrict__ lval = reinterpret_cast<float*>(lists + big);
  int* __restrict__ rpos = lists + 2 * big;
  float* __restrict__ rval = reinterpret_cast<float*>(lists + 3 * big);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float* __restrict__ a = sd.work;
  const float p = T.pivot;
  const Segs sg(T.sfirst + 1, T.slast);
  const int nseg = sg.nseg;
  const int total_le = T.seg_le[nseg];
  for (int g = blockIdx.x * kRoundWarps + warp; g < nseg; g += gridDim.x * kRoundWarps) {
    int rge = T.seg_ge[g], rle = T.seg_le[g];
    if (rge >= K && total_le - T.seg_le[g + 1] >= K) continue;
    const int x0 = sg.x0(g), x1 = sg.x1(g);
    for (int a0 = sg.start(g); a0 < x1; a0 += kStep) {
      VChunk w;
      w.load(a, a0, x0, x1);
#pragma unroll
      for (int q = 0; q < kV4; ++q) {
        unsigned mg, ml;
        w.masks(q, a0, x0, x1, p, mg, ml);
        const int packed = __popc(mg) | (__popc(ml) << 16);
        const int inc = warp_incl_scan(packed);
        const int eg = rge + ((inc - packed) & 0xffff), el = rle + ((inc - packed) >> 16);
        const int base = a0 + 128 * q + 4 * lane;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const unsigned below = (1u << c) - 1u;
          if ((mg >> c) & 1u) {
            const int r = eg + __popc(mg & below);
            if (r < K) {
              lpos[r] = base + c;
              lval[r] = w.at(q, c);
            }
          }
          if ((ml >> c) & 1u) {
            const int rd = total_le - 1 - (el + __popc(ml & below));
            if (rd < K) {
              rpos[rd] = base + c;
              rval[rd] = w.at(q, c);
            }
          }
        }
        const int tot = __shfl_sync(0xffffffffu, inc, 31);
        rge += tot & 0xffff;
        rle += tot >> 16;
      }
    }
  }
}

// Round, launch 3: the swaps; the last CTA of a task starts its next step.
__global__ void __launch_bounds__(kRoundThreads) round_swap_kernel(const __grid_constant__ SearchBatch b, int t0,
                                                                   int nt) {
  const int t = t0 + (int)(blockIdx.y % nt);
  const SearchDesc& sd = b.s[blockIdx.y / nt];
  OrderTask& T = order_tasks(sd)[t];
  if (!*(volatile int*)&T.active) return;
  const int K = T.K;
  int big;
  int* lists = task_lists(sd, t, &big);
  const int* __restrict__ lpos = lists;
  const float* __restrict__ lval = reinterpret_cast<const float*>(lists + big);
  const int* __restrict__ rpos = lists + 2 * big;
  const float* __restrict__ rval = reinterpret_cast<const float*>(lists + 3 * big);
  float* __restrict__ a = sd.work;
  const int stride = gridDim.x * kRoundThreads;
  for (int k0 = blockIdx.x * kRoundThreads + threadIdx.x; k0 < K; k0 += 4 * stride) {
    int i[4], j[4];
    float vi[4], vj[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = k0 + u * stride;
      if (k < K) {
        i[u] = __ldcg(lpos + k);
        j[u] = __ldcg(rpos + k);
        vi[u] = __ldcg(lval + k);
        vj[u] = __ldcg(rval + k);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (k0 + u * stride < K) {
        a[i[u]] = vj[u];
        a[j[u]] = vi[u];
      }
    }
  }
  if (last_cta(&T.ticket, gridDim.x) && threadIdx.x == 0) {
    T.ticket = 0;
    task_next_step(a, T);
  }
}

// The rest of each call after the rounds, one CTA per call: blockIdx.x selects the call of
// this launch (t0 + blockIdx.x).  After the middle call, its CTA starts both end calls.
__global__ void __launch_bounds__(kOrdThreads, 1) order_finish_kernel(const __grid_constant__ SearchBatch b, int t0,
                                                                     int min_ties) {
  const SearchDesc& sd = b.s[blockIdx.y];
  const int N = sd.N;
  if (N <= 0 || sd.hdr->ties < min_ties || *(volatile int*)&sd.hdr->error) return;
  __shared__ OrdShared S;
  extern __shared__ __align__(16) float dyn[];
  float* sdata = dyn;                                      // kSmemRange values
  int* slists = reinterpret_cast<int*>(dyn + kSmemRange);  // 4 * kSmemPairs entries
  const int t = t0 + (int)blockIdx.x;
  OrderTask* tasks = order_tasks(sd);
  OrderTask& T = tasks[t];
  bool bad = T.error != 0;
  int big;
  int* lists = task_lists(sd, t, &big);
  // A task still active after the rounds has its next step prepared: the range of that step
  // is [sfirst, slast) = [first, last).
  introselect_from(sd.work, T.first, T.nth, T.last, T.depth, T.active != 0, lists, big, sdata, slists, S, &bad);
  if (bad) {
    if (threadIdx.x == 0) atomicExch(&sd.hdr->error, 2);  // the results of this search are invalid
    return;
  }
  if (t == 0 && threadIdx.x == 0) {
    task_init(sd.work, tasks[1], 0, sd.first, sd.mid - 1);
    task_init(sd.work, tasks[2], sd.mid + 1, sd.last, N);
  }
}

// Kernel 3, one CTA per search: the median, the mean and the deviation exactly as the
// reference forms them, from the work array in its nth_element order.
__global__ void __launch_bounds__(kOrdThreads, 1) order_moments_kernel(const __grid_constant__ SearchBatch b,
                                                                      int min_ties) {
  const SearchDesc& sd = b.s[blockIdx.y];
  const int N = sd.N;
  if (N <= 0 || sd.hdr->ties < min_ties || *(volatile int*)&sd.hdr->error) return;
  __shared__ OrdShared S;
  extern __shared__ __align__(16) float dyn[];
  float* sbuf = dyn;  // kSumBuf floats
  const float* __restrict__ a = sd.work;
  const int first = sd.first, last = sd.last;
  const float median = __ldcg(a + sd.mid);
  const int n = last + 1 - first;
  // float sum = std::accumulate(a + first, a + last + 1, 0.0): a double sum in order.
  const double dsum = ordered_double_sum(a, first, last, sbuf, S);
  const float m = __fdiv_rn((float)dsum, (float)n);
  // accum += (f - m) * (f - m), float, in order.
  const float accum = exact_sequential_sum<float>(a, first, last, [m](float f) {
    const float d = __fsub_rn(f, m);
    return __fmul_rn(d, d);
  }, sbuf, S);
  if (threadIdx.x == 0) {
    const float std_dev = sqrtf(__fdiv_rn(accum, (float)n));
    SearchHeader* hdr = sd.hdr;
    hdr->median = median;
    hdr->mean = m;
    hdr->std_dev = std_dev;
    hdr->threshold = (float)(sd.snr_threshold * (double)std_dev + (double)median);  // dedoppler.cu:273
    hdr->order_exact = 1;
  }
}

}  // namespace

namespace {
// Rounds that bring a range of n values to kSmemRange, with slack (a task that needs more
// finishes in its finisher's own steps).
int rounds_for(long long n) {
  int r = 0;
  while (n > kSmemRange) {
    n = n / 2 + 1;
    ++r;
  }
  return r + 1;
}
}  // namespace

cudaError_t search_stats_exact(const SearchBatch& b, int num_sms, cudaStream_t stream) {
  if (b.count <= 0) return cudaSuccess;
  const int smem_sel = (int)(sizeof(float) * kSmemRange + sizeof(int) * 4 * kSmemPairs);
  const int smem_sum = (int)(sizeof(float) * kSumBuf);
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(order_finish_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_sel)) !=
          cudaSuccess ||
      (e = cudaFuncSetAttribute(order_moments_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_sum)) !=
          cudaSuccess)
    return e;
  const int n = b.count;
  const long long max_steps = (b.maxN + kStep - 1) / kStep;  // warp steps of the largest range
  auto grid_x = [&](int tasks) {
    long long g = (4ll * num_sms + (long long)tasks * n - 1) / ((long long)tasks * n);
    const long long cap = std::max(1ll, (max_steps + kRoundWarps - 1) / kRoundWarps);
    return (int)std::max(1ll, std::min(g, cap));
  };
  const int min_ties = exact_statistics_always() ? INT_MIN : kExactStatsTies;
  order_reset_kernel<<<dim3(1, n), 32, 0, stream>>>(b);
  const int g1 = grid_x(1);
  order_init_kernel<<<dim3(g1, n), kRoundThreads, 0, stream>>>(b, min_ties);
  for (int r = rounds_for(b.maxN); r > 0; --r) {
    round_count_kernel<<<dim3(g1, n), kRoundThreads, 0, stream>>>(b, 0, 1);
    round_lists_kernel<<<dim3(g1, n), kRoundThreads, 0, stream>>>(b, 0, 1);
    round_swap_kernel<<<dim3(g1, n), kRoundThreads, 0, stream>>>(b, 0, 1);
  }
  order_finish_kernel<<<dim3(1, n), kOrdThreads, smem_sel, stream>>>(b, 0, min_ties);
  const int g2 = grid_x(2);
  for (int r = rounds_for(b.maxN / 2 + 1); r > 0; --r) {
    round_count_kernel<<<dim3(g2, 2 * n), kRoundThreads, 0, stream>>>(b, 1, 2);
    round_lists_kernel<<<dim3(g2, 2 * n), kRoundThreads, 0, stream>>>(b, 1, 2);
    round_swap_kernel<<<dim3(g2, 2 * n), kRoundThreads, 0, stream>>>(b, 1, 2);
  }
  order_finish_kernel<<<dim3(2, n), kOrdThreads, smem_sel, stream>>>(b, 1, min_ties);
  order_moments_kernel<<<dim3(1, n), kOrdThreads, smem_sum, stream>>>(b, min_ties);
  return cudaGetLastError();
}

namespace {
std::atomic<bool> g_exact_always{false};
}
void set_exact_statistics_always(bool always) { g_exact_always.store(always); }
bool exact_statistics_always() { return g_exact_always.load(); }

cudaError_t search_stats_batch(const SearchBatch& b, int num_sms, cudaStream_t stream) {
  cudaError_t e = search_stats_emulated(b, num_sms, stream);
  if (e == cudaSuccess) e = search_stats_exact(b, num_sms, stream);
  return e;
}

}  // namespace scb
