// Bounding-volume tree of every block's cells: a 4-ary radix tree over the
// cells' Morton keys (storage order), built on the device once per
// registration and refitted to the current coordinates on every call.
//
// A node's range of storage cells is split at the highest bit in which the
// first and last keys differ (in the middle when they are equal), and each
// half again, giving two to four children; a range of at most kMaxLeafCells
// cells is a leaf.  Nodes therefore follow the Morton prefixes: no node mixes
// cells from two distant parts of the curve, as fixed-count groups do on
// sparse or curved blocks.
//
// Layout: slot s holds two float4, (lo.x, lo.y, lo.z, hi.x) and
// (hi.y, hi.z, link, count) with link and count stored as int bits:
//   count > 0   leaf of `count` storage cells starting at cell `link`;
//   count < 0   internal node with -count children in slots link .. link+3;
//   count == 0  empty slot (empty box, never entered).
// The children of a node fill one group of four slots, one 128-byte line.
// Group b (slots 4b .. 4b+3) holds the root of block b in slot 4b.
#include "kernels.cuh"

namespace tb {

// first index in [a, b) whose key is >= v (keys sorted)
__device__ __forceinline__ int lower_bound_key(const unsigned long long* __restrict__ key, int a, int b,
                                               unsigned long long v) {
  while (a < b) {
    const int m = a + ((b - a) >> 1);
    if (key[m] < v) a = m + 1;
    else b = m;
  }
  return a;
}

__device__ __forceinline__ int split_range(const unsigned long long* __restrict__ key, int a, int b) {
  const unsigned long long ka = key[a], kb = key[b - 1];
  if (ka == kb) return a + ((b - a) >> 1);
  const int hb = 63 - __clzll((long long)(ka ^ kb));
  const unsigned long long thr = (kb >> hb) << hb;  // the common prefix with bit hb set
  return lower_bound_key(key, a, b, thr);
}

// One level of the build: every node of the level is either a leaf (its link
// written now, its first cell marked) or an internal node whose two to four
// child ranges go to kids.
__global__ void k_tree_split(const unsigned long long* __restrict__ key, int n, const int* __restrict__ ca,
                             const int* __restrict__ cb, const int* __restrict__ cslot, int2* __restrict__ kids,
                             int* __restrict__ nk, int* __restrict__ isint, int2* __restrict__ tlink,
                             int* __restrict__ leaf_at) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int a = ca[i], b = cb[i];
    if (b - a <= kMaxLeafCells) {
      tlink[cslot[i]] = make_int2(a, b - a);
      leaf_at[a] = cslot[i];
      nk[i] = 0;
      isint[i] = 0;
      continue;
    }
    const int s = split_range(key, a, b);
    int2 half[2] = {make_int2(a, s), make_int2(s, b)};
    int k = 0;
    for (int h = 0; h < 2; h++) {
      const int ha = half[h].x, hb = half[h].y;
      if (hb - ha <= kMaxLeafCells) {
        kids[4 * i + k++] = half[h];
      } else {
        const int t = split_range(key, ha, hb);
        kids[4 * i + k++] = make_int2(ha, t);
        kids[4 * i + k++] = make_int2(t, hb);
      }
    }
    nk[i] = k;
    isint[i] = 1;
  }
}

// Internal nodes of the level get child group g = g0 + ioff[i]: their link,
// the group's parent and child count, and the next level's entries.
__global__ void k_tree_link(int n, const int* __restrict__ cslot, const int2* __restrict__ kids,
                            const int* __restrict__ nk, const int* __restrict__ isint,
                            const int* __restrict__ ioff, const int* __restrict__ koff, int g0,
                            int2* __restrict__ tlink, int* __restrict__ gparent, int* __restrict__ gnk,
                            int* __restrict__ na, int* __restrict__ nb, int* __restrict__ nslot) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!isint[i]) continue;
    const int g = g0 + ioff[i];
    const int k = nk[i];
    tlink[cslot[i]] = make_int2(4 * g, -k);
    gparent[g] = cslot[i];
    gnk[g] = k;
    for (int c = 0; c < k; c++) {
      const int2 r = kids[4 * i + c];
      na[koff[i] + c] = r.x;
      nb[koff[i] + c] = r.y;
      nslot[koff[i] + c] = 4 * g + c;
    }
  }
}

// every slot: empty box plus its link
__global__ void k_tree_init(const int2* __restrict__ tlink, long long nslots, float4* __restrict__ tnode) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nslots;
       s += (long long)gridDim.x * blockDim.x) {
    const int2 l = tlink[s];
    tnode[2 * s] = make_float4(INFINITY, INFINITY, INFINITY, -INFINITY);
    tnode[2 * s + 1] = make_float4(-INFINITY, -INFINITY, __int_as_float(l.x), __int_as_float(l.y));
  }
}

__global__ void k_tree_init64(long long nslots, double* __restrict__ t64) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nslots;
       s += (long long)gridDim.x * blockDim.x)
    for (int k = 0; k < 6; k++) t64[6 * s + k] = (k < 3) ? 1e300 : -1e300;
}

// leaves in storage order: (first cell, cell count, slot, block)
__global__ void k_leaf_flags(const int* __restrict__ leaf_at, long long ctot, int* __restrict__ flag) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x)
    flag[c] = leaf_at[c] >= 0;
}

__global__ void k_leaf_list(const int* __restrict__ leaf_at, const int* __restrict__ loff, long long ctot,
                            const int2* __restrict__ tlink, const blk_t* __restrict__ cell_blk,
                            int4* __restrict__ leaves) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x) {
    const int s = leaf_at[c];
    if (s >= 0) leaves[loff[c]] = make_int4((int)c, tlink[s].y, s, cell_blk[c]);
  }
}

// One-launch refit.  At build time every child group g >= g_root (the root
// groups hold the blocks' roots and have no parent) counts its internal
// slots (nint[g]); the groups with none start the refit.  Per call, each
// starting group writes the union of its four slots into its parent slot,
// then counts itself done at the parent's group; the child that completes a
// group (its nint-th) refits that group too, and so on up to a root group.
// No thread waits for another: the last one to arrive carries on, and the
// fence before the count makes its children's unions visible to it (the
// slots are read through L2).
__global__ void k_group_nint(const float4* __restrict__ tnode, int g_root, int ngroups, int* __restrict__ nint,
                             int* __restrict__ start, int* __restrict__ nstart) {
  for (int g = g_root + blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += gridDim.x * blockDim.x) {
    int n = 0;
    for (int k = 0; k < 4; k++) n += __float_as_int(tnode[2 * (4ll * g + k) + 1].w) < 0;
    nint[g] = n;
    if (n == 0) start[atomicAdd(nstart, 1)] = g;
  }
}

__global__ void k_refit_fused(const int* __restrict__ start, int nstart, const int* __restrict__ gparent,
                              const int* __restrict__ nint, int g_root, int* __restrict__ cnt, float4* tnode,
                              double* tnode64) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nstart; i += gridDim.x * blockDim.x) {
    int g = start[i];
    for (int guard = 0; guard < 64; guard++) {  // at most one step per tree level
      const int p = gparent[g];
      float b[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
      for (int k = 0; k < 4; k++) {
        const float4 A = __ldcg(&tnode[2 * (4ll * g + k)]), B = __ldcg(&tnode[2 * (4ll * g + k) + 1]);
        b[0] = fminf(b[0], A.x); b[1] = fminf(b[1], A.y); b[2] = fminf(b[2], A.z);
        b[3] = fmaxf(b[3], A.w); b[4] = fmaxf(b[4], B.x); b[5] = fmaxf(b[5], B.y);
      }
      tnode[2 * (long long)p] = make_float4(b[0], b[1], b[2], b[3]);
      *reinterpret_cast<float2*>(&tnode[2 * (long long)p + 1]) = make_float2(b[4], b[5]);  // keep the link
      if (tnode64) {
        double d[6] = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300};
        for (int k = 0; k < 4; k++) {
          const double* c = tnode64 + 6 * (4ll * g + k);
          for (int j = 0; j < 3; j++) {
            d[j] = dmin(d[j], __ldcg(c + j));
            d[j + 3] = dmax(d[j + 3], __ldcg(c + j + 3));
          }
        }
        for (int j = 0; j < 6; j++) tnode64[6 * (long long)p + j] = d[j];
      }
      const int G = p >> 2;  // the group holding the parent slot
      if (G < g_root) break;   // a block's root: done
      __threadfence();
      if (atomicAdd(&cnt[G], 1) + 1 != nint[G]) break;  // a sibling subtree is still being refitted
      __threadfence();
      g = G;
    }
  }
}

// first leaf of every block that has leaves (leaves are in storage order,
// which is block-major)
__global__ void k_block_leaves(const int4* __restrict__ leaves, long long nleaf, int* __restrict__ first) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nleaf;
       i += (long long)gridDim.x * blockDim.x) {
    const int b = leaves[i].w;
    if (i == 0 || leaves[i - 1].w != b) first[b] = (int)i;
  }
}

}  // namespace tb
