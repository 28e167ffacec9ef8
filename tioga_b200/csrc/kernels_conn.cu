// Connectivity kernels: hole maps (src/holeMap.C:40-188, MeshBlock.C:637-772,
// utils.c:192-295), box pairs (exchangeBoxes.C:34-272, utils.c:297-384,
// MeshBlock.C:774-838), query gathering (exchangeSearchData.C:27-263,
// MeshBlock.C:953-1117), the bounding-volume tree refit and the fused
// tree-search + Newton containment kernel (search.C:78-269,
// searchADTrecursion.C:26-101, checkContainment.C:27-96, math.c:25-294).
#include <cub/block/block_scan.cuh>

#include "kernels.cuh"

namespace tb {

// ===========================================================================
// hole maps
// ===========================================================================
// Wall-node bounds of every wall-bearing block: blockIdx.y indexes the wall
// table (first wall node, wall nodes, cells: first, count; hole map index)
__global__ void k_wall_bounds(const double* __restrict__ x, const int* __restrict__ wall_list,
                              const WallBlock* __restrict__ wt, unsigned long long* __restrict__ bb_all) {
  const WallBlock W = wt[blockIdx.y];
  unsigned long long* bb = bb_all + 6 * W.hm;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < W.nwall; i += gridDim.x * blockDim.x) {
    const double* p = x + 3 * (long long)wall_list[W.wall_off + i];
    for (int j = 0; j < 3; j++) {
      lo[j] = dmin(lo[j], p[j]);
      hi[j] = dmax(hi[j], p[j]);
    }
  }
  for (int j = 0; j < 3; j++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[j] = dmin(lo[j], __shfl_xor_sync(0xffffffffu, lo[j], o));
      hi[j] = dmax(hi[j], __shfl_xor_sync(0xffffffffu, hi[j], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int j = 0; j < 3; j++) {
      atomicMin(&bb[j], dkey(lo[j]));
      atomicMax(&bb[j + 3], dkey(hi[j]));
    }
  }
}

// extents and sizes exactly as holeMap.C:118-140, one thread per hole map
__global__ void k_holemap_setup(const unsigned long long* __restrict__ bb, HoleMapInfo* __restrict__ hm, int nhm) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nhm) return;
  HoleMapInfo& h = hm[t];
  double ds[3];
  for (int j = 0; j < 3; j++) {
    h.ext[j] = dkey_inv(bb[6 * t + j]);
    h.ext[j + 3] = dkey_inv(bb[6 * t + j + 3]);
    ds[j] = h.ext[j + 3] - h.ext[j];
  }
  double dsmax = dmax(ds[0], ds[1]);
  dsmax = dmax(dsmax, ds[2]);
  double dsbox = dsmax / kHoleMapSize;
  for (int j = 0; j < 3; j++) {
    h.ext[j] -= (2 * dsbox);
    h.ext[j + 3] += (2 * dsbox);
    h.nx[j] = (int)floor(dmax((h.ext[j + 3] - h.ext[j]) / dsbox, 1));
  }
  h.exist = 1;
}

// wall-touching cells mark their index box with 2 (MeshBlock.C:666-772):
// one thread per cell of the wall-cell list (cells of wall-bearing blocks
// with a wall node).  Maps past the slab are left alone (the host rejects
// such a map before it is used).
__global__ void k_holemap_mark(const double* __restrict__ x, const int* __restrict__ conn8,
                               const unsigned char* __restrict__ cell_nv, const int* __restrict__ wall_cells,
                               int nwc, const blk_t* __restrict__ cell_blk, const BlockInfo* __restrict__ bi,
                               const HoleMapInfo* __restrict__ hm_all, unsigned char* __restrict__ sam_all,
                               size_t cap) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nwc; i += gridDim.x * blockDim.x) {
    const long long c = wall_cells[i];
    const int t = bi[cell_blk[c]].hm;
    const HoleMapInfo h = hm_all[t];
    if ((size_t)h.nx[0] * h.nx[1] * h.nx[2] > cap) continue;
    unsigned char* __restrict__ sam = sam_all + (size_t)t * cap;
    double ds[3];
    for (int k = 0; k < 3; k++) ds[k] = (h.ext[k + 3] - h.ext[k]) / h.nx[k];
    const int nv = cell_nv[c];
    const int* cv = conn8 + 8 * c;
    int imin[3] = {kBigInt, kBigInt, kBigInt}, imax[3] = {-kBigInt, -kBigInt, -kBigInt};
    for (int m = 0; m < nv; m++) {
      const double* p = x + 3 * (long long)cv[m];
      for (int k = 0; k < 3; k++) {
        int iv = (int)floor((p[k] - h.ext[k]) / ds[k]);
        imin[k] = min(imin[k], iv);
        imax[k] = max(imax[k], iv);
      }
    }
    for (int j = 0; j < 3; j++) {
      imin[j] = max(imin[j], 0);
      imax[j] = min(imax[j], h.nx[j] - 1);
    }
    for (int kk = imin[2]; kk < imax[2] + 1; kk++)
      for (int jj = imin[1]; jj < imax[1] + 1; jj++)
        for (int ii = imin[0]; ii < imax[0] + 1; ii++)
          sam[(size_t)kk * h.nx[1] * h.nx[0] + (size_t)jj * h.nx[0] + ii] = 2;
  }
}

// cells of wall-bearing blocks that touch a wall node
__global__ void k_wall_cell_flags(const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
                                  const blk_t* __restrict__ cell_blk, const BlockInfo* __restrict__ bi,
                                  const unsigned char* __restrict__ wallf, long long ctot, int* __restrict__ flag) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x) {
    int w = 0;
    if (bi[cell_blk[c]].hm >= 0) {
      const int nv = cell_nv[c];
      for (int m = 0; m < nv; m++) w |= wallf[conn8[8 * c + m]];
    }
    flag[c] = w ? 1 : 0;
  }
}

__global__ void k_wall_cell_list(const int* __restrict__ flag, const int* __restrict__ off, long long ctot,
                                 int* __restrict__ list) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x)
    if (flag[c]) list[off[c]] = (int)c;
}

// first wall cell of every hole map (the list is block-major, and maps are
// numbered in block order)
__global__ void k_wall_map_first(const int* __restrict__ wall_cells, int nwc, const blk_t* __restrict__ cell_blk,
                                 const BlockInfo* __restrict__ bi, int* __restrict__ first) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nwc; i += gridDim.x * blockDim.x) {
    const int t = bi[cell_blk[wall_cells[i]]].hm;
    if (i == 0 || bi[cell_blk[wall_cells[i - 1]]].hm != t) first[t] = i;
  }
}

// The index box every wall cell marks (MeshBlock.C:666-772, the same
// floor((x - lo) / ds) per vertex, clamped to the map), packed into 48 bits:
// imin x, y, z | imax x, y, z, a byte each (maps have at most 197 cells per
// axis).  An empty box gets imin z = 255, imax z = 0.
__global__ void k_holemap_boxes(const double* __restrict__ x, const int* __restrict__ conn8,
                                const unsigned char* __restrict__ cell_nv, const int* __restrict__ wall_cells, int nwc,
                                const blk_t* __restrict__ cell_blk, const BlockInfo* __restrict__ bi,
                                const HoleMapInfo* __restrict__ hm_all, unsigned long long* __restrict__ box) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nwc; i += gridDim.x * blockDim.x) {
    const long long c = wall_cells[i];
    const HoleMapInfo h = hm_all[bi[cell_blk[c]].hm];
    double ds[3];
    for (int k = 0; k < 3; k++) ds[k] = (h.ext[k + 3] - h.ext[k]) / h.nx[k];
    const int nv = cell_nv[c];
    const int* cv = conn8 + 8 * c;
    int imin[3] = {kBigInt, kBigInt, kBigInt}, imax[3] = {-kBigInt, -kBigInt, -kBigInt};
    for (int m = 0; m < nv; m++) {
      const double* p = x + 3 * (long long)cv[m];
      for (int k = 0; k < 3; k++) {
        int iv = (int)floor((p[k] - h.ext[k]) / ds[k]);
        imin[k] = min(imin[k], iv);
        imax[k] = max(imax[k], iv);
      }
    }
    bool empty = false;
    for (int j = 0; j < 3; j++) {
      imin[j] = max(imin[j], 0);
      imax[j] = min(imax[j], h.nx[j] - 1);
      empty = empty || imin[j] > imax[j] || h.nx[j] > 255;
    }
    unsigned long long v = 0;
    if (empty) {
      v = 255ull << 16;
    } else {
      for (int j = 0; j < 3; j++)
        v |= ((unsigned long long)imin[j] << (8 * j)) | ((unsigned long long)imax[j] << (24 + 8 * j));
    }
    box[i] = v;
  }
}

// ---------------------------------------------------------------------------
// Bit-parallel plane fill for isym = 1, 2, 3 (utils.c:192-295 with the
// in-plane 4-neighbour sweeps): one CTA per plane normal to the symmetry
// axis.  Every line of the plane is a 224-bit mask (7 words): passable cells
// (not wall-marked, or seeded) and filled cells (seeds: the six box faces,
// utils.c:206-226).  A line is filled in one step: adding the seeds to the
// passable mask carries through each run of passable cells above its lowest
// seed, and the same on the bit-reversed line covers the run below its
// highest seed, so every run holding a seed becomes filled.  Rows and columns
// alternate (a shuffle bit transpose between them) until a round changes
// nothing: the closure of the seeds through unmarked cells, the fixed point
// of the reference's Gauss-Seidel sweeps.  The plane is written back as the
// final map (1 = hole: wall-marked or unreached), so no separate pass is
// needed, and cells that are not marked 2 by this call count as unmarked
// whatever the map held before.
// ---------------------------------------------------------------------------
constexpr int kHW = 7;            // words per line: 224 >= 197 cells
constexpr int kHL = 32 * kHW;     // lines per plane at most (row and column tables)

__device__ __forceinline__ bool line_fill(unsigned* __restrict__ F, const unsigned* __restrict__ M) {
  unsigned S[kHW], U[kHW], Mr[kHW], Sr[kHW];
#pragma unroll
  for (int w = 0; w < kHW; w++) S[w] = F[w] & M[w];
  unsigned long long c = 0;
#pragma unroll
  for (int w = 0; w < kHW; w++) {  // upwards from the lowest seed of every run
    const unsigned long long t = (unsigned long long)M[w] + S[w] + c;
    U[w] = (((unsigned)t ^ M[w]) & M[w]) | S[w];
    c = t >> 32;
  }
#pragma unroll
  for (int w = 0; w < kHW; w++) {
    Mr[w] = __brev(M[kHW - 1 - w]);
    Sr[w] = __brev(S[kHW - 1 - w]);
  }
  c = 0;
  bool ch = false;
#pragma unroll
  for (int w = 0; w < kHW; w++) {  // downwards from the highest seed (on the reversed line)
    const unsigned long long t = (unsigned long long)Mr[w] + Sr[w] + c;
    Sr[w] = (((unsigned)t ^ Mr[w]) & Mr[w]) | Sr[w];
    c = t >> 32;
  }
#pragma unroll
  for (int w = 0; w < kHW; w++) {
    const unsigned v = U[w] | __brev(Sr[kHW - 1 - w]);
    ch = ch || (v != F[w]);
    F[w] = v;
  }
  return ch;
}

// dst[c][w'] bit b' = src[32 w' + b'][w] bit (c - 32 w) for source lines <
// nsrc and destination lines < ndst: one warp per 32x32 tile, transposed in
// five shuffle stages (off-diagonal half blocks swapped, then recursively).
__device__ __forceinline__ void bit_transpose(const unsigned (*__restrict__ src)[kHW], int nsrc,
                                              unsigned (*__restrict__ dst)[kHW], int ndst) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int wmax = (ndst + 31) >> 5, lmax = (nsrc + 31) >> 5;  // tiles that hold any line
  for (int t = warp; t < wmax * lmax; t += nwarps) {
    const int w = t % wmax, wp = t / wmax;  // source word, source line block
    const int r = 32 * wp + lane;
    unsigned x = (r < nsrc) ? src[r][w] : 0u;
#pragma unroll
    for (int j = 16, m = 0x0000ffff; j > 0; j >>= 1, m ^= (m << j)) {
      const unsigned y = __shfl_xor_sync(0xffffffffu, x, j);
      x = (lane & j) ? ((x & ~(unsigned)m) | ((y & ~(unsigned)m) >> j)) : ((x & (unsigned)m) | ((y & (unsigned)m) << j));
    }
    if (32 * w + lane < ndst) dst[32 * w + lane][wp] = x;
  }
}

__global__ void __launch_bounds__(256, 4) k_holemap_fill_bits(unsigned char* __restrict__ sam_all,
                                                           const HoleMapInfo* __restrict__ hm_all, size_t cap,
                                                           const unsigned long long* __restrict__ box,
                                                           const int* __restrict__ box_first, int isym,
                                                           int round_cap, unsigned* __restrict__ err) {
  __shared__ unsigned pr[kHL][kHW], fr[kHL][kHW], pc[kHL][kHW], fc[kHL][kHW];
  const HoleMapInfo h = hm_all[blockIdx.y];
  unsigned char* __restrict__ sam = sam_all + (size_t)blockIdx.y * cap;
  const int b0 = box_first[blockIdx.y], b1 = box_first[blockIdx.y + 1];
  const int n[3] = {h.nx[0], h.nx[1], h.nx[2]};
  const long long st[3] = {1, n[0], (long long)n[0] * n[1]};
  int pa, a0, a1;  // plane-normal axis and the two in-plane axes
  if (isym == 1) { pa = 0; a0 = 1; a1 = 2; }
  else if (isym == 2) { pa = 1; a0 = 0; a1 = 2; }
  else { pa = 2; a0 = 0; a1 = 1; }
  const int n0 = n[a0], n1 = n[a1];
  if (n0 > kHL || n1 > kHL) {
    if (threadIdx.x == 0) atomicOr(err, kErrFloodFillBound);
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int plane = blockIdx.x; plane < n[pa]; plane += gridDim.x) {
    const bool face_plane = (plane == 0 || plane == n[pa] - 1);
    const long long base = plane * st[pa];
    // rows (lines along a0): every cell passable, the box faces seeded
    for (int r = threadIdx.x; r < n1; r += blockDim.x)
      for (int w = 0; w < kHW; w++) {
        const int lo = 32 * w, hi = min(32 * w + 32, n0);  // cells [lo, hi) of this word
        const unsigned all = (hi <= lo) ? 0u : (hi - lo == 32 ? 0xffffffffu : ((1u << (hi - lo)) - 1u));
        unsigned seed = 0u;
        if (face_plane || r == 0 || r == n1 - 1) seed = all;
        else {
          if (lo == 0 && hi > 0) seed |= 1u;                                 // i0 = 0
          if (n0 - 1 >= lo && n0 - 1 < hi) seed |= 1u << (n0 - 1 - lo);     // i0 = n0 - 1
        }
        pr[r][w] = all;
        fr[r][w] = seed;
      }
    __syncthreads();
    // wall-marked cells of this plane: the boxes that reach it, cleared
    // from the passable masks (utils.c:192-205 marks them 2)
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
      const unsigned long long v = box[i];
      int lo3[3], hi3[3];
      for (int j = 0; j < 3; j++) {
        lo3[j] = (int)((v >> (8 * j)) & 255u);
        hi3[j] = (int)((v >> (24 + 8 * j)) & 255u);
      }
      if (plane < lo3[pa] || plane > hi3[pa]) continue;
      const int c0 = lo3[a0], c1 = hi3[a0];
      for (int r = lo3[a1]; r <= hi3[a1]; r++)
        for (int w = c0 >> 5; w <= (c1 >> 5); w++) {
          const int lo = max(c0, 32 * w) - 32 * w, hi = min(c1, 32 * w + 31) - 32 * w;  // bits [lo, hi]
          const unsigned m = (hi - lo == 31) ? 0xffffffffu : (((1u << (hi - lo + 1)) - 1u) << lo);
          atomicAnd(&pr[r][w], ~m);
        }
    }
    __syncthreads();
    // seeds overwrite wall marks on the box faces (utils.c:206-226)
    for (int r = threadIdx.x; r < n1; r += blockDim.x)
      for (int w = 0; w < kHW; w++) pr[r][w] |= fr[r][w];
    __syncthreads();
    bit_transpose(pr, n1, pc, n0);
    __syncthreads();
    // rows, then columns, alternately: every run of passable cells that holds
    // a filled cell fills.  A pass that changes nothing ends the fill (the
    // state is then a fixed point of both, a fill being idempotent); the
    // row masks hold the state when it ends.
    // A fill needs fewer rounds than the plane has cells; round_cap > 0
    // lowers the bound to round_cap line passes that change something
    // (tioga_b200_set_test_bound_).
    for (int rounds = 0;; rounds++) {
      bool ch = false;
      for (int r = threadIdx.x; r < n1; r += blockDim.x) ch = line_fill(fr[r], pr[r]) || ch;
      const bool rch = __syncthreads_or(ch);
      if (!rch && rounds > 0) break;
      if (round_cap > 0 && rch && 2 * rounds + 1 >= round_cap) {
        if (threadIdx.x == 0) atomicOr(err, kErrFloodFillBound);
        break;
      }
      bit_transpose(fr, n1, fc, n0);
      __syncthreads();
      ch = false;
      for (int c = threadIdx.x; c < n0; c += blockDim.x) ch = line_fill(fc[c], pc[c]) || ch;
      if (!__syncthreads_or(ch)) break;  // fr already holds this state
      bit_transpose(fc, n0, fr, n1);
      __syncthreads();
      if (round_cap > 0 ? 2 * rounds + 2 >= round_cap : rounds > n0 * n1 + 2) {
        if (threadIdx.x == 0) atomicOr(err, kErrFloodFillBound);
        break;
      }
    }
    // final map: hole = wall-marked or unreached (utils.c:291-294)
    for (int r = warp; r < n1; r += nwarps) {
      if (pa == 2) {  // rows are contiguous
        unsigned char* __restrict__ row = sam + base + (size_t)r * n0;
        for (int w = 0; w < kHW && 32 * w < n0; w++)
          if (32 * w + lane < n0) row[32 * w + lane] = ((fr[r][w] >> lane) & 1u) ? 0 : 1;
      } else {
        for (int w = 0; w < kHW; w++) {
          const int i0 = 32 * w + lane;
          if (i0 < n0) sam[base + i0 * st[a0] + r * st[a1]] = ((fr[r][w] >> lane) & 1u) ? 0 : 1;
        }
      }
    }
    __syncthreads();
  }
}

// Plane-wise flood fill for isym = 1, 2, 3 (4-neighbour fills inside planes
// normal to x, y, z).  One CTA owns one plane in shared memory, seeds the
// six box faces with 1 (utils.c:206-226) and alternates forward/backward line
// sweeps along both in-plane axes until nothing changes.  The painted set is
// the closure of the seeds through unmarked cells, the same fixed point as
// the reference's Gauss-Seidel sweeps (utils.c:227-290), which is
// independent of the visiting order.  With seed == 2 (6-neighbour mode) the
// kernel only seeds the faces.
__global__ void k_holemap_fill_planes(unsigned char* __restrict__ sam_all, const HoleMapInfo* __restrict__ hm_all,
                                      size_t cap, int isym, int seed_only, unsigned* __restrict__ err) {
  extern __shared__ unsigned char s[];
  const HoleMapInfo h = hm_all[blockIdx.y];
  unsigned char* __restrict__ sam = sam_all + (size_t)blockIdx.y * cap;
  const int n[3] = {h.nx[0], h.nx[1], h.nx[2]};
  const long long st[3] = {1, n[0], (long long)n[0] * n[1]};
  int pa, a0, a1;  // plane-normal axis and the two in-plane axes
  if (isym == 1) { pa = 0; a0 = 1; a1 = 2; }
  else if (isym == 2) { pa = 1; a0 = 0; a1 = 2; }
  else { pa = 2; a0 = 0; a1 = 1; }
  const int n0 = n[a0], n1 = n[a1];
  for (int plane = blockIdx.x; plane < n[pa]; plane += gridDim.x) {
    const bool face_plane = (plane == 0 || plane == n[pa] - 1);
    const long long base = plane * st[pa];
    for (int t = threadIdx.x; t < n0 * n1; t += blockDim.x) {
      int i0 = t % n0, i1 = t / n0;
      unsigned char v = sam[base + i0 * st[a0] + i1 * st[a1]];
      if (face_plane || i0 == 0 || i0 == n0 - 1 || i1 == 0 || i1 == n1 - 1) v = 1;
      s[t] = v;
    }
    __syncthreads();
    if (!seed_only && !face_plane) {
      int rounds = 0;
      const int max_rounds = n0 * n1 + 2;
      for (;;) {
        int ch = 0;
        // lines along a0 (fixed i1)
        for (int i1 = 1 + threadIdx.x; i1 < n1 - 1; i1 += blockDim.x) {
          unsigned char* L = s + i1 * n0;
          for (int i0 = 1; i0 < n0 - 1; i0++)
            if (L[i0] == 0 && L[i0 - 1] == 1) { L[i0] = 1; ch = 1; }
          for (int i0 = n0 - 2; i0 >= 1; i0--)
            if (L[i0] == 0 && L[i0 + 1] == 1) { L[i0] = 1; ch = 1; }
        }
        __syncthreads();
        // lines along a1 (fixed i0)
        for (int i0 = 1 + threadIdx.x; i0 < n0 - 1; i0 += blockDim.x) {
          for (int i1 = 1; i1 < n1 - 1; i1++)
            if (s[i1 * n0 + i0] == 0 && s[(i1 - 1) * n0 + i0] == 1) { s[i1 * n0 + i0] = 1; ch = 1; }
          for (int i1 = n1 - 2; i1 >= 1; i1--)
            if (s[i1 * n0 + i0] == 0 && s[(i1 + 1) * n0 + i0] == 1) { s[i1 * n0 + i0] = 1; ch = 1; }
        }
        int any = __syncthreads_or(ch);
        if (!any) break;
        if (++rounds > max_rounds) {
          if (threadIdx.x == 0) atomicOr(err, kErrFloodFillBound);
          break;
        }
      }
    }
    for (int t = threadIdx.x; t < n0 * n1; t += blockDim.x) {
      int i0 = t % n0, i1 = t / n0;
      sam[base + i0 * st[a0] + i1 * st[a1]] = s[t];
    }
    __syncthreads();
  }
}

// 6-neighbour mode: one forward and one backward sweep along `axis` for every
// line of interior cells; repeated over the three axes until no change.
__global__ void k_holemap_lines(unsigned char* __restrict__ sam_all, const HoleMapInfo* __restrict__ hm_all,
                                size_t cap, int axis, unsigned* __restrict__ changed) {
  const HoleMapInfo h = hm_all[blockIdx.y];
  unsigned char* __restrict__ sam = sam_all + (size_t)blockIdx.y * cap;
  const int n[3] = {h.nx[0], h.nx[1], h.nx[2]};
  const long long st[3] = {1, n[0], (long long)n[0] * n[1]};
  int b0 = (axis == 0) ? 1 : 0, b1 = (axis == 2) ? 1 : 2;
  long long nlines = (long long)n[b0] * n[b1];
  int ch = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nlines;
       t += (long long)gridDim.x * blockDim.x) {
    int i0 = (int)(t % n[b0]), i1 = (int)(t / n[b0]);
    if (i0 == 0 || i0 == n[b0] - 1 || i1 == 0 || i1 == n[b1] - 1) continue;
    unsigned char* L = sam + i0 * st[b0] + i1 * st[b1];
    long long s = st[axis];
    for (int k = 1; k < n[axis] - 1; k++)
      if (L[k * s] == 0 && L[(k - 1) * s] == 1) { L[k * s] = 1; ch = 1; }
    for (int k = n[axis] - 2; k >= 1; k--)
      if (L[k * s] == 0 && L[(k + 1) * s] == 1) { L[k * s] = 1; ch = 1; }
  }
  if (ch) atomicOr(changed, 1u);
}

// hole = unreached or wall-marked (utils.c:291-294)
__global__ void k_holemap_final(unsigned char* __restrict__ sam_all, const HoleMapInfo* __restrict__ hm_all,
                                size_t cap) {
  const HoleMapInfo h = hm_all[blockIdx.y];
  unsigned char* __restrict__ sam = sam_all + (size_t)blockIdx.y * cap;
  long long n = (long long)h.nx[0] * h.nx[1] * h.nx[2];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    unsigned char v = sam[i];
    sam[i] = (v == 0 || v == 2) ? 1 : 0;
  }
}

// ===========================================================================
// box pairs
// ===========================================================================
// src/utils.c:297-384: separating-axis test of two oriented boxes
__device__ int obb_intersect(const double vA[3][3], const double xA[3], const double dxA[3],
                             const double vB[3][3], const double xB[3], const double dxB[3]) {
  const double eps = 1e-12;
  double D[3], c[3][3], r, r0, r1, d1, d2;
  for (int i = 0; i < 3; i++) D[i] = xB[i] - xA[i];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      c[i][j] = 0;
      for (int k = 0; k < 3; k++) c[i][j] = c[i][j] + vA[i][k] * vB[j][k];
    }
  for (int i = 0; i < 3; i++) {
    r0 = dxA[i];
    r1 = 0;
    r = 0;
    for (int j = 0; j < 3; j++) {
      r1 += dxB[j] * fabs(c[i][j]);
      r += fabs(vA[i][j]) * D[j];
    }
    if (r > (r0 + r1 + eps)) return 0;
  }
  for (int i = 0; i < 3; i++) {
    r1 = dxB[i];
    r0 = 0;
    r = 0;
    for (int j = 0; j < 3; j++) {
      r0 += dxA[j] * fabs(c[j][i]);
      r += fabs(vB[i][j]) * D[j];
    }
    if (r > (r0 + r1 + eps)) return 0;
  }
  for (int i = 0; i < 3; i++) {
    int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    for (int j = 0; j < 3; j++) {
      int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      r0 = dxA[i1] * fabs(c[i2][j]) + dxA[i2] * fabs(c[i1][j]);
      r1 = dxB[j1] * fabs(c[i][j2]) + dxB[j2] * fabs(c[i][j1]);
      d2 = 0;
      d1 = 0;
      for (int k = 0; k < 3; k++) {
        d2 += vA[i2][k] * D[k];
        d1 += vA[i1][k] * D[k];
      }
      r = fabs(c[i1][j] * d2 - c[i2][j] * d1);
      if (r > (r0 + r1 + eps)) return 0;
    }
  }
  return 1;
}

// pairs listed donor-outer, receptor-inner as in exchangeBoxes.C:133-160:
// the candidates (donor, receptor) of different mesh tags within a system
// come in that order, and one CTA keeps those whose boxes intersect, in
// order.  pfirst[b] = first pair whose donor is block b (pairs are sorted by
// donor), pfirst[nb] = the pair count.
constexpr int kPairThreads = 1024;
__global__ void __launch_bounds__(kPairThreads) k_pairs(const BlockInfo* __restrict__ bi, int nb,
                                                        const int2* __restrict__ cand, int ncand,
                                                        PairInfo* __restrict__ pairs, int* __restrict__ npairs,
                                                        int* __restrict__ pfirst) {
  typedef cub::BlockScan<int, kPairThreads> Scan;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ int s_base;
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  for (int c0 = 0; c0 < ncand; c0 += kPairThreads) {
    const int i = c0 + threadIdx.x;
    int hit = 0, ob = 0, ib = 0;
    if (i < ncand) {
      ob = cand[i].x;
      ib = cand[i].y;
      const Obb& a = bi[ib].obb;
      const Obb& o = bi[ob].obb;
      hit = obb_intersect(a.vec, a.xc, a.dxc, o.vec, o.xc, o.dxc) ||
            obb_intersect(o.vec, o.xc, o.dxc, a.vec, a.xc, a.dxc);
    }
    int pos, total;
    Scan(tmp).ExclusiveSum(hit, pos, total);
    const int base = s_base;
    if (hit) {
      pairs[base + pos].rec = ib;
      pairs[base + pos].don = ob;
    }
    __syncthreads();
    if (threadIdx.x == 0) s_base = base + total;
    __syncthreads();
  }
  const int np = s_base;
  for (int b = threadIdx.x; b <= nb; b += blockDim.x) {
    int lo = 0, hi = np;  // first pair with donor >= b
    while (lo < hi) {
      const int m = (lo + hi) >> 1;
      if (pairs[m].don < b) lo = m + 1;
      else hi = m;
    }
    pfirst[b] = lo;
  }
  if (threadIdx.x == 0) *npairs = np;
}

__global__ void k_pair_finish(const BlockInfo* __restrict__ bi, PairInfo* __restrict__ pairs, int npairs,
                              const unsigned long long* __restrict__ acc) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const Obb& o = bi[pairs[p].don].obb;
  double rd[6];
  for (int k = 0; k < 6; k++) rd[k] = dkey_inv(acc[6 * p + k]);
  Obb r;
  for (int j = 0; j < 3; j++) {
    r.xc[j] = o.xc[j];
    for (int k = 0; k < 3; k++) r.xc[j] += ((rd[k] + rd[k + 3]) * 0.5) * o.vec[k][j];
    r.dxc[j] = (rd[j + 3] - rd[j]) * 0.51;
    for (int k = 0; k < 3; k++) r.vec[j][k] = o.vec[j][k];
  }
  for (int k = 0; k < 6; k++) pairs[p].rd[k] = rd[k];
  pairs[p].region = r;
  // world box of the region, widened so rounding can never exclude a node
  // the exact test keeps
  for (int k = 0; k < 3; k++) {
    double h = 0;
    for (int j = 0; j < 3; j++) h += fabs(r.dxc[j]) * fabs(r.vec[j][k]);
    const double slack = 1e-9 * (fabs(r.xc[k]) + h) + 1e-12;
    pairs[p].wbox[k] = r.xc[k] - h - slack;
    pairs[p].wbox[k + 3] = r.xc[k] + h + slack;
  }
}

// ===========================================================================
// bounding-volume tree: cell boxes in Morton order, leaves of up to
// kMaxLeafCells cells, implicit complete 4-ary tree (heap order) per block
// ===========================================================================
__device__ __forceinline__ float f_rd(double v) { return __double2float_rd(v); }
__device__ __forceinline__ float f_ru(double v) { return __double2float_ru(v); }

// Bounds of every double that rounds to nearest onto v: it lies within half
// an ulp of v, at most 2^-24 |v| (or 2^-150 below the normal range).
__device__ __forceinline__ float f_down(float v) { return __fsub_rd(__fmaf_rd(fabsf(v), -6.0e-8f, v), 1e-44f); }
__device__ __forceinline__ float f_up(float v) { return __fadd_ru(__fmaf_ru(fabsf(v), 6.0e-8f, v), 1e-44f); }

// float -> int key with the same order (-0 taken as +0), for shared-memory
// atomicMin / atomicMax
__device__ __forceinline__ int fkey(float f) {
  const int i = __float_as_int(__fadd_rn(f, 0.0f));
  return i >= 0 ? i : i ^ 0x7fffffff;
}

// FP32 bounds [lo_j, hi_j] of the projections onto axes vec (rows) about
// origin o of every point of the box with centre cc and half sizes hh.  The
// slack covers, with a wide margin, the rounding of this FP32 arithmetic, of
// the FP32 axes and half sizes, and of the reference's FP64 projections of the
// vertices: every error term is below 2^-22 times the magnitudes summed into
// it (sd, sh, ext, and |cc| for the FP64 centre).
__device__ __forceinline__ void proj_bounds(const double cc[3], const double o[3], const float vec[9],
                                            const float hh[3], float sc, const float ext[3], float lo[3],
                                            float hi[3]) {
  float dc[3], sd = 0.f;
  for (int k = 0; k < 3; k++) {
    dc[k] = (float)(cc[k] - o[k]);
    sd += fabsf(dc[k]);
  }
  const float sh = hh[0] + hh[1] + hh[2];
  for (int jx = 0; jx < 3; jx++) {
    float cp = 0.f, rad = 0.f;
    for (int k = 0; k < 3; k++) {
      cp = __fmaf_rn(dc[k], vec[3 * jx + k], cp);
      rad = __fmaf_rn(hh[k], fabsf(vec[3 * jx + k]), rad);
    }
    const float slack = 2e-6f * (sd + sh + ext[jx]) + 1e-12f * sc + 1e-30f;
    lo[jx] = cp - rad - slack;
    hi[jx] = cp + rad + slack;
  }
}

// Extents of a cell's vertices projected onto a box's axes about its centre,
// in the reference's FP64 arithmetic and order (MeshBlock.C:800-833): lo/hi
// of axis j in pb[j], pb[j + 3] (pb holds the start values).
__device__ __forceinline__ void project_cell64(const double* __restrict__ x, const int* __restrict__ conn8,
                                               long long c, int nv, const Obb& B, double pb[6]) {
  for (int m = 0; m < nv; m++) {
    const double* v = x + 3 * (long long)conn8[8 * c + m];
    const double v0 = v[0], v1 = v[1], v2 = v[2];
    for (int jx = 0; jx < 3; jx++) {
      double xd = 0;
      xd += (v0 - B.xc[0]) * B.vec[jx][0];
      xd += (v1 - B.xc[1]) * B.vec[jx][1];
      xd += (v2 - B.xc[2]) * B.vec[jx][2];
      pb[jx] = dmin(pb[jx], xd);
      pb[jx + 3] = dmax(pb[jx + 3], xd);
    }
  }
}

// The reduced boxes (getReducedOBB, MeshBlock.C:774-838): for every pair,
// the extents along the donor's axes of the donor's cells that overlap the
// receptor's box.  FP32 bounds of a cell's or a leaf's projections (box
// centre and half sizes, widened by far more than their rounding error and
// the reference's) decide what needs FP64:
//  * a cell or leaf clearly outside the receptor box is skipped, one clearly
//    inside overlaps it; only cells across its faces get the reference's
//    FP64 test;
//  * for the extents, an FP32 upper bound of every axis minimum (the least
//    upper bound of the projections of any leaf inside the receptor box, or
//    the exact minimum of any overlapping cell rounded up) and a lower bound
//    of every maximum are kept per pair.  A cell or leaf whose
//    projections lie strictly between them on every axis cannot hold an
//    extreme, whether it overlaps or not; the cell that does hold one always
//    has its lower bound under every such upper bound, so it is always
//    projected exactly.  The exact extents are combined per warp and by
//    min/max atomics on order-preserving keys, so their order is free.
// Each CTA keeps the bounds of its chunk's pairs in shared memory; the split
// form starts them from seeds taken over every leaf inside a receptor box
// (k_leaf_seeds), the FP64 form (k_cell_pass64) from open bounds.
// A leaf (centre lc, half sizes lh) that is not outside pair q's receptor
// box, against the pair's extent bounds (s_ext: per donor axis, in fkey
// order, an upper bound of the reduced box's minimum and a lower bound of its
// maximum): true when its projections on the donor's axes reach a bound, so
// that its cells must be tested one by one.  A leaf whose projections lie
// strictly between the bounds on every axis cannot hold an extreme, whether
// its cells take part in the reduced box or not.  Every cell of a leaf
// inside the receptor box takes part, so such a leaf (`inside`) then
// tightens the bounds with its own projections (the minimum is at most the
// leaf's upper bound, the maximum at least its lower bound).
__device__ __forceinline__ bool leaf_reaches_extents(int* __restrict__ s_ext, int q, const double lc[3],
                                                     const float lh[3], float lsc, const PairCull& Q, bool inside) {
  volatile int* v_ext = s_ext;
  const float zero[3] = {0.f, 0.f, 0.f};
  float blo[3], bhi[3];
  proj_bounds(lc, Q.dxc, Q.dvec, lh, lsc, zero, blo, bhi);
  bool mix = false;
  for (int jx = 0; jx < 3; jx++) {
    const int kl = fkey(blo[jx]), ku = fkey(bhi[jx]);
    const int umin = v_ext[6 * q + jx], lmax = v_ext[6 * q + 3 + jx];
    mix = mix || (kl <= umin) || (ku >= lmax);
    if (inside && ku < umin) atomicMin(&s_ext[6 * q + jx], ku);
    if (inside && kl > lmax) atomicMax(&s_ext[6 * q + 3 + jx], kl);
  }
  return mix;
}

// First part: every leaf tests its box f against the pairs of its block,
// lane g of the leaf taking pairs qa+g, qa+g+LC, ...; returns the mask of
// pairs (bit q - qa) that need cell-by-cell work, the same in every lane of
// the leaf, and the pair range [qa, qb) the lane's leaf takes part in.
__device__ __forceinline__ unsigned leaf_pairs_mixed(const PairCull* __restrict__ s_pc, int* __restrict__ s_ext,
                                                     int lane, bool leaf_ok, int qa0, int qb0, const float f[6],
                                                     int& qa, int& qb) {
  constexpr int LC = kMaxLeafCells;
  const bool leaf_live = leaf_ok && f[0] <= f[3];
  qa = leaf_live ? qa0 : 0;
  qb = leaf_live ? qb0 : 0;
  const int g = lane % LC;
  unsigned mixed = 0u;
  {
    const int nqw = __reduce_max_sync(0xffffffffu, qb - qa);
    if (nqw > 32) {
      mixed = 0xffffffffu;  // more pairs than mask bits: cell by cell
    } else if (nqw > 0) {
      double lc[3];
      float lh[3], lsc = 0.f;
      for (int k = 0; k < 3; k++) {
        lc[k] = 0.5 * ((double)f[k] + (double)f[k + 3]);
        lh[k] = leaf_live ? __fmul_ru(__fsub_ru(f[k + 3], f[k]), 0.5f) : 0.f;
        lsc += leaf_live ? fabsf((float)lc[k]) : 0.f;
      }
      for (int r = 0; LC * r < nqw; r++) {
        const int q = qa + g + LC * r;
        if (q < qb) {
          const PairCull& Q = s_pc[q];
          float blo[3], bhi[3];
          proj_bounds(lc, Q.rxc, Q.rvec, lh, lsc, Q.rdxc, blo, bhi);
          bool out = false, inside = true;
          for (int jx = 0; jx < 3; jx++) {
            out = out || (blo[jx] > Q.rdxc[jx]) || (bhi[jx] < -Q.rdxc[jx]);
            inside = inside && (bhi[jx] <= Q.rdxc[jx]) && (blo[jx] >= -Q.rdxc[jx]);
          }
          const bool mix = !out && leaf_reaches_extents(s_ext, q, lc, lh, lsc, Q, inside);
          if (mix) mixed |= 1u << (q - qa);
        }
      }
      for (int o = 1; o < LC; o <<= 1) mixed |= __shfl_xor_sync(0xffffffffu, mixed, o);
    }
  }
  return mixed;
}

// Second part: the cells of the mixed (leaf, pair) combinations, with the
// cell's box (centre cc, half sizes hh), exactly as getReducedOBB decides.
__device__ __forceinline__ void cell_pairs_exact(const double* __restrict__ x, const int* __restrict__ conn8,
                                                 const BlockInfo* __restrict__ bi, const PairInfo* __restrict__ pairs,
                                                 const PairCull* __restrict__ s_pc, int* __restrict__ s_ext,
                                                 unsigned long long* __restrict__ s_acc, int lane, bool valid,
                                                 long long c, int nv, unsigned mixed, int qa, int qb,
                                                 const double cc[3], const float hh[3]) {
  volatile int* v_ext = s_ext;
  float sc = 0.f;
  for (int k = 0; k < 3; k++) sc += valid ? fabsf((float)cc[k]) : 0.f;
  const int q0 = __reduce_min_sync(0xffffffffu, (valid && mixed) ? qa : 0x7fffffff);
  const int q1 = __reduce_max_sync(0xffffffffu, (valid && mixed) ? qb : 0);
  for (int q = q0; q < q1; q++) {
    const bool mine = valid && q >= qa && q < qb && ((mixed >> min(q - qa, 31)) & 1u);
    if (!__any_sync(0xffffffffu, mine)) continue;
    bool contrib = false;
    double rlo[3] = {1e300, 1e300, 1e300}, rhi[3] = {-1e300, -1e300, -1e300};
    if (mine) {
      const PairCull& Q = s_pc[q];
      float blo[3], bhi[3];
      proj_bounds(cc, Q.rxc, Q.rvec, hh, sc, Q.rdxc, blo, bhi);
      bool out = false, inside = true;
      for (int jx = 0; jx < 3; jx++) {
        out = out || (blo[jx] > Q.rdxc[jx]) || (bhi[jx] < -Q.rdxc[jx]);
        inside = inside && (bhi[jx] <= Q.rdxc[jx]) && (blo[jx] >= -Q.rdxc[jx]);
      }
      // a cell whose projections on the donor's axes lie strictly between
      // the extents' bounds cannot hold an extreme: neither its overlap nor
      // its projections matter
      bool need = false;
      if (!out) {
        const float zero[3] = {0.f, 0.f, 0.f};
        proj_bounds(cc, Q.dxc, Q.dvec, hh, sc, zero, blo, bhi);
        for (int jx = 0; jx < 3; jx++)
          need = need || (fkey(blo[jx]) <= v_ext[6 * q + jx]) || (fkey(bhi[jx]) >= v_ext[6 * q + 3 + jx]);
      }
      bool ov = need && inside;
      if (need && !inside) {  // across a face: the reference's test, MeshBlock.C:800-821
        const Obb& R = bi[pairs[Q.pair].rec].obb;
        double bb[6] = {kBig, kBig, kBig, -kBig, -kBig, -kBig};
        project_cell64(x, conn8, c, nv, R, bb);
        ov = true;
        for (int jx = 0; jx < 3; jx++) ov = ov && !(bb[jx] > R.dxc[jx]);
        for (int jx = 0; jx < 3; jx++) ov = ov && !(bb[jx + 3] < -R.dxc[jx]);
      }
      if (ov) {
        double pb[6] = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300};  // the reference's projections,
        project_cell64(x, conn8, c, nv, bi[Q.don].obb, pb);               // MeshBlock.C:822-833
        for (int jx = 0; jx < 3; jx++) {  // a cell that takes part tightens the bounds with its
          const int eu = fkey(__double2float_ru(pb[jx]));      // exact extremes, rounded outward
          const int el = fkey(__double2float_rd(pb[jx + 3]));
          if (eu < v_ext[6 * q + jx]) atomicMin(&s_ext[6 * q + jx], eu);
          if (el > v_ext[6 * q + 3 + jx]) atomicMax(&s_ext[6 * q + 3 + jx], el);
        }
        for (int jx = 0; jx < 3; jx++) {
          rlo[jx] = pb[jx];
          rhi[jx] = pb[jx + 3];
        }
        contrib = true;
      }
    }
    if (__any_sync(0xffffffffu, contrib)) {
      for (int jx = 0; jx < 3; jx++)
        for (int o = 16; o > 0; o >>= 1) {
          rlo[jx] = dmin(rlo[jx], __shfl_xor_sync(0xffffffffu, rlo[jx], o));
          rhi[jx] = dmax(rhi[jx], __shfl_xor_sync(0xffffffffu, rhi[jx], o));
        }
      if (lane == 0)
        for (int jx = 0; jx < 3; jx++) {
          atomicMin(&s_acc[6 * q + jx], dkey(rlo[jx]));
          atomicMax(&s_acc[6 * q + jx + 3], dkey(rhi[jx]));
        }
    }
  }
}


// Both parts, for the kernels that hold every cell's box in registers.
__device__ __forceinline__ void cell_pass_pairs(
    const double* __restrict__ x, const int* __restrict__ conn8, const BlockInfo* __restrict__ bi,
    const PairInfo* __restrict__ pairs, const PairCull* __restrict__ s_pc, int* __restrict__ s_ext,
    unsigned long long* __restrict__ s_acc, int lane, bool leaf_ok, bool valid, long long c, int nv, int qa0, int qb0,
    const float f[6], const double cc[3], const float hh[3]) {
  int qa, qb;
  const unsigned mixed = leaf_pairs_mixed(s_pc, s_ext, lane, leaf_ok, qa0, qb0, f, qa, qb);
  cell_pairs_exact(x, conn8, bi, pairs, s_pc, s_ext, s_acc, lane, valid, c, nv, mixed, qa, qb, cc, hh);
}

// this CTA's chunk: the last one whose first CTA is <= blockIdx.x.  Work
// comes in chunks of consecutive blocks (chunk = work items [x, y), pairs
// z .. z+w-1: all the pairs whose donor is one of the chunk's blocks, as the
// pairs are sorted by donor); CTAs chunk_cta[k] .. chunk_cta[k+1]-1 share
// chunk k, whose pairs sit in their shared memory.
__device__ __forceinline__ int chunk_of_cta(const int* __restrict__ chunk_cta, int nchunks) {
  int kc = 0, hi = nchunks - 1;
  while (kc < hi) {
    const int m = (kc + hi + 1) >> 1;
    if (chunk_cta[m] <= (int)blockIdx.x) kc = m;
    else hi = m - 1;
  }
  return kc;
}

// the chunk's pairs into shared memory, the extents' accumulators cleared,
// the extents' bounds from ext (the seeds) or open
__device__ __forceinline__ void cell_pass_setup(const int4& CH, int kc, const int* __restrict__ chunk_cta,
                                                const BlockInfo* __restrict__ bi, const PairInfo* __restrict__ pairs,
                                                unsigned long long* s_acc, PairCull* s_pc, int* s_ext, int& cta,
                                                int& ncta, const int* __restrict__ ext = nullptr) {
  const int p0 = CH.z, np = CH.w;
  cta = (int)blockIdx.x - chunk_cta[kc];
  ncta = chunk_cta[kc + 1] - chunk_cta[kc];
  const int tid = threadIdx.x;
  for (int i = tid; i < 6 * np; i += blockDim.x) {
    s_acc[i] = (i % 6 < 3) ? ~0ull : 0ull;
    s_ext[i] = ext ? ext[6 * (long long)p0 + i] : ((i % 6 < 3) ? 0x7fffffff : (int)0x80000000);
  }
  for (int i = tid; i < np; i += blockDim.x) {
    const PairInfo& P = pairs[p0 + i];
    const Obb& R = bi[P.rec].obb;
    const Obb& D = bi[P.don].obb;
    PairCull q;
    for (int k = 0; k < 3; k++) {
      q.rxc[k] = R.xc[k];
      q.dxc[k] = D.xc[k];
      q.rdxc[k] = (float)R.dxc[k];
      for (int j = 0; j < 3; j++) {
        q.rvec[3 * j + k] = (float)R.vec[j][k];
        q.dvec[3 * j + k] = (float)D.vec[j][k];
      }
    }
    q.don = P.don;
    q.pair = p0 + i;
    s_pc[i] = q;
  }
  __syncthreads();
}

// the CTA's exact extents into the pairs' accumulators
__device__ __forceinline__ void cell_pass_flush(const unsigned long long* s_acc, int p0, int np,
                                                unsigned long long* __restrict__ acc) {
  __syncthreads();
  for (int i = threadIdx.x; i < 6 * np; i += blockDim.x) {
    const unsigned long long v = s_acc[i];
    unsigned long long* dst = &acc[6 * (long long)(p0 + i / 6) + i % 6];
    if (i % 6 < 3) {
      if (v != ~0ull) atomicMin(dst, v);
    } else if (v != 0ull) {
      atomicMax(dst, v);
    }
  }
}

// One lane's leaf (box f) against the pairs [qa, qb) of its block, as
// leaf_pairs_mixed does for a leaf spread over kMaxLeafCells lanes: the mask
// of pairs (bit q - qa) whose cells need the exact test.
__device__ __forceinline__ unsigned leaf_lane_mixed(const PairCull* __restrict__ s_pc, int* __restrict__ s_ext,
                                                    const float f[6], int qa, int qb) {
  if (qb - qa > 32) return 0xffffffffu;  // more pairs than mask bits: cell by cell
  unsigned mixed = 0u;
  if (qb > qa) {
    double lc[3];
    float lh[3], lsc = 0.f;
    for (int k = 0; k < 3; k++) {
      lc[k] = 0.5 * ((double)f[k] + (double)f[k + 3]);
      lh[k] = __fmul_ru(__fsub_ru(f[k + 3], f[k]), 0.5f);
      lsc += fabsf((float)lc[k]);
    }
    for (int q = qa; q < qb; q++) {
      const PairCull& Q = s_pc[q];
      float blo[3], bhi[3];
      proj_bounds(lc, Q.rxc, Q.rvec, lh, lsc, Q.rdxc, blo, bhi);
      bool out = false, inside = true;
      for (int jx = 0; jx < 3; jx++) {
        out = out || (blo[jx] > Q.rdxc[jx]) || (bhi[jx] < -Q.rdxc[jx]);
        inside = inside && (bhi[jx] <= Q.rdxc[jx]) && (blo[jx] >= -Q.rdxc[jx]);
      }
      const bool mix = !out && leaf_reaches_extents(s_ext, q, lc, lh, lsc, Q, inside);
      if (mix) mixed |= 1u << (q - qa);
    }
  }
  return mixed;
}

// One lane per leaf of the CTA's share of its chunk: the leaf's box and
// block from lbox (a warp loads 32 consecutive leaves) and its block's pair
// range within the chunk, [qa, qb); an empty range past the chunk's end.
__device__ __forceinline__ void leaf_lane_load(const float4* __restrict__ lbox, const int* __restrict__ pfirst,
                                               long long leaf, long long leaf_hi, int p0, float f[6], int& qa,
                                               int& qb) {
  f[0] = f[1] = f[2] = INFINITY;
  f[3] = f[4] = f[5] = -INFINITY;
  qa = qb = 0;
  if (leaf < leaf_hi) {
    const float4 A = lbox[2 * leaf], B = lbox[2 * leaf + 1];
    f[0] = A.x; f[1] = A.y; f[2] = A.z; f[3] = A.w; f[4] = B.x; f[5] = B.y;
    const int b = __float_as_int(B.z);
    qa = pfirst[b] - p0;
    qb = pfirst[b + 1] - p0;
  }
}

// A cell's FP32 box is three float2 (24 bytes): (lo.x, lo.y), (lo.z, hi.x),
// (hi.y, hi.z); as the (lo.xyz, hi.x) / (hi.yz) pair of float4 the box tests
// take.
__device__ __forceinline__ void cell_box_load(const float2* __restrict__ cbox, long long c, float4& A, float4& B) {
  const float2 a = cbox[3 * c], b = cbox[3 * c + 1], d = cbox[3 * c + 2];
  A = make_float4(a.x, a.y, b.x, b.y);
  B = make_float4(d.x, d.y, 0.f, 0.f);
}

// Cell pass of the split form, in three kernels.
//
// k_cell_boxes: leaf by leaf (32 / kMaxLeafCells leaves per warp, one lane per
// cell), each lane gathers its cell's eight FP32 vertices (xf, rounded to
// nearest by k_node_tiles; slots past the vertex count read vertex 0 again,
// so the eight loads are unconditional and in flight together), rounds the
// box outward (f_down/f_up cover every double that rounds onto a vertex) into
// cbox, and the leaf's lanes write the union to the leaf's tree slot and,
// with the leaf's block, to lbox (leaf order).  It holds nothing else, so it
// runs at a high occupancy that hides the gathers.  With ids it takes only the
// nleaf leaves listed there (those whose coordinates have been uploaded).
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_cell_boxes(const float4* __restrict__ xf,
                                                          const int* __restrict__ conn8,
                                                          const unsigned char* __restrict__ cell_nv,
                                                          const int4* __restrict__ leaves,
                                                          const int* __restrict__ ids, long long nleaf,
                                                          float2* __restrict__ cbox, float4* __restrict__ tnode,
                                                          float4* __restrict__ lbox) {
  constexpr int LC = kMaxLeafCells, LPW = 32 / kMaxLeafCells;
  const int lane = threadIdx.x & 31;
  const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long base = LPW * warp0; base < nleaf; base += LPW * nwarps) {
    const long long li = base + lane / LC;
    const bool leaf_ok = li < nleaf;
    const long long leaf = (ids && leaf_ok) ? ids[li] : li;  // the leaves listed in ids, else all
    const int4 L = leaf_ok ? leaves[leaf] : make_int4(0, 0, 0, 0);  // first cell, cells, slot, block
    const bool valid = leaf_ok && lane % LC < L.y;
    const long long c = (long long)L.x + lane % LC;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (valid) {
      const int nv = cell_nv[c];
      const int4 c0 = *reinterpret_cast<const int4*>(conn8 + 8 * c);
      const int4 c1 = *reinterpret_cast<const int4*>(conn8 + 8 * c + 4);
      const int cv[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
#pragma unroll
      for (int m = 0; m < 8; m++) {
        const float4 v = xf[m < nv ? cv[m] : cv[0]];
        lo[0] = fminf(lo[0], v.x); lo[1] = fminf(lo[1], v.y); lo[2] = fminf(lo[2], v.z);
        hi[0] = fmaxf(hi[0], v.x); hi[1] = fmaxf(hi[1], v.y); hi[2] = fmaxf(hi[2], v.z);
      }
    }
    float f[6];
    for (int k = 0; k < 3; k++) {
      f[k] = valid ? f_down(lo[k]) : INFINITY;
      f[k + 3] = valid ? f_up(hi[k]) : -INFINITY;
    }
    if (valid) {
      cbox[3 * c] = make_float2(f[0], f[1]);
      cbox[3 * c + 1] = make_float2(f[2], f[3]);
      cbox[3 * c + 2] = make_float2(f[4], f[5]);
    }
    for (int o = 1; o < LC; o <<= 1)
      for (int k = 0; k < 3; k++) {
        f[k] = fminf(f[k], __shfl_xor_sync(0xffffffffu, f[k], o));
        f[k + 3] = fmaxf(f[k + 3], __shfl_xor_sync(0xffffffffu, f[k + 3], o));
      }
    if (leaf_ok && lane % LC == 0) {
      const long long sl = L.z;
      tnode[2 * sl] = make_float4(f[0], f[1], f[2], f[3]);
      *reinterpret_cast<float2*>(&tnode[2 * sl + 1]) = make_float2(f[4], f[5]);  // keep the link
      lbox[2 * leaf] = make_float4(f[0], f[1], f[2], f[3]);
      lbox[2 * leaf + 1] = make_float4(f[4], f[5], __int_as_float(L.w), 0.f);
    }
  }
}

// k_leaf_seeds: over the chunks of k_cell_pairs, one lane per leaf tests the
// leaf against its block's pairs (leaf_lane_mixed) for the bounds alone:
// each CTA's tightest bounds, merged over the CTAs into ext (fkey order).
// k_cell_pairs starts every CTA from them, so only the leaves and cells near
// a pair's extremes are projected one by one, wherever they lie.
__global__ void __launch_bounds__(256) k_leaf_seeds(const BlockInfo* __restrict__ bi,
                                                    const int4* __restrict__ chunks,
                                                    const int* __restrict__ chunk_cta, int nchunks,
                                                    const int* __restrict__ pfirst,
                                                    const PairInfo* __restrict__ pairs,
                                                    const float4* __restrict__ lbox, int* __restrict__ ext) {
  extern __shared__ unsigned long long s_dyn[];
  int cta, ncta;
  const int kc = chunk_of_cta(chunk_cta, nchunks);
  const int4 CH = chunks[kc];  // first leaf, end leaf, first pair, pairs
  unsigned long long* s_acc = s_dyn;
  PairCull* s_pc = reinterpret_cast<PairCull*>(s_dyn + 6 * CH.w);
  int* s_ext = reinterpret_cast<int*>(s_pc + CH.w);
  cell_pass_setup(CH, kc, chunk_cta, bi, pairs, s_acc, s_pc, s_ext, cta, ncta);
  const long long leaf_lo = CH.x, leaf_hi = CH.y;
  const int p0 = CH.z;
  const long long t0 = (long long)cta * blockDim.x + threadIdx.x;
  const long long nt = (long long)ncta * blockDim.x;
  for (long long base = leaf_lo + (t0 & ~31ll); base < leaf_hi; base += nt) {
    float f[6];
    int qa, qb;
    leaf_lane_load(lbox, pfirst, base + (threadIdx.x & 31), leaf_hi, p0, f, qa, qb);
    leaf_lane_mixed(s_pc, s_ext, f, qa, qb);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 6 * CH.w; i += blockDim.x) {
    const int v = s_ext[i];
    int* dst = &ext[6 * (long long)p0 + i];
    if (i % 6 < 3) {
      if (v != 0x7fffffff) atomicMin(dst, v);
    } else if (v != (int)0x80000000) {
      atomicMax(dst, v);
    }
  }
}

// k_cell_pairs: over the same chunks, one lane per leaf, the bounds starting
// from the seeds: each leaf is tested against its block's pairs
// (leaf_lane_mixed); then the warp's leaves with a (leaf, pair) combination
// that needs its cells tested, four at a time, a lane per cell: their cells'
// boxes are read back from cbox for the exact cell-by-cell work
// (cell_pairs_exact).  The boxes are the ones k_cell_boxes wrote, so every
// decision is the one-kernel form's.
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_cell_pairs(
    const double* __restrict__ x, const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
    const BlockInfo* __restrict__ bi, const int4* __restrict__ leaves, const int4* __restrict__ chunks,
    const int* __restrict__ chunk_cta, int nchunks, const int* __restrict__ pfirst,
    const PairInfo* __restrict__ pairs, const float2* __restrict__ cbox, const float4* __restrict__ lbox,
    const int* __restrict__ ext, unsigned long long* __restrict__ acc) {
  extern __shared__ unsigned long long s_dyn[];
  int cta, ncta;
  const int kc = chunk_of_cta(chunk_cta, nchunks);
  const int4 CH = chunks[kc];  // first leaf, end leaf, first pair, pairs
  unsigned long long* s_acc = s_dyn;
  PairCull* s_pc = reinterpret_cast<PairCull*>(s_dyn + 6 * CH.w);
  int* s_ext = reinterpret_cast<int*>(s_pc + CH.w);
  cell_pass_setup(CH, kc, chunk_cta, bi, pairs, s_acc, s_pc, s_ext, cta, ncta, ext);
  const long long leaf_lo = CH.x, leaf_hi = CH.y;
  const int p0 = CH.z;
  const int lane = threadIdx.x & 31;
  const long long t0 = (long long)cta * blockDim.x + threadIdx.x;
  const long long nt = (long long)ncta * blockDim.x;
  constexpr int LC = kMaxLeafCells;
  for (long long base = leaf_lo + (t0 & ~31ll); base < leaf_hi; base += nt) {
    float f[6];
    int qa, qb;
    leaf_lane_load(lbox, pfirst, base + lane, leaf_hi, p0, f, qa, qb);
    const unsigned mixed = leaf_lane_mixed(s_pc, s_ext, f, qa, qb);
    // the mixed leaves, four at a time, a lane per cell
    unsigned todo = __ballot_sync(0xffffffffu, mixed != 0u);
    while (todo) {
      int src = -1;  // the leaf (lane of the scan) this lane's quarter takes
      unsigned t = todo;
      for (int j = 0; j < 32 / LC; j++) {
        const int l = t ? __ffs(t) - 1 : -1;
        if (j == lane / LC) src = l;
        if (t) t &= t - 1;
      }
      todo = t;
      const int s_lane = src < 0 ? 0 : src;
      const unsigned m = __shfl_sync(0xffffffffu, mixed, s_lane);
      const int sqa = __shfl_sync(0xffffffffu, qa, s_lane), sqb = __shfl_sync(0xffffffffu, qb, s_lane);
      int4 L = make_int4(0, 0, 0, 0);
      if (src >= 0) L = leaves[base + src];  // first cell, cells, slot, block
      const bool valid = src >= 0 && lane % LC < L.y;
      const long long c = (long long)L.x + lane % LC;
      int nv = 0;
      double cc[3] = {0.0, 0.0, 0.0};
      float hh[3] = {0.f, 0.f, 0.f};
      if (valid) {
        nv = cell_nv[c];
        float4 A, B;
        cell_box_load(cbox, c, A, B);
        const float fb[6] = {A.x, A.y, A.z, A.w, B.x, B.y};
        for (int k = 0; k < 3; k++) {
          cc[k] = 0.5 * ((double)fb[k] + (double)fb[k + 3]);
          hh[k] = __fmul_ru(__fsub_ru(fb[k + 3], fb[k]), 0.5f);
        }
      }
      cell_pairs_exact(x, conn8, bi, pairs, s_pc, s_ext, s_acc, lane, valid, c, nv, valid ? m : 0u,
                       valid ? sqa : 0, valid ? sqb : 0, cc, hh);
    }
  }
  cell_pass_flush(s_acc, p0, CH.w, acc);
}

// Upload chunk of every leaf: the chunk (of `chunk` consecutive global node
// ids) holding the largest vertex id of its cells, so the leaf's cell boxes
// can be computed once that chunk has landed.
__global__ void k_leaf_chunk(const int4* __restrict__ leaves, long long nleaf, const int* __restrict__ conn8,
                             const unsigned char* __restrict__ cell_nv, int chunk, int* __restrict__ key,
                             int* __restrict__ id) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < nleaf;
       l += (long long)gridDim.x * blockDim.x) {
    const int4 L = leaves[l];
    int vmax = 0;
    for (int j = 0; j < L.y; j++) {
      const long long c = (long long)L.x + j;
      const int nv = cell_nv[c];
      for (int m = 0; m < nv; m++) vmax = max(vmax, conn8[8 * c + m]);
    }
    key[l] = vmax / chunk;
    id[l] = (int)l;
  }
}

// Upload chunk of every node tile: the chunk holding the largest node id of
// the tile (its kNodeTile Morton-ordered nodes), as for the leaves.
__global__ void k_tile_chunk(const BlockInfo* __restrict__ bi, int nb, const long long* __restrict__ tile_base,
                             const int* __restrict__ node_order, int chunk, int* __restrict__ key,
                             int* __restrict__ id) {
  const long long ntile = tile_base[nb];
  for (long long T = blockIdx.x * (long long)blockDim.x + threadIdx.x; T < ntile;
       T += (long long)gridDim.x * blockDim.x) {
    const int b = block_of_tile(tile_base, nb, T);
    const BlockInfo& B = bi[b];
    const int t0 = (int)(T - tile_base[b]) * kNodeTile;
    int vmax = 0;
    for (int i = t0; i < min(t0 + kNodeTile, B.nnodes); i++) vmax = max(vmax, node_order[B.node_off + i]);
    key[T] = vmax / chunk;
    id[T] = (int)T;
  }
}

// FP32 copy (rounded to nearest) of the coordinates of nodes [lo, hi)
__global__ void k_round_nodes(const double* __restrict__ x, long long lo, long long hi, float4* __restrict__ xf) {
  for (long long i = lo + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < hi;
       i += (long long)gridDim.x * blockDim.x)
    xf[i] = make_float4(__double2float_rn(x[3 * i]), __double2float_rn(x[3 * i + 1]), __double2float_rn(x[3 * i + 2]),
                        0.f);
}

// Cell pass of the FP64 form, leaf by leaf (32 / kMaxLeafCells leaves per
// warp, one lane per cell; chunk work items are leaves): the FP64 element
// box of every cell (cbox64, exact) and of every leaf (tnode64), their FP32
// roundings outward for the leaf slots (links), and the reduced boxes.
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_cell_pass64(
    const double* __restrict__ x, const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
    const BlockInfo* __restrict__ bi, const int4* __restrict__ leaves, const int4* __restrict__ chunks,
    const int* __restrict__ chunk_cta, int nchunks, const int* __restrict__ pfirst,
    const PairInfo* __restrict__ pairs, double* __restrict__ cbox64, float4* __restrict__ tnode,
    double* __restrict__ tnode64, unsigned long long* __restrict__ acc) {
  extern __shared__ unsigned long long s_dyn[];
  int cta, ncta;
  const int kc = chunk_of_cta(chunk_cta, nchunks);
  const int4 CH = chunks[kc];  // first leaf, end leaf, first pair, pairs
  unsigned long long* s_acc = s_dyn;
  PairCull* s_pc = reinterpret_cast<PairCull*>(s_dyn + 6 * CH.w);
  int* s_ext = reinterpret_cast<int*>(s_pc + CH.w);
  cell_pass_setup(CH, kc, chunk_cta, bi, pairs, s_acc, s_pc, s_ext, cta, ncta);
  const long long leaf_lo = CH.x, leaf_hi = CH.y;
  const int p0 = CH.z;
  const int tid = threadIdx.x, lane = tid & 31;
  const long long warp0 = ((long long)cta * blockDim.x + tid) >> 5;
  const long long nwarps = ((long long)ncta * blockDim.x) >> 5;
  constexpr int LC = kMaxLeafCells, LPW = 32 / kMaxLeafCells;  // cells per leaf, leaves per warp
  for (long long base = leaf_lo + LPW * warp0; base < leaf_hi; base += LPW * nwarps) {
    const long long leaf = base + lane / LC;
    const bool leaf_ok = leaf < leaf_hi;
    const int4 L = leaf_ok ? leaves[leaf] : make_int4(0, 0, 0, 0);  // first cell, cells, slot, block
    const int b = L.w;
    const bool valid = leaf_ok && lane % LC < L.y;
    const long long c = (long long)L.x + lane % LC;
    const long long sl = L.z;
    int nv = 0;
    float fb[6];
    double cc[3];
    float hh[3];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    if (valid) {
      nv = cell_nv[c];
      const int4 c0 = *reinterpret_cast<const int4*>(conn8 + 8 * c);
      const int4 c1 = *reinterpret_cast<const int4*>(conn8 + 8 * c + 4);
      const int cv[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
#pragma unroll
      for (int m = 0; m < 8; m++) {
        if (m < nv) {
          const double* v = x + 3 * (long long)cv[m];
          for (int k = 0; k < 3; k++) {
            const double t = v[k];
            lo[k] = fmin(lo[k], t);
            hi[k] = fmax(hi[k], t);
          }
        }
      }
    }
    for (int k = 0; k < 3; k++) {
      fb[k] = valid ? f_rd(lo[k]) : INFINITY;
      fb[k + 3] = valid ? f_ru(hi[k]) : -INFINITY;
      cc[k] = 0.5 * (lo[k] + hi[k]);
      hh[k] = valid ? __double2float_ru(0.5 * (hi[k] - lo[k])) : 0.f;
    }
    if (valid) {
      double* o = cbox64 + 6 * c;
      o[0] = lo[0]; o[1] = lo[1]; o[2] = lo[2];
      o[3] = hi[0]; o[4] = hi[1]; o[5] = hi[2];
    }
    for (int o = 1; o < LC; o <<= 1)
      for (int k = 0; k < 3; k++) {
        lo[k] = dmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
        hi[k] = dmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
      }
    if (leaf_ok && lane % LC == 0)
      for (int k = 0; k < 3; k++) {
        tnode64[6 * sl + k] = lo[k];
        tnode64[6 * sl + k + 3] = hi[k];
      }
    float f[6];
    for (int k = 0; k < 6; k++) f[k] = fb[k];
    for (int o = 1; o < LC; o <<= 1)
      for (int k = 0; k < 3; k++) {
        f[k] = fminf(f[k], __shfl_xor_sync(0xffffffffu, f[k], o));
        f[k + 3] = fmaxf(f[k + 3], __shfl_xor_sync(0xffffffffu, f[k + 3], o));
      }
    if (leaf_ok && lane % LC == 0) {
      tnode[2 * sl] = make_float4(f[0], f[1], f[2], f[3]);
      *reinterpret_cast<float2*>(&tnode[2 * sl + 1]) = make_float2(f[4], f[5]);  // keep the link
    }
    cell_pass_pairs(x, conn8, bi, pairs, s_pc, s_ext, s_acc, lane, leaf_ok, valid, c, nv,
                    leaf_ok ? pfirst[b] - p0 : 0, leaf_ok ? pfirst[b + 1] - p0 : 0, f, cc, hh);
  }
  cell_pass_flush(s_acc, p0, CH.w, acc);
}

// minb: CTAs per SM the kernel's register budget is cut for (2, 3 or 4;
// more CTAs hide more load latency, fewer keep more values in registers).
// The dynamic shared memory (the chunk's pairs) may take the static part
// over 48 KB, so the kernels opt in to the size they are launched with.
template <class K>
static void set_smem(K kern, size_t smem) {
  // Above the default 48 KB the limit is raised to the largest a CTA may
  // have, never set to this launch's size: engines on other host threads
  // (the server's slots) launch the same kernels, and a smaller limit set
  // between another thread's call and its launch would fail that launch.
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
}

void launch_cell_boxes(int minb, int grid, cudaStream_t st, const float4* xf, const int* conn8,
                       const unsigned char* cell_nv, const int4* leaves, const int* ids, long long nleaf, float2* cbox,
                       float4* tnode, float4* lbox) {
#define TB_CB(MB) k_cell_boxes<MB><<<grid, 256, 0, st>>>(xf, conn8, cell_nv, leaves, ids, nleaf, cbox, tnode, lbox)
  if (minb <= 4) TB_CB(4);
  else if (minb <= 6) TB_CB(6);
  else TB_CB(8);
#undef TB_CB
}

void launch_cell_pairs(int minb, int grid, size_t smem, cudaStream_t st, const double* x, const int* conn8,
                       const unsigned char* cell_nv, const BlockInfo* bi, const int4* leaves, const int4* chunks,
                       const int* chunk_cta, int nchunks, const int* pfirst, const PairInfo* pairs,
                       const float2* cbox, const float4* lbox, int* ext, unsigned long long* acc) {
  set_smem(k_leaf_seeds, smem);
  k_leaf_seeds<<<grid, 256, smem, st>>>(bi, chunks, chunk_cta, nchunks, pfirst, pairs, lbox, ext);
#define TB_CPP(MB)                                                                                           \
  do {                                                                                                       \
    set_smem(k_cell_pairs<MB>, smem);                                                                        \
    k_cell_pairs<MB><<<grid, 256, smem, st>>>(x, conn8, cell_nv, bi, leaves, chunks, chunk_cta, nchunks, pfirst, \
                                              pairs, cbox, lbox, ext, acc);                                  \
  } while (0)
  if (minb <= 2) TB_CPP(2);
  else if (minb == 3) TB_CPP(3);
  else TB_CPP(4);
#undef TB_CPP
}

void launch_cell_pass64(int minb, int grid, size_t smem, cudaStream_t st, const double* x, const int* conn8,
                        const unsigned char* cell_nv, const BlockInfo* bi, const int4* leaves, const int4* chunks,
                        const int* chunk_cta, int nchunks, const int* pfirst, const PairInfo* pairs, double* cbox64,
                        float4* tnode, double* tnode64, unsigned long long* acc) {
#define TB_CP64(MB)                                                                                       \
  do {                                                                                                    \
    set_smem(k_cell_pass64<MB>, smem);                                                                    \
    k_cell_pass64<MB><<<grid, 256, smem, st>>>(x, conn8, cell_nv, bi, leaves, chunks, chunk_cta, nchunks, \
                                               pfirst, pairs, cbox64, tnode, tnode64, acc);               \
  } while (0)
  if (minb <= 2) TB_CP64(2);
  else if (minb == 3) TB_CP64(3);
  else TB_CP64(4);
#undef TB_CP64
}

// Bounding box of every tile of kNodeTile consecutive nodes of a block (FP32,
// rounded outward), so the query gathering can skip tiles far from a region;
// with xf, every node's coordinates rounded to nearest FP32 (k_cell_boxes).
// With ids, one CTA per tile listed there (those whose nodes have landed).
__global__ void __launch_bounds__(256) k_node_tiles(const double* __restrict__ x, const BlockInfo* __restrict__ bi,
                                                    int nb, const long long* __restrict__ tile_base,
                                                    float4* __restrict__ tbox, const int* __restrict__ node_order,
                                                    float4* __restrict__ xf, const int* __restrict__ ids) {
  __shared__ float sh[6][8];
  const long long T = ids ? ids[blockIdx.x] : blockIdx.x;  // the tiles listed in ids, else all
  const int b = block_of_tile(tile_base, nb, T);
  const BlockInfo& B = bi[b];
  const int t0 = (int)(T - tile_base[b]) * kNodeTile;
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i = t0 + threadIdx.x; i < min(t0 + kNodeTile, B.nnodes); i += blockDim.x) {
    const int nd = node_order[B.node_off + i];
    const double* p = x + 3 * (long long)nd;
    const float4 v = make_float4(__double2float_rn(p[0]), __double2float_rn(p[1]), __double2float_rn(p[2]), 0.f);
    if (xf) xf[nd] = v;
    lo[0] = fminf(lo[0], v.x); lo[1] = fminf(lo[1], v.y); lo[2] = fminf(lo[2], v.z);
    hi[0] = fmaxf(hi[0], v.x); hi[1] = fmaxf(hi[1], v.y); hi[2] = fmaxf(hi[2], v.z);
  }
  for (int k = 0; k < 3; k++)
    for (int o = 16; o > 0; o >>= 1) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; k++) {
      sh[k][w] = lo[k];
      sh[k + 3][w] = hi[k];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int ww = 1; ww < (int)(blockDim.x >> 5); ww++)
      for (int k = 0; k < 3; k++) {
        sh[k][0] = fminf(sh[k][0], sh[k][ww]);
        sh[k + 3][0] = fmaxf(sh[k + 3][0], sh[k + 3][ww]);
      }
    tbox[2 * T] = make_float4(f_down(sh[0][0]), f_down(sh[1][0]), f_down(sh[2][0]), f_up(sh[3][0]));
    tbox[2 * T + 1] = make_float4(f_up(sh[4][0]), f_up(sh[5][0]), 0.f, 0.f);
  }
}

// ===========================================================================
// query points: receptor nodes inside each pair's donor region
// (getQueryPoints2's exact test, |xd| <= dxc on all three axes), written in
// pair order then node order by an ordered two-pass compaction
// ===========================================================================
constexpr int kQThreads = 256;
constexpr int kQItems = 8;

__device__ __forceinline__ bool in_region(const double* p, const Obb& r) {
  double xd[3];
  for (int j = 0; j < 3; j++) {
    xd[j] = 0;
    for (int k = 0; k < 3; k++) xd[j] += (p[k] - r.xc[k]) * r.vec[j][k];
  }
  return fabs(xd[0]) <= r.dxc[0] && fabs(xd[1]) <= r.dxc[1] && fabs(xd[2]) <= r.dxc[2];
}

// A tile is skipped when its box misses the region's world box (the region
// is an oriented box inside it), so only tiles that may hold a query point are
// tested node by node.
__device__ __forceinline__ bool tile_may_hit(const float4* __restrict__ tbox, long long T, const PairInfo& P) {
  const float4 A = tbox[2 * T], C = tbox[2 * T + 1];
  return !((double)A.x > P.wbox[3] || (double)A.y > P.wbox[4] || (double)A.z > P.wbox[5] ||
           (double)A.w < P.wbox[0] || (double)C.x < P.wbox[1] || (double)C.y < P.wbox[2]);
}

// Tiles of all pairs in one list: pair p owns tiles pair_t0[p] .. pair_t0[p+1]-1
// (its receptor block's node tiles), so a launch covers every pair whatever
// the sizes of their receptor blocks.
__device__ __forceinline__ int pair_of_tile(const long long* __restrict__ pair_t0, int npairs, long long T) {
  int lo = 0, hi = npairs - 1;  // the last pair whose first tile is <= T
  while (lo < hi) {
    const int m = (lo + hi + 1) >> 1;
    if (pair_t0[m] <= T) lo = m;
    else hi = m - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(kQThreads) k_query_count(const double* __restrict__ x,
                                                           const BlockInfo* __restrict__ bi,
                                                           const PairInfo* __restrict__ pairs, int npairs,
                                                           const long long* __restrict__ pair_t0, int tile,
                                                           int* __restrict__ tile_cnt,
                                                           const float4* __restrict__ tbox,
                                                           const long long* __restrict__ tile_base,
                                                           const int* __restrict__ node_order,
                                                           unsigned char* __restrict__ tile_mask) {
  __shared__ int sh[kQThreads / 32];
  const long long ntiles = pair_t0[npairs];
  for (long long T = blockIdx.x; T < ntiles; T += gridDim.x) {
    const int p = pair_of_tile(pair_t0, npairs, T);
    const int t = (int)(T - pair_t0[p]);
    const PairInfo& P = pairs[p];
    const BlockInfo& R = bi[P.rec];
    const int n0 = t * tile;
    if (!tile_may_hit(tbox, tile_base[P.rec] + t, P)) {
      if (threadIdx.x == 0) tile_cnt[T] = 0;
      continue;
    }
    const Obb reg = P.region;
    unsigned mask = 0;
    for (int k = 0; k < kQItems; k++) {
      int i = n0 + threadIdx.x * kQItems + k;
      if (i < R.nnodes && in_region(x + 3 * (long long)node_order[R.node_off + i], reg)) mask |= 1u << k;
    }
    tile_mask[T * kQThreads + threadIdx.x] = (unsigned char)mask;  // for k_query_write
    int w = __popc(mask);
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = w;
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
      for (int k = 0; k < kQThreads / 32; k++) s += sh[k];
      tile_cnt[T] = s;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kQThreads) k_query_write(const BlockInfo* __restrict__ bi,
                                                           const PairInfo* __restrict__ pairs, int npairs,
                                                           const long long* __restrict__ pair_t0, int tile,
                                                           const int* __restrict__ tile_off,
                                                           const double* __restrict__ node_res,
                                                           int* __restrict__ qnode, int* __restrict__ qdon,
                                                           double* __restrict__ qres,
                                                           const int* __restrict__ node_order,
                                                           const unsigned char* __restrict__ tile_mask) {
  typedef cub::BlockScan<int, kQThreads> Scan;
  __shared__ typename Scan::TempStorage tmp;
  const long long ntiles = pair_t0[npairs];
  for (long long T = blockIdx.x; T < ntiles; T += gridDim.x) {
    if (tile_off[T + 1] == tile_off[T]) continue;  // culled, or no node inside
    const int p = pair_of_tile(pair_t0, npairs, T);
    const int t = (int)(T - pair_t0[p]);
    const PairInfo& P = pairs[p];
    const BlockInfo& R = bi[P.rec];
    const int n0 = t * tile;
    const unsigned mask = tile_mask[T * kQThreads + threadIdx.x];  // k_query_count's test
    int pos;
    Scan(tmp).ExclusiveSum(__popc(mask), pos);
    long long o = (long long)tile_off[T] + pos;
    for (int k = 0; k < kQItems; k++) {
      if (mask & (1u << k)) {
        int g = node_order[R.node_off + n0 + threadIdx.x * kQItems + k];
        qnode[o] = g;
        qdon[o] = P.don;
        qres[o] = node_res[g];
        o++;
      }
    }
    __syncthreads();
  }
}

// ===========================================================================
// fused tree search + containment
// ===========================================================================
// FP32 screen of the Newton inversion (hex 8, prism 6, pyramid 5) on
// coordinates relative to vertex 0.  Returns 0 reject, 1 clean interior
// accept, -1 undecided (the FP64 path decides).
// FP32 core on vertex offsets y[m] = x_m - x_0 and point offset yp = p - x_0.
// Margins: the residual is evaluated in FP32 on offsets of size h (the
// cell's), with an error below about 5e-7 h; the map's conditioning
// |det J| / (|J1| |J2| |J3|), checked every step, is at least 1e-2 (else
// FP64 decides), so the error it makes in (u, v, w) is below 5e-5.  The
// iterate stops once a step is below 3e-5, leaving a truncation error of
// the step's square over the conditioning, below 1e-7.  Every weight is then
// off by less than 2e-4, a fifth of kEps: a point classified clean inside
// has every true weight above 8e-4, one rejected a true weight below -8e-4.
__device__ __forceinline__ int screen32f(const float y[8][3], const float yp[3], int nv) {
  constexpr float kEps = 1e-3f;
  float f[8][3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    f[0][j] = -yp[j];
    if (nv == 8) {
      f[1][j] = y[1][j];
      f[2][j] = y[3][j];
      f[3][j] = y[4][j];
      f[4][j] = -y[1][j] + y[2][j] - y[3][j];
      f[5][j] = -y[3][j] + y[7][j] - y[4][j];
      f[6][j] = -y[1][j] + y[5][j] - y[4][j];
      f[7][j] = y[1][j] - y[2][j] + y[3][j] + y[4][j] - y[5][j] + y[6][j] - y[7][j];
    } else if (nv == 6) {
      f[1][j] = y[1][j];
      f[2][j] = y[2][j];
      f[3][j] = y[3][j];
      f[4][j] = 0.f;
      f[5][j] = -y[2][j] - y[3][j] + y[5][j];
      f[6][j] = -y[1][j] - y[3][j] + y[4][j];
      f[7][j] = 0.f;
    } else {
      f[1][j] = y[1][j];
      f[2][j] = y[3][j];
      f[3][j] = y[4][j];
      f[4][j] = -y[1][j] + y[2][j] - y[3][j];
      f[5][j] = -y[3][j];
      f[6][j] = -y[1][j];
      f[7][j] = y[1][j] - y[2][j] + y[3][j];
    }
  }
  float u = 0.5f, v = 0.5f, w = 0.5f;
  bool conv = false;
  float cond = 0.f;
  for (int it = 0; it < 16; it++) {
    float uv = u * v, vw = v * w, wu = w * u, uvw = uv * w;
    float r[3], J[3][3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      r[j] = __fmaf_rn(f[7][j], uvw, __fmaf_rn(f[6][j], wu, __fmaf_rn(f[5][j], vw, __fmaf_rn(f[4][j], uv,
             __fmaf_rn(f[3][j], w, __fmaf_rn(f[2][j], v, __fmaf_rn(f[1][j], u, f[0][j])))))));
      J[j][0] = __fmaf_rn(f[7][j], vw, __fmaf_rn(f[6][j], w, __fmaf_rn(f[4][j], v, f[1][j])));
      J[j][1] = __fmaf_rn(f[7][j], wu, __fmaf_rn(f[4][j], u, __fmaf_rn(f[5][j], w, f[2][j])));
      J[j][2] = __fmaf_rn(f[7][j], uv, __fmaf_rn(f[5][j], v, __fmaf_rn(f[6][j], u, f[3][j])));
    }
    float c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    float c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    float c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    float det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    float n0 = sqrtf(J[0][0] * J[0][0] + J[1][0] * J[1][0] + J[2][0] * J[2][0]);
    float n1 = sqrtf(J[0][1] * J[0][1] + J[1][1] * J[1][1] + J[2][1] * J[2][1]);
    float n2 = sqrtf(J[0][2] * J[0][2] + J[1][2] * J[1][2] + J[2][2] * J[2][2]);
    float scale = n0 * n1 * n2;
    if (!(scale > 0.f)) return -1;
    cond = fabsf(det) / scale;
    if (cond < 1e-2f) return -1;  // ill-conditioned map: let FP64 decide
    float id = 1.f / det;
    float du = (r[0] * c00 + r[1] * (J[0][2] * J[2][1] - J[0][1] * J[2][2]) +
                r[2] * (J[0][1] * J[1][2] - J[0][2] * J[1][1])) * id;
    float dv = (r[0] * c01 + r[1] * (J[0][0] * J[2][2] - J[0][2] * J[2][0]) +
                r[2] * (J[0][2] * J[1][0] - J[0][0] * J[1][2])) * id;
    float dw = (r[0] * c02 + r[1] * (J[0][1] * J[2][0] - J[0][0] * J[2][1]) +
                r[2] * (J[0][0] * J[1][1] - J[0][1] * J[1][0])) * id;
    u -= du;
    v -= dv;
    w -= dw;
    if (!(fabsf(u) < 1e3f && fabsf(v) < 1e3f && fabsf(w) < 1e3f)) return -1;
    if (fabsf(du) + fabsf(dv) + fabsf(dw) < 3e-5f) {
      conv = true;
      break;
    }
  }
  if (!conv) return -1;
  float fr[8];
  int n;
  if (nv == 8) {
    float a = 1.f - u, b = 1.f - v, c = 1.f - w;
    fr[0] = a * b * c; fr[1] = u * b * c; fr[2] = u * v * c; fr[3] = a * v * c;
    fr[4] = a * b * w; fr[5] = u * b * w; fr[6] = u * v * w; fr[7] = a * v * w;
    n = 8;
  } else if (nv == 6) {
    float a = 1.f - u - v, c = 1.f - w;
    fr[0] = a * c; fr[1] = u * c; fr[2] = v * c; fr[3] = a * w; fr[4] = u * w; fr[5] = v * w;
    n = 6;
  } else {
    float a = 1.f - u, b = 1.f - v, c = 1.f - w;
    fr[0] = a * b * c; fr[1] = u * b * c; fr[2] = u * v * c; fr[3] = a * v * c; fr[4] = w;
    n = 5;
  }
  bool interior = true;
  for (int m = 0; m < n; m++) {
    if (fr[m] < -kEps || fr[m] > 1.f + kEps) return 0;
    if (fr[m] < kEps || fr[m] > 1.f - kEps) interior = false;
  }
  return interior ? 1 : -1;
}

__device__ __forceinline__ int screen32(const double xv[8][3], const double p[3], int nv) {
  float y[8][3], yp[3];
#pragma unroll
  for (int m = 0; m < 8; m++)
    if (m < nv)
#pragma unroll
      for (int j = 0; j < 3; j++) y[m][j] = (float)(xv[m][j] - xv[0][j]);
#pragma unroll
  for (int j = 0; j < 3; j++) yp[j] = (float)(p[j] - xv[0][j]);
  return screen32f(y, yp, nv);
}

// ---------------------------------------------------------------------------
// Search, stage 1: stack-free traversal of the donor block's tree.  Every
// cell whose (conservative) box holds the point is appended to the candidate
// list as (query, sorted cell position).  FORM 0 tests FP64 boxes with the
// reference's +-TOL (exact candidates); FORM 1 tests FP32 boxes rounded
// outward with a relative margin (a superset, filtered exactly in stage 2).
// ---------------------------------------------------------------------------
// Candidates of a query go to kSlots inline slots of that query; the rare
// extra ones (thin cells crowding a pole axis) go to an overflow list.  No
// global counter is touched for the common case.
__device__ __forceinline__ void add_candidate(int q, int s, int& n, int* __restrict__ slots,
                                              int3* __restrict__ ovf, int ovf_cap, unsigned* __restrict__ novf) {
  if (n < kSlots) {
    slots[(long long)q * kSlots + n] = s;
  } else {
    const unsigned i = atomicAdd(novf, 1u);
    if (i < (unsigned)ovf_cap) ovf[i] = make_int3(q, s, n);
  }
  n++;
}

// box [A.xyz, (A.w, B.x, B.y)] against the point interval [lo, hi] = p -+ e
__device__ __forceinline__ bool hit32(const float4* __restrict__ tn, long long slot, const float* lo,
                                      const float* hi) {
  const float4 A = tn[2 * slot], B = tn[2 * slot + 1];
  return A.x <= hi[0] && A.y <= hi[1] && A.z <= hi[2] && A.w >= lo[0] && B.x >= lo[1] && B.y >= lo[2];
}
__device__ __forceinline__ bool hit64(const double* __restrict__ tn, long long slot, const double* p) {
  const double* b = tn + 6 * slot;
  return p[0] >= b[0] - kTol && p[1] >= b[1] - kTol && p[2] >= b[2] - kTol && p[0] <= b[3] + kTol &&
         p[1] <= b[4] + kTol && p[2] <= b[5] + kTol;
}

// FP32 node or cell box [A.xyz, (A.w, B.x, B.y)] against the point interval
__device__ __forceinline__ bool hit_ab(const float4& A, const float4& B, const float* lo, const float* hi) {
  return A.x <= hi[0] && A.y <= hi[1] && A.z <= hi[2] && A.w >= lo[0] && B.x >= lo[1] && B.y >= lo[2];
}
__device__ __forceinline__ int pick4(int k, int a0, int a1, int a2, int a3) {
  return k == 0 ? a0 : (k == 1 ? a1 : (k == 2 ? a2 : a3));
}

// Depth-first walk of the donor block's radix tree.  Every step tests the
// four slots of one child group (one 128-byte line) against the point; hit
// leaves have their cells tested at once, the first hit internal child is
// entered and the other hit ones are kept as a 4-bit mask for the current
// depth in the trail (two 64-bit words, 32 depths), with the group's base
// slot in shared memory.  The next node after a subtree is always in the
// deepest non-empty mask.
template <int FORM>
__global__ void __launch_bounds__(256) k_traverse(
    const double* __restrict__ x, const BlockInfo* __restrict__ bi, const float2* __restrict__ cbox,
    const double* __restrict__ cbox64, const float4* __restrict__ tnode, const double* __restrict__ tnode64,
    const int* __restrict__ qnode, const int* __restrict__ qdon, long long nq, int* __restrict__ slots,
    int* __restrict__ ncand_q, int3* __restrict__ ovf, int ovf_cap, unsigned* __restrict__ novf,
    unsigned* __restrict__ err, int skip_uhex) {
  __shared__ int s_base[kMaxTreeDepth][256];
  const int t = threadIdx.x;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    int n = 0;
    const int g = qnode[q];
    const int root = bi[qdon[q]].root;
    if (skip_uhex && bi[qdon[q]].uhex) {  // searched by k_uhex_search instead
      ncand_q[q] = 0;
      continue;
    }
    double p[3];
    float plo[3], phi[3];  // the point widened by a margin that covers TOL and FP32 rounding
    p[0] = x[3 * (long long)g];
    p[1] = x[3 * (long long)g + 1];
    p[2] = x[3 * (long long)g + 2];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float p32 = (float)p[k];
      const float e = fabsf(p32) * 9.6e-7f + 2e-9f;
      plo[k] = p32 - e;
      phi[k] = p32 + e;
    }
    // cells [c0, c0 + nc) of a hit leaf (1 <= nc <= kMaxLeafCells).  FP32
    // boxes: the loop is unrolled and every slot reads a cell of the leaf
    // (the last one again past nc), so all the box loads are issued before
    // the first test, one memory round trip per leaf.  Hits are added in
    // cell order.
    auto leaf_cells = [&](int c0, int ncell) {
      unsigned hit = 0;
      if (FORM == 0) {  // (FP64 boxes: 48 B a cell, tested one at a time)
        for (int j = 0; j < ncell; j++) {
          const double* bb = cbox64 + 6 * (long long)(c0 + j);
          const double lo[3] = {bb[0], bb[1], bb[2]}, hi[3] = {bb[3], bb[4], bb[5]};
          hit |= (unsigned)in_box64(p, lo, hi) << j;
        }
      } else {
        float4 A[kMaxLeafCells], B[kMaxLeafCells];
#pragma unroll
        for (int j = 0; j < kMaxLeafCells; j++) {
          cell_box_load(cbox, c0 + min(j, ncell - 1), A[j], B[j]);
        }
#pragma unroll
        for (int j = 0; j < kMaxLeafCells; j++) hit |= (unsigned)(hit_ab(A[j], B[j], plo, phi) && j < ncell) << j;
      }
      while (hit) {
        const int j = __ffs(hit) - 1;
        hit &= hit - 1;
        add_candidate((int)q, c0 + j, n, slots, ovf, ovf_cap, novf);
      }
    };
    if (root >= 0) {
      const float4 RA = tnode[2 * root], RB = tnode[2 * root + 1];
      const bool rh = (FORM == 0) ? hit64(tnode64, root, p) : hit_ab(RA, RB, plo, phi);
      const int rlink = __float_as_int(RB.z), rcnt = __float_as_int(RB.w);
      if (rh && rcnt > 0) leaf_cells(rlink, rcnt);
      if (rh && rcnt < 0) {
        int base = rlink, depth = 0;
        unsigned long long tr0 = 0, tr1 = 0;  // masks of depths 0-15 and 16-31
        for (;;) {
          int lk[4], lc[4];
          unsigned mi = 0, ml = 0;
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const long long sl = base + k;
            const float4 A = tnode[2 * sl], B = tnode[2 * sl + 1];
            lk[k] = __float_as_int(B.z);
            lc[k] = __float_as_int(B.w);
            const bool h = (FORM == 0) ? (lc[k] != 0 && hit64(tnode64, sl, p)) : hit_ab(A, B, plo, phi);
            if (h) {
              if (lc[k] > 0) ml |= 1u << k;
              else mi |= 1u << k;
            }
          }
          while (ml) {
            const int k = __ffs(ml) - 1;
            ml &= ml - 1;
            leaf_cells(pick4(k, lk[0], lk[1], lk[2], lk[3]), pick4(k, lc[0], lc[1], lc[2], lc[3]));
          }
          if (mi) {
            const int c = __ffs(mi) - 1;
            mi &= mi - 1;
            if (mi) {
              if (depth < 16) tr0 |= (unsigned long long)mi << (4 * depth);
              else tr1 |= (unsigned long long)mi << (4 * (depth - 16));
              s_base[depth][t] = base;
            }
            base = pick4(c, lk[0], lk[1], lk[2], lk[3]);
            if (++depth >= kMaxTreeDepth) {  // deeper than the trail (the build refuses such trees)
              atomicOr(err, kErrTraversalOverflow);
              break;
            }
            continue;
          }
          int d2;
          unsigned mm;
          if (tr1) {
            d2 = 16 + ((63 - __clzll((long long)tr1)) >> 2);
            mm = (unsigned)(tr1 >> (4 * (d2 - 16))) & 0xFu;
            tr1 &= ~(1ull << (4 * (d2 - 16) + __ffs(mm) - 1));
          } else if (tr0) {
            d2 = (63 - __clzll((long long)tr0)) >> 2;
            mm = (unsigned)(tr0 >> (4 * d2)) & 0xFu;
            tr0 &= ~(1ull << (4 * d2 + __ffs(mm) - 1));
          } else {
            break;
          }
          const long long sl = s_base[d2][t] + __ffs(mm) - 1;
          base = __float_as_int(tnode[2 * sl + 1].z);
          depth = d2 + 1;
        }
      }
    }
    ncand_q[q] = n;
  }
}

// The split form's traversal with postponed leaves: each lane walks its
// query's tree until it holds a hit leaf or has nothing left, and only when no
// lane of the warp still walks (every lane holds a leaf or is done) does the
// warp test the held leaves' cells together; then the walk resumes.  Node
// visits and leaf tests each run with the lanes that need them side by side,
// where the walk of k_traverse mixes them within a warp.  The trail keeps,
// per depth, the hit children (leaves and internal nodes) still to visit;
// the deepest goes first, so the order is a depth-first one as in
// k_traverse, and every hit leaf's cells are tested, so each query gets the
// same candidates (in another order, which the selection does not see).
__global__ void __launch_bounds__(256) k_traverse_ww(
    const double* __restrict__ x, const BlockInfo* __restrict__ bi, const float2* __restrict__ cbox,
    const float4* __restrict__ tnode, const int* __restrict__ qnode, const int* __restrict__ qdon, long long nq,
    int* __restrict__ slots, int* __restrict__ ncand_q, int3* __restrict__ ovf, int ovf_cap,
    unsigned* __restrict__ novf, unsigned* __restrict__ err, int skip_uhex) {
  __shared__ int s_base[kMaxTreeDepth][256];
  const int t = threadIdx.x, lane = t & 31;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q0 = blockIdx.x * (long long)blockDim.x + (t & ~31); q0 < nq; q0 += stride) {
    const long long q = q0 + lane;
    bool active = q < nq;
    int root = -1;
    if (active) {
      const BlockInfo& B = bi[qdon[q]];
      root = B.root;
      if (skip_uhex && B.uhex) {  // searched by k_uhex_search instead
        ncand_q[q] = 0;
        active = false;
      }
    }
    int n = 0;
    float plo[3] = {0.f, 0.f, 0.f}, phi[3] = {0.f, 0.f, 0.f};  // the point widened as in k_traverse
    if (active) {
      const int g = qnode[q];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const float p32 = (float)x[3 * (long long)g + k];
        const float e = fabsf(p32) * 9.6e-7f + 2e-9f;
        plo[k] = p32 - e;
        phi[k] = p32 + e;
      }
    }
    int base = -1, depth = 0;             // the next group to visit and its depth
    unsigned long long tr0 = 0, tr1 = 0;  // hit children still to visit, 4 bits per depth (0-15, 16-31)
    int lf0 = 0, lfn = 0;                 // the held leaf: first cell, cells
    if (active && root >= 0) {
      const float4 RA = tnode[2 * root], RB = tnode[2 * root + 1];
      const int rlink = __float_as_int(RB.z), rcnt = __float_as_int(RB.w);
      if (hit_ab(RA, RB, plo, phi)) {
        if (rcnt > 0) {
          lf0 = rlink;
          lfn = rcnt;
        } else if (rcnt < 0) {
          base = rlink;
        }
      }
    }
    for (;;) {
      for (;;) {  // walk until every lane holds a leaf or is done
        const bool walk = lfn == 0 && (base >= 0 || (tr0 | tr1) != 0ull);
        if (!__any_sync(0xffffffffu, walk)) break;
        if (!walk) continue;
        if (base < 0) {  // the deepest child still to visit
          int d2;
          unsigned mm;
          if (tr1) {
            d2 = 16 + ((63 - __clzll((long long)tr1)) >> 2);
            mm = (unsigned)(tr1 >> (4 * (d2 - 16))) & 0xFu;
            tr1 &= ~(1ull << (4 * (d2 - 16) + __ffs(mm) - 1));
          } else {
            d2 = (63 - __clzll((long long)tr0)) >> 2;
            mm = (unsigned)(tr0 >> (4 * d2)) & 0xFu;
            tr0 &= ~(1ull << (4 * d2 + __ffs(mm) - 1));
          }
          const long long sl = s_base[d2][t] + __ffs(mm) - 1;
          const float4 B = tnode[2 * sl + 1];
          const int lk = __float_as_int(B.z), cnt = __float_as_int(B.w);
          if (cnt > 0) {
            lf0 = lk;
            lfn = cnt;
          } else if (d2 + 1 < kMaxTreeDepth) {
            base = lk;
            depth = d2 + 1;
          } else {  // deeper than the trail (the build refuses such trees)
            atomicOr(err, kErrTraversalOverflow);
            tr0 = tr1 = 0ull;
          }
          continue;
        }
        int lk[4], lc[4];
        unsigned h = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const long long sl = base + k;
          const float4 A = tnode[2 * sl], B = tnode[2 * sl + 1];
          lk[k] = __float_as_int(B.z);
          lc[k] = __float_as_int(B.w);
          if (hit_ab(A, B, plo, phi)) h |= 1u << k;
        }
        const int gbase = base;
        base = -1;
        if (h) {
          const int k = __ffs(h) - 1;
          h &= h - 1;
          if (h) {
            if (depth < 16) tr0 |= (unsigned long long)h << (4 * depth);
            else tr1 |= (unsigned long long)h << (4 * (depth - 16));
            s_base[depth][t] = gbase;
          }
          const int ck = pick4(k, lk[0], lk[1], lk[2], lk[3]), cc = pick4(k, lc[0], lc[1], lc[2], lc[3]);
          if (cc > 0) {
            lf0 = ck;
            lfn = cc;
          } else if (depth + 1 < kMaxTreeDepth) {
            base = ck;
            depth++;
          } else {  // deeper than the trail (the build refuses such trees)
            atomicOr(err, kErrTraversalOverflow);
            tr0 = tr1 = 0ull;
          }
        }
      }
      if (lfn > 0) {  // the held leaves, side by side: all box loads first, then the tests
        float4 A[kMaxLeafCells], B[kMaxLeafCells];
#pragma unroll
        for (int j = 0; j < kMaxLeafCells; j++) {
          cell_box_load(cbox, lf0 + min(j, lfn - 1), A[j], B[j]);
        }
        unsigned hit = 0;
#pragma unroll
        for (int j = 0; j < kMaxLeafCells; j++) hit |= (unsigned)(hit_ab(A[j], B[j], plo, phi) && j < lfn) << j;
        while (hit) {
          const int j = __ffs(hit) - 1;
          hit &= hit - 1;
          add_candidate((int)q, lf0 + j, n, slots, ovf, ovf_cap, novf);
        }
        lfn = 0;
      }
      if (!__any_sync(0xffffffffu, base >= 0 || (tr0 | tr1) != 0ull)) break;
    }
    if (active) ncand_q[q] = n;
  }
}

// Dense, query-ordered candidate list from the slots and the overflow list
// (off = exclusive scan of the per-query counts).
__global__ void k_gather_candidates(const int* __restrict__ slots, const int* __restrict__ ncand_q,
                                    const int* __restrict__ off, long long nq, const int3* __restrict__ ovf,
                                    const unsigned* __restrict__ novf, int ovf_cap, int2* __restrict__ cand) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const int n = min(ncand_q[q], kSlots);
    const int o = off[q];
    for (int k = 0; k < n; k++) cand[o + k] = make_int2((int)q, slots[q * kSlots + k]);
  }
  const int no = min((int)*novf, ovf_cap);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < no; i += gridDim.x * blockDim.x) {
    const int3 e = ovf[i];
    cand[off[e.x] + e.z] = make_int2(e.x, e.y);
  }
}

// The query's outcome is the lowest cell id among clean accepts, else among
// accepts on a no-donor cell's face: one ordered 64-bit key per query,
// (face accept) << 32 | cell, merged with atomicMin.  The accept counters
// (low half: accepts, high half: face accepts) flag order-dependent ties.
__device__ __forceinline__ void record_accept(int q, int c, int cls, unsigned long long* __restrict__ qkey,
                                              unsigned* __restrict__ qacc) {
  if (cls <= 0) return;
  const unsigned long long key = ((unsigned long long)(cls == 2) << 32) | (unsigned)c;
  atomicMin(&qkey[q], key);
  atomicAdd(&qacc[q], cls == 2 ? 0x10001u : 1u);
}

// ---------------------------------------------------------------------------
// Search, stage 2: one thread per candidate.  The exact FP64 element box
// (searchADTrecursion.C:63-66) filters the superset; FORM 1 screens the
// Newton inversion in FP32 and defers undecided candidates and tets to stage
// 3; FORM 0 decides everything with the reference's FP64 arithmetic.
// ---------------------------------------------------------------------------
template <int FORM>
__global__ void __launch_bounds__(256, FORM == 1 ? 3 : 2) k_candidates(
    const double* __restrict__ x, const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
    const double* __restrict__ cell_res, const int* __restrict__ sorted_cell, const int* __restrict__ qnode,
    const int2* __restrict__ cand, int ncand, unsigned long long* __restrict__ qkey,
    unsigned* __restrict__ qacc, int* __restrict__ refine, unsigned* __restrict__ nrefine,
    unsigned long long* __restrict__ counters) {
  unsigned long long my_cand = 0, my_verts = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncand; i += gridDim.x * blockDim.x) {
    const int2 qs = cand[i];
    const int q = qs.x;
    const int c = qs.y;  // storage position; the tie rule uses the registration id
    const int nv = cell_nv[c];
    const int4 c0 = *reinterpret_cast<const int4*>(conn8 + 8 * (long long)c);
    const int4 c1 = *reinterpret_cast<const int4*>(conn8 + 8 * (long long)c + 4);
    const int cv[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    const int g = qnode[q];
    const double p[3] = {x[3 * (long long)g], x[3 * (long long)g + 1], x[3 * (long long)g + 2]};
    int cls;
    if (FORM == 1) {
      // exact FP64 element box while streaming the vertices; keep only the
      // FP32 offsets from vertex 0 for the screen.  Slots past nv read
      // vertex 0 again (a no-op for the box, offsets unused), so every load
      // is unconditional and all of them are in flight at once.
      const double* v0p = x + 3 * (long long)cv[0];
      const double v0[3] = {v0p[0], v0p[1], v0p[2]};
      double lo[3] = {v0[0], v0[1], v0[2]}, hi[3] = {v0[0], v0[1], v0[2]};
      float y[8][3];
      y[0][0] = y[0][1] = y[0][2] = 0.f;
#pragma unroll
      for (int m = 1; m < 8; m++) {
        const double* vp = x + 3 * (long long)(m < nv ? cv[m] : cv[0]);
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const double v = vp[k];
          lo[k] = dmin(lo[k], v);
          hi[k] = dmax(hi[k], v);
          y[m][k] = (float)(v - v0[k]);
        }
      }
      if (!in_box64(p, lo, hi)) continue;
      my_cand++;
      my_verts += nv;
      const float yp[3] = {(float)(p[0] - v0[0]), (float)(p[1] - v0[1]), (float)(p[2] - v0[2])};
      cls = (nv == 4) ? -1 : screen32f(y, yp, nv);
      if (cls < 0) {
        const unsigned r = atomicAdd(nrefine, 1u);
        refine[r] = i;  // capacity: one slot per candidate
        continue;
      }
    } else {
      double xv[8][3];
      gather_vertices(x, cv, nv, xv);
      my_cand++;
      my_verts += nv;
      double frac[8];
      nodal_weights64(xv, p, frac, nv);
      cls = classify64(frac, nv, cell_res[c] == kBig);
    }
    record_accept(q, sorted_cell[c], cls, qkey, qacc);
  }
  for (int o = 16; o > 0; o >>= 1) {
    my_cand += __shfl_xor_sync(0xffffffffu, my_cand, o);
    my_verts += __shfl_xor_sync(0xffffffffu, my_verts, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&counters[0], my_cand);
    atomicAdd(&counters[6], my_verts);
  }
}

// Search, stage 3: the reference's FP64 Newton for the deferred candidates.
__global__ void __launch_bounds__(128) k_refine(const double* __restrict__ x, const int* __restrict__ conn8,
                                                const unsigned char* __restrict__ cell_nv,
                                                const double* __restrict__ cell_res,
                                                const int* __restrict__ sorted_cell, const int* __restrict__ qnode,
                                                const int2* __restrict__ cand, const int* __restrict__ refine,
                                                const unsigned* __restrict__ nrefine,
                                                unsigned long long* __restrict__ qkey, unsigned* __restrict__ qacc) {
  const int n = (int)*nrefine;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int2 qs = cand[refine[k]];
    const int q = qs.x;
    const int c = qs.y;
    const int nv = cell_nv[c];
    double xv[8][3];
    gather_vertices(x, conn8 + 8 * (long long)c, nv, xv);
    const int g = qnode[q];
    const double p[3] = {x[3 * (long long)g], x[3 * (long long)g + 1], x[3 * (long long)g + 2]};
    double frac[8];
    nodal_weights64(xv, p, frac, nv);
    record_accept(q, sorted_cell[c], classify64(frac, nv, cell_res[c] == kBig), qkey, qacc);
  }
}

// Search, stage 4: per query outcome and tie flags.
__global__ void k_search_finish(const unsigned long long* __restrict__ qkey, const unsigned* __restrict__ qacc,
                                long long nq, const int* __restrict__ inv_sorted, int* __restrict__ qcell,
                                unsigned char* __restrict__ qtie, unsigned long long* __restrict__ counters) {
  unsigned long long my_tie = 0, my_found = 0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const unsigned long long key = qkey[q];
    const int donor = (key == ~0ull) ? -1 : inv_sorted[(int)(key & 0xffffffffull)];
    const unsigned acc = qacc[q];
    const unsigned nacc = acc & 0xffffu, nprov = acc >> 16;
    const unsigned char tie = (unsigned char)((nacc >= 2 ? 1 : 0) | (nprov >= 1 ? 2 : 0));
    qcell[q] = donor;
    qtie[q] = tie;
    my_tie += (tie != 0);
    my_found += (donor >= 0);
  }
  for (int o = 16; o > 0; o >>= 1) {
    my_tie += __shfl_xor_sync(0xffffffffu, my_tie, o);
    my_found += __shfl_xor_sync(0xffffffffu, my_found, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&counters[2], my_tie);
    atomicAdd(&counters[3], my_found);
  }
}

void launch_traverse(int form, int variant, int blocks, cudaStream_t st, const double* x, const BlockInfo* bi,
                     const float2* cbox, const double* cbox64, const float4* tnode, const double* tnode64,
                     const int* qnode, const int* qdon, long long nq, int* slots, int* ncand_q, int3* ovf,
                     int ovf_cap, unsigned* novf, unsigned* err, int skip_uhex) {
  if (form == 1 && variant == 1)
    k_traverse_ww<<<blocks, 256, 0, st>>>(x, bi, cbox, tnode, qnode, qdon, nq, slots, ncand_q, ovf, ovf_cap, novf,
                                          err, skip_uhex);
  else if (form == 0)
    k_traverse<0><<<blocks, 256, 0, st>>>(x, bi, cbox, cbox64, tnode, tnode64, qnode, qdon, nq, slots, ncand_q,
                                          ovf, ovf_cap, novf, err, skip_uhex);
  else
    k_traverse<1><<<blocks, 256, 0, st>>>(x, bi, cbox, cbox64, tnode, tnode64, qnode, qdon, nq, slots, ncand_q,
                                          ovf, ovf_cap, novf, err, skip_uhex);
}

void launch_candidates(int form, int blocks, cudaStream_t st, const double* x, const int* conn8,
                       const unsigned char* cell_nv, const double* cell_res, const int* sorted_cell,
                       const int* qnode, const int2* cand, int ncand, unsigned long long* qkey, unsigned* qacc,
                       int* refine, unsigned* nrefine, unsigned long long* counters) {
  if (form == 0)
    k_candidates<0><<<blocks, 256, 0, st>>>(x, conn8, cell_nv, cell_res, sorted_cell, qnode, cand, ncand, qkey,
                                            qacc, refine, nrefine, counters);
  else
    k_candidates<1><<<blocks, 256, 0, st>>>(x, conn8, cell_nv, cell_res, sorted_cell, qnode, cand, ncand, qkey,
                                            qacc, refine, nrefine, counters);
}

}  // namespace tb
