// tree_dev.cu -- refinement marking and the tree of a regrid on the device.
//
// The same rules as the host restatement (tree.cu, amr.regrid): FLASH's
// marking (Grid_markRefineDerefine.F90, paramesh4/gr_markRefineDerefine.F90)
// from the estimator's errors, then PARAMESH's amr_refine_derefine: marked
// leaves below the top level are split, refinement spreads until every
// leaf's neighbours (diagonals included) are within one level, and a
// parent's children are removed when all of them are unrefined leaves
// marked for derefinement and no neighbour's child touching the parent stays
// refined.  The tree lives in a dense table per level over every block
// position (0 absent, 1 leaf, 2 inner), the layout of the context's
// node-by-position table; each rule is a kernel over the positions, repeated
// until nothing changes (the result does not depend on the order in which a
// pass applies its changes: balance only adds splits, and derefinement
// removes candidates monotonically towards the largest unblocked set).  The
// new nodes are numbered by level and then Morton index through a scan over
// Morton-ordered slots of each level.
#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <stdint.h>
#include "hy_launch.h"

namespace fhy {

namespace {

struct Lv {
  int L, ndim;
  int off[18];          // position table offset of level l (the context's at_off)
  int ext[18][3];
  long moff[18];        // Morton slot offset of level l
  int mbits[18];        // bits per coordinate of level l's Morton slots
  int per[3];           // periodic axes
};

__device__ __forceinline__ long pos_of(const Lv &V, int l, int x, int y, int z) {
  return V.off[l] + ((long)z * V.ext[l][1] + y) * V.ext[l][0] + x;
}
__device__ __forceinline__ void coords_of(const Lv &V, int l, long q, int c[3]) {
  const long r = q - V.off[l];
  c[0] = (int)(r % V.ext[l][0]);
  c[1] = (int)((r / V.ext[l][0]) % V.ext[l][1]);
  c[2] = (int)(r / ((long)V.ext[l][0] * V.ext[l][1]));
}
__device__ __forceinline__ int level_of(const Lv &V, long q) {
  int l = 1;
  while (l < V.L && q >= V.off[l + 1]) ++l;
  return l;
}
// neighbour position at offset o on level l (periodic wrap), false outside
__device__ __forceinline__ bool nb_pos(const Lv &V, int l, const int c[3], const int o[3], int p[3]) {
  for (int d = 0; d < 3; ++d) {
    int v = c[d] + (d < V.ndim ? o[d] : 0);
    if (d < V.ndim && (v < 0 || v >= V.ext[l][d])) {
      if (!V.per[d]) return false;
      v = ((v % V.ext[l][d]) + V.ext[l][d]) % V.ext[l][d];
    }
    p[d] = v;
  }
  return true;
}
// does neighbour p (level l, offset o from the block) have a child touching
// the block that is inner (T == 2) and, with `cand`, not a candidate?
__device__ __forceinline__ bool touching_inner_child(const Lv &V, const unsigned char *T, const unsigned char *cand,
                                                     int l, const int p[3], const int o[3]) {
  for (int q = 0; q < (1 << V.ndim); ++q) {
    const int ch[3] = {2 * p[0] + (q & 1), V.ndim > 1 ? 2 * p[1] + ((q >> 1) & 1) : 0,
                       V.ndim > 2 ? 2 * p[2] + ((q >> 2) & 1) : 0};
    bool touch = true;
    for (int d = 0; d < V.ndim; ++d) {
      const int co = ch[d] - 2 * p[d];
      if ((o[d] == 1 && co != 0) || (o[d] == -1 && co != 1)) touch = false;
    }
    if (!touch) continue;
    const long cq = pos_of(V, l + 1, ch[0], ch[1], ch[2]);
    if (T[cq] == 2 && !(cand && cand[cq])) return true;
  }
  return false;
}
__device__ __forceinline__ void split_at(const Lv &V, unsigned char *T, int l, const int c[3]) {
  T[pos_of(V, l, c[0], c[1], c[2])] = 2;
  for (int q = 0; q < (1 << V.ndim); ++q)
    T[pos_of(V, l + 1, 2 * c[0] + (q & 1), V.ndim > 1 ? 2 * c[1] + ((q >> 1) & 1) : 0,
             V.ndim > 2 ? 2 * c[2] + ((q >> 2) & 1) : 0)] = 1;
}
template <class F>
__device__ __forceinline__ bool any_offset(const Lv &V, F f) {
  for (int z = -1; z <= (V.ndim > 2 ? 1 : -1); ++z)
    for (int y = -1; y <= (V.ndim > 1 ? 1 : -1); ++y)
      for (int x = -1; x <= 1; ++x) {
        const int o[3] = {x, V.ndim > 1 ? y : 0, V.ndim > 2 ? z : 0};
        if (!o[0] && !o[1] && !o[2]) continue;
        if (f(o)) return true;
      }
  return false;
}

// FLASH's marking rules, per node, variable by variable (amr.mark_refine_derefine)
__global__ void k_mark(const double *err, int nvar, int nblocks, const double *rc, const double *dc,
                       const int *level, const int *leaf, const int *parent, int max_refine, unsigned char *refine,
                       unsigned char *derefine) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  bool r = false, d = false, stay = false;
  const bool lf = leaf[b] != 0, top = level[b] >= max_refine;
  for (int v = 0; v < nvar; ++v) {
    const double e = err[(size_t)v * nblocks + b];
    const double ep = parent[b] >= 0 ? err[(size_t)v * nblocks + parent[b]] : 0.0;
    d = lf && !r && !stay && e <= dc[v] && ep <= dc[v];
    const bool up = e > rc[v];
    d = d && !up;
    r = r || up;
    stay = stay || (lf && e > dc[v]) || ep > dc[v];
    r = r && !top;
  }
  refine[b] = r && lf;
  derefine[b] = d && lf;
}

__global__ void k_tree_init(Lv V, int nblocks, const int *level, const int *coord, const int *leaf, unsigned char *T) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  T[pos_of(V, level[b], coord[3 * b], coord[3 * b + 1], coord[3 * b + 2])] = leaf[b] ? 1 : 2;
}

__global__ void k_tree_split_marked(Lv V, int nblocks, const int *level, const int *coord, const int *leaf,
                                    const unsigned char *refine, unsigned char *T) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks || !refine[b] || !leaf[b] || level[b] >= V.L) return;
  const int c[3] = {coord[3 * b], coord[3 * b + 1], coord[3 * b + 2]};
  split_at(V, T, level[b], c);
}

// balance pass, part 1: leaves (below the top level) next to an inner
// neighbour with an inner child touching them
__global__ void k_balance_mark(Lv V, long npos, const unsigned char *T, unsigned char *flag, int *changed) {
  const long q = V.off[1] + blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= V.off[1] + npos || T[q] != 1) return;
  const int l = level_of(V, q);
  if (l >= V.L) return;
  int c[3];
  coords_of(V, l, q, c);
  const bool need = any_offset(V, [&](const int o[3]) {
    int p[3];
    if (!nb_pos(V, l, c, o, p) || T[pos_of(V, l, p[0], p[1], p[2])] != 2) return false;
    return touching_inner_child(V, T, nullptr, l, p, o);
  });
  if (need) { flag[q] = 1; *changed = 1; }
}
// part 2: split the flagged leaves
__global__ void k_balance_apply(Lv V, long npos, unsigned char *T, unsigned char *flag) {
  const long q = V.off[1] + blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= V.off[1] + npos || !flag[q]) return;
  flag[q] = 0;
  const int l = level_of(V, q);
  int c[3];
  coords_of(V, l, q, c);
  split_at(V, T, l, c);
}

// derefinement candidates: old parents at or above min_level whose children
// are all (still) leaves that were old leaves marked for derefinement
__global__ void k_deref_cand(Lv V, long npos, int min_level, const unsigned char *T, const int *old_at,
                             const int *old_leaf, const unsigned char *derefine, unsigned char *cand) {
  const long q = V.off[1] + blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= V.off[1] + npos) return;
  const int b = old_at[q];
  cand[q] = 0;
  if (b < 0 || old_leaf[b]) return;
  const int l = level_of(V, q);
  if (l < min_level || l >= V.L) return;
  int c[3];
  coords_of(V, l, q, c);
  for (int o = 0; o < (1 << V.ndim); ++o) {
    const long cq = pos_of(V, l + 1, 2 * c[0] + (o & 1), V.ndim > 1 ? 2 * c[1] + ((o >> 1) & 1) : 0,
                           V.ndim > 2 ? 2 * c[2] + ((o >> 2) & 1) : 0);
    const int cb = old_at[cq];
    if (T[cq] != 1 || cb < 0 || !old_leaf[cb] || !derefine[cb]) return;
  }
  cand[q] = 1;
}
// one pass: candidates next to an inner neighbour whose touching child stays
// refined (inner and not a candidate) are dropped
__global__ void k_deref_block(Lv V, long npos, const unsigned char *T, const unsigned char *cand, unsigned char *drop,
                              int *changed) {
  const long q = V.off[1] + blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= V.off[1] + npos || !cand[q]) return;
  const int l = level_of(V, q);
  int c[3];
  coords_of(V, l, q, c);
  const bool blocked = any_offset(V, [&](const int o[3]) {
    int p[3];
    if (!nb_pos(V, l, c, o, p) || T[pos_of(V, l, p[0], p[1], p[2])] != 2) return false;
    return touching_inner_child(V, T, cand, l, p, o);
  });
  if (blocked) { drop[q] = 1; *changed = 1; }
}
__global__ void k_deref_drop(long off1, long npos, unsigned char *cand, unsigned char *drop) {
  const long q = off1 + blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= off1 + npos || !drop[q]) return;
  drop[q] = 0;
  cand[q] = 0;
}
__global__ void k_deref_merge(Lv V, long npos, const unsigned char *cand, unsigned char *T) {
  const long q = V.off[1] + blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= V.off[1] + npos || !cand[q]) return;
  const int l = level_of(V, q);
  int c[3];
  coords_of(V, l, q, c);
  T[q] = 1;
  for (int o = 0; o < (1 << V.ndim); ++o)
    T[pos_of(V, l + 1, 2 * c[0] + (o & 1), V.ndim > 1 ? 2 * c[1] + ((o >> 1) & 1) : 0,
             V.ndim > 2 ? 2 * c[2] + ((o >> 2) & 1) : 0)] = 0;
}

// Morton slot m of level l -> coordinates (bits interleaved x, y[, z])
__device__ __forceinline__ void demorton(const Lv &V, long m, int c[3]) {
  c[0] = c[1] = c[2] = 0;
  for (int bit = 0; bit < 20; ++bit)
    for (int d = 0; d < V.ndim; ++d) c[d] |= (int)((m >> (V.ndim * bit + d)) & 1) << bit;
}
__device__ __forceinline__ long enmorton(const Lv &V, const int c[3]) {
  long m = 0;
  for (int bit = 0; bit < 20; ++bit)
    for (int d = 0; d < V.ndim; ++d) m |= (long)((c[d] >> bit) & 1) << (V.ndim * bit + d);
  return m;
}
__device__ __forceinline__ int slot_level(const Lv &V, long s) {
  int l = 1;
  while (l < V.L && s >= V.moff[l + 1]) ++l;
  return l;
}
__global__ void k_slot_flags(Lv V, long nslots, const unsigned char *T, int *flag) {
  const long s = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  const int l = slot_level(V, s);
  int c[3];
  demorton(V, s - V.moff[l], c);
  bool in = true;
  for (int d = 0; d < 3; ++d) in = in && c[d] < V.ext[l][d];
  flag[s] = in && T[pos_of(V, l, c[0], c[1], c[2])] != 0;
}
__global__ void k_emit(Lv V, long nslots, const int *flag, const int *idx, const unsigned char *T, const int *old_at,
                       const int *old_leaf, int *levels, int *coords, int *parent, int *src, int *how, int *bad) {
  const long s = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (s >= nslots || !flag[s]) return;
  const int l = slot_level(V, s);
  int c[3];
  demorton(V, s - V.moff[l], c);
  const int q = idx[s];
  levels[q] = l;
  coords[3 * q] = c[0]; coords[3 * q + 1] = c[1]; coords[3 * q + 2] = c[2];
  const int pc[3] = {c[0] / 2, c[1] / 2, c[2] / 2};
  parent[q] = l > 1 ? idx[V.moff[l - 1] + enmorton(V, pc)] : -1;
  const long pq = pos_of(V, l, c[0], c[1], c[2]);
  const int ob = old_at[pq];
  if (ob >= 0) {
    src[q] = ob;
    how[q] = (!old_leaf[ob] && T[pq] == 1) ? 2 : 0;
  } else {
    const int pb = l > 1 ? old_at[pos_of(V, l - 1, pc[0], pc[1], pc[2])] : -1;
    if (pb < 0 || !old_leaf[pb]) *bad = 1;
    src[q] = pb;
    how[q] = 1;
  }
}

}  // namespace

int tree_update_dev(const TreeArgs &a) {
  cudaStream_t st = a.stream;
  Lv V;
  memset(&V, 0, sizeof V);
  V.L = a.L;
  V.ndim = a.ndim;
  for (int l = 0; l <= a.L + 1 && l < 18; ++l) {
    V.off[l] = a.at_off[l];
    for (int d = 0; d < 3; ++d) V.ext[l][d] = l <= 16 ? a.at_ext[l][d] : 1;
  }
  for (int d = 0; d < 3; ++d) V.per[d] = a.periodic[d];
  long nslots = 0;
  for (int l = 1; l <= a.L; ++l) {
    int m = 0;
    for (int d = 0; d < a.ndim; ++d)
      while ((1 << m) < V.ext[l][d]) ++m;
    V.mbits[l] = m;
    V.moff[l] = nslots;
    nslots += 1L << (m * a.ndim);
  }
  V.moff[a.L + 1] = nslots;
  const long npos = (long)a.at_off[a.L + 1] - a.at_off[1];
  const long ntab = a.at_off[a.L + 1];
  unsigned char *T = nullptr, *flag = nullptr, *cand = nullptr, *refine = nullptr, *deref = nullptr;
  int *d_changed = nullptr, *sflag = nullptr, *sidx = nullptr, *d_bad = nullptr;
  int *o_lev = nullptr, *o_coord = nullptr, *o_par = nullptr, *o_src = nullptr, *o_how = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0;
  int rc = 0, n = 0, h_changed = 0, h_bad = 0;
  const int B = 256;
  auto grid = [&](long m) { return (unsigned)((m + B - 1) / B); };
#define TCHK(x)                                   \
  do {                                            \
    if ((x) != cudaSuccess) { rc = -2; goto out; } \
  } while (0)
  TCHK(cudaMalloc((void **)&T, ntab));
  TCHK(cudaMalloc((void **)&flag, ntab));
  TCHK(cudaMalloc((void **)&cand, ntab));
  TCHK(cudaMalloc((void **)&refine, a.nblocks));
  TCHK(cudaMalloc((void **)&deref, a.nblocks));
  TCHK(cudaMalloc((void **)&d_changed, 2 * sizeof(int)));
  d_bad = d_changed + 1;
  TCHK(cudaMalloc((void **)&sflag, (nslots + 1) * sizeof(int)));
  TCHK(cudaMalloc((void **)&sidx, (nslots + 1) * sizeof(int)));
  TCHK(cudaMemsetAsync(T, 0, ntab, st));
  TCHK(cudaMemsetAsync(flag, 0, ntab, st));
  TCHK(cudaMemsetAsync(cand, 0, ntab, st));
  TCHK(cudaMemsetAsync(d_changed, 0, 2 * sizeof(int), st));
  k_mark<<<grid(a.nblocks), B, 0, st>>>(a.err, a.nvar, a.nblocks, a.rc, a.dc, a.level, a.leaf, a.parent,
                                        a.max_refine, refine, deref);
  k_tree_init<<<grid(a.nblocks), B, 0, st>>>(V, a.nblocks, a.level, a.coord, a.leaf, T);
  k_tree_split_marked<<<grid(a.nblocks), B, 0, st>>>(V, a.nblocks, a.level, a.coord, a.leaf, refine, T);
  TCHK(cudaGetLastError());
  // balance: each pass splits, from the tree at its start, every leaf next to
  // an inner neighbour with an inner child touching it (at most one pass per
  // level of spreading plus one)
  for (int it = 0; it < 64; ++it) {
    TCHK(cudaMemsetAsync(d_changed, 0, sizeof(int), st));
    k_balance_mark<<<grid(npos), B, 0, st>>>(V, npos, T, flag, d_changed);
    k_balance_apply<<<grid(npos), B, 0, st>>>(V, npos, T, flag);
    TCHK(cudaMemcpyAsync(&h_changed, d_changed, sizeof(int), cudaMemcpyDeviceToHost, st));
    TCHK(cudaStreamSynchronize(st));
    if (!h_changed) break;
    if (it == 63) { rc = -3; goto out; }
  }
  k_deref_cand<<<grid(npos), B, 0, st>>>(V, npos, a.min_level, T, a.old_at, a.leaf, deref, cand);
  for (int it = 0; it < 1024; ++it) {
    TCHK(cudaMemsetAsync(d_changed, 0, sizeof(int), st));
    k_deref_block<<<grid(npos), B, 0, st>>>(V, npos, T, cand, flag, d_changed);
    k_deref_drop<<<grid(npos), B, 0, st>>>(V.off[1], npos, cand, flag);
    TCHK(cudaMemcpyAsync(&h_changed, d_changed, sizeof(int), cudaMemcpyDeviceToHost, st));
    TCHK(cudaStreamSynchronize(st));
    if (!h_changed) break;
    if (it == 1023) { rc = -3; goto out; }
  }
  k_deref_merge<<<grid(npos), B, 0, st>>>(V, npos, cand, T);
  // number the nodes by level and Morton index
  k_slot_flags<<<grid(nslots), B, 0, st>>>(V, nslots, T, sflag);
  TCHK(cudaGetLastError());
  TCHK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, sflag, sidx, (int)(nslots + 1), st));
  TCHK(cudaMalloc(&tmp, tmp_bytes));
  TCHK(cudaMemsetAsync(sflag + nslots, 0, sizeof(int), st));
  TCHK(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, sflag, sidx, (int)(nslots + 1), st));
  TCHK(cudaMemcpyAsync(&n, sidx + nslots, sizeof(int), cudaMemcpyDeviceToHost, st));
  TCHK(cudaStreamSynchronize(st));
  *a.new_n = n;
  if (n > a.cap) { rc = -4; goto out; }
  TCHK(cudaMalloc((void **)&o_lev, (size_t)n * 7 * sizeof(int)));
  o_coord = o_lev + n; o_par = o_coord + 3 * (size_t)n; o_src = o_par + n; o_how = o_src + n;
  k_emit<<<grid(nslots), B, 0, st>>>(V, nslots, sflag, sidx, T, a.old_at, a.leaf, o_lev, o_coord, o_par, o_src,
                                     o_how, d_bad);
  TCHK(cudaGetLastError());
  TCHK(cudaMemcpyAsync(a.new_levels, o_lev, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st));
  TCHK(cudaMemcpyAsync(a.new_coords, o_coord, (size_t)n * 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
  TCHK(cudaMemcpyAsync(a.new_parent, o_par, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st));
  TCHK(cudaMemcpyAsync(a.src, o_src, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st));
  TCHK(cudaMemcpyAsync(a.how, o_how, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st));
  TCHK(cudaMemcpyAsync(&h_bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
  TCHK(cudaStreamSynchronize(st));
  if (h_bad) rc = -5;
out:
#undef TCHK
  cudaFree(T); cudaFree(flag); cudaFree(cand); cudaFree(refine); cudaFree(deref); cudaFree(d_changed);
  cudaFree(sflag); cudaFree(sidx); cudaFree(o_lev); cudaFree(tmp);
  return rc;
}

}  // namespace fhy
