// nb_list.cu -- link-cell binning and Verlet-list build on the GPU.
//
// Replaces get_ngbr (energy/control/ngbr_list.c:297-581), ngbr_list
// (ngbr_list.c:35-101), get_ngbr_e (energy/control/elec_ngbr.c:220-358),
// ngbr_liste (ngbr_list.c:103-143) and the link-cell helpers get_lnklist /
// get_lnklist_e (energy/control/set_link.c:203-300).
//
// Pair membership is decided exactly as CM3D decides it: the displacement is
// taken in FP64, folded with CM3D's period() arithmetic (md_period.new.c:39-52,
// CM3D's anint and operation order, no FMA contraction -- this file is
// compiled with -fmad=false as well) and compared with the per-interaction
// radius rmaxl_skin2[map[ti][tj]] / rmaxs_skin2 (LJ, after the map == -1 and
// exclusion tests) or rmaxl_skin2_e / rmaxs_skin2_e (charged atoms, after the
// charge-exclusion test).  The resulting pair sets are bit-identical to
// CM3D's.  The cell grid itself is our own: cells at least one list radius
// wide, atoms counting-sorted by cell (inside a cell by atom type, then atom
// index), and a stencil of unique neighbour cells, so every pair within range
// is seen exactly once per direction whatever CM3D's ncell_div is.
//
// A context may hold several independent systems (SysP, nb_common.cuh): each
// has its own box, cell grid and parameters, its cells and atoms occupy
// contiguous ranges, and a system is rebuilt only when its own displacement
// test asked for it (sreb[s]) unless the build covers every system (`all`).
//
// Outputs
//   lst[0..3]  CM3D's four half lists t, s, te, se as (i, j) with i < j
//   nbr        (mixed mode) a full list per atom in cell-sorted order; each
//              32-bit entry holds j's sorted index, the code of the cell shift
//              that turns cell-relative coordinates into the minimum-image
//              displacement, and whether the pair is in the t/s/te/se lists
//   xq, styp   cell-relative FP32 coordinates + charge and type, sorted order
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "nb_common.cuh"

namespace cm3d {

__device__ __forceinline__ bool sys_skip(int s, const int *__restrict__ sreb, int all) {
  return !all && sreb[s] == 0;
}

// ----------------------------------------------------------------- binning
// zero the cell counters of the systems being rebuilt
__global__ void k_cell_zero(int ncells, const int *__restrict__ cell_sys, const int *__restrict__ sreb, int all,
                            int *__restrict__ cell_count, const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells || sys_skip(cell_sys[c], sreb, all)) return;
  cell_count[c] = 0;
}

__global__ void k_cell_assign(int n, const double *__restrict__ pos, const SysP *__restrict__ sp,
                              const int *__restrict__ sys_of, const int *__restrict__ sreb, int all,
                              int *__restrict__ cell_of, int *__restrict__ cell_count, int4 *__restrict__ cimg,
                              const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = sys_of[i];
  if (sys_skip(s, sreb, all)) return;
  const SysP &P = sp[s];
  double x = pos[i], y = pos[n + i], z = pos[2 * n + i];
  double sv[3];
  for (int d = 0; d < 3; d++)
    sv[d] = __dadd_rn(__dadd_rn(__dmul_rn(x, P.hi[3 * d]), __dmul_rn(y, P.hi[3 * d + 1])),
                      __dmul_rn(z, P.hi[3 * d + 2]));
  int img[3], cc[3];
  for (int d = 0; d < 3; d++) {
    const int ncd = P.nc[d];
    double fl = floor(sv[d]);
    double fr = sv[d] - fl;                      // [0, 1]
    int c = (int)(fr * ncd);
    c = c < 0 ? 0 : (c >= ncd ? ncd - 1 : c);
    img[d] = (int)fl;
    cc[d] = c;
  }
  int cell = P.c0 + (cc[0] * P.nc[1] + cc[1]) * P.nc[2] + cc[2];
  cell_of[i] = cell;
  cimg[i] = make_int4(cc[0] | (cc[1] << 10) | (cc[2] << 20), img[0], img[1], img[2]);
  atomicAdd(cell_count + cell, 1);
}

// one block per system: cell_start[c0 ..] = a0 + exclusive scan of the
// system's cell counts; the counters are then reset for the fill
__global__ void __launch_bounds__(256) k_cell_scan(const SysP *__restrict__ sp, const int *__restrict__ sreb,
                                                   int all, int *__restrict__ cell_count,
                                                   int *__restrict__ cell_start, const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  const int s = blockIdx.x;
  if (sys_skip(s, sreb, all)) return;
  const int c0 = sp[s].c0, m = sp[s].ncells, a0 = sp[s].a0;
  __shared__ int part[256];
  const int t = threadIdx.x, nt = blockDim.x;
  const int chunk = (m + nt - 1) / nt;
  const int lo = t * chunk, hi = min(m, lo + chunk);
  int sum = 0;
  for (int k = lo; k < hi; k++) sum += cell_count[c0 + k];
  part[t] = sum;
  __syncthreads();
  for (int d = 1; d < nt; d <<= 1) {
    int v = t >= d ? part[t - d] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = a0 + (t > 0 ? part[t - 1] : 0);
  for (int k = lo; k < hi; k++) {
    const int cnt = cell_count[c0 + k];
    cell_start[c0 + k] = run;
    cell_count[c0 + k] = 0;
    run += cnt;
  }
  if (t == nt - 1) cell_start[c0 + m] = a0 + part[nt - 1];
}

// exclusive scan of `m` ints in one block; `nseg` independent segments laid
// out back to back, one per blockIdx.y; segment totals go to tot[blockIdx.y]
template <typename TI, typename TO>
__global__ void k_scan(const TI *__restrict__ in, TO *__restrict__ out, long long *__restrict__ tot,
                       int m, const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  const TI *a = in + (size_t)blockIdx.y * m;
  TO *o = out + (size_t)blockIdx.y * (m + 1);
  __shared__ TO part[1024];
  int t = threadIdx.x, nt = blockDim.x;
  int chunk = (m + nt - 1) / nt;
  int lo = t * chunk, hi = min(m, lo + chunk);
  TO s = 0;
  for (int k = lo; k < hi; k++) s += (TO)a[k];
  part[t] = s;
  __syncthreads();
  for (int d = 1; d < nt; d <<= 1) {
    TO v = t >= d ? part[t - d] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  TO run = t > 0 ? part[t - 1] : 0;
  for (int k = lo; k < hi; k++) {
    o[k] = run;
    run += (TO)a[k];
  }
  if (t == nt - 1) {
    o[m] = part[nt - 1];
    if (tot) tot[blockIdx.y] = (long long)part[nt - 1];
  }
}

__global__ void k_cell_fill(int n, const int *__restrict__ sys_of, const int *__restrict__ sreb, int all,
                            const int *__restrict__ cell_of, const int *__restrict__ cell_start,
                            int *__restrict__ cursor, int *__restrict__ cell_atoms, const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || sys_skip(sys_of[i], sreb, all)) return;
  int c = cell_of[i];
  int slot = atomicAdd(cursor + c, 1);
  cell_atoms[cell_start[c] + slot] = i;
}

// order every cell's atoms by (atom type, atom index): deterministic lists,
// and the atoms of one type are neighbours in sorted order, so the lane
// groups of a warp in the pair kernels mostly hold atoms of one type and
// walk lists of the same make-up.  One block per cell ranks each atom among
// its cell's atoms (keys are distinct).
__device__ __forceinline__ long long sort_key(const int *__restrict__ itype, int i) {
  return ((long long)itype[i] << 32) | (unsigned)i;
}

constexpr int SORT_CELLS = 8;      // most cells per block of k_cell_sort
constexpr int SORT_THREADS = 128;

__global__ void __launch_bounds__(SORT_THREADS) k_cell_sort(int ncells, int per_block, const int *__restrict__ cell_sys,
                                                             const int *__restrict__ sreb, int all,
                                                             const int *__restrict__ cell_start,
                                                             const int *__restrict__ itype,
                                                             int *__restrict__ cell_atoms,
                                                             const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  __shared__ long long s[1024];
  // per_block consecutive cells per block: up to SORT_CELLS where a batch has
  // tens of thousands of cells of a few atoms each, one where a grid of few,
  // crowded cells would otherwise leave most SMs idle
  const int c_end = min(ncells, (blockIdx.x + 1) * per_block);
  for (int c = blockIdx.x * per_block; c < c_end; c++) {
    if (sys_skip(cell_sys[c], sreb, all)) continue;     // whole blocks
    const int lo = cell_start[c], hi = cell_start[c + 1], m = hi - lo;
    if (m <= 1) continue;
    __syncthreads();                                     // the previous cell's keys are no longer read
    if (m <= 1024) {
      for (int k = threadIdx.x; k < m; k += blockDim.x) s[k] = sort_key(itype, cell_atoms[lo + k]);
      __syncthreads();
      for (int k = threadIdx.x; k < m; k += blockDim.x) {
        const long long v = s[k];
        int r = 0;
        for (int u = 0; u < m; u++) r += s[u] < v;
        cell_atoms[lo + r] = (int)(v & 0xffffffffLL);
      }
      continue;
    }
    // a cell with more than 1024 atoms: odd-even transposition sort in place
    for (int pass = 0; pass < m; pass++) {
      for (int k = lo + (pass & 1) + 2 * threadIdx.x; k + 1 < hi; k += 2 * blockDim.x) {
        int a0 = cell_atoms[k], a1 = cell_atoms[k + 1];
        if (sort_key(itype, a0) > sort_key(itype, a1)) {
          cell_atoms[k] = a1;
          cell_atoms[k + 1] = a0;
        }
      }
      __syncthreads();
    }
  }
}

// Exact membership test of one candidate pair, in CM3D's FP64 operation
// order.  Returns flags (bit0 t, bit1 s, bit2 te, bit3 se, bit4 bad shift)
// and the cell-shift code of the pair for the full list.
__device__ __forceinline__ int exact_flags(const SysP &P, int n, int i, int j, int4 ci,
                                           const double *__restrict__ pos, double xi, double yi, double zi, int ti,
                                           bool qi, const int *__restrict__ itype, const int *__restrict__ map,
                                           const double *__restrict__ icut, const double *__restrict__ q,
                                           const int *__restrict__ excl_off, const int *__restrict__ excl_idx,
                                           const int *__restrict__ cexcl_off, const int *__restrict__ cexcl_idx,
                                           const int4 *__restrict__ cimg, int &code) {
  const int intr = map[P.map0 + ti * P.ntypes + itype[j]];
  const bool lj_ok = intr >= 0;
  const bool el_ok = qi && q[j] != 0.0;
  if (!lj_ok && !el_ok) return 0;
  double dx = xi - pos[j], dy = yi - pos[n + j], dz = zi - pos[2 * n + j];
  double sx = __dadd_rn(__dadd_rn(__dmul_rn(dx, P.hi[0]), __dmul_rn(dy, P.hi[1])), __dmul_rn(dz, P.hi[2]));
  double sy = __dadd_rn(__dadd_rn(__dmul_rn(dx, P.hi[3]), __dmul_rn(dy, P.hi[4])), __dmul_rn(dz, P.hi[5]));
  double sz = __dadd_rn(__dadd_rn(__dmul_rn(dx, P.hi[6]), __dmul_rn(dy, P.hi[7])), __dmul_rn(dz, P.hi[8]));
  const double mx = anint_ref(sx), my = anint_ref(sy), mz = anint_ref(sz);
  sx = __dsub_rn(sx, mx);
  sy = __dsub_rn(sy, my);
  sz = __dsub_rn(sz, mz);
  const double ex = __dadd_rn(__dadd_rn(__dmul_rn(sx, P.h[0]), __dmul_rn(sy, P.h[1])), __dmul_rn(sz, P.h[2]));
  const double ey = __dadd_rn(__dadd_rn(__dmul_rn(sx, P.h[3]), __dmul_rn(sy, P.h[4])), __dmul_rn(sz, P.h[5]));
  const double ez = __dadd_rn(__dadd_rn(__dmul_rn(sx, P.h[6]), __dmul_rn(sy, P.h[7])), __dmul_rn(sz, P.h[8]));
  const double r2 = r2_ref(ex, ey, ez);
  int flags = 0;
  if (lj_ok && r2 < icut[8 * intr + 5] && !(P.excl && excluded(i, j, excl_off, excl_idx))) {
    flags |= 1;
    if (r2 < icut[8 * intr + 4]) flags |= 2;
  }
  if (el_ok && r2 < P.rmaxl_skin2_e && !(P.cexcl && excluded(i, j, cexcl_off, cexcl_idx))) {
    flags |= 4;
    if (r2 < P.rmaxs_skin2_e) flags |= 8;
  }
  if (!flags) return 0;
  // small boxes: the atoms may move skin/2 each before the next rebuild, so a
  // pair whose fractional displacement is within skin / plane spacing of 1/2
  // may change its nearest image; the pair kernel checks those pairs
  if (P.smallbox && (fabs(sx) > P.near_s[0] || fabs(sy) > P.near_s[1] || fabs(sz) > P.near_s[2])) flags |= 32;
  // shift code: k = (n_i - n_j - m) nc + (c_i - c_j) per dimension; |k| <= 1
  // whenever r < rlist <= cell width.  Anything else means the geometry
  // assumption broke: flag it and use the zero shift rather than index past
  // the shift table.
  const int4 cj = cimg[j];
  const int kx = (ci.y - cj.y - (int)mx) * P.nc[0] + ((ci.x & 1023) - (cj.x & 1023));
  const int ky = (ci.z - cj.z - (int)my) * P.nc[1] + (((ci.x >> 10) & 1023) - ((cj.x >> 10) & 1023));
  const int kz = (ci.w - cj.w - (int)mz) * P.nc[2] + (((ci.x >> 20) & 1023) - ((cj.x >> 20) & 1023));
  code = (kx + 1) * 9 + (ky + 1) * 3 + (kz + 1);
  if (kx < -1 || kx > 1 || ky < -1 || ky > 1 || kz < -1 || kz > 1) {
    code = 13;
    flags |= 16;
  }
  return flags;
}

// The candidate walk shared by both list kernels.  One warp owns the
// cell-sorted atom t; its lanes walk the stencil cells 32 candidates at a
// time (consecutive sorted atoms: coalesced FP32 loads) and drop those
// clearly beyond the largest list radius with an FP32 distance from
// cell-relative coordinates (margin 1e-3 A, far above FP32 rounding).  The
// survivors -- typically a few of every 32 -- are queued in shared memory in
// candidate order, and whenever 32 are waiting the whole warp runs the exact
// FP64 test on them at once (`decide(first, m)`: lane l < m takes queue entry
// first + l), so the expensive test runs on full warps.
//
// With qr (the full lists of a grid of 3 or more cells per axis) the queue
// also keeps each survivor's FP32 squared distance and its stencil cell's
// shift code (bits ENT_CODE_SHIFT and up of the queue entry), for the
// FP32-first flags (fast_flags); with `prune` (an orthorhombic such grid of
// cells cw wide) stencil cells wholly beyond lim2 from the atom, by the gaps
// to their faces less 1e-3 A, are skipped -- none of their atoms would pass
// the prefilter, so the lists are the same.
constexpr int LQ = 64;                     // queue entries per warp (> 2 * 32 - 1)

template <class Decide>
__device__ __forceinline__ void walk_candidates(const SysP &P, int i, int4 ci, float4 xi4, bool half_only,
                                                const int *__restrict__ cell_atoms,
                                                const int *__restrict__ cell_start,
                                                const float4 *__restrict__ xq, int *qbuf, Decide &decide,
                                                float *qr = nullptr, bool prune = false,
                                                float3 cw = make_float3(0.f, 0.f, 0.f), int t = -1) {
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const int cx = ci.x & 1023, cy = (ci.x >> 10) & 1023, cz = (ci.x >> 20) & 1023;
  const float lim2 = P.lim2;
  // the stencil cells in walk order (x offsets outermost), one per lane:
  // their sorted-atom ranges (empty where pruned) and shift codes, loaded
  // together up front
  const int nw = P.nsx * P.nsy * P.nsz;
  int my_lo = 0, my_hi = 0, my_code = 13;
  if (lane < nw) {
    const int ox = P.sx[lane / (P.nsy * P.nsz)], oy = P.sy[(lane / P.nsz) % P.nsy], oz = P.sz[lane % P.nsz];
    bool vis = true;
    if (prune) {
      const float gx = fmaxf((ox > 0 ? cw.x - xi4.x : ox < 0 ? xi4.x : 0.f) - 1e-3f, 0.f);
      const float gy = fmaxf((oy > 0 ? cw.y - xi4.y : oy < 0 ? xi4.y : 0.f) - 1e-3f, 0.f);
      const float gz = fmaxf((oz > 0 ? cw.z - xi4.z : oz < 0 ? xi4.z : 0.f) - 1e-3f, 0.f);
      vis = gx * gx + gy * gy + gz * gz < lim2;
    }
    int jx = cx + ox, jy = cy + oy, jz = cz + oz;
    jx = jx < 0 ? jx + P.nc[0] : (jx >= P.nc[0] ? jx - P.nc[0] : jx);
    jy = jy < 0 ? jy + P.nc[1] : (jy >= P.nc[1] ? jy - P.nc[1] : jy);
    jz = jz < 0 ? jz + P.nc[2] : (jz >= P.nc[2] ? jz - P.nc[2] : jz);
    const int cell = P.c0 + (jx * P.nc[1] + jy) * P.nc[2] + jz;
    // cell-corner shift of this stencil offset (k = -offset)
    my_code = (1 - ox) * 9 + (1 - oy) * 3 + (1 - oz);
    if (vis) {
      my_lo = cell_start[cell];
      my_hi = cell_start[cell + 1];
    }
  }
  unsigned left = __ballot_sync(0xffffffffu, my_hi > my_lo);
  // the chunks of 32 candidates in walk order; the next chunk's positions
  // are loaded while the current one is tested
  int w = left ? __ffs(left) - 1 : -1;
  int u0 = 0, hi = 0, code = 13;
  float4 S = make_float4(0.f, 0.f, 0.f, 0.f), xn = S;
  if (w >= 0) {
    u0 = __shfl_sync(0xffffffffu, my_lo, w);
    hi = __shfl_sync(0xffffffffu, my_hi, w);
    code = __shfl_sync(0xffffffffu, my_code, w);
    S = P.shift[code];
    if (u0 + lane < hi) xn = xq[u0 + lane];
  }
  int head = 0, tail = 0;
  while (w >= 0) {
    const int u = u0 + lane, hcur = hi, ccur = code;
    const float4 Sc = S, xj = xn;
    u0 += 32;
    if (u0 >= hi) {
      left &= ~(1u << w);
      w = left ? __ffs(left) - 1 : -1;
      if (w >= 0) {
        u0 = __shfl_sync(0xffffffffu, my_lo, w);
        hi = __shfl_sync(0xffffffffu, my_hi, w);
        code = __shfl_sync(0xffffffffu, my_code, w);
        S = P.shift[code];
      }
    }
    if (w >= 0 && u0 + lane < hi) xn = xq[u0 + lane];
    bool keep = false;
    float r2f = 0.f;
    if (u < hcur) {
      const float dx = (xi4.x - xj.x) + Sc.x, dy = (xi4.y - xj.y) + Sc.y, dz = (xi4.z - xj.z) + Sc.z;
      r2f = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      keep = r2f < lim2;
      if (keep) {
        // the atom itself (sorted index t when given); half lists: j > i
        if (half_only || t < 0) {
          const int j = cell_atoms[u];
          keep = j != i && (!half_only || j > i);
        } else {
          keep = u != t;
        }
      }
    }
    const unsigned bk = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      const int slot = (tail + __popc(bk & lt_mask)) & (LQ - 1);
      qbuf[slot] = qr ? (u | (ccur << ENT_CODE_SHIFT)) : u;
      if (qr) qr[slot] = r2f;
    }
    tail += __popc(bk);
    __syncwarp();
    if (tail - head >= 32) {
      decide(head, 32);
      head += 32;
      __syncwarp();
    }
  }
  while (tail > head) {
    const int m = tail - head < 32 ? tail - head : 32;
    decide(head, m);
    head += m;
  }
}

struct ListCaps {
  long long cap[4];
};

// CM3D's four half lists (i < j): FILL = false counts the pairs of every
// list per atom, FILL = true writes them at the scanned offsets, compacted
// with warp ballots in candidate order (deterministic).  Always built for
// every system (host-driven builds and the single-system plain engine).
template <bool FILL>
__global__ void __launch_bounds__(256) k_list_half(
    int n, const SysP *__restrict__ sp, const int *__restrict__ sys_of, ListCaps C,
    const int *__restrict__ cell_atoms, const int *__restrict__ cell_start, const float4 *__restrict__ xq,
    const double *__restrict__ pos, const int *__restrict__ itype, const int *__restrict__ map,
    const double *__restrict__ icut, const double *__restrict__ q, const int *__restrict__ excl_off,
    const int *__restrict__ excl_idx, const int *__restrict__ cexcl_off, const int *__restrict__ cexcl_idx,
    const int4 *__restrict__ cimg, int *__restrict__ cnt, const long long *__restrict__ off,
    const long long *__restrict__ tot, int2 *__restrict__ l0, int2 *__restrict__ l1, int2 *__restrict__ l2,
    int2 *__restrict__ l3, long long *__restrict__ stat, int *__restrict__ halt, const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  __shared__ int qs[256 / 32][LQ];
  const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= n) return;                                     // whole warps
  const unsigned lt_mask = (1u << lane) - 1u;
  long long p[4] = {0, 0, 0, 0};
  if (FILL) {
    bool fits = true;
    for (int k = 0; k < 4; k++) {
      fits = fits && tot[k] <= C.cap[k];
      p[k] = off[(size_t)k * (n + 1) + t];
    }
    if (!fits) {
      // a list outgrew its buffer: write nothing, halt the step (the host
      // grows the buffers and finishes it, see run_step)
      if (t == 0 && lane == 0) {
        atomicAdd((unsigned long long *)(stat + ST_OVERFLOW), 1ull);
        if (halt) *halt = 1;
      }
      return;
    }
  }
  int *qbuf = qs[threadIdx.x >> 5];
  const SysP &P = sp[sys_of[t]];
  const int i = cell_atoms[t];
  const int4 ci = cimg[i];
  const double xi = pos[i], yi = pos[n + i], zi = pos[2 * n + i];
  const int ti = itype[i];
  const bool qi = q[i] != 0.0;
  int c[4] = {0, 0, 0, 0};
  unsigned bad = 0;
  auto decide = [&](int first, int m) {
    int fl = 0, code = 13, j = -1;
    if (lane < m) {
      j = cell_atoms[qbuf[(first + lane) & (LQ - 1)]];
      fl = exact_flags(P, n, i, j, ci, pos, xi, yi, zi, ti, qi, itype, map, icut, q, excl_off, excl_idx,
                       cexcl_off, cexcl_idx, cimg, code);
    }
    bad |= (fl >> 4) & 1;
    const unsigned b0 = __ballot_sync(0xffffffffu, fl & 1), b1 = __ballot_sync(0xffffffffu, fl & 2);
    const unsigned b2 = __ballot_sync(0xffffffffu, fl & 4), b3 = __ballot_sync(0xffffffffu, fl & 8);
    if (!FILL) {
      c[0] += __popc(b0); c[1] += __popc(b1); c[2] += __popc(b2); c[3] += __popc(b3);
    } else {
      const int2 pr = make_int2(i, j);
      if (fl & 1) l0[p[0] + __popc(b0 & lt_mask)] = pr;
      if (fl & 2) l1[p[1] + __popc(b1 & lt_mask)] = pr;
      if (fl & 4) l2[p[2] + __popc(b2 & lt_mask)] = pr;
      if (fl & 8) l3[p[3] + __popc(b3 & lt_mask)] = pr;
      p[0] += __popc(b0); p[1] += __popc(b1); p[2] += __popc(b2); p[3] += __popc(b3);
    }
  };
  walk_candidates(P, i, ci, xq[t], true, cell_atoms, cell_start, xq, qbuf, decide);
  if (FILL) {
    if (bad && lane == 0) atomicAdd((unsigned long long *)(stat + ST_BADSHIFT), 1ull);
  } else if (lane == 0) {
    for (int k = 0; k < 4; k++) cnt[(size_t)k * n + t] = c[k];
  }
}

// Candidates from a staged neighbourhood (k_list_win): `cnt` atoms with FP32
// positions moved by their cell's shift into the frame of atom t's cell
// (s_x) and their sorted indices (s_u, low ENT_JBITS bits), walked 32 at a
// time with the same prefilter and in the same order as walk_candidates.  The
// queue holds the staged index, and qr its FP32 squared distance.
//
// With `prune` (an orthorhombic cell grid of three or more cells per axis,
// cells cw wide), the lanes first bound atom t's distance from each stencil
// cell (the gaps to the cell's faces, each shortened by 1e-3 A) and the walk
// skips the cells that lie wholly beyond lim2: none of their atoms would pass
// the prefilter, and the others keep their order, so the lists are the same.
// s_off holds the stencil cells' first staged index, s_code their shift code.
template <class Decide>
__device__ __forceinline__ void walk_staged(int t, float4 xi4, float lim2, const float4 *s_x, const int *s_u,
                                            int cnt, int *qbuf, float *qr, Decide &decide, const int *s_off,
                                            const int *s_code, int nw, bool prune, float3 cw) {
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  unsigned vis = nw >= 32 ? 0xffffffffu : (1u << nw) - 1u;
  if (prune) {
    bool v = false;
    if (lane < nw) {
      const int code = s_code[lane];
      const int ox = 1 - code / 9, oy = 1 - (code / 3) % 3, oz = 1 - code % 3;
      const float gx = fmaxf((ox > 0 ? cw.x - xi4.x : ox < 0 ? xi4.x : 0.f) - 1e-3f, 0.f);
      const float gy = fmaxf((oy > 0 ? cw.y - xi4.y : oy < 0 ? xi4.y : 0.f) - 1e-3f, 0.f);
      const float gz = fmaxf((oz > 0 ? cw.z - xi4.z : oz < 0 ? xi4.z : 0.f) - 1e-3f, 0.f);
      v = gx * gx + gy * gy + gz * gz < lim2;
    }
    vis = __ballot_sync(0xffffffffu, v);
  }
  int head = 0, tail = 0;
  for (int w = 0; w < nw;) {
    if (!((vis >> w) & 1u)) {
      w++;
      continue;
    }
    // a run of visited stencil cells is one contiguous span of staged atoms
    int e = w;
    while (e + 1 < nw && ((vis >> (e + 1)) & 1u)) e++;
    const int a = s_off[w], b = e + 1 < nw ? s_off[e + 1] : cnt;
    w = e + 1;
  for (int k0 = a; k0 < b; k0 += 32) {
    const int k = k0 + lane;
    bool keep = false;
    float r2f = 0.f;
    if (k < b) {
      const float4 xs = s_x[k];
      const int u = s_u[k] & (int)ENT_JMASK;
      const float dx = xi4.x - xs.x, dy = xi4.y - xs.y, dz = xi4.z - xs.z;
      r2f = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      keep = u != t && r2f < lim2;
    }
    const unsigned bk = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      const int slot = (tail + __popc(bk & lt_mask)) & (LQ - 1);
      qbuf[slot] = k;
      qr[slot] = r2f;
    }
    tail += __popc(bk);
    __syncwarp();
    if (tail - head >= 32) {
      decide(head, 32);
      head += 32;
      __syncwarp();
    }
  }
  }
  while (tail > head) {
    const int m = tail - head < 32 ? tail - head : 32;
    decide(head, m);
    head += m;
  }
}

// List flags from the FP32 squared distance of a staged pair (cell grid of 3
// or more cells per axis, where the stencil image is the only image within
// the list radius and its shift code the pair's).  Each comparison with a
// list radius R^2 matches CM3D's FP64 one unless the FP32 value lies within
// 4e-5 R^2 + 2e-3 A^2 of R^2 -- a margin ten times the FP32 error of a
// squared distance formed from cell-relative coordinates (cells are narrower
// than two list radii) -- and then *exact is set and the caller decides in
// FP64 (exact_flags).  Same tests, same order as exact_flags.
__device__ __forceinline__ int fast_flags(const SysP &P, int i, int j, int ti, int tj, bool qi, bool qj,
                                          float r2f, const int *__restrict__ map, const double *__restrict__ icut,
                                          const int *__restrict__ excl_off, const int *__restrict__ excl_idx,
                                          const int *__restrict__ cexcl_off, const int *__restrict__ cexcl_idx,
                                          bool *exact) {
  const int intr = map[P.map0 + ti * P.ntypes + tj];
  const bool lj_ok = intr >= 0;
  const bool el_ok = qi && qj;
  if (!lj_ok && !el_ok) return 0;
  bool near = false;
  auto below = [&](double R2d) {
    const float R2 = (float)R2d;
    near |= fabsf(r2f - R2) < fmaf(4e-5f, R2, 2e-3f);
    return r2f < R2;
  };
  int flags = 0;
  if (lj_ok && below(icut[8 * intr + 5]) && !(P.excl && excluded(i, j, excl_off, excl_idx))) {
    flags |= 1;
    if (below(icut[8 * intr + 4])) flags |= 2;
  }
  if (el_ok && below(P.rmaxl_skin2_e) && !(P.cexcl && excluded(i, j, cexcl_off, cexcl_idx))) {
    flags |= 4;
    if (below(P.rmaxs_skin2_e)) flags |= 8;
  }
  *exact = near;
  return flags;
}

// The full list of sorted atom t (mixed mode; one warp): both directions,
// every pair in CM3D's t or te list, written straight into its fixed slot
// nbr[t * stride ...] in two segments, each in candidate order: the pairs in
// an LJ list (t or s) from the front of the slot, their count in nlen[t], and
// the electrostatics-only pairs from the back (the last one at the slot's
// end), their count in nlen[n + t].  A pair kernel then runs the LJ arithmetic
// only over the front segment.  An atom with more than `stride` pairs writes
// none past its slot, records the length it needed (ST_NEED_STRIDE) and halts
// a captured step; the host then widens the slots and builds again.
// STAGED: candidates from the block's staged neighbourhood (s_x, s_u, scnt),
// otherwise from global memory through the stencil walk.
template <bool STAGED>
__device__ __forceinline__ void full_list_atom(
    const SysP &P, int n, int t, int stride, const int *__restrict__ cell_atoms,
    const int *__restrict__ cell_start, const float4 *__restrict__ xq, const double *__restrict__ pos,
    const int *__restrict__ itype, const int *__restrict__ map, const double *__restrict__ icut,
    const double *__restrict__ q, const int *__restrict__ excl_off, const int *__restrict__ excl_idx,
    const int *__restrict__ cexcl_off, const int *__restrict__ cexcl_idx, const int4 *__restrict__ cimg,
    uint32_t *__restrict__ nbr, int *__restrict__ nlen, long long *__restrict__ stat, int *__restrict__ halt,
    int *qbuf, float *qr, const float4 *s_x, const int *s_u, const int *s_j, int scnt,
    bool fast, const int *s_off = nullptr, const int *s_code = nullptr, int nw = 0, bool prune = false,
    float3 cw = make_float3(0.f, 0.f, 0.f)) {
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const int i = cell_atoms[t];
  const int4 ci = cimg[i];
  const double xi = pos[i], yi = pos[n + i], zi = pos[2 * n + i];
  const int ti = itype[i];
  const bool qi = q[i] != 0.0;
  uint32_t *out = nbr + (size_t)t * stride;
  int na = 0, nb = 0;
  unsigned bad = 0;
  auto decide = [&](int first, int m) {
    int fl = 0, code = 13, u = 0;
    if (lane < m) {
      const int slot = (first + lane) & (LQ - 1);
      if (STAGED) {
        const int k = qbuf[slot];
        const int uc = s_u[k];
        u = uc & (int)ENT_JMASK;
        const int j = s_j[k];
        bool exact = !fast;
        if (fast) {
          const int meta = __float_as_int(s_x[k].w);
          fl = fast_flags(P, i, j, ti, meta >> 1, qi, (meta & 1) != 0, qr[slot], map, icut, excl_off, excl_idx,
                          cexcl_off, cexcl_idx, &exact);
          code = (int)((unsigned)uc >> ENT_CODE_SHIFT);
        }
        if (exact)
          fl = exact_flags(P, n, i, j, ci, pos, xi, yi, zi, ti, qi, itype, map, icut, q, excl_off, excl_idx,
                           cexcl_off, cexcl_idx, cimg, code);
      } else {
        const int uc = qbuf[slot];
        u = fast ? (uc & (int)ENT_JMASK) : uc;
        const int j = cell_atoms[u];
        bool exact = !fast;
        if (fast) {
          fl = fast_flags(P, i, j, ti, itype[j], qi, q[j] != 0.0, qr[slot], map, icut, excl_off, excl_idx,
                          cexcl_off, cexcl_idx, &exact);
          code = (int)((unsigned)uc >> ENT_CODE_SHIFT);
        }
        if (exact)
          fl = exact_flags(P, n, i, j, ci, pos, xi, yi, zi, ti, qi, itype, map, icut, q, excl_off, excl_idx,
                           cexcl_off, cexcl_idx, cimg, code);
      }
    }
    bad |= (fl >> 4) & 1;
    const bool fa = (fl & 3) != 0;                   // in an LJ list: front segment
    const bool fb = !fa && (fl & 12) != 0;           // electrostatics only: back segment
    const unsigned ba = __ballot_sync(0xffffffffu, fa), bb = __ballot_sync(0xffffffffu, fb);
    if (fa || fb) {
      uint32_t e = (uint32_t)u | ((uint32_t)code << ENT_CODE_SHIFT);
      if (fl & 1) e |= ENT_LJ;
      if (fl & 2) e |= ENT_LJS;
      if (fl & 4) e |= ENT_EL;
      if (fl & 8) e |= ENT_ELS;
      if (fl & 32) e |= ENT_NEAR;
      // every write lands inside the slot; once the two segments meet (an
      // overflow) the slot's contents no longer matter: the lengths are set
      // to zero below and the list is built again with wider slots
      if (fa) {
        const int slot = na + __popc(ba & lt_mask);
        if (slot < stride - nb) out[slot] = e;
      } else {
        const int slot = nb + __popc(bb & lt_mask);
        if (slot < stride - na) out[stride - 1 - slot] = e;
      }
    }
    na += __popc(ba);
    nb += __popc(bb);
  };
  if (STAGED) walk_staged(t, xq[t], P.lim2, s_x, s_u, scnt, qbuf, qr, decide, s_off, s_code, nw, prune, cw);
  else walk_candidates(P, i, ci, xq[t], false, cell_atoms, cell_start, xq, qbuf, decide, fast ? qr : nullptr,
                       prune, cw, t);
  const int count = na + nb;
  if (lane == 0) {
    if (count <= stride) {
      nlen[t] = na;
      nlen[n + t] = nb;
    } else {
      nlen[t] = 0;
      nlen[n + t] = 0;
    }
    if (count > stride) {
      atomicMax((unsigned long long *)(stat + ST_NEED_STRIDE), (unsigned long long)count);
      if (halt) {
        atomicAdd((unsigned long long *)(stat + ST_OVERFLOW), 1ull);
        *halt = 1;
      }
    }
    if (bad) atomicAdd((unsigned long long *)(stat + ST_BADSHIFT), 1ull);
  }
}

// Mixed mode, warp per atom over every atom (the candidates walked in global
// memory): the fallback of k_list_win.
__global__ void __launch_bounds__(256, 3) k_list_full(
    int n, const SysP *__restrict__ sp, const int *__restrict__ sys_of, const int *__restrict__ sreb, int all,
    int stride, const int *__restrict__ cell_atoms, const int *__restrict__ cell_start,
    const float4 *__restrict__ xq, const double *__restrict__ pos, const int *__restrict__ itype,
    const int *__restrict__ map, const double *__restrict__ icut, const double *__restrict__ q,
    const int *__restrict__ excl_off, const int *__restrict__ excl_idx, const int *__restrict__ cexcl_off,
    const int *__restrict__ cexcl_idx, const int4 *__restrict__ cimg, uint32_t *__restrict__ nbr,
    int *__restrict__ nlen, long long *__restrict__ stat, int *__restrict__ halt, const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  __shared__ int qs[256 / 32][LQ];
  __shared__ float qrs[256 / 32][LQ];
  const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (t >= n) return;                                     // whole warps
  const int s = sys_of[t];
  if (sys_skip(s, sreb, all)) return;                     // whole warps
  // FP32-first flags and stencil pruning where the grid allows them (as in
  // k_list_win: 3 or more cells per axis, no near-image pairs)
  const SysP &P = sp[s];
  const bool fast = P.nc[0] >= 3 && P.nc[1] >= 3 && P.nc[2] >= 3 && !P.smallbox;
  const bool ortho = P.h[1] == 0. && P.h[2] == 0. && P.h[3] == 0. && P.h[5] == 0. && P.h[6] == 0. && P.h[7] == 0.;
  const float3 cw = make_float3(P.hF[0] / (float)P.nc[0], P.hF[4] / (float)P.nc[1], P.hF[8] / (float)P.nc[2]);
  full_list_atom<false>(P, n, t, stride, cell_atoms, cell_start, xq, pos, itype, map, icut, q, excl_off,
                        excl_idx, cexcl_off, cexcl_idx, cimg, nbr, nlen, stat, halt, qs[threadIdx.x >> 5],
                        qrs[threadIdx.x >> 5], nullptr, nullptr, nullptr, 0, fast, nullptr, nullptr, 0,
                        fast && ortho, cw);
}

// The cells of the systems being rebuilt, as one index range: rb_scan[s] is
// the number of such cells in systems before s, rb_scan[nsys] their total.
// A batch rebuilds a few of its systems on most steps; the list kernel then
// walks those cells only instead of skipping every other system's.
__global__ void k_rebuild_cells(int nsys, const SysP *__restrict__ sp, const int *__restrict__ sreb, int all,
                                int *__restrict__ rb_scan, const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  __shared__ int warp_tot[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < nsys; base += blockDim.x) {
    const int sy = base + threadIdx.x;
    const int v = sy < nsys && (all || sreb[sy] != 0) ? sp[sy].ncells : 0;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
      int t = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += u;
      }
      warp_tot[lane] = t;                              // inclusive over warps
    }
    __syncthreads();
    const int before = carry + (w > 0 ? warp_tot[w - 1] : 0);
    if (sy < nsys) rb_scan[sy] = before + incl - v;
    __syncthreads();
    if (threadIdx.x == 0) carry += warp_tot[(blockDim.x >> 5) - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) rb_scan[nsys] = carry;
}

// Mixed mode, block per cell: the block stages the cell's stencil
// neighbourhood (every candidate of every atom of the cell: FP32 positions
// moved by their cell's shift, sorted index + the cell's shift code, atom
// index, type and charge flag) in shared memory once, then its warps build
// the cell's atoms' lists from it: the prefilter reads shared memory, and in
// a grid of 3 or more cells per axis the list flags come from the FP32
// distance (fast_flags) except within a margin of a list radius, where the
// FP64 test decides -- the same lists as the FP64 test of every candidate.
// Blocks walk the cells of the systems being rebuilt; a cell whose
// neighbourhood holds more than `cap` atoms is walked in global memory
// instead (same decisions).
constexpr int LW_THREADS = 256;
constexpr size_t LW_BYTES_PER_ATOM = sizeof(float4) + 2 * sizeof(int);   // s_x (w: type, charge), s_u, s_j
constexpr long long LW_MAX_CAP = 2048;     // largest staged neighbourhood (48 KB)

__global__ void __launch_bounds__(LW_THREADS) k_list_win(
    int nsys, const int *__restrict__ rb_scan, const SysP *__restrict__ sp, int n, int stride, int cap,
    const int *__restrict__ cell_atoms, const int *__restrict__ cell_start,
    const float4 *__restrict__ xq, const double *__restrict__ pos, const int *__restrict__ itype,
    const int *__restrict__ map, const double *__restrict__ icut, const double *__restrict__ q,
    const int *__restrict__ excl_off, const int *__restrict__ excl_idx, const int *__restrict__ cexcl_off,
    const int *__restrict__ cexcl_idx, const int4 *__restrict__ cimg, uint32_t *__restrict__ nbr,
    int *__restrict__ nlen, long long *__restrict__ stat, int *__restrict__ halt, const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  extern __shared__ float4 s_x[];                        // cap
  int *s_u = reinterpret_cast<int *>(s_x + cap);         // cap: sorted index | shift code << ENT_CODE_SHIFT
  int *s_j = s_u + cap;                                  // cap: atom index
  __shared__ int qs[LW_THREADS / 32][LQ];
  __shared__ float qrs[LW_THREADS / 32][LQ];
  __shared__ int s_cs[27], s_off[27], s_code[27], s_tot, s_nw;
  __shared__ float4 s_sh[27];
  const int warp = threadIdx.x >> 5;
  const int total = rb_scan[nsys];
  for (int v = blockIdx.x; v < total; v += gridDim.x) {
    // the system of rebuilt cell v: the last s with rb_scan[s] <= v (systems
    // without rebuilt cells share their successor's value and are passed)
    int sa = 0, sb = nsys;
    while (sb - sa > 1) {
      const int mid = (sa + sb) >> 1;
      if (rb_scan[mid] <= v) sa = mid;
      else sb = mid;
    }
    const int s = sa;
    const SysP &P = sp[s];
    const int c = P.c0 + (v - rb_scan[s]);
    __syncthreads();                                     // the previous neighbourhood is no longer read
    if (threadIdx.x < 32) {
      // the system's stencil around cell c, one stencil cell per lane, in
      // walk_candidates' order (x offsets outermost), and the prefix of
      // their atom counts
      const int w = threadIdx.x;
      const int nw = P.nsx * P.nsy * P.nsz;
      int cn = 0;
      if (w < nw) {
        const int lc = c - P.c0;
        const int cz = lc % P.nc[2], cy = (lc / P.nc[2]) % P.nc[1], cx = lc / (P.nc[2] * P.nc[1]);
        const int ox = P.sx[w / (P.nsy * P.nsz)], oy = P.sy[(w / P.nsz) % P.nsy], oz = P.sz[w % P.nsz];
        int jx = cx + ox, jy = cy + oy, jz = cz + oz;
        jx = jx < 0 ? jx + P.nc[0] : (jx >= P.nc[0] ? jx - P.nc[0] : jx);
        jy = jy < 0 ? jy + P.nc[1] : (jy >= P.nc[1] ? jy - P.nc[1] : jy);
        jz = jz < 0 ? jz + P.nc[2] : (jz >= P.nc[2] ? jz - P.nc[2] : jz);
        const int cell = P.c0 + (jx * P.nc[1] + jy) * P.nc[2] + jz;
        const int cs = cell_start[cell];
        cn = cell_start[cell + 1] - cs;
        s_cs[w] = cs;
        s_code[w] = (1 - ox) * 9 + (1 - oy) * 3 + (1 - oz);
        s_sh[w] = P.shift[s_code[w]];
      }
      int incl = cn;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (w >= o) incl += v;
      }
      if (w < nw) s_off[w] = incl - cn;
      if (w == 31) {
        s_nw = nw;
        s_tot = incl;
      }
    }
    __syncthreads();
    const int tot = s_tot, nw = s_nw;
    const bool staged = tot <= cap;
    if (staged) {
      // one pass over the whole neighbourhood, so that every thread's loads
      // are in flight at once: staged atom g lies in the last stencil cell w
      // with s_off[w] <= g (empty cells share their successor's offset)
      for (int g = threadIdx.x; g < tot; g += blockDim.x) {
        int wa = 0, wb = nw;
        while (wb - wa > 1) {
          const int mid = (wa + wb) >> 1;
          if (s_off[mid] <= g) wa = mid;
          else wb = mid;
        }
        const int u = s_cs[wa] + (g - s_off[wa]);
        const float4 x = xq[u];
        const int j = cell_atoms[u];
        const float4 sh = s_sh[wa];
        s_x[g] = make_float4(x.x - sh.x, x.y - sh.y, x.z - sh.z, __int_as_float(itype[j] * 2 + (q[j] != 0.0 ? 1 : 0)));
        s_u[g] = u | (s_code[wa] << ENT_CODE_SHIFT);
        s_j[g] = j;
      }
    }
    __syncthreads();
    const int lo = cell_start[c], hi = cell_start[c + 1];
    const bool fast = P.nc[0] >= 3 && P.nc[1] >= 3 && P.nc[2] >= 3 && !P.smallbox;
    const bool ortho = P.h[1] == 0. && P.h[2] == 0. && P.h[3] == 0. && P.h[5] == 0. && P.h[6] == 0. && P.h[7] == 0.;
    const float3 cw = make_float3(P.hF[0] / (float)P.nc[0], P.hF[4] / (float)P.nc[1], P.hF[8] / (float)P.nc[2]);
    for (int t = lo + warp; t < hi; t += LW_THREADS / 32) {
      if (staged)
        full_list_atom<true>(P, n, t, stride, cell_atoms, cell_start, xq, pos, itype, map, icut, q, excl_off,
                             excl_idx, cexcl_off, cexcl_idx, cimg, nbr, nlen, stat, halt, qs[warp], qrs[warp], s_x,
                             s_u, s_j, tot, fast, s_off, s_code, nw, fast && ortho && nw == 27, cw);
      else
        full_list_atom<false>(P, n, t, stride, cell_atoms, cell_start, xq, pos, itype, map, icut, q, excl_off,
                              excl_idx, cexcl_off, cexcl_idx, cimg, nbr, nlen, stat, halt, qs[warp], nullptr,
                              nullptr, nullptr, nullptr, 0, false);
    }
  }
}

// sorted-order arrays: rank, type, the FP64 corner of the atom's cell (held
// fixed until the next rebuild) and FP32 cell-relative coordinates + charge
__global__ void k_sorted_init(int n, const SysP *__restrict__ sp, const int *__restrict__ sys_of,
                              const int *__restrict__ sreb, int all, const int *__restrict__ cell_atoms,
                              const int4 *__restrict__ cimg, const int *__restrict__ itype,
                              const double *__restrict__ pos, const double *__restrict__ q, int *__restrict__ rank,
                              int *__restrict__ styp, double *__restrict__ corner, float4 *__restrict__ xq,
                              const int *__restrict__ gate) {
  if (gated_off(gate, 1)) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int s = sys_of[t];
  if (sys_skip(s, sreb, all)) return;
  const SysP &P = sp[s];
  int i = cell_atoms[t];
  int4 ci = cimg[i];
  const double *h = P.h;
  double o0 = (double)ci.y + (double)(ci.x & 1023) / P.nc[0];
  double o1 = (double)ci.z + (double)((ci.x >> 10) & 1023) / P.nc[1];
  double o2 = (double)ci.w + (double)((ci.x >> 20) & 1023) / P.nc[2];
  double c0 = h[0] * o0 + h[1] * o1 + h[2] * o2;
  double c1 = h[3] * o0 + h[4] * o1 + h[5] * o2;
  double c2 = h[6] * o0 + h[7] * o1 + h[8] * o2;
  corner[t] = c0;
  corner[n + t] = c1;
  corner[2 * n + t] = c2;
  xq[t] = make_float4((float)(pos[i] - c0), (float)(pos[n + i] - c1), (float)(pos[2 * n + i] - c2), (float)q[i]);
  rank[i] = t;
  styp[t] = itype[i];
}

// The cell corners (and FP32 cell-relative positions) under a new box: every
// atom keeps its cell and image, its corner moves with H (mixed mode; the
// pair kernels' shifts, also H-derived, are updated beside this).
int refresh_corners(Ctx *c) {
  if (c->mode != CM3D_NB_MIXED || !c->lists_built) return CM3D_NB_OK;
  k_sorted_init<<<grid_for(c->n, 256), 256, 0, c->st>>>(c->n, c->sp, c->sys_of, c->sreb, 1, c->cell_atoms,
                                                        c->cimg, c->itype, c->pos, c->q, c->rank, c->styp,
                                                        c->corner, c->xq, nullptr);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

// dxn = pos of the rebuilt systems (ngbr_list.c:577-580) and, per rebuilt
// system, isteplast = istep (md_finter.c:98)
__global__ void k_snapshot(int n, const SysP *__restrict__ sp, const int *__restrict__ sys_of,
                           const int *__restrict__ sreb, int all, const double *__restrict__ pos,
                           double *__restrict__ dxn, int *__restrict__ slast, long long *__restrict__ sstat,
                           const int *__restrict__ gate, const int *__restrict__ istate,
                           long long *__restrict__ stat) {
  if (gated_off(gate, 1)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) atomicAdd((unsigned long long *)(stat + ST_REBUILDS), 1ull);
  if (i >= n) return;
  const int s = sys_of[i];
  if (sys_skip(s, sreb, all)) return;
  dxn[i] = pos[i];
  dxn[n + i] = pos[n + i];
  dxn[2 * n + i] = pos[2 * n + i];
  if (i == sp[s].a0) {
    slast[s] = istate[IS_ISTEP];
    sstat[(size_t)s * SS_COUNT + SS_REBUILDS] += 1;
  }
}

// --------------------------------------------------------------- host side
static void stencil(int nc, int *s, int *ns) {
  if (nc >= 3) {
    s[0] = -1; s[1] = 0; s[2] = 1; *ns = 3;
  } else if (nc == 2) {
    s[0] = 0; s[1] = 1; *ns = 2;
  } else {
    s[0] = 0; *ns = 1;
  }
}

// Cell grids of every system (cells at least one list radius wide in every
// fractional direction: plane spacing 1 / |row d of hmati|), their stencils,
// the 27 cell-corner shifts and the FP32 prefilter radius; fills the cell
// fields of c->h_sp and allocates the binning and list arrays.
// the 27 neighbour-cell displacements of a system's grid (one cell step
// along each box vector), as FP32 hi + lo parts
void cell_shifts(SysP &P, const SysH &H) {
  for (int a = -1; a <= 1; a++)
    for (int b = -1; b <= 1; b++)
      for (int d = -1; d <= 1; d++) {
        double f0 = (double)a / P.nc[0], f1 = (double)b / P.nc[1], f2 = (double)d / P.nc[2];
        const double *h = H.hmat;
        const double v0 = h[0] * f0 + h[1] * f1 + h[2] * f2, v1 = h[3] * f0 + h[4] * f1 + h[5] * f2,
                     v2 = h[6] * f0 + h[7] * f1 + h[8] * f2;
        const int k = (a + 1) * 9 + (b + 1) * 3 + (d + 1);
        P.shift[k] = make_float4((float)v0, (float)v1, (float)v2, 0.f);
        P.shift_lo[k] = make_float4((float)(v0 - (double)(float)v0), (float)(v1 - (double)(float)v1),
                                    (float)(v2 - (double)(float)v2), 0.f);
      }
}

int list_setup(Ctx *c) {
  int c0 = 0;
  double est_max = 32.0;
  for (int s = 0; s < c->nsys; s++) {
    SysP &P = c->h_sp[s];
    const SysH &H = c->hs[s];
    int tot = 1;
    for (int d = 0; d < 3; d++) {
      double w = 1.0 / sqrt(H.hmati[3 * d] * H.hmati[3 * d] + H.hmati[3 * d + 1] * H.hmati[3 * d + 1] +
                            H.hmati[3 * d + 2] * H.hmati[3 * d + 2]);
      int m = H.rlist > 0 ? (int)floor(w / (H.rlist * c->cell_scale)) : 1;
      m = m < 1 ? 1 : (m > 1000 ? 1000 : m);
      P.nc[d] = m;
      tot *= m;
    }
    P.c0 = c0;
    P.ncells = tot;
    c0 += tot;
    stencil(P.nc[0], P.sx, &P.nsx);
    stencil(P.nc[1], P.sy, &P.nsy);
    stencil(P.nc[2], P.sz, &P.nsz);
    // with three or more cells per direction the stencil neighbour's image
    // is the minimum image of every pair in range, so the FP32 prefilter is
    // exact up to rounding; with fewer cells every candidate goes to the
    // FP64 test
    const bool pre = P.nc[0] >= 3 && P.nc[1] >= 3 && P.nc[2] >= 3;
    const double rl = H.rlist + 1e-3;
    P.lim2 = pre ? (float)(rl * rl) : INFINITY;
    cell_shifts(P, H);
    // first guess of the full-list slot: 1.3 x the mean number of atoms in
    // a list sphere, plus 64
    double vol = fabs(H.hmat[0] * (H.hmat[4] * H.hmat[8] - H.hmat[5] * H.hmat[7]) +
                      H.hmat[1] * (H.hmat[5] * H.hmat[6] - H.hmat[3] * H.hmat[8]) +
                      H.hmat[2] * (H.hmat[3] * H.hmat[7] - H.hmat[4] * H.hmat[6]));
    double r = H.rlist;
    double est = 1.3 * (double)H.n / vol * (4.0 / 3.0) * M_PI * r * r * r + 64.0;
    if (est > (double)H.n + 31.0) est = (double)H.n + 31.0;
    if (est > est_max) est_max = est;
  }
  c->ncells = c0;
  c->nc[0] = c->h_sp[0].nc[0];
  c->nc[1] = c->h_sp[0].nc[1];
  c->nc[2] = c->h_sp[0].nc[2];
  std::vector<int> cell_sys(c0);
  for (int s = 0; s < c->nsys; s++)
    for (int k = 0; k < c->h_sp[s].ncells; k++) cell_sys[c->h_sp[s].c0 + k] = s;
  CK(cudaMalloc(&c->cell_sys, sizeof(int) * (size_t)c0));
  CK(cudaMemcpy(c->cell_sys, cell_sys.data(), sizeof(int) * (size_t)c0, cudaMemcpyHostToDevice));
  CK(cudaMalloc(&c->cell_of, sizeof(int) * (size_t)c->n));
  CK(cudaMalloc(&c->cell_start, sizeof(int) * ((size_t)c0 + 1)));
  CK(cudaMalloc(&c->cell_cursor, sizeof(int) * ((size_t)c0 + 1)));
  CK(cudaMemset(c->cell_cursor, 0, sizeof(int) * ((size_t)c0 + 1)));
  CK(cudaMalloc(&c->cell_atoms, sizeof(int) * (size_t)c->n));
  CK(cudaMalloc(&c->rank, sizeof(int) * (size_t)c->n));
  CK(cudaMalloc(&c->cnt, sizeof(int) * 4 * (size_t)c->n));
  CK(cudaMalloc(&c->off, sizeof(long long) * 4 * ((size_t)c->n + 1)));
  CK(cudaMalloc(&c->ltot, sizeof(long long) * LT_COUNT));
  CK(cudaMallocHost(&c->h_ltot, sizeof(long long) * LT_COUNT));
  CK(cudaMalloc(&c->styp, sizeof(int) * (size_t)c->n));
  CK(cudaMalloc(&c->corner, sizeof(double) * 3 * (size_t)c->n));
  CK(cudaMalloc(&c->xq, sizeof(float4) * (size_t)c->n));
  CK(cudaMalloc(&c->cimg, sizeof(int4) * (size_t)c->n));
  // system 0's shifts (the single-system pair kernel keeps them in shared memory)
  CK(cudaMalloc(&c->shift, sizeof(float4) * 54));
  CK(cudaMemcpy(c->shift, c->h_sp[0].shift, sizeof(float4) * 27, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->shift + 27, c->h_sp[0].shift_lo, sizeof(float4) * 27, cudaMemcpyHostToDevice));
  if (c->mode == CM3D_NB_MIXED) {
    // staged list build: room for 1.6x the largest mean stencil neighbourhood
    // (+64), within the shared memory a block may opt into
    double nb_max = 0;
    for (int sy = 0; sy < c->nsys; sy++) {
      const SysP &S = c->h_sp[sy];
      const double per_cell = (double)S.n / (double)(S.ncells > 0 ? S.ncells : 1);
      nb_max = std::max(nb_max, per_cell * S.nsx * S.nsy * S.nsz);
    }
    c->lw_smem_max = c->smem_optin > 8192 ? c->smem_optin - 8192 : 0;
    long long cap = (long long)(1.6 * nb_max) + 64;
    const long long cap_max = (long long)(c->lw_smem_max / LW_BYTES_PER_ATOM);
    c->lw_cap = (int)std::min(cap, cap_max);
    // a neighbourhood of thousands of atoms leaves one block per SM: the
    // warp-per-atom walk through global memory keeps more warps in flight
    if (c->lw_cap < 64 || cap > LW_MAX_CAP) c->lw_cap = 0;
    const char *lk = getenv("CM3D_NB_LIST_KERNEL");
    if (lk && strcmp(lk, "walk") == 0) c->lw_cap = 0;
    CK(cudaMalloc(&c->rb_scan, sizeof(int) * ((size_t)c->nsys + 1)));
    CK(cudaMalloc(&c->nlen, sizeof(int) * 2 * (size_t)c->n));
    CK(cudaMemset(c->nlen, 0, sizeof(int) * 2 * (size_t)c->n));
    long long s = ((long long)est_max + 31) / 32 * 32;
    if (s < 32) s = 32;
    c->nbr_stride = (int)s;
    CK(cudaMalloc(&c->nbr, sizeof(uint32_t) * (size_t)c->n * (size_t)s));
    c->lcap[LT_FULL] = (long long)c->n * s;
  }
  return CM3D_NB_OK;
}

// one warp per atom: its front segment (nlen[t] entries) and back segment
// (nlen[n + t]) from a slot of `old_s` entries into one of `new_s`
__global__ void k_regrow_copy(int n, int old_s, int new_s, const int *__restrict__ nlen,
                              const uint32_t *__restrict__ src, uint32_t *__restrict__ dst) {
  const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (t >= n) return;
  const int na = min(nlen[t], old_s), nb = min(nlen[n + t], old_s - na);
  const uint32_t *a = src + (size_t)t * old_s;
  uint32_t *b = dst + (size_t)t * new_s;
  for (int k = lane; k < na; k += 32) b[k] = a[k];
  for (int k = lane; k < nb; k += 32) b[new_s - nb + k] = a[old_s - nb + k];
}

// grow list buffers to hold at least `need` entries (with 50% headroom)
static int grow(Ctx *c, int which, long long need) {
  if (need <= c->lcap[which]) return CM3D_NB_OK;
  DevLock lock(device_mutex());
  long long cap = need + need / 2 + 4096;
  if (c->graph) {
    // a captured step holds the old buffer addresses
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  if (c->lst[which]) cudaFree(c->lst[which]);
  c->lst[which] = nullptr;
  cudaError_t e = cudaMalloc(&c->lst[which], sizeof(int2) * (size_t)cap);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(list)");
  c->lcap[which] = cap;
  return CM3D_NB_OK;
}

// widen the full-list slots to hold `need` entries (+1/8 and 32 spare)
static int grow_full(Ctx *c, long long need) {
  DevLock lock(device_mutex());
  long long s = (need + need / 8 + 32 + 31) / 32 * 32;
  if (s <= c->nbr_stride) s = c->nbr_stride + 32;
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  CK(cudaStreamSynchronize(c->st));
  uint32_t *wider = nullptr;
  cudaError_t e = cudaMalloc(&wider, sizeof(uint32_t) * (size_t)c->n * (size_t)s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(full list)");
  // the lists of the systems not being rebuilt stay valid: both segments of
  // every slot move into the wider slots (a rebuilt system's are rewritten)
  if (c->nbr)
    k_regrow_copy<<<grid_for((long long)c->n * 32, 256), 256, 0, c->st>>>(c->n, c->nbr_stride, (int)s, c->nlen,
                                                                           c->nbr, wider);
  CK(cudaStreamSynchronize(c->st));
  if (c->nbr) cudaFree(c->nbr);
  c->nbr = wider;
  c->nbr_stride = (int)s;
  c->lcap[LT_FULL] = (long long)c->n * s;
  return CM3D_NB_OK;
}

static ListCaps caps(Ctx *c) {
  ListCaps C;
  for (int k = 0; k < 4; k++) C.cap[k] = c->lcap[k];
  return C;
}

// Build the lists from the current positions.  `all`: every system (set-up,
// get_ngbr, export); otherwise only the systems whose displacement test
// asked for it (sreb).  With device_flag the kernels are also gated on the
// device rebuild flag (graph replay) and the capacities are not re-checked on
// the host.  The plain engine always builds CM3D's half lists (its pair
// kernels walk them); the mixed engine builds its full list and the half
// lists only when asked (export / parity checks).
int build_lists(Ctx *c, bool device_flag, bool all) {
  const int n = c->n;
  const int B = 256;
  const int *gate = device_flag ? c->istate : nullptr;
  const int al = all ? 1 : 0;
  const bool want_half = c->mode == CM3D_NB_PLAIN_FP64 || c->want_half;
  cudaEvent_t e0;
  tbegin(c, 2, &e0);
  int4 *cimg = c->cimg;
  k_cell_zero<<<grid_for(c->ncells, B), B, 0, c->st>>>(c->ncells, c->cell_sys, c->sreb, al, c->cell_cursor, gate);
  k_cell_assign<<<grid_for(n, B), B, 0, c->st>>>(n, c->pos, c->sp, c->sys_of, c->sreb, al, c->cell_of,
                                                  c->cell_cursor, cimg, gate);
  k_cell_scan<<<c->nsys, 256, 0, c->st>>>(c->sp, c->sreb, al, c->cell_cursor, c->cell_start, gate);
  k_cell_fill<<<grid_for(n, B), B, 0, c->st>>>(n, c->sys_of, c->sreb, al, c->cell_of, c->cell_start,
                                                c->cell_cursor, c->cell_atoms, gate);
  {
    // enough blocks for four per SM where the grid allows it
    const int per_block = std::max(1, std::min(SORT_CELLS, c->ncells / std::max(1, 4 * c->num_sms)));
    k_cell_sort<<<(c->ncells + per_block - 1) / per_block, SORT_THREADS, 0, c->st>>>(
        c->ncells, per_block, c->cell_sys, c->sreb, al, c->cell_start, c->itype, c->cell_atoms, gate);
  }
  k_sorted_init<<<grid_for(n, B), B, 0, c->st>>>(n, c->sp, c->sys_of, c->sreb, al, c->cell_atoms, cimg, c->itype,
                                                  c->pos, c->q, c->rank, c->styp, c->corner, c->xq, gate);
  c->launches += 6;
  const long long warps_threads = 32LL * n;
  if (c->mode == CM3D_NB_MIXED) {
    for (;;) {
      if (c->lw_cap > 0) {
        // block per cell over the cells of the systems being rebuilt, the
        // stencil neighbourhood staged in shared memory
        const size_t smem = (size_t)c->lw_cap * LW_BYTES_PER_ATOM;
        static unsigned long long attr_devs = 0;
        if (c->dev < 64 && !(attr_devs & (1ull << c->dev))) {
          cudaFuncSetAttribute(k_list_win, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->lw_smem_max);
          attr_devs |= 1ull << c->dev;
        }
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_list_win, LW_THREADS, smem);
        long long grid = (long long)c->num_sms * (per_sm > 0 ? per_sm : 1);
        if (grid > c->ncells) grid = c->ncells;
        k_rebuild_cells<<<1, 1024, 0, c->st>>>(c->nsys, c->sp, c->sreb, al, c->rb_scan, gate);
        k_list_win<<<(int)grid, LW_THREADS, smem, c->st>>>(
            c->nsys, c->rb_scan, c->sp, n, c->nbr_stride, c->lw_cap, c->cell_atoms, c->cell_start, c->xq, c->pos,
            c->itype, c->map, c->icut, c->q, c->excl_off, c->excl_idx, c->cexcl_off, c->cexcl_idx, cimg, c->nbr,
            c->nlen, c->stat, device_flag ? c->istate + IS_HALT : nullptr, gate);
        c->launches++;
      } else {
        k_list_full<<<grid_for(warps_threads, 256), 256, 0, c->st>>>(
            n, c->sp, c->sys_of, c->sreb, al, c->nbr_stride, c->cell_atoms, c->cell_start, c->xq, c->pos,
            c->itype, c->map, c->icut, c->q, c->excl_off, c->excl_idx, c->cexcl_off, c->cexcl_idx, cimg, c->nbr,
            c->nlen, c->stat, device_flag ? c->istate + IS_HALT : nullptr, gate);
      }
      c->launches++;
      CKL(c);
      if (device_flag) break;
      // host-driven build: widen the slots and build again if a list did not fit
      CK(cudaMemcpyAsync(c->h_stat, c->stat, sizeof(long long) * ST_COUNT, cudaMemcpyDeviceToHost, c->st));
      CK(cudaStreamSynchronize(c->st));
      if (c->h_stat[ST_NEED_STRIDE] <= c->nbr_stride) break;
      int rc = grow_full(c, c->h_stat[ST_NEED_STRIDE]);
      if (rc) return rc;
    }
  }
  if (c->mode == CM3D_NB_MIXED) {
    int rc = cw_convert(c, device_flag, all);
    if (rc) return rc;
  }
  if (want_half) {
    k_list_half<false><<<grid_for(warps_threads, 256), 256, 0, c->st>>>(
        n, c->sp, c->sys_of, caps(c), c->cell_atoms, c->cell_start, c->xq, c->pos, c->itype, c->map, c->icut,
        c->q, c->excl_off, c->excl_idx, c->cexcl_off, c->cexcl_idx, cimg, c->cnt, nullptr, nullptr, nullptr,
        nullptr, nullptr, nullptr, c->stat, nullptr, gate);
    k_scan<int, long long><<<dim3(1, 4), 1024, 0, c->st>>>(c->cnt, c->off, c->ltot, n, gate);
    c->launches += 2;
    CKL(c);
    if (!device_flag) {
      CK(cudaMemcpyAsync(c->h_ltot, c->ltot, sizeof(long long) * 4, cudaMemcpyDeviceToHost, c->st));
      CK(cudaStreamSynchronize(c->st));
      for (int k = 0; k < 4; k++) {
        int rc = grow(c, k, c->h_ltot[k] > 0 ? c->h_ltot[k] : 1);
        if (rc) return rc;
        c->hcount[k] = c->h_ltot[k];
      }
    }
    k_list_half<true><<<grid_for(warps_threads, 256), 256, 0, c->st>>>(
        n, c->sp, c->sys_of, caps(c), c->cell_atoms, c->cell_start, c->xq, c->pos, c->itype, c->map, c->icut,
        c->q, c->excl_off, c->excl_idx, c->cexcl_off, c->cexcl_idx, cimg, nullptr, c->off, c->ltot, c->lst[0],
        c->lst[1], c->lst[2], c->lst[3], c->stat, device_flag ? c->istate + IS_HALT : nullptr, gate);
    c->launches++;
  }
  if (!c->no_snapshot) {
    k_snapshot<<<grid_for(n, B), B, 0, c->st>>>(n, c->sp, c->sys_of, c->sreb, al, c->pos, c->dxn, c->slast,
                                                 c->sstat, gate, c->istate, c->stat);
    c->launches++;
  }
  CKL(c);
  tend(c, 2, e0);
  if (!device_flag) {
    c->lists_built = true;
    c->rebuilds_host++;
  }
  return CM3D_NB_OK;
}

}  // namespace cm3d
