// nb_cwin.cu -- compact-window pair kernel for one large system.
//
// The physics is that of force_npol (energy/inter/md_fnopol.c:46-255) and
// force_e (energy/inter/finter_e.c:42-233): CM3D's tables on the r^2 grid,
// its 3-point interpolation f = f0 + p (A + p B) (finter_e.c:122-136), the
// cut-off test `dis2 < rmax2` (finter_e.c:119) and its energy shifts -- the
// same sums as nb_pair.cu, laid out so that the kernel's shared-memory
// traffic per pair is close to the minimum.
//
// The master full list (nb_list.cu: per cell-sorted atom, 32-bit entries of
// sorted index + cell-shift code + list flags) is rewritten after every
// rebuild into a compact list (k_cw_convert):
//
//   * a 16-bit entry holds the index of j in the 27-cell window of i's cell
//     (the window a pair-kernel block stages in shared memory, each cell
//     already moved by its periodic shift), so an entry names j's staged
//     position directly: no shift code, no index translation per pair; and
//     the list is half the bytes;
//   * every segment (LJ-list pairs first, then electrostatics-only pairs) is
//     stored in blocks of 128 entries interleaved by lane: the 8-byte word
//     `w` of a block holds entries w, w + 32, w + 64, w + 96, so that in each
//     of the four passes over a block the 32 lanes of a warp read 32
//     consecutive entries -- mostly consecutive window slots of one cell,
//     which spreads a warp's window loads over the shared-memory banks.
//
// The pair kernel (k_pair_cw) keeps the tables in shared memory replicated
// RF (RG) times, lane l reading copy l % RF: with RF = 8 the 16-byte force
// coefficients a lane reads always lie in bank group l % 8, so a warp's 32
// random table reads take 4 shared-memory wavefronts -- the minimum for 512
// bytes -- instead of the ~7 that random 16-byte reads cost.
//
// Precision and order: distances, interpolation and the per-pair products
// are FP32 (cell-relative coordinates, as in nb_pair.cu); each lane sums its
// pairs of one atom in FP32 (about 20 pairs for 32 lanes per atom) and then
// adds that chunk in FP64: forces across the atom's lanes (fixed shuffle
// tree), energies and virials into per-lane FP64 sums that the block adds up
// per work item and k_cw_ereduce adds over items, all in a fixed order.  The
// results do not depend on timing: a run repeats bit for bit.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <type_traits>
#include <vector>

#include "nb_common.cuh"

namespace cm3d {

constexpr int CW_THREADS = 512;            // threads of a pair-kernel block (or CW_THREADS_WIDE)
constexpr int CW_THREADS_WIDE = 640;       // 20 warps at 96 registers: the autotuner picks either
constexpr int CW_ROW = CM3D_CW_ROW;         // interleave width (entries per pass of a block)
constexpr int CW_BLOCK = 4 * CW_ROW;        // entries per block: one 8-byte word per lane
constexpr uint32_t CW_IDX = 0x3FFFu;        // window index bits of an entry
constexpr uint32_t CW_EL = 0x4000u;         // LJ-segment entry: the pair is also in CM3D's te list
constexpr int CW_MAX_CAP = 16382;           // window slots (the dummy slot `cap` must fit 14 bits)
constexpr float CW_MAGIC = 12582912.0f;     // 1.5 * 2^23: p + MAGIC rounded toward zero holds floor(p)
constexpr unsigned CW_MAGIC_BITS = 0x4B400000u;
constexpr int CW_STATIC_SMEM = 6144;        // >= the kernel's static shared arrays (5.2 KB)
constexpr int CW_RF = 8;                    // copies of the erfc force table (lane l reads copy l % 8)
constexpr int CW_RG = 8;                    // copies of the erfc energy table

// per-item FP64 sums (each pair is seen from both ends: k_cw_ereduce halves)
enum { CQ_EEL = 0, CQ_QQ_UNUSED, CQ_VE0, CQ_VE1, CQ_VE2, CQ_VE4, CQ_VE5, CQ_VE8,
       CQ_ELJ, CQ_VSH, CQ_VL0, CQ_VL1, CQ_VL2, CQ_VL4, CQ_VL5, CQ_VL8, CQ_COUNT };

struct CwP {
  int n, ncx, ncy, ncz, nitems, nsplit, cap, words;   // words: 8-byte words per atom slot
  int ntable, ntypes, ninter;
  float rc2_el, dx2c, offc, pmax;
  float sat_a, sat_b;        // dx2 / pmax, -rmin^2 dx2 / pmax: the saturated table coordinate
  float r2under;             // r^2 below which the erfc table underflows (p < 1)
  // one LJ interaction (LJM 1): cut-off^2, dx2tab, rmins_cut2 * dx2tab, vtab[ntable-4]
  float rc2_l, dx2l, offl, vtl;
  int map0, inter0;          // a batch group: the type map and cut-offs of its first system
};

// ------------------------------------------------------------------
// Master list -> compact list.  Warp per cell-sorted atom t (one system:
// every atom; a batch: the atoms of the compact systems being rebuilt): the 27-cell
// window layout of t's cell (stencil cell w = shift code, j-cell = i-cell -
// k_w, cells in code order) gives delta[w] = window offset - first sorted
// index (lane w holds it), so entry (u, w) becomes window index u +
// delta[w].  A window larger than `cap` cannot be indexed: the cell's atoms
// get empty lists, ST_CWIN counts it (once per cell) and a captured step
// halts (the host then turns the compact path off).
__device__ __forceinline__ void cw_convert_atom(const int t, const int lane, int ncx, int ncy, int ncz, int c0,
                                                int cap, int n, int words, int row,
                                                const int *__restrict__ cell_start, const int *__restrict__ cell_of,
                                                const int *__restrict__ sorig, const int *__restrict__ nlen,
                                                int stride, const uint32_t *__restrict__ nbr, uint2 *__restrict__ cwl,
                                                int2 *__restrict__ cwn, long long *__restrict__ stat,
                                                int *__restrict__ halt) {
  const uint32_t dummy = (uint32_t)cap;
  const int c = cell_of[sorig[t]] - c0;
  int delta = 0, tot = 0;
  {
    const int cz = c % ncz, cy = (c / ncz) % ncy, cx = c / (ncz * ncy);
    int cnt = 0, cs = 0;
    if (lane < 27) {
      int jx = cx - (lane / 9 - 1), jy = cy - ((lane / 3) % 3 - 1), jz = cz - (lane % 3 - 1);
      jx = jx < 0 ? jx + ncx : (jx >= ncx ? jx - ncx : jx);
      jy = jy < 0 ? jy + ncy : (jy >= ncy ? jy - ncy : jy);
      jz = jz < 0 ? jz + ncz : (jz >= ncz ? jz - ncz : jz);
      const int jc = c0 + (jx * ncy + jy) * ncz + jz;
      cs = cell_start[jc];
      cnt = cell_start[jc + 1] - cs;
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    delta = lane < 27 ? incl - cnt - cs : 0;
    tot = __shfl_sync(0xffffffffu, incl, 26);
  }
  const bool fits = tot <= cap;
  if (!fits && lane == 0 && t == cell_start[c0 + c]) {
    atomicAdd((unsigned long long *)(stat + ST_CWIN), 1ull);
    if (halt) *halt = 1;
  }
  {
    {
      const int na = fits ? nlen[t] : 0, nb = fits ? nlen[n + t] : 0;
      const uint32_t *src = nbr + (size_t)t * stride;
      uint2 *dst = cwl + (size_t)t * words;
      // blocks of 4 row entries: row 32 lanes per atom (k_pair_cw) or 8 (k_pair_cs)
      const int blk = 4 * row;
      const int nba = (na + blk - 1) / blk, nbb = (nb + blk - 1) / blk;
      // padding first: every slot of the atom's blocks holds the dummy
      for (int w = lane; w < (nba + nbb) * row; w += 32)
        dst[w] = make_uint2(dummy | (dummy << 16), dummy | (dummy << 16));
      __syncwarp();
      for (int sg = 0; sg < 2; sg++) {
        const bool front = sg == 0;
        const int m = front ? na : nb;
        const uint32_t *in = front ? src : src + (stride - nb);   // the back segment ends at the slot's end
        unsigned short *out = reinterpret_cast<unsigned short *>(dst + (front ? 0 : nba * row));
        // every lane calls it (the delta comes by shuffle); -1 past the end
        auto window_index_of = [&](bool v, uint32_t en, uint32_t &o) -> int {
          const int code = (en >> ENT_CODE_SHIFT) & 31;
          const int wi = (int)(en & ENT_JMASK) + __shfl_sync(0xffffffffu, delta, code);
          // inside the window by construction (a pair's shift code names
          // j's stencil cell); anything else would index past the staged
          // atoms, so it becomes the dummy
          o = wi >= 0 && wi < tot ? (uint32_t)wi : dummy;
          if (front && (en & ENT_EL) && o != dummy) o |= CW_EL;
          return v ? (int)(o & 7u) : -1;
        };
        auto window_index = [&](int e, uint32_t &o) -> int {
          const bool v = e < m;
          return window_index_of(v, v ? in[e] : 0u, o);
        };
        // bank classes: the window slot mod 8 (the 16-byte bank group of
        // the staged position).  Position j of the segment is read by lane
        // j % row (of the atom's lanes), so putting a class-(j % 8) entry at
        // j gives the 8 lanes of each quarter-warp 8 different bank groups;
        // the entries that do not fit their own class's positions fill the
        // rest.  Ranks within a class go lane by lane (lane l's entries l,
        // l + 32, ... after those of the lanes before it): each lane counts
        // its classes in 16-bit fields (classes 0-3 in c03, 4-7 in c47), one
        // warp scan gives the bases -- no warp vote per entry.
        // a segment of up to CW_KEEP x 32 entries keeps its window indices
        // in registers between the passes (16 bits each, two per register;
        // 0xFFFF past the segment's end), with every entry's load issued
        // up front; longer segments read the master list twice
        constexpr int CW_KEEP = 24;
        const bool kept = m <= 32 * CW_KEEP;
        unsigned pk[CW_KEEP / 2];
        unsigned long long c03 = 0ull, c47 = 0ull;
        auto count = [&](int cl) {
          if (cl < 4) c03 += 1ull << (16 * cl);
          else c47 += 1ull << (16 * (cl - 4));
        };
        if (kept) {
          uint32_t en[CW_KEEP];
#pragma unroll
          for (int k = 0; k < CW_KEEP; k++) en[k] = k * 32 + lane < m ? in[k * 32 + lane] : 0u;
#pragma unroll
          for (int k = 0; k < CW_KEEP; k++) {
            unsigned ok = 0xFFFFu;
            if (k * 32 < m) {
              uint32_t o;
              const int cl = window_index_of(k * 32 + lane < m, en[k], o);
              if (cl >= 0) {
                ok = o;
                count(cl);
              }
            }
            if (k & 1) pk[k >> 1] |= ok << 16;
            else pk[k >> 1] = ok;
          }
        } else {
          for (int e0 = 0; e0 < m; e0 += 32) {
            uint32_t o;
            const int cl = window_index(e0 + lane, o);
            if (cl >= 0) count(cl);
          }
        }
        unsigned long long i03 = c03, i47 = c47;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const unsigned long long a = __shfl_up_sync(0xffffffffu, i03, o);
          const unsigned long long b = __shfl_up_sync(0xffffffffu, i47, o);
          if (lane >= o) {
            i03 += a;
            i47 += b;
          }
        }
        const unsigned long long t03 = __shfl_sync(0xffffffffu, i03, 31), t47 = __shfl_sync(0xffffffffu, i47, 31);
        int cnt[8];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          cnt[q] = (int)((t03 >> (16 * q)) & 0xFFFFull);
          cnt[q + 4] = (int)((t47 >> (16 * q)) & 0xFFFFull);
        }
        const int Q = m >> 3;
        // running ranks: this lane's bases, advanced per entry
        unsigned long long r03 = i03 - c03, r47 = i47 - c47;
        auto place = [&](int cl, uint32_t o) {
          int rank;
          if (cl < 4) {
            rank = (int)((r03 >> (16 * cl)) & 0xFFFFull);
            r03 += 1ull << (16 * cl);
          } else {
            rank = (int)((r47 >> (16 * (cl - 4))) & 0xFFFFull);
            r47 += 1ull << (16 * (cl - 4));
          }
          int pos;
          if (rank < Q) {
            pos = cl + 8 * rank;
          } else {
            // the L-th free position: the unused class positions of the
            // classes short of Q entries, in class order, then the tail
            int L = rank - Q;
#pragma unroll
            for (int q = 0; q < 8; q++)
              if (q < cl) L += max(0, cnt[q] - Q);
            pos = -1;
#pragma unroll
            for (int q = 0; q < 8; q++) {
              const int d = max(0, Q - cnt[q]);
              if (pos < 0) {
                if (L < d) pos = q + 8 * (cnt[q] + L);
                else L -= d;
              }
            }
            if (pos < 0) pos = 8 * Q + L;
          }
          // position -> (block, lane, k): 16-bit entry k of the block's
          // word for lane r % row (row is 8 or 32: a power of two)
          const int bb = pos / blk, r = pos - bb * blk;
          out[(bb * row + (r & (row - 1))) * 4 + r / row] = (unsigned short)o;
        };
        if (kept) {
#pragma unroll
          for (int k = 0; k < CW_KEEP; k++) {
            if (k * 32 < m) {
              const unsigned o = (k & 1) ? pk[k >> 1] >> 16 : pk[k >> 1] & 0xFFFFu;
              if (o != 0xFFFFu) place((int)(o & 7u), o);
            }
          }
        } else {
          for (int e0 = 0; e0 < m; e0 += 32) {
            uint32_t o = dummy;
            const int cl = window_index(e0 + lane, o);
            if (cl >= 0) place(cl, o);
          }
        }
      }
      if (lane == 0) cwn[t] = make_int2(na, nb);
    }
  }
}

__global__ void __launch_bounds__(256, 2) k_cw_convert(int ncx, int ncy, int ncz, int cap, int n, int words, int row,
                                                    const int *__restrict__ cell_start,
                                                    const int *__restrict__ cell_of,
                                                    const int *__restrict__ sorig,
                                                    const int *__restrict__ nlen, int stride,
                                                    const uint32_t *__restrict__ nbr, uint2 *__restrict__ cwl,
                                                    int2 *__restrict__ cwn, long long *__restrict__ stat,
                                                    int *__restrict__ halt, const int *__restrict__ gs) {
  if (gated_off(gs, 1)) return;
  const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (t >= n) return;                                  // whole warps
  cw_convert_atom(t, threadIdx.x & 31, ncx, ncy, ncz, 0, cap, n, words, row, cell_start, cell_of, sorig, nlen,
                  stride, nbr, cwl, cwn, stat, halt);
}

// The atoms to convert in a batch, as one index range: scan[s] is the
// number of atoms of compact systems being rebuilt (all: every compact
// system) before system s, scan[nsys] their total.  One block.
__global__ void __launch_bounds__(1024) k_cw_scan(int nsys, const SysP *__restrict__ sp,
                                                  const int *__restrict__ cwsys, const int *__restrict__ sreb,
                                                  int all, int *__restrict__ scan, const int *__restrict__ gs) {
  if (gated_off(gs, 1)) return;
  __shared__ int warp_tot[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < nsys; base += blockDim.x) {
    const int sy = base + threadIdx.x;
    const int v = sy < nsys && cwsys[sy] && (all || sreb[sy] != 0) ? sp[sy].n : 0;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
      int x = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += u;
      }
      warp_tot[lane] = x;
    }
    __syncthreads();
    if (sy < nsys) scan[sy] = carry + (w > 0 ? warp_tot[w - 1] : 0) + incl - v;
    __syncthreads();
    if (threadIdx.x == 0) carry += warp_tot[nw - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) scan[nsys] = carry;
}

// A batch: warps walk the scanned range (a fixed grid, so that a captured
// step converts whatever the device-side rebuild flags select); atom v of the
// range lies in the last system s with scan[s] <= v, each on its own grid.
__global__ void __launch_bounds__(256, 2) k_cw_convert_sys(int nsys, const int *__restrict__ scan,
                                                        const SysP *__restrict__ sp, int cap, int n, int words,
                                                        int row, const int *__restrict__ cell_start,
                                                        const int *__restrict__ cell_of,
                                                        const int *__restrict__ sorig,
                                                        const int *__restrict__ nlen, int stride,
                                                        const uint32_t *__restrict__ nbr, uint2 *__restrict__ cwl,
                                                        int2 *__restrict__ cwn, long long *__restrict__ stat,
                                                        int *__restrict__ halt, const int *__restrict__ gs) {
  if (gated_off(gs, 1)) return;
  const int total = scan[nsys];
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < total; v += nwarps) {
    int sa = 0, sb = nsys;
    while (sb - sa > 1) {
      const int mid = (sa + sb) >> 1;
      if (scan[mid] <= v) sa = mid;
      else sb = mid;
    }
    const SysP &P = sp[sa];
    cw_convert_atom(P.a0 + (v - scan[sa]), threadIdx.x & 31, P.nc[0], P.nc[1], P.nc[2], P.c0, cap, n, words, row,
                    cell_start, cell_of, sorig, nlen, stride, nbr, cwl, cwn, stat, halt);
  }
}

// ------------------------------------------------------------------
// Pair kernel.  Block per work item (a cell, or one of `nsplit` parts of
// its atoms); the block stages the cell's window, then each warp takes one
// i-atom at a time and its 32 lanes walk the atom's list blocks (every
// branch is warp-uniform).  The next two blocks' list words are loaded
// while a block is being evaluated.
//   HAS_EL: the system has charges; LJM: 0 no LJ, 1 one LJ interaction (its
//   parameters in CwP), 2 several (type map, cut-offs and tables per pair).
//
// Electrostatic table lookup without a range test: the table coordinate
// p = (r^2 - rmin^2) dx2 is formed as pmax * sat((r^2 - rmin^2) dx2 / pmax),
// saturated to [0, pmax] by the FMA itself; knot 0 holds CM3D's clamp below
// the table (k = 1, fraction 0: the value at knot 1), knot pmax = ntable - 3
// holds zeros.  A pair at or beyond the cut-off (CM3D's `dis2 < rmax2`
// test: p < ntable - 3 exactly when r^2 < rc^2) and the padding entries
// therefore read zero coefficients and contribute nothing.
struct CwAcc {
  float fx, fy, fz;              // sum qj f d over the electrostatic pairs (x qi at the end)
  float gx, gy, gz;              // sum f d over the LJ pairs
  float eel, ve[6];              // sum qj V, sum qj f d d
  float elo, vsh, vl[6];         // LJ: energy lo parts, sum vt, sum f d d
  double elj_hi;                 // LJ: energy hi parts (FP64)
  float r2min, pminl;            // underflow tests: smallest r^2 (electrostatics), LJ table coordinate
};

__device__ __forceinline__ void cw_zero(CwAcc &A) {
  A.fx = A.fy = A.fz = A.gx = A.gy = A.gz = 0.f;
  A.eel = A.elo = A.vsh = 0.f;
#pragma unroll
  for (int k = 0; k < 6; k++) A.ve[k] = A.vl[k] = 0.f;
  A.elj_hi = 0.0;
  A.r2min = A.pminl = 3.0e38f;
}

// floor of p in [1, 2^22) by the rounding of one FP32 add (RZ mode); returns
// the fraction and leaves the float bits MAGIC + floor(p) in kb
__device__ __forceinline__ float cw_split(float p, unsigned &kb) {
  const float t = __fadd_rz(p, CW_MAGIC);
  kb = __float_as_uint(t);
  return p - (t - CW_MAGIC);
}

// Shared-memory loads from 32-bit shared-window addresses (the hot loop's
// address arithmetic stays in 32 bits: one shift-and-add per address).
__device__ __forceinline__ float4 lds_f4(unsigned a) {
  float4 v;
  asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
  return v;
}
__device__ __forceinline__ float2 lds_f2(unsigned a) {
  float2 v;
  asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
  return v;
}

// Window staging by bulk copies (TMA, cp.async.bulk, no multicast: the
// source is this GPU's own memory) completing on a block mbarrier.
__device__ __forceinline__ void mbar_init(unsigned bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Generic-proxy accesses of the window (the previous item's reads) before
// the async-proxy writes of the next copies.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void *src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// Waits for the phase of the given parity to complete; false after `limit`
// polls (each try_wait may suspend the thread for a while first).
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, int limit) {
  for (int it = 0; it < limit; it++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
constexpr int CW_WAIT_LIMIT = 1 << 22;

// One electrostatic pair: qj = j's charge, or 0 for an LJ-segment pair
// outside the te list.  tfb / tgb: this lane's table copies as 32-bit shared
// addresses less MAGIC_BITS knots, so that the float bits of the split
// coordinate address the knot directly (k * stride = bits * stride - MAGIC_BITS
// * stride, mod 2^32).
template <int RF = CW_RF, int RG = CW_RG>
__device__ __forceinline__ void cw_elec(const CwP &P, float qj, float dx, float dy, float dz, float r2,
                                        unsigned tfb, unsigned tgb, CwAcc &A) {
  A.r2min = fminf(A.r2min, r2);
  const float ps = __saturatef(fmaf(r2, P.sat_a, P.sat_b));
  const float t = __fmaf_rz(ps, P.pmax, CW_MAGIC);
  const float kf = t - CW_MAGIC;
  const float fr = fmaf(ps, P.pmax, -kf);
  const unsigned kb = __float_as_uint(t);
  const float4 c = lds_f4(tfb + kb * (unsigned)(RF * sizeof(float4)));
  const float2 d = lds_f2(tgb + kb * (unsigned)(RG * sizeof(float2)));
  const float fe = qj * fmaf(fr, fmaf(fr, c.z, c.y), c.x);
  A.eel = fmaf(qj, fmaf(fr, fmaf(fr, d.y, d.x), c.w), A.eel);
  const float ux = fe * dx, uy = fe * dy, uz = fe * dz;
  A.fx += ux;
  A.fy += uy;
  A.fz += uz;
  A.ve[0] = fmaf(ux, dx, A.ve[0]);
  A.ve[1] = fmaf(ux, dy, A.ve[1]);
  A.ve[2] = fmaf(ux, dz, A.ve[2]);
  A.ve[3] = fmaf(uy, dy, A.ve[3]);
  A.ve[4] = fmaf(uy, dz, A.ve[4]);
  A.ve[5] = fmaf(uz, dz, A.ve[5]);
}

// One LJ pair of interaction parameters {rc2, dx2, off, vt}; tl holds 2
// float4 per knot {d0, dA, dB, v0 hi} {vA, vB, v0 lo, -}.
__device__ __forceinline__ void cw_lj(const CwP &P, float dx, float dy, float dz, float r2, float rc2, float dx2,
                                      float off, float vt, const float4 *__restrict__ tl, CwAcc &A) {
  const bool ok = r2 < rc2;
  float p = fmaf(r2, dx2, -off);
  A.pminl = fminf(A.pminl, ok ? p : 3.0e38f);
  p = fminf(fmaxf(p, 1.f), P.pmax);
  unsigned kb;
  const float fr = cw_split(p, kb);
  const unsigned k = kb - CW_MAGIC_BITS;
  const float4 a = tl[2 * k], b = tl[2 * k + 1];
  const float okf = ok ? 1.f : 0.f;
  const float f = okf * fmaf(fr, fmaf(fr, a.z, a.y), a.x);
  A.elj_hi += ok ? (double)a.w : 0.0;
  A.elo = fmaf(okf, fmaf(fr, fmaf(fr, b.y, b.x), b.z), A.elo);
  A.vsh = fmaf(okf, vt, A.vsh);
  const float ux = f * dx, uy = f * dy, uz = f * dz;
  A.gx += ux;
  A.gy += uy;
  A.gz += uz;
  A.vl[0] = fmaf(ux, dx, A.vl[0]);
  A.vl[1] = fmaf(ux, dy, A.vl[1]);
  A.vl[2] = fmaf(ux, dz, A.vl[2]);
  A.vl[3] = fmaf(uy, dy, A.vl[3]);
  A.vl[4] = fmaf(uy, dz, A.vl[4]);
  A.vl[5] = fmaf(uz, dz, A.vl[5]);
}

// BATCH: the work items of one group of a batch's systems -- systems whose
// tables and pair parameters are the same, so that P and the staged tables
// serve them all -- given as {system, cell of the system, part, parts};
// each item's cell grid and shifts come from its system's SysP, and its
// partial sums go to item0 + item.
template <bool HAS_EL, int LJM, bool BATCH = false, int NT = CW_THREADS>
__global__ void __launch_bounds__(NT, 1) k_pair_cw(
    CwP P, const float4 *__restrict__ xq, const int *__restrict__ styp, const int *__restrict__ sorig,
    const int *__restrict__ cell_start, const int2 *__restrict__ cwn, const uint2 *__restrict__ cwl,
    const float4 *__restrict__ gshift, const int *__restrict__ gmap, const float *__restrict__ gfcut,
    const float4 *__restrict__ gtf, const float2 *__restrict__ gtg, const float4 *__restrict__ gtl,
    double *__restrict__ fout, double *__restrict__ ipart, long long *__restrict__ stat,
    const int *__restrict__ gs, const int4 *__restrict__ items = nullptr, const SysP *__restrict__ sp = nullptr,
    int item0 = 0) {
  if (gated_off(gs, 0)) return;
  extern __shared__ float4 sm[];
  // tables first (16-byte aligned), then the window
  float4 *tf = sm;                                                    // ntable * CW_RF
  float2 *tg = reinterpret_cast<float2 *>(tf + (HAS_EL ? P.ntable * CW_RF : 0));   // ntable * CW_RG
  float4 *tl = reinterpret_cast<float4 *>(tg + (HAS_EL ? P.ntable * CW_RG : 0));   // 2 ninter ntable
  const int nl = LJM ? 2 * P.ninter * P.ntable : 0;
  float4 *wx = tl + nl;                                               // cap + 1 staged atoms
  unsigned char *wt = reinterpret_cast<unsigned char *>(wx + P.cap + 1);   // LJM 2: their types
  __shared__ int s_cs[27], s_off[28];
  __shared__ float4 s_shift[54];
  __shared__ int s_map[256];
  __shared__ float4 s_cut[64];                                        // LJM 2: {rc2, dx2, off, vt}
  __shared__ double s_red[NT / 32][CQ_COUNT];
  __shared__ __align__(8) unsigned long long s_mbar;
  static_assert(CQ_COUNT == 16, "the transposing reduction gives lane pair q quantity q of 16");

  if (!BATCH)
    for (int k = threadIdx.x; k < 54; k += blockDim.x) s_shift[k] = gshift[k];
  if (HAS_EL) {
    for (int k = threadIdx.x; k < P.ntable * CW_RF; k += blockDim.x) tf[k] = gtf[k / CW_RF];
    for (int k = threadIdx.x; k < P.ntable * CW_RG; k += blockDim.x) tg[k] = gtg[k / CW_RG];
  }
  for (int k = threadIdx.x; k < nl; k += blockDim.x) tl[k] = gtl[k];
  if (LJM == 2) {
    // the type map as local interaction indices (a batch's global map holds
    // inter0 + local); the cut-offs of those interactions
    for (int k = threadIdx.x; k < P.ntypes * P.ntypes; k += blockDim.x) {
      const int in = gmap[P.map0 + k];
      s_map[k] = in >= 0 ? in - P.inter0 : -1;
    }
    for (int k = threadIdx.x; k < P.ninter; k += blockDim.x) {
      const float *f = gfcut + 8 * (P.inter0 + k);
      s_cut[k] = make_float4(f[0], f[2], f[1], f[3]);
    }
  }
  const unsigned bar = (unsigned)__cvta_generic_to_shared(&s_mbar);
  unsigned phase = 0;
  if (threadIdx.x == 0) {
    wx[P.cap] = make_float4(1.0e6f, 1.0e6f, 1.0e6f, 0.f);   // the dummy entry's partner: out of range
    if (LJM == 2) wt[P.cap] = 0;
    mbar_init(bar);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NWARP = NT / 32;
  // this lane's table copies and the window as 32-bit shared addresses
  const unsigned tfb = (unsigned)__cvta_generic_to_shared(tf + (lane & (CW_RF - 1))) -
                       CW_MAGIC_BITS * (unsigned)(CW_RF * sizeof(float4));
  const unsigned tgb = (unsigned)__cvta_generic_to_shared(tg + (lane & (CW_RG - 1))) -
                       CW_MAGIC_BITS * (unsigned)(CW_RG * sizeof(float2));
  const unsigned wxb = (unsigned)__cvta_generic_to_shared(wx);
  unsigned long long under = 0;

  for (int item = blockIdx.x; item < P.nitems; item += gridDim.x) {
    int c, part, nsplit, ncx = P.ncx, ncy = P.ncy, ncz = P.ncz, c0 = 0, sys = 0;
    if (BATCH) {
      const int4 it = items[item];
      sys = it.x;
      c = it.y;
      part = it.z;
      nsplit = it.w;
      ncx = sp[sys].nc[0];
      ncy = sp[sys].nc[1];
      ncz = sp[sys].nc[2];
      c0 = sp[sys].c0;
    } else {
      c = item / P.nsplit;
      part = item - c * P.nsplit;
      nsplit = P.nsplit;
    }
    const int cz = c % ncz, cy = (c / ncz) % ncy, cx = c / (ncz * ncy);
    __syncthreads();                                       // the previous window is no longer read
    if (BATCH)
      for (int k = threadIdx.x; k < 54; k += blockDim.x) s_shift[k] = k < 27 ? sp[sys].shift[k] : sp[sys].shift_lo[k - 27];
    if (warp == 0) {
      int cnt = 0, cs = 0;
      if (lane < 27) {
        int jx = cx - (lane / 9 - 1), jy = cy - ((lane / 3) % 3 - 1), jz = cz - (lane % 3 - 1);
        jx = jx < 0 ? jx + ncx : (jx >= ncx ? jx - ncx : jx);
        jy = jy < 0 ? jy + ncy : (jy >= ncy ? jy - ncy : jy);
        jz = jz < 0 ? jz + ncz : (jz >= ncz ? jz - ncz : jz);
        const int jc = c0 + (jx * ncy + jy) * ncz + jz;
        cs = cell_start[jc];
        cnt = cell_start[jc + 1] - cs;
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      if (lane < 27) {
        s_cs[lane] = cs;
        s_off[lane] = incl - cnt;
      }
      if (lane == 26) s_off[27] = incl;
    }
    __syncthreads();
    const int tot = s_off[27];
    // a window that does not fit was given empty lists by k_cw_convert
    const bool staged = tot <= P.cap;
    if (staged) {
      // each stencil cell's atoms are a contiguous run of the cell-sorted
      // positions: one bulk copy per cell into its window range (16-byte
      // rows, so every address and size is a multiple of 16), all
      // completing on the block's mbarrier
      if (warp == 0) {
        fence_async_smem();
        if (lane == 0) mbar_expect(bar, (unsigned)tot * (unsigned)sizeof(float4));
        __syncwarp();
        if (lane < 27) {
          const int cnt = s_off[lane + 1] - s_off[lane];
          if (cnt > 0)
            bulk_g2s(wxb + (unsigned)s_off[lane] * (unsigned)sizeof(float4), xq + s_cs[lane],
                     (unsigned)cnt * (unsigned)sizeof(float4), bar);
        }
      }
      const bool arrived = mbar_wait(bar, phase, CW_WAIT_LIMIT);
      phase ^= 1u;
      if (!__syncthreads_and(arrived)) {
        // the copies did not complete (never seen): count it, wait once
        // more for copies still in flight, and leave the block's remaining
        // items undone; the host reads the count in the status
        if (threadIdx.x == 0) atomicAdd((unsigned long long *)(stat + ST_STAGE_TIMEOUT), 1ull);
        mbar_wait(bar, phase ^ 1u, CW_WAIT_LIMIT);
        return;
      }
      // the cell's periodic shift and the cell-relative origin, in place
      // (and the types of a multi-type system)
      for (int w = warp; w < 27; w += NWARP) {
        const float4 sh = s_shift[w], shl = s_shift[27 + w];
        const int g0 = s_off[w], g1 = s_off[w + 1], u0 = s_cs[w] - g0;
        for (int g = g0 + lane; g < g1; g += 32) {
          const float4 x = wx[g];
          wx[g] = make_float4((x.x - sh.x) - shl.x, (x.y - sh.y) - shl.y, (x.z - sh.z) - shl.z, x.w);
          if (LJM == 2) wt[g] = (unsigned char)styp[u0 + g];
        }
      }
    }
    __syncthreads();
    // energy and virial sums: lane l keeps quantity (l >> 1) of CQ_* in
    // FP64 (both lanes of a pair hold it), plus its own FP64 LJ hi parts
    double Eq = 0.0, Ehi = 0.0;
    const int ci0 = s_cs[13], cin = s_off[14] - s_off[13], ioff = s_off[13];
    // the item's atoms r * NWARP + warp, r = part, part + nsplit, ...; the
    // next atom's lengths and first two list words are loaded while this
    // one is evaluated (every slot holds at least two blocks)
    const int astep = nsplit * NWARP;
    int2 nn_nx = make_int2(0, 0);
    uint2 p0 = make_uint2(0u, 0u), p1 = make_uint2(0u, 0u);
    if (staged && part * NWARP + warp < cin) {
      const int tn = ci0 + part * NWARP + warp;
      nn_nx = cwn[tn];
      p0 = __ldg(cwl + (size_t)tn * P.words + lane);
      p1 = __ldg(cwl + (size_t)tn * P.words + CW_ROW + lane);
    }
    for (int a = part * NWARP + warp; staged && a < cin; a += astep) {
      const int t = ci0 + a;
      const int2 nn = nn_nx;
      uint2 w0 = p0, w1 = p1;
      if (a + astep < cin) {
        const int tn = t + astep;
        nn_nx = cwn[tn];
        p0 = __ldg(cwl + (size_t)tn * P.words + lane);
        p1 = __ldg(cwl + (size_t)tn * P.words + CW_ROW + lane);
      }
      CwAcc A;
      cw_zero(A);
      const float4 xi = wx[ioff + a];
      const int ti = LJM == 2 ? wt[ioff + a] : 0;
      const int nba = (nn.x + CW_BLOCK - 1) / CW_BLOCK, nbt = nba + (nn.y + CW_BLOCK - 1) / CW_BLOCK;
      const uint2 *words = cwl + (size_t)t * P.words + lane;
      auto geom = [&](uint32_t e, float4 &xj, float &dx, float &dy, float &dz) {
        xj = lds_f4(wxb + ((e & CW_IDX) << 4));
        dx = xi.x - xj.x;
        dy = xi.y - xj.y;
        dz = xi.z - xj.z;
        return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      };
      auto lj_pair = [&](uint32_t e, float dx, float dy, float dz, float r2, CwAcc &Acc) {
        if (LJM == 1) {
          cw_lj(P, dx, dy, dz, r2, P.rc2_l, P.dx2l, P.offl, P.vtl, tl, Acc);
        } else if (LJM == 2) {
          const int tj = wt[e & CW_IDX];
          const int in = s_map[ti * P.ntypes + tj];
          const float4 cut = s_cut[in < 0 ? 0 : in];
          // a pair without an LJ interaction (map -1) never reaches the LJ
          // segment; a padding entry may, with an out-of-range distance
          cw_lj(P, dx, dy, dz, in < 0 ? 3.0e38f : r2, cut.x, cut.y, cut.z, cut.w,
                tl + (size_t)2 * (in < 0 ? 0 : in) * P.ntable, Acc);
        }
      };
      auto front_pair = [&](uint32_t e, CwAcc &Acc) {
        float4 xj;
        float dx, dy, dz;
        const float r2 = geom(e, xj, dx, dy, dz);
        if (HAS_EL) cw_elec(P, (e & CW_EL) ? xj.w : 0.f, dx, dy, dz, (e & CW_EL) ? r2 : 3.0e38f, tfb, tgb, Acc);
        lj_pair(e, dx, dy, dz, r2, Acc);
      };
      auto back_pair = [&](uint32_t e, CwAcc &Acc) {
        if (HAS_EL) {
          float4 xj;
          float dx, dy, dz;
          const float r2 = geom(e, xj, dx, dy, dz);
          cw_elec(P, xj.w, dx, dy, dz, r2, tfb, tgb, Acc);
        }
      };
      // block b's word of this lane; the next two are in flight
      const uint2 pad = make_uint2((uint32_t)P.cap | ((uint32_t)P.cap << 16), (uint32_t)P.cap | ((uint32_t)P.cap << 16));
      if (nbt < 2) w1 = pad;
      for (int b = 0; b < nbt; b++) {
        const uint2 w2 = b + 2 < nbt ? __ldg(words + (b + 2) * CW_ROW) : pad;
        const bool front = b < nba;
        const int m = front ? min(CW_BLOCK, nn.x - b * CW_BLOCK) : min(CW_BLOCK, nn.y - (b - nba) * CW_BLOCK);
        const uint32_t e[4] = {w0.x & 0xFFFFu, w0.x >> 16, w0.y & 0xFFFFu, w0.y >> 16};
        if (front && m == CW_BLOCK) {
#pragma unroll
          for (int k = 0; k < 4; k++) front_pair(e[k], A);
        } else if (front) {
          front_pair(e[0], A);
#pragma unroll
          for (int k = 1; k < 4; k++)
            if (k * CW_ROW < m) front_pair(e[k], A);
        } else if (m == CW_BLOCK) {
#pragma unroll
          for (int k = 0; k < 4; k++) back_pair(e[k], A);
        } else {
          back_pair(e[0], A);
#pragma unroll
          for (int k = 1; k < 4; k++)
            if (k * CW_ROW < m) back_pair(e[k], A);
        }
        w0 = w1;
        w1 = w2;
      }
      // CM3D's table underflow (k < 1) is counted per pair; the walk only
      // tracks the smallest distance and LJ table coordinate, and an atom
      // with an underflow (none in a sane system) is walked again to count
      // them
      if (__any_sync(0xffffffffu, (HAS_EL && A.r2min < P.r2under) || (LJM && A.pminl < 1.f))) {
        unsigned cnt = 0;
        for (int b = 0; b < nbt; b++) {
          const uint2 w = __ldg(words + b * CW_ROW);
          const uint32_t e[4] = {w.x & 0xFFFFu, w.x >> 16, w.y & 0xFFFFu, w.y >> 16};
          const bool front = b < nba;
#pragma unroll
          for (int k = 0; k < 4; k++) {
            float4 xj;
            float dx, dy, dz;
            const float r2 = geom(e[k], xj, dx, dy, dz);
            const bool el = HAS_EL && (!front || (e[k] & CW_EL));
            cnt += (el && r2 < P.rc2_el && fmaf(r2, P.dx2c, -P.offc) < 1.f) ? 1u : 0u;
            if (front && LJM) {
              CwAcc B;
              cw_zero(B);
              lj_pair(e[k], dx, dy, dz, r2, B);
              cnt += B.pminl < 1.f ? 1u : 0u;
            }
          }
        }
        under += cnt;
      }
      // forces: F_i = -(qi sum qj f d + sum f_lj d), the chunk in FP64 and
      // summed over the atom's lanes
      // (a transposing reduction: after the first two levels each lane
      // carries one component, lanes 0-7 x, 8-15 y, 16-23 z)
      const double qi = (double)xi.w;
      const double Fx = -(qi * (double)A.fx + (double)A.gx);
      const double Fy = -(qi * (double)A.fy + (double)A.gy);
      const double Fz = -(qi * (double)A.fz + (double)A.gz);
      const bool up = (lane & 16) != 0, odd = (lane & 8) != 0;
      const double k0 = (up ? Fz : Fx) + __shfl_xor_sync(0xffffffffu, up ? Fx : Fz, 16);
      const double k1 = (up ? 0.0 : Fy) + __shfl_xor_sync(0xffffffffu, up ? Fy : 0.0, 16);
      double Fc = (odd ? k1 : k0) + __shfl_xor_sync(0xffffffffu, odd ? k0 : k1, 8);
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) Fc += __shfl_xor_sync(0xffffffffu, Fc, o);
      if ((lane & 7) == 0 && lane < 24) {
        const int comp = lane >> 3;                   // 0 x, 1 y, 2 z
        fout[(size_t)comp * P.n + sorig[t]] += Fc;
      }
      // the atom's 16 quantities (CQ_* order) over the warp: three
      // transposing FP32 levels (8 lanes' chunks, about 160 pairs, then each
      // lane carries two quantities), FP64 for the last two levels, so lane
      // pair (2q, 2q + 1) ends with quantity q's atom total
      {
        const float qf = xi.w;
        float v[16] = {qf * A.eel, 0.f, qf * A.ve[0], qf * A.ve[1], qf * A.ve[2], qf * A.ve[3], qf * A.ve[4],
                       qf * A.ve[5], A.elo, A.vsh, A.vl[0], A.vl[1], A.vl[2], A.vl[3], A.vl[4], A.vl[5]};
#pragma unroll
        for (int h = 8, o = 16; h >= 2; h >>= 1, o >>= 1) {
          const bool hi = (lane & o) != 0;
#pragma unroll
          for (int i = 0; i < h; i++) {
            const float snd = hi ? v[i] : v[i + h];
            const float kp = hi ? v[i + h] : v[i];
            v[i] = kp + __shfl_xor_sync(0xffffffffu, snd, o);
          }
        }
        const bool b1 = (lane & 2) != 0;
        const double d0 = (double)v[0], d1 = (double)v[1];
        double dq = (b1 ? d1 : d0) + __shfl_xor_sync(0xffffffffu, b1 ? d0 : d1, 2);
        dq += __shfl_xor_sync(0xffffffffu, dq, 1);
        Eq += dq;
        Ehi += A.elj_hi;
      }
    }
    // the item's sums: warps, then the block, in a fixed order
    {
      const double hi = warp_sum(Ehi);
      if ((lane & 1) == 0) s_red[warp][lane >> 1] = Eq + ((lane >> 1) == CQ_ELJ ? hi : 0.0);
    }
    __syncthreads();
    if (threadIdx.x < CQ_COUNT) {
      double s = 0.0;
      for (int w = 0; w < NWARP; w++) s += s_red[w][threadIdx.x];
      ipart[(size_t)(item0 + item) * CQ_COUNT + threadIdx.x] = s;
    }
  }
  if (lane == 0 && under) atomicAdd((unsigned long long *)(stat + ST_UNDERFLOW), under);
}

// ------------------------------------------------------------------
// Pair kernel for small cells (k_pair_cs): boxes whose cells hold a few
// tens of atoms, as in a batch of small LJ boxes.  There a block per cell
// spends most of its time staging the window and waiting for it, and a
// warp per atom leaves most lanes idle on lists of ~70 entries.  Here
//   * a block is NG groups of GW warps, each group working through
//     its own items (cells) with its own window, mbarrier and named
//     barrier, so one group's staging overlaps the others' pairs;
//   * an atom has CS_LPA = 8 lanes (four atoms per warp) and its compact
//     list comes in blocks of 32 entries (k_cw_convert with row 8: the
//     8-byte word of lane l of a block holds entries l, l + 8, l + 16,
//     l + 24), so a list of n entries pads to a multiple of 32, not 128;
//   * both segments go through one pair body (the segment is a per-lane
//     condition here), and every entry of a block is evaluated: padding
//     names the dummy slot, which contributes exact zeros.
// The sums are the same as k_pair_cw's: FP32 per lane and pair chunk, FP64
// across an atom's lanes (forces) and per lane, warp, group and item (the
// 16 energy/virial quantities), all in a fixed order.
constexpr int CS_LPA = CM3D_CS_LPA;         // lanes per atom (the list row)
constexpr int CS_BLOCK = 4 * CS_LPA;        // list entries per block
// a block: NG groups of GW warps, 512 threads -- 4 x 4 where the tables
// leave room for four windows only, else 8 x 2 (more cells in flight, fewer
// idle atom slots on cells of ~20 atoms)
constexpr int CS_NG = 4, CS_GW = 4;
constexpr int CS_NG_WIDE = 8, CS_GW_WIDE = 2;
static_assert(CS_NG * CS_GW * 32 == CM3D_CS_THREADS && CS_NG_WIDE * CS_GW_WIDE * 32 == CM3D_CS_THREADS,
              "k_pair_cs block size");
constexpr int CS_STATIC_SMEM = 16384;       // >= k_pair_cs's static shared arrays
constexpr int CS_RF = 4;                    // erfc table copies (four groups' windows need the room)
constexpr int CS_RG = 4;

__device__ __forceinline__ void group_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
// group barrier that also returns whether `p` holds in every thread of it
__device__ __forceinline__ bool group_and(int id, int nthreads, bool p) {
  unsigned r;
  asm volatile(
      "{\n .reg .pred a, b;\n setp.ne.u32 a, %1, 0;\n bar.red.and.pred b, %2, %3, a;\n selp.u32 %0, 1, 0, b;\n}"
      : "=r"(r)
      : "r"((unsigned)p), "r"(id), "r"(nthreads)
      : "memory");
  return r != 0;
}

template <bool HAS_EL, int LJM, bool BATCH, int NG = CS_NG, int GW = CS_GW>
__global__ void __launch_bounds__(NG *GW * 32, 1) k_pair_cs(
    CwP P, const float4 *__restrict__ xq, const int *__restrict__ styp, const int *__restrict__ sorig,
    const int *__restrict__ cell_start, const int2 *__restrict__ cwn, const uint2 *__restrict__ cwl,
    const float4 *__restrict__ gshift, const int *__restrict__ gmap, const float *__restrict__ gfcut,
    const float4 *__restrict__ gtf, const float2 *__restrict__ gtg, const float4 *__restrict__ gtl,
    double *__restrict__ fout, double *__restrict__ ipart, long long *__restrict__ stat,
    const int *__restrict__ gs, const int4 *__restrict__ items = nullptr, const SysP *__restrict__ sp = nullptr,
    int item0 = 0) {
  if (gated_off(gs, 0)) return;
  extern __shared__ float4 sm[];
  // tables (as k_pair_cw), then NG windows of cap + 1 slots, then (LJM 2)
  // NG type arrays
  float4 *tf = sm;
  float2 *tg = reinterpret_cast<float2 *>(tf + (HAS_EL ? P.ntable * CS_RF : 0));
  float4 *tl = reinterpret_cast<float4 *>(tg + (HAS_EL ? P.ntable * CS_RG : 0));
  const int nl = LJM ? 2 * P.ninter * P.ntable : 0;
  constexpr int GT = GW * 32;                     // threads per group
  const int g = threadIdx.x / GT, gt = threadIdx.x % GT, gw = gt >> 5;
  const int lane = threadIdx.x & 31, l8 = lane & (CS_LPA - 1), sub = lane / CS_LPA;
  const int bar_id = 1 + g;
  float4 *wx = tl + nl + (size_t)g * (P.cap + 1);
  unsigned char *wt = reinterpret_cast<unsigned char *>(tl + nl + (size_t)NG * (P.cap + 1)) + (size_t)g * (P.cap + 1);
  __shared__ int s_cs[NG][27], s_off[NG][28];
  __shared__ float4 s_shift[BATCH ? NG : 1][54];
  __shared__ int s_map[256];
  __shared__ float4 s_cut[64];
  __shared__ double s_red[NG][GW][CQ_COUNT];
  __shared__ __align__(8) unsigned long long s_mbar[NG];
  static_assert(CQ_COUNT == 2 * CS_LPA, "the transposing reduction gives lane l quantities 2l and 2l + 1");

  if (!BATCH)
    for (int k = threadIdx.x; k < 54; k += blockDim.x) s_shift[0][k] = gshift[k];
  if (HAS_EL) {
    for (int k = threadIdx.x; k < P.ntable * CS_RF; k += blockDim.x) tf[k] = gtf[k / CS_RF];
    for (int k = threadIdx.x; k < P.ntable * CS_RG; k += blockDim.x) tg[k] = gtg[k / CS_RG];
  }
  for (int k = threadIdx.x; k < nl; k += blockDim.x) tl[k] = gtl[k];
  if (LJM == 2) {
    for (int k = threadIdx.x; k < P.ntypes * P.ntypes; k += blockDim.x) {
      const int in = gmap[P.map0 + k];
      s_map[k] = in >= 0 ? in - P.inter0 : -1;
    }
    for (int k = threadIdx.x; k < P.ninter; k += blockDim.x) {
      const float *f = gfcut + 8 * (P.inter0 + k);
      s_cut[k] = make_float4(f[0], f[2], f[1], f[3]);
    }
  }
  const unsigned bar = (unsigned)__cvta_generic_to_shared(&s_mbar[g]);
  unsigned phase = 0;
  if (gt == 0) {
    wx[P.cap] = make_float4(1.0e6f, 1.0e6f, 1.0e6f, 0.f);   // the dummy entry's partner: out of range
    if (LJM == 2) wt[P.cap] = 0;
    mbar_init(bar);
  }
  __syncthreads();
  const unsigned tfb = (unsigned)__cvta_generic_to_shared(tf + (lane & (CS_RF - 1))) -
                       CW_MAGIC_BITS * (unsigned)(CS_RF * sizeof(float4));
  const unsigned tgb = (unsigned)__cvta_generic_to_shared(tg + (lane & (CS_RG - 1))) -
                       CW_MAGIC_BITS * (unsigned)(CS_RG * sizeof(float2));
  const unsigned wxb = (unsigned)__cvta_generic_to_shared(wx);
  const float4 *shift = s_shift[BATCH ? g : 0];
  unsigned long long under = 0;

  for (int item = blockIdx.x * NG + g; item < P.nitems; item += gridDim.x * NG) {
    int c, ncx = P.ncx, ncy = P.ncy, ncz = P.ncz, c0 = 0, sys = 0;
    if (BATCH) {
      const int4 it = items[item];
      sys = it.x;
      c = it.y;
      ncx = sp[sys].nc[0];
      ncy = sp[sys].nc[1];
      ncz = sp[sys].nc[2];
      c0 = sp[sys].c0;
    } else {
      c = item;
    }
    const int cz = c % ncz, cy = (c / ncz) % ncy, cx = c / (ncz * ncy);
    group_sync(bar_id, GT);                                    // the previous window is no longer read
    if (BATCH)
      for (int k = gt; k < 54; k += GT)
        s_shift[g][k] = k < 27 ? sp[sys].shift[k] : sp[sys].shift_lo[k - 27];
    if (gw == 0) {
      int cnt = 0, cs = 0;
      if (lane < 27) {
        int jx = cx - (lane / 9 - 1), jy = cy - ((lane / 3) % 3 - 1), jz = cz - (lane % 3 - 1);
        jx = jx < 0 ? jx + ncx : (jx >= ncx ? jx - ncx : jx);
        jy = jy < 0 ? jy + ncy : (jy >= ncy ? jy - ncy : jy);
        jz = jz < 0 ? jz + ncz : (jz >= ncz ? jz - ncz : jz);
        const int jc = c0 + (jx * ncy + jy) * ncz + jz;
        cs = cell_start[jc];
        cnt = cell_start[jc + 1] - cs;
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      if (lane < 27) {
        s_cs[g][lane] = cs;
        s_off[g][lane] = incl - cnt;
      }
      if (lane == 26) s_off[g][27] = incl;
    }
    group_sync(bar_id, GT);
    const int tot = s_off[g][27];
    const bool staged = tot <= P.cap;
    if (staged) {
      if (gw == 0) {
        fence_async_smem();
        if (lane == 0) mbar_expect(bar, (unsigned)tot * (unsigned)sizeof(float4));
        __syncwarp();
        if (lane < 27) {
          const int cnt = s_off[g][lane + 1] - s_off[g][lane];
          if (cnt > 0)
            bulk_g2s(wxb + (unsigned)s_off[g][lane] * (unsigned)sizeof(float4), xq + s_cs[g][lane],
                     (unsigned)cnt * (unsigned)sizeof(float4), bar);
        }
      }
      const bool arrived = mbar_wait(bar, phase, CW_WAIT_LIMIT);
      phase ^= 1u;
      if (!group_and(bar_id, GT, arrived)) {
        // the copies did not complete (never seen): count it, wait once
        // more for copies still in flight, and leave the group's remaining
        // items undone; the host reads the count in the status
        if (gt == 0) atomicAdd((unsigned long long *)(stat + ST_STAGE_TIMEOUT), 1ull);
        mbar_wait(bar, phase ^ 1u, CW_WAIT_LIMIT);
        break;
      }
      for (int w = gw; w < 27; w += GW) {
        const float4 sh = shift[w], shl = shift[27 + w];
        const int g0 = s_off[g][w], g1 = s_off[g][w + 1], u0 = s_cs[g][w] - g0;
        for (int k = g0 + lane; k < g1; k += 32) {
          const float4 x = wx[k];
          wx[k] = make_float4((x.x - sh.x) - shl.x, (x.y - sh.y) - shl.y, (x.z - sh.z) - shl.z, x.w);
          if (LJM == 2) wt[k] = (unsigned char)styp[u0 + k];
        }
      }
    }
    group_sync(bar_id, GT);
    // lane l8 of an atom keeps quantities 2 l8 and 2 l8 + 1 of CQ_* in FP64
    double Eq0 = 0.0, Eq1 = 0.0, Ehi = 0.0;
    const int ci0 = s_cs[g][13], cin = staged ? s_off[g][14] - s_off[g][13] : 0, ioff = s_off[g][13];
    const uint32_t dm = (uint32_t)P.cap | ((uint32_t)P.cap << 16);
    const uint2 pad = make_uint2(dm, dm);
    // the group's 4 GW atom slots (warp gw, quarter sub) over the cell's atoms
    for (int a0 = 0; a0 < cin; a0 += GW * 4) {
      const int a = a0 + gw * 4 + sub;
      const bool act = a < cin;
      const int t = ci0 + (act ? a : 0);
      const uint2 *words = cwl + (size_t)t * P.words + l8;
      // the lengths, the first two blocks' words (every slot holds at least
      // two blocks) and the atom's original index, all in flight together
      const int2 nn = act ? cwn[t] : make_int2(0, 0);
      uint2 w0 = __ldg(words);
      uint2 w1 = __ldg(words + CS_LPA);
      const int io = sorig[t];
      const int nba = (nn.x + CS_BLOCK - 1) / CS_BLOCK, nbt = nba + (nn.y + CS_BLOCK - 1) / CS_BLOCK;
      const int nbw = __reduce_max_sync(0xffffffffu, nbt);
      if (nbt < 1) w0 = pad;
      if (nbt < 2) w1 = pad;
      // an idle quarter sits far from every staged atom: its sums stay zero
      const float4 xi = act ? wx[ioff + a] : make_float4(-1.0e6f, -1.0e6f, -1.0e6f, 0.f);
      const int ti = LJM == 2 && act ? wt[ioff + a] : 0;
      CwAcc A;
      cw_zero(A);
      auto geom = [&](uint32_t e, float4 &xj, float &dx, float &dy, float &dz) {
        xj = lds_f4(wxb + ((e & CW_IDX) << 4));
        dx = xi.x - xj.x;
        dy = xi.y - xj.y;
        dz = xi.z - xj.z;
        return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      };
      auto lj_pair = [&](uint32_t e, float dx, float dy, float dz, float r2, CwAcc &Acc) {
        if (LJM == 1) {
          cw_lj(P, dx, dy, dz, r2, P.rc2_l, P.dx2l, P.offl, P.vtl, tl, Acc);
        } else if (LJM == 2) {
          const int tj = wt[e & CW_IDX];
          const int in = s_map[ti * P.ntypes + tj];
          const float4 cut = s_cut[in < 0 ? 0 : in];
          cw_lj(P, dx, dy, dz, in < 0 ? 3.0e38f : r2, cut.x, cut.y, cut.z, cut.w,
                tl + (size_t)2 * (in < 0 ? 0 : in) * P.ntable, Acc);
        }
      };
      // one entry: the front segment (LJ list; electrostatics where the te
      // flag is set) or the back segment (electrostatics only)
      auto pair = [&](uint32_t e, bool front, CwAcc &Acc) {
        float4 xj;
        float dx, dy, dz;
        const float r2 = geom(e, xj, dx, dy, dz);
        if (HAS_EL) {
          const bool el = !front || (e & CW_EL);
          cw_elec<CS_RF, CS_RG>(P, el ? xj.w : 0.f, dx, dy, dz, el ? r2 : 3.0e38f, tfb, tgb, Acc);
        }
        if (LJM) lj_pair(e, dx, dy, dz, front ? r2 : 3.0e38f, Acc);
      };
      for (int b = 0; b < nbw; b++) {
        const uint2 w2 = b + 2 < nbt ? __ldg(words + (b + 2) * CS_LPA) : pad;
        const bool front = b < nba;
        pair(w0.x & 0xFFFFu, front, A);
        pair(w0.x >> 16, front, A);
        pair(w0.y & 0xFFFFu, front, A);
        pair(w0.y >> 16, front, A);
        w0 = w1;
        w1 = w2;
      }
      // CM3D's table underflow (k < 1), counted per pair: an atom whose
      // smallest distance or LJ coordinate says it has some is walked again
      if (__any_sync(0xffffffffu, (HAS_EL && A.r2min < P.r2under) || (LJM && A.pminl < 1.f))) {
        unsigned cnt = 0;
        for (int b = 0; b < nbw; b++) {
          const uint2 w = b < nbt ? __ldg(words + b * CS_LPA) : pad;
          const uint32_t e[4] = {w.x & 0xFFFFu, w.x >> 16, w.y & 0xFFFFu, w.y >> 16};
          const bool front = b < nba;
#pragma unroll
          for (int k = 0; k < 4; k++) {
            float4 xj;
            float dx, dy, dz;
            const float r2 = geom(e[k], xj, dx, dy, dz);
            const bool el = HAS_EL && (!front || (e[k] & CW_EL));
            cnt += (el && r2 < P.rc2_el && fmaf(r2, P.dx2c, -P.offc) < 1.f) ? 1u : 0u;
            if (front && LJM) {
              CwAcc B;
              cw_zero(B);
              lj_pair(e[k], dx, dy, dz, r2, B);
              cnt += B.pminl < 1.f ? 1u : 0u;
            }
          }
        }
        under += cnt;
      }
      // forces: F_i = -(qi sum qj f d + sum f_lj d), each lane's chunk in
      // FP64, summed over the atom's 8 lanes
      const double qi = (double)xi.w;
      double Fx = -(qi * (double)A.fx + (double)A.gx);
      double Fy = -(qi * (double)A.fy + (double)A.gy);
      double Fz = -(qi * (double)A.fz + (double)A.gz);
#pragma unroll
      for (int o = CS_LPA / 2; o > 0; o >>= 1) {
        Fx += __shfl_xor_sync(0xffffffffu, Fx, o);
        Fy += __shfl_xor_sync(0xffffffffu, Fy, o);
        Fz += __shfl_xor_sync(0xffffffffu, Fz, o);
      }
      if (act && l8 < 3) {
        // the only addition to this element in the launch, so the result
        // does not depend on timing; a reduction needs no round trip
        const double Fc = l8 == 0 ? Fx : (l8 == 1 ? Fy : Fz);
        atomicAdd(fout + (size_t)l8 * P.n + io, Fc);
      }
      // the atom's 16 quantities over its 8 lanes: three transposing FP32
      // levels leave lane l8 with quantities 2 l8 and 2 l8 + 1
      {
        const float qf = xi.w;
        float v[16] = {qf * A.eel, 0.f, qf * A.ve[0], qf * A.ve[1], qf * A.ve[2], qf * A.ve[3], qf * A.ve[4],
                       qf * A.ve[5], A.elo, A.vsh, A.vl[0], A.vl[1], A.vl[2], A.vl[3], A.vl[4], A.vl[5]};
#pragma unroll
        for (int h = 8, o = 4; h >= 2; h >>= 1, o >>= 1) {
          const bool hi = (lane & o) != 0;
#pragma unroll
          for (int i = 0; i < h; i++) {
            const float snd = hi ? v[i] : v[i + h];
            const float kp = hi ? v[i + h] : v[i];
            v[i] = kp + __shfl_xor_sync(0xffffffffu, snd, o);
          }
        }
        Eq0 += (double)v[0];
        Eq1 += (double)v[1];
        Ehi += A.elj_hi;
      }
    }
    // the item's sums: the four atom quarters of a warp, the group's warps,
    // in a fixed order
    {
      Eq0 += __shfl_xor_sync(0xffffffffu, Eq0, 8);
      Eq0 += __shfl_xor_sync(0xffffffffu, Eq0, 16);
      Eq1 += __shfl_xor_sync(0xffffffffu, Eq1, 8);
      Eq1 += __shfl_xor_sync(0xffffffffu, Eq1, 16);
      const double hi = warp_sum(Ehi);
      if (lane < CS_LPA) {
        s_red[g][gw][2 * lane] = Eq0 + (2 * lane == CQ_ELJ ? hi : 0.0);
        s_red[g][gw][2 * lane + 1] = Eq1 + (2 * lane + 1 == CQ_ELJ ? hi : 0.0);
      }
    }
    group_sync(bar_id, GT);
    if (gt < CQ_COUNT) {
      double s = 0.0;
      for (int w = 0; w < GW; w++) s += s_red[g][w][gt];
      ipart[(size_t)(item0 + item) * CQ_COUNT + gt] = s;
    }
  }
  if (lane == 0 && under) atomicAdd((unsigned long long *)(stat + ST_UNDERFLOW), under);
}

// Sum of the items' partials into CM3D's accumulators: one block, warp q
// sums quantity q over the items (fixed order), then one thread applies the
// sums in a fixed order (several quantities feed one accumulator); each pair
// was counted from both ends, hence 1/2.
__device__ void cw_apply(int mask, const double *v, double *acc) {
  if (mask & 2) {
    // (CM3D's shifted sum spothe, finter_e.c:197, is read by nothing --
    // getsvirter_e reports spote -- and this path does not form it)
    acc[ACC_SPOTE] += v[CQ_EEL];
    acc[ACC_SPRSE] -= v[CQ_VE0] + v[CQ_VE4] + v[CQ_VE8];
    acc[ACC_SPRSET + 0] -= v[CQ_VE0];
    acc[ACC_SPRSET + 1] -= v[CQ_VE1];
    acc[ACC_SPRSET + 2] -= v[CQ_VE2];
    acc[ACC_SPRSET + 4] -= v[CQ_VE4];
    acc[ACC_SPRSET + 5] -= v[CQ_VE5];
    acc[ACC_SPRSET + 8] -= v[CQ_VE8];
  }
  if (mask & 1) {
    acc[ACC_SPOTL] += v[CQ_ELJ];
    acc[ACC_SPOTHL] += v[CQ_ELJ] - v[CQ_VSH];
    acc[ACC_SPRSL] -= v[CQ_VL0] + v[CQ_VL4] + v[CQ_VL8];
    acc[ACC_SPRSLT + 0] -= v[CQ_VL0];
    acc[ACC_SPRSLT + 1] -= v[CQ_VL1];
    acc[ACC_SPRSLT + 2] -= v[CQ_VL2];
    acc[ACC_SPRSLT + 4] -= v[CQ_VL4];
    acc[ACC_SPRSLT + 5] -= v[CQ_VL5];
    acc[ACC_SPRSLT + 8] -= v[CQ_VL8];
  }
}

__global__ void __launch_bounds__(CQ_COUNT * 32) k_cw_ereduce(int nitems, int mask, double tablast_e,
                                                               const double *__restrict__ ipart,
                                                               double *__restrict__ acc, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  __shared__ double s_q[CQ_COUNT];
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double s = 0.0;
  for (int it = lane; it < nitems; it += 32) s += ipart[(size_t)it * CQ_COUNT + q];
  s = warp_sum(s);
  if (lane == 0) s_q[q] = 0.5 * s;
  __syncthreads();
  if (threadIdx.x == 0) cw_apply(mask, s_q, acc);
}

// The same for a batch's compact systems: block per system, its items
// {first, count} (none: a gather-kernel system, nothing to do), its own
// accumulators; LJ sums where it has LJ interactions, electrostatic ones
// where it has charges.
__global__ void __launch_bounds__(CQ_COUNT * 32) k_cw_ereduce_sys(int mask, const int2 *__restrict__ sitems,
                                                                   const SysP *__restrict__ sp,
                                                                   const double *__restrict__ ipart,
                                                                   double *__restrict__ acc,
                                                                   const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  const int sy = blockIdx.x;
  const int2 r = sitems[sy];
  if (r.y == 0) return;
  __shared__ double s_q[CQ_COUNT];
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double s = 0.0;
  for (int it = lane; it < r.y; it += 32) s += ipart[(size_t)(r.x + it) * CQ_COUNT + q];
  s = warp_sum(s);
  if (lane == 0) s_q[q] = 0.5 * s;
  __syncthreads();
  if (threadIdx.x == 0) {
    const int m = mask & ((sp[sy].ninter > 0 ? 1 : 0) | (sp[sy].coul >= 0 ? 2 : 0));
    cw_apply(m, s_q, acc + (size_t)sy * ACC_STRIDE);
  }
}

// ------------------------------------------------------------------ host
static int cw_ljm_of(int ninter) { return ninter == 0 ? 0 : (ninter == 1 ? 1 : 2); }

static size_t cw_table_bytes(bool el, int ljm, int ninter, int ntable, int rf = CW_RF, int rg = CW_RG) {
  size_t b = 0;
  if (el) b += (size_t)ntable * (rf * sizeof(float4) + rg * sizeof(float2));
  if (ljm) b += (size_t)2 * ninter * ntable * sizeof(float4);
  return b;
}

// The compact tables of one system: erfc force coefficients + base energy
// and energy slope/curvature (knot 0: CM3D's clamp below the table, the
// value at knot 1 with no slope; knots ntable - 3 and up: zeros, which the
// saturated coordinate of a pair at or beyond the cut-off reads); LJ 2 float4
// per knot {d0, dA, dB, v0 hi} {vA, vB, v0 lo, -} for its interactions.
static void cw_build_tables(int nt, const double *ct, const double *dct, const double *vt, const double *dv,
                            int ninter, std::vector<float4> &tf, std::vector<float2> &tg, std::vector<float4> &tl) {
  tf.clear();
  tg.clear();
  tl.clear();
  if (ct) {
    tf.assign(nt, make_float4(0.f, 0.f, 0.f, 0.f));
    tg.assign(nt, make_float2(0.f, 0.f));
    tf[0] = make_float4((float)dct[1], 0.f, 0.f, (float)ct[1]);
    for (int k = 1; k <= nt - 4; k++) {
      const double d0 = dct[k], da = 0.5 * (dct[k + 1] - dct[k - 1]),
                   db = 0.5 * (dct[k - 1] - 2.0 * dct[k] + dct[k + 1]);
      const double v0 = ct[k], va = 0.5 * (ct[k + 1] - ct[k - 1]), vb = 0.5 * (ct[k - 1] - 2.0 * ct[k] + ct[k + 1]);
      tf[k] = make_float4((float)d0, (float)da, (float)db, (float)v0);
      tg[k] = make_float2((float)va, (float)vb);
    }
  }
  tl.assign((size_t)2 * ninter * nt, make_float4(0.f, 0.f, 0.f, 0.f));
  for (int in = 0; in < ninter; in++)
    for (int k = 1; k <= nt - 2; k++) {
      const double *d = dv + (size_t)in * nt, *v = vt + (size_t)in * nt;
      const double d0 = d[k], da = 0.5 * (d[k + 1] - d[k - 1]), db = 0.5 * (d[k - 1] - 2.0 * d[k] + d[k + 1]);
      const double v0 = v[k], va = 0.5 * (v[k + 1] - v[k - 1]), vb = 0.5 * (v[k - 1] - 2.0 * v[k] + v[k + 1]);
      // v0 as hi + lo: the kernel sums the hi parts in FP64
      const float hi = (float)v0;
      tl[2 * ((size_t)in * nt + k)] = make_float4((float)d0, (float)da, (float)db, hi);
      tl[2 * ((size_t)in * nt + k) + 1] = make_float4((float)va, (float)vb, (float)(v0 - (double)hi), 0.f);
    }
}

// the erfc part of the pair parameters of a system with charges
static void cw_coul_params(CwP &P, int nt, double rmaxl_coul2, double dx2coul, double rmins_coul2) {
  P.rc2_el = (float)rmaxl_coul2;
  P.dx2c = (float)dx2coul;
  P.offc = (float)(rmins_coul2 * dx2coul);
  P.pmax = (float)(nt - 3);
  P.sat_a = (float)(dx2coul / (nt - 3));
  P.sat_b = (float)(-rmins_coul2 * dx2coul / (nt - 3));
  P.r2under = (float)(rmins_coul2 + 1.0 / dx2coul);
}

// the one-interaction LJ parameters from its 8 cut-off doubles (icut)
static void cw_lj1_params(CwP &P, const double *q) {
  P.rc2_l = (float)q[2];          // rmaxl_cut2
  P.dx2l = (float)q[6];           // dx2tab
  P.offl = (float)(q[1] * q[6]);  // rmins_cut2 * dx2tab
  P.vtl = (float)q[7];            // vtab[ntable - 4]
}

// A group of a batch's compact systems: the same tables and parameters.
struct CwGroup {
  bool el = false;
  int ljm = 0;
  CwP P;                   // parameters; nitems = the group's items
  int item0 = 0;           // first item (global item index)
  size_t smem = 0;         // k_pair_cw's dynamic shared memory
  size_t smem8 = 0;        // k_pair_cs's (0: its windows do not fit)
  int ng8 = 0;             // k_pair_cs's groups per block (CS_NG or CS_NG_WIDE)
  size_t tf0 = 0, tl0 = 0; // offsets of its tables in cw_tf / cw_tg (knots) and cw_tl (float4)
  std::string key;         // tables + parameters, byte for byte
};

static std::vector<CwGroup> &cw_groups(Ctx *c) { return *reinterpret_cast<std::vector<CwGroup> *>(c->cw_grp); }

void cw_destroy(Ctx *c) {
  delete reinterpret_cast<std::vector<CwGroup> *>(c->cw_grp);
  c->cw_grp = nullptr;
}

static bool cw_env_off() {
  const char *pk = getenv("CM3D_NB_PAIR_KERNEL");
  return pk && (strcmp(pk, "list") == 0 || strcmp(pk, "window") == 0);
}

// CM3D_NB_CW_CAP lowers the window capacity (tests of the fall-back)
static long long cw_env_cap(long long cap) {
  const char *ce = getenv("CM3D_NB_CW_CAP");
  if (ce && atoi(ce) > 0) cap = std::min<long long>(cap, atoi(ce));
  return cap;
}

// the compact list's 8-byte words per atom slot: each segment rounded up to
// whole blocks of 4 row entries (row lanes per atom: 32 or 8)
static int cw_words_row(long long stride, int row) {
  return (int)(((stride + 4 * row - 1) / (4 * row) + 1) * row);
}
// room for either layout, so that the autotuner can switch without
// reallocating
static int cw_words_for(long long stride) {
  return std::max(cw_words_row(stride, CW_ROW), cw_words_row(stride, CS_LPA));
}

static int cw_setup_batch(Ctx *c);

// Whether the compact path can run this context, and its tables and window
// size: one system with at least 3 cells per axis (a batch: cw_setup_batch),
// the full force level without the RESPA switch copy, a window of the mean
// size (x 1.25, + 64) next to the tables in the shared memory a block may use.
int cw_setup(Ctx *c) {
  c->cw_ok = 0;
  if (c->mode != CM3D_NB_MIXED) return CM3D_NB_OK;
  if (c->need_short || c->nres_lrf > 1) return CM3D_NB_OK;
  if (cw_env_off()) return CM3D_NB_OK;
  if (c->nsys > 1) return cw_setup_batch(c);
  if (c->nc[0] < 3 || c->nc[1] < 3 || c->nc[2] < 3) return CM3D_NB_OK;
  if (c->ntypes > 16 || c->ninter > 64) return CM3D_NB_OK;       // static map / cut-off arrays
  const int ljm = cw_ljm_of(c->ninter);
  const bool el = c->ncharge > 0;
  const double mean_window = 27.0 * (double)c->n / (double)c->ncells;
  const size_t want_cap = (size_t)(1.25 * mean_window) + 64;
  const size_t budget = c->smem_optin > CW_STATIC_SMEM ? c->smem_optin - CW_STATIC_SMEM : 0;
  const size_t per_slot = sizeof(float4) + (ljm == 2 ? 1 : 0);
  const size_t tb = cw_table_bytes(el, ljm, c->ninter, c->ntable);
  if (tb + (want_cap + 1) * per_slot + 16 > budget) return CM3D_NB_OK;
  long long cap = (long long)((budget - tb - 16) / per_slot) - 1;
  cap = cw_env_cap(std::min<long long>(cap, CW_MAX_CAP));
  c->cw_cap = c->cw_cap32 = (int)cap;
  c->cw_row = CW_ROW;
  c->cw_smem = tb + ((size_t)cap + 1) * sizeof(float4) + (ljm == 2 ? (size_t)cap + 1 : 0);
  c->cw_smem = (c->cw_smem + 15) / 16 * 16;
  c->cw_words = cw_words_for(c->nbr_stride);
  CK(cudaMalloc(&c->cwl, sizeof(uint2) * (size_t)c->n * (size_t)c->cw_words));
  CK(cudaMalloc(&c->cwn, sizeof(int2) * (size_t)c->n));
  CK(cudaMemset(c->cwn, 0, sizeof(int2) * (size_t)c->n));
  const int nt = c->ntable;
  std::vector<double> ct, dct, vt, dv, cut;
  if (el) {
    ct.resize(nt);
    dct.resize(nt);
    CK(cudaMemcpy(ct.data(), c->coultab, sizeof(double) * nt, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dct.data(), c->dcoultab, sizeof(double) * nt, cudaMemcpyDeviceToHost));
  }
  if (ljm) {
    vt.resize((size_t)c->ninter * nt);
    dv.resize(vt.size());
    cut.resize(8 * (size_t)c->ninter);
    CK(cudaMemcpy(vt.data(), c->vtab, sizeof(double) * vt.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dv.data(), c->dvtab, sizeof(double) * dv.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(cut.data(), c->icut, sizeof(double) * cut.size(), cudaMemcpyDeviceToHost));
  }
  std::vector<float4> tf, tl;
  std::vector<float2> tg;
  cw_build_tables(nt, el ? ct.data() : nullptr, el ? dct.data() : nullptr, vt.data(), dv.data(), ljm ? c->ninter : 0,
                  tf, tg, tl);
  if (el) {
    CK(cudaMalloc(&c->cw_tf, sizeof(float4) * nt));
    CK(cudaMalloc(&c->cw_tg, sizeof(float2) * nt));
    CK(cudaMemcpy(c->cw_tf, tf.data(), sizeof(float4) * nt, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->cw_tg, tg.data(), sizeof(float2) * nt, cudaMemcpyHostToDevice));
  }
  if (ljm) {
    CK(cudaMalloc(&c->cw_tl, sizeof(float4) * tl.size()));
    CK(cudaMemcpy(c->cw_tl, tl.data(), sizeof(float4) * tl.size(), cudaMemcpyHostToDevice));
    if (ljm == 1) {
      CwP q;
      cw_lj1_params(q, &cut[0]);
      c->cw_lj1[0] = q.rc2_l;
      c->cw_lj1[1] = q.dx2l;
      c->cw_lj1[2] = q.offl;
      c->cw_lj1[3] = q.vtl;
    }
  }
  // work items: cells, split into parts where the cells are fewer than four
  // per SM (each part stages its cell's window again); the autotuner may
  // choose another split (room for the largest)
  const int want = (4 * c->num_sms + c->ncells - 1) / c->ncells;
  CK(cudaMalloc(&c->cw_part, sizeof(double) * CQ_COUNT * (size_t)c->ncells * CW_MAX_SPLIT));
  cw_set_split(c, std::max(1, std::min(want, CW_MAX_SPLIT)));
  c->cw_ok = 1;
  c->cw_use = 1;
  return CM3D_NB_OK;
}

// A batch: every system with at least 3 cells per axis (and at most 16 atom
// types and 64 interactions) runs in the compact kernel; the systems whose
// tables and pair parameters agree byte for byte form a group, one launch
// each with the group's tables staged once per block; the other systems run
// in the gather kernel.  Items: one per cell, in system order within a group.
static int cw_setup_batch(Ctx *c) {
  const int nt = c->ntable, nsys = c->nsys;
  std::vector<double> ct, dct, vt((size_t)c->ninter * nt), dv(vt.size()), cut(8 * (size_t)c->ninter);
  if (c->ninter > 0) {
    CK(cudaMemcpy(vt.data(), c->vtab, sizeof(double) * vt.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dv.data(), c->dvtab, sizeof(double) * dv.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(cut.data(), c->icut, sizeof(double) * cut.size(), cudaMemcpyDeviceToHost));
  }
  if (c->ncoul > 0) {
    ct.resize((size_t)c->ncoul * nt);
    dct.resize(ct.size());
    CK(cudaMemcpy(ct.data(), c->coultab, sizeof(double) * ct.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dct.data(), c->dcoultab, sizeof(double) * dct.size(), cudaMemcpyDeviceToHost));
  }
  size_t nmap = 0;
  for (int s = 0; s < nsys; s++) nmap = std::max(nmap, (size_t)(c->h_sp[s].map0 + c->h_sp[s].ntypes * c->h_sp[s].ntypes));
  std::vector<int> gmap(nmap > 0 ? nmap : 1);
  if (nmap) CK(cudaMemcpy(gmap.data(), c->map, sizeof(int) * nmap, cudaMemcpyDeviceToHost));

  auto *groups = new std::vector<CwGroup>();
  c->cw_grp = groups;
  std::vector<int> gid(nsys, -1), cwsys(nsys, 0);
  std::vector<std::vector<float4>> gtf, gtl;
  std::vector<std::vector<float2>> gtg;
  double want_window = 0.0;
  for (int s = 0; s < nsys; s++) {
    const SysP &S = c->h_sp[s];
    const SysH &H = c->hs[s];
    if (S.nc[0] < 3 || S.nc[1] < 3 || S.nc[2] < 3) continue;
    if (S.ntypes > 16 || S.ninter > 64) continue;
    const bool el = S.coul >= 0;
    const int ljm = cw_ljm_of(S.ninter);
    if (!el && !ljm) continue;
    std::vector<float4> tf, tl;
    std::vector<float2> tg;
    cw_build_tables(nt, el ? &ct[(size_t)S.coul * nt] : nullptr, el ? &dct[(size_t)S.coul * nt] : nullptr,
                    S.ninter ? &vt[(size_t)S.inter0 * nt] : nullptr, S.ninter ? &dv[(size_t)S.inter0 * nt] : nullptr,
                    S.ninter, tf, tg, tl);
    CwP P;
    memset(&P, 0, sizeof P);
    P.ntable = nt;
    P.ntypes = S.ntypes;
    P.ninter = S.ninter;
    P.pmax = (float)(nt - 3);
    if (el) cw_coul_params(P, nt, H.rmaxl_coul2, H.dx2coul, H.rmins_coul2);
    if (ljm == 1) cw_lj1_params(P, &cut[8 * (size_t)S.inter0]);
    // the group key: everything the kernel reads besides the geometry
    std::string key;
    auto put = [&](const void *p, size_t b) { key.append(reinterpret_cast<const char *>(p), b); };
    const int hdr[4] = {el ? 1 : 0, ljm, S.ntypes, S.ninter};
    put(hdr, sizeof hdr);
    const float prm[11] = {P.rc2_el, P.dx2c, P.offc, P.pmax, P.sat_a, P.sat_b, P.r2under, P.rc2_l, P.dx2l, P.offl, P.vtl};
    put(prm, sizeof prm);
    put(tf.data(), sizeof(float4) * tf.size());
    put(tg.data(), sizeof(float2) * tg.size());
    put(tl.data(), sizeof(float4) * tl.size());
    for (int k = 0; k < S.ntypes * S.ntypes; k++) {
      const int in = gmap[S.map0 + k];
      const int loc = in >= 0 ? in - S.inter0 : -1;
      put(&loc, sizeof loc);
    }
    for (int k = 0; k < S.ninter; k++) {
      const double *q = &cut[8 * ((size_t)S.inter0 + k)];
      const float f4[4] = {(float)q[0], (float)q[2], (float)q[1], (float)q[3]};
      put(f4, sizeof f4);
    }
    int g = -1;
    for (size_t k = 0; k < groups->size(); k++)
      if ((*groups)[k].key == key) g = (int)k;
    if (g < 0) {
      CwGroup G;
      G.el = el;
      G.ljm = ljm;
      P.map0 = S.map0;
      P.inter0 = S.inter0;
      G.P = P;
      G.key = key;
      groups->push_back(G);
      gtf.push_back(tf);
      gtg.push_back(tg);
      gtl.push_back(tl);
      g = (int)groups->size() - 1;
    }
    gid[s] = g;
    cwsys[s] = 1;
    want_window = std::max(want_window, 27.0 * (double)S.n / (double)S.ncells);
  }
  if (groups->empty()) return CM3D_NB_OK;
  // one window capacity for all groups: what shared memory leaves next to
  // the largest tables, and at least the largest mean window x 1.25 + 64
  const size_t budget = c->smem_optin > CW_STATIC_SMEM ? c->smem_optin - CW_STATIC_SMEM : 0;
  long long cap = CW_MAX_CAP;
  for (const CwGroup &G : *groups) {
    const size_t tb = cw_table_bytes(G.el, G.ljm, G.P.ninter, nt);
    const size_t per_slot = sizeof(float4) + (G.ljm == 2 ? 1 : 0);
    const long long room = budget > tb + 16 ? (long long)((budget - tb - 16) / per_slot) - 1 : 0;
    cap = std::min(cap, room);
  }
  cap = cw_env_cap(cap);
  if ((double)cap < 1.25 * want_window + 64.0) {
    groups->clear();
    return CM3D_NB_OK;
  }
  c->cw_cap32 = (int)cap;
  // k_pair_cs: CS_NG windows per block next to the tables
  const size_t budget8 = c->smem_optin > CS_STATIC_SMEM ? c->smem_optin - CS_STATIC_SMEM : 0;
  long long cap8 = CW_MAX_CAP;
  for (const CwGroup &G : *groups) {
    const size_t tb = cw_table_bytes(G.el, G.ljm, G.P.ninter, nt, CS_RF, CS_RG);
    const size_t per_slot = sizeof(float4) + (G.ljm == 2 ? 1 : 0);
    const long long room = budget8 > tb + 16 * CS_NG ? (long long)((budget8 - tb - 16 * CS_NG) / (per_slot * CS_NG)) - 1 : 0;
    cap8 = std::min(cap8, room);
  }
  cap8 = cw_env_cap(cap8);
  c->cw_cap8 = (double)cap8 >= 1.25 * want_window + 64.0 ? (int)cap8 : 0;
  // the layout: 32 lanes per atom (a system runs as it does alone) until
  // the autotuner finds the 8-lane kernel faster (cells of a few tens of
  // atoms); CM3D_NB_CW_ROW=8 starts there
  c->cw_row = CW_ROW;
  if (const char *r = getenv("CM3D_NB_CW_ROW"))
    if (atoi(r) == CS_LPA && c->cw_cap8 > 0) c->cw_row = CS_LPA;
  c->cw_cap = c->cw_row == CS_LPA ? c->cw_cap8 : c->cw_cap32;
  // items by group, systems in order; tables back to back
  std::vector<int4> items;
  std::vector<int2> sitems(nsys, make_int2(0, 0));
  std::vector<float4> atf, atl;
  std::vector<float2> atg;
  for (size_t g = 0; g < groups->size(); g++) {
    CwGroup &G = (*groups)[g];
    G.item0 = (int)items.size();
    for (int s = 0; s < nsys; s++) {
      if (gid[s] != (int)g) continue;
      const SysP &S = c->h_sp[s];
      sitems[s] = make_int2((int)items.size(), S.ncells);
      for (int k = 0; k < S.ncells; k++) items.push_back(make_int4(s, k, 0, 1));
    }
    G.P.nitems = (int)items.size() - G.item0;
    G.P.nsplit = 1;
    G.tf0 = atf.size();
    G.tl0 = atl.size();
    atf.insert(atf.end(), gtf[g].begin(), gtf[g].end());
    atg.insert(atg.end(), gtg[g].begin(), gtg[g].end());
    atl.insert(atl.end(), gtl[g].begin(), gtl[g].end());
    const size_t tb = cw_table_bytes(G.el, G.ljm, G.P.ninter, nt);
    G.smem = (tb + ((size_t)c->cw_cap32 + 1) * sizeof(float4) + (G.ljm == 2 ? (size_t)c->cw_cap32 + 1 : 0) + 15) /
             16 * 16;
    if (c->cw_cap8 > 0) {
      // eight groups of two warps where their windows fit next to the
      // group's tables, else four of four
      const size_t tb8 = cw_table_bytes(G.el, G.ljm, G.P.ninter, nt, CS_RF, CS_RG);
      auto bytes = [&](int ng) {
        const size_t w8 = (size_t)ng * ((size_t)c->cw_cap8 + 1);
        return (tb8 + w8 * sizeof(float4) + (G.ljm == 2 ? w8 : 0) + 15) / 16 * 16;
      };
      G.ng8 = bytes(CS_NG_WIDE) <= budget8 ? CS_NG_WIDE : CS_NG;
      G.smem8 = bytes(G.ng8);
    }
  }
  // the gather kernel's atoms: the other systems' (a system's sorted
  // indices span its own atom range)
  std::vector<int> gidx;
  for (int s = 0; s < nsys; s++)
    if (!cwsys[s])
      for (int a = c->h_sp[s].a0; a < c->h_sp[s].a0 + c->h_sp[s].n; a++) gidx.push_back(a);
  c->cw_ng = (int)gidx.size();
  auto upload_v = [&](auto **dst, const auto &v) -> int {
    using T = typename std::remove_reference<decltype(v)>::type::value_type;
    CK(cudaMalloc((void **)dst, sizeof(T) * (v.empty() ? 1 : v.size())));
    if (!v.empty()) CK(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return CM3D_NB_OK;
  };
  int rc;
  if ((rc = upload_v(&c->cw_items, items)) || (rc = upload_v(&c->cw_sitems, sitems)) ||
      (rc = upload_v(&c->cw_sys, cwsys)) || (rc = upload_v(&c->cw_gidx, gidx)) || (rc = upload_v(&c->cw_tf, atf)) ||
      (rc = upload_v(&c->cw_scan, std::vector<int>(nsys + 1, 0))) ||
      (rc = upload_v(&c->cw_tg, atg)) || (rc = upload_v(&c->cw_tl, atl)))
    return rc;
  c->cw_words = cw_words_for(c->nbr_stride);
  CK(cudaMalloc(&c->cwl, sizeof(uint2) * (size_t)c->n * (size_t)c->cw_words));
  CK(cudaMalloc(&c->cwn, sizeof(int2) * (size_t)c->n));
  CK(cudaMemset(c->cwn, 0, sizeof(int2) * (size_t)c->n));
  c->cw_nitems = (int)items.size();
  c->cw_nsplit = 1;
  CK(cudaMalloc(&c->cw_part, sizeof(double) * CQ_COUNT * (size_t)c->cw_nitems));
  c->cw_batch = 1;
  c->cw_ok = 1;
  c->cw_use = 1;
  return CM3D_NB_OK;
}

// work items of the compact kernel (one system): each cell's atoms in
// `nsplit` parts
void cw_set_split(Ctx *c, int nsplit) {
  if (c->cw_batch) return;
  c->cw_nsplit = std::max(1, std::min(nsplit, CW_MAX_SPLIT));
  c->cw_nitems = c->ncells * c->cw_nsplit;
}

// A batch's compact-list layout and the kernel that reads it: row 32
// (k_pair_cw) or 8 lanes per atom (k_pair_cs).  The lists in use are
// converted again; a window beyond the 8-lane kernel's smaller capacity
// returns the batch to 32 lanes for good.
int cw_set_row(Ctx *c, int row) {
  if (!c->cw_ok || !c->cw_batch) return CM3D_NB_OK;
  if (row == CS_LPA && c->cw_cap8 == 0) row = CW_ROW;
  if (row == c->cw_row) return CM3D_NB_OK;
  c->cw_row = row;
  c->cw_cap = row == CS_LPA ? c->cw_cap8 : c->cw_cap32;
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);       // it holds the other kernel
    c->graph = nullptr;
  }
  if (!c->cw_use) return CM3D_NB_OK;      // converted when the compact path is taken up
  int rc = cw_convert(c, false, true);
  if (rc || c->cw_ok || row != CS_LPA) return rc;
  c->cw_ok = c->cw_use = 1;
  c->cw_cap8 = 0;
  c->cw_row = CW_ROW;
  c->cw_cap = c->cw_cap32;
  return cw_convert(c, false, true);
}

// after a (gated) rebuild of the master list: the compact list (a batch:
// of the compact systems being rebuilt, or of all after the slots widened)
int cw_convert(Ctx *c, bool device_flag, bool all) {
  // (a context whose autotuner chose another kernel keeps no compact lists;
  // the autotuner converts them all before it times the compact path)
  if (!c->cw_ok || !c->cw_use) return CM3D_NB_OK;
  // the master slots widen on overflow (host-driven builds only): so do ours
  if (cw_words_row(c->nbr_stride, c->cw_row) > c->cw_words) {
    const int words = cw_words_for(c->nbr_stride);
    DevLock lock(device_mutex());
    CK(cudaStreamSynchronize(c->st));
    cudaFree(c->cwl);
    c->cwl = nullptr;
    CK(cudaMalloc(&c->cwl, sizeof(uint2) * (size_t)c->n * (size_t)words));
    c->cw_words = words;
    all = true;
    if (c->graph) {
      cudaGraphExecDestroy(c->graph);
      c->graph = nullptr;
    }
  }
  const int *gate = device_flag ? c->istate : nullptr;
  int *halt = device_flag ? c->istate + IS_HALT : nullptr;
  if (c->cw_batch) {
    // only the atoms of the compact systems being rebuilt (all: every one)
    k_cw_scan<<<1, 1024, 0, c->st>>>(c->nsys, c->sp, c->cw_sys, c->sreb, all ? 1 : 0, c->cw_scan, gate);
    k_cw_convert_sys<<<8 * c->num_sms, 256, 0, c->st>>>(c->nsys, c->cw_scan, c->sp, c->cw_cap, c->n, c->cw_words,
                                                         c->cw_row, c->cell_start, c->cell_of, c->cell_atoms, c->nlen,
                                                         c->nbr_stride, c->nbr, c->cwl, c->cwn, c->stat, halt, gate);
    c->launches += 2;
  } else {
    k_cw_convert<<<grid_for(32LL * c->n, 256), 256, 0, c->st>>>(
        c->nc[0], c->nc[1], c->nc[2], c->cw_cap, c->n, c->cw_words, c->cw_row, c->cell_start, c->cell_of,
        c->cell_atoms, c->nlen, c->nbr_stride, c->nbr, c->cwl, c->cwn, c->stat, halt, gate);
    c->launches++;
  }
  CKL(c);
  if (!device_flag) {
    // a host-driven build: a window that did not fit turns the compact path
    // off for this context (the gather/window kernels read the master list)
    CK(cudaMemcpyAsync(c->h_stat, c->stat, sizeof(long long) * ST_COUNT, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (c->h_stat[ST_CWIN] > 0) {
      c->cw_ok = 0;
      c->cw_use = 0;
      long long zero = 0;
      CK(cudaMemcpy(c->stat + ST_CWIN, &zero, sizeof(long long), cudaMemcpyHostToDevice));
    }
  }
  return CM3D_NB_OK;
}

template <bool EL, int LJM, bool BATCH, int NT>
static void cw_launch_nt(Ctx *c, const CwP &P, size_t smem, double *fout, const float4 *tf, const float2 *tg,
                         const float4 *tl, const int4 *items, int item0) {
  auto kern = k_pair_cw<EL, LJM, BATCH, NT>;
  static unsigned long long attr_devs = 0;
  if (c->dev < 64 && !(attr_devs & (1ull << c->dev))) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(c->smem_optin - CW_STATIC_SMEM));
    attr_devs |= 1ull << c->dev;
  }
  const int grid = std::min(P.nitems, c->num_sms);
  kern<<<grid, NT, smem, c->st>>>(P, c->xq, c->styp, c->cell_atoms, c->cell_start, c->cwn, c->cwl, c->shift,
                                          c->map, c->fcut, tf, tg, tl, fout, c->cw_part, c->stat, c->gate, items,
                                          c->sp, item0);
}

template <bool EL, int LJM, bool BATCH>
static void cw_launch_t(Ctx *c, const CwP &P, size_t smem, double *fout, const float4 *tf, const float2 *tg,
                        const float4 *tl, const int4 *items, int item0) {
  if (c->cw_nt == CW_THREADS_WIDE) cw_launch_nt<EL, LJM, BATCH, CW_THREADS_WIDE>(c, P, smem, fout, tf, tg, tl, items, item0);
  else cw_launch_nt<EL, LJM, BATCH, CW_THREADS>(c, P, smem, fout, tf, tg, tl, items, item0);
}

template <bool BATCH>
static void cw_launch(Ctx *c, bool el, int ljm, const CwP &P, size_t smem, double *fout, const float4 *tf,
                      const float2 *tg, const float4 *tl, const int4 *items, int item0) {
  if (el) {
    if (ljm == 0) cw_launch_t<true, 0, BATCH>(c, P, smem, fout, tf, tg, tl, items, item0);
    else if (ljm == 1) cw_launch_t<true, 1, BATCH>(c, P, smem, fout, tf, tg, tl, items, item0);
    else cw_launch_t<true, 2, BATCH>(c, P, smem, fout, tf, tg, tl, items, item0);
  } else {
    if (ljm == 1) cw_launch_t<false, 1, BATCH>(c, P, smem, fout, tf, tg, tl, items, item0);
    else if (ljm == 2) cw_launch_t<false, 2, BATCH>(c, P, smem, fout, tf, tg, tl, items, item0);
  }
}

// k_pair_cs over a batch group's items (NG groups of items per block)
template <bool EL, int LJM, int NG, int GW>
static void cs_launch_g(Ctx *c, const CwP &P, size_t smem, double *fout, const float4 *tf, const float2 *tg,
                        const float4 *tl, const int4 *items, int item0) {
  auto kern = k_pair_cs<EL, LJM, true, NG, GW>;
  static unsigned long long attr_devs = 0;
  if (c->dev < 64 && !(attr_devs & (1ull << c->dev))) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(c->smem_optin - CS_STATIC_SMEM));
    attr_devs |= 1ull << c->dev;
  }
  const int grid = std::min((P.nitems + NG - 1) / NG, c->num_sms);
  kern<<<grid, NG * GW * 32, smem, c->st>>>(P, c->xq, c->styp, c->cell_atoms, c->cell_start, c->cwn, c->cwl,
                                             c->shift, c->map, c->fcut, tf, tg, tl, fout, c->cw_part, c->stat,
                                             c->gate, items, c->sp, item0);
}

template <bool EL, int LJM>
static void cs_launch_t(Ctx *c, int ng, const CwP &P, size_t smem, double *fout, const float4 *tf,
                        const float2 *tg, const float4 *tl, const int4 *items, int item0) {
  if (ng == CS_NG_WIDE) cs_launch_g<EL, LJM, CS_NG_WIDE, CS_GW_WIDE>(c, P, smem, fout, tf, tg, tl, items, item0);
  else cs_launch_g<EL, LJM, CS_NG, CS_GW>(c, P, smem, fout, tf, tg, tl, items, item0);
}

static void cs_launch(Ctx *c, int ng, bool el, int ljm, const CwP &P, size_t smem, double *fout, const float4 *tf,
                      const float2 *tg, const float4 *tl, const int4 *items, int item0) {
  if (el) {
    if (ljm == 0) cs_launch_t<true, 0>(c, ng, P, smem, fout, tf, tg, tl, items, item0);
    else if (ljm == 1) cs_launch_t<true, 1>(c, ng, P, smem, fout, tf, tg, tl, items, item0);
    else cs_launch_t<true, 2>(c, ng, P, smem, fout, tf, tg, tl, items, item0);
  } else {
    if (ljm == 1) cs_launch_t<false, 1>(c, ng, P, smem, fout, tf, tg, tl, items, item0);
    else if (ljm == 2) cs_launch_t<false, 2>(c, ng, P, smem, fout, tf, tg, tl, items, item0);
  }
}

bool cw_applies(Ctx *c, int iflg, bool ns) { return c->cw_ok && c->cw_use && iflg == 1 && !ns; }

// full force level through the compact path (the caller checked cw_applies):
// one system, or a batch's compact groups (the caller runs the gather kernel
// over the other systems' atoms); mask bit0 LJ, bit1 charges
int cw_pairs(Ctx *c, int mask, double *fout) {
  if (c->cw_batch) {
    for (const CwGroup &G : cw_groups(c)) {
      CwP P = G.P;
      P.n = c->n;
      P.words = c->cw_words;
      P.cap = c->cw_cap;
      const bool el = G.el && (mask & 2);
      const int ljm = (mask & 1) ? G.ljm : 0;
      if (!el && !ljm) continue;
      if (c->cw_row == CS_LPA)
        cs_launch(c, G.ng8, el, ljm, P, G.smem8, fout, c->cw_tf + G.tf0, c->cw_tg + G.tf0, c->cw_tl + G.tl0,
                  c->cw_items + G.item0, G.item0);
      else
        cw_launch<true>(c, el, ljm, P, G.smem, fout, c->cw_tf + G.tf0, c->cw_tg + G.tf0, c->cw_tl + G.tl0,
                        c->cw_items + G.item0, G.item0);
      c->launches++;
    }
    CKL(c);
    return CM3D_NB_OK;
  }
  CwP P;
  memset(&P, 0, sizeof P);
  P.n = c->n;
  P.ncx = c->nc[0];
  P.ncy = c->nc[1];
  P.ncz = c->nc[2];
  P.nsplit = c->cw_nsplit;
  P.nitems = c->cw_nitems;
  P.cap = c->cw_cap;
  P.words = c->cw_words;
  P.ntable = c->ntable;
  P.ntypes = c->ntypes;
  P.ninter = c->ninter;
  cw_coul_params(P, c->ntable, c->rmaxl_coul2, c->dx2coul, c->rmins_coul2);
  P.rc2_l = c->cw_lj1[0];
  P.dx2l = c->cw_lj1[1];
  P.offl = c->cw_lj1[2];
  P.vtl = c->cw_lj1[3];
  const bool el = (mask & 2) != 0;
  const int ljm = (mask & 1) ? cw_ljm_of(c->ninter) : 0;
  cw_launch<false>(c, el, ljm, P, c->cw_smem, fout, c->cw_tf, c->cw_tg, c->cw_tl, nullptr, 0);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

int cw_ereduce(Ctx *c, int mask) {
  if (c->cw_batch)
    k_cw_ereduce_sys<<<c->nsys, CQ_COUNT * 32, 0, c->st>>>(mask, c->cw_sitems, c->sp, c->cw_part, c->acc, c->gate);
  else
    k_cw_ereduce<<<1, CQ_COUNT * 32, 0, c->st>>>(c->cw_nitems, mask, c->tablast_e, c->cw_part, c->acc, c->gate);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

}  // namespace cm3d
