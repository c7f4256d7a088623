// nb_pair.cu -- mixed-precision fused LJ + real-space Ewald pair kernel.
//
// The same physics as force_npol (energy/inter/md_fnopol.c:46-255) and
// force_e (energy/inter/finter_e.c:42-233) -- table lookups with CM3D's
// 3-point interpolation f = f0 + p (A + p B), A = (f1 - f-1)/2,
// B = (f-1 - 2 f0 + f1)/2 (md_fnopol.c:148), the RESPA switch, CM3D's energy
// shifts -- computed in one pass over one list:
//
//   * atoms are cell-sorted; each carries FP32 coordinates relative to its
//     cell's corner (fixed between list rebuilds), so distances are formed
//     from numbers of at most a cell width instead of absolute coordinates;
//     the minimum-image shift of a pair is a per-entry 5-bit code into a
//     27-entry table of cell shifts;
//   * the list is full (both directions), so a group of TPA lanes owns atom i
//     and reduces its force with warp shuffles: no atomics, every force is
//     written exactly once;
//   * interpolation coefficients are FP32 float4 tables held in shared memory,
//     loaded once per block: the grid is persistent (resident blocks walk
//     the atoms), so the table load is paid once per SM, not per atom group;
//   * forces are summed per lane in FP32 over chunks of 16 pairs and then in
//     FP64; energies and virials are summed per atom in FP32 and written as
//     per-atom partials that k_ereduce adds up in FP64 in a fixed order --
//     except the table base values of the LJ energy, whose hi parts are
//     summed in FP64 (an LJ energy is a sum of terms of both signs that can
//     nearly cancel).
#include "nb_common.cuh"

namespace cm3d {

struct MixedP {
  int n, ntypes, ninter, ntable, iflg, mask;  // mask: bit0 LJ, bit1 charges
  float rc2_el, dx2c, offc, tablast_e;
  float hF[9], hiF[9];
  int tab_smem;
};

__global__ void k_xq_update(int n, const int *__restrict__ sorig, const double *__restrict__ pos,
                            const double *__restrict__ corner, const double *__restrict__ q,
                            float4 *__restrict__ xq, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int i = sorig[t];
  xq[t] = make_float4((float)(pos[i] - corner[t]), (float)(pos[n + i] - corner[n + t]),
                      (float)(pos[2 * n + i] - corner[2 * n + t]), (float)q[i]);
}

__device__ __forceinline__ float poly(float p, float c0, float a, float b) {
  return fmaf(p, fmaf(p, b, a), c0);
}

// Per-atom energy/virial partials (EP_* rows of epart, FP32, half-weighted
// because every pair is seen from both ends), summed by k_ereduce in FP64.
enum { EP_ELJ = 0, EP_ELJH, EP_VL0, EP_VL1, EP_VL2, EP_VL4, EP_VL5, EP_VL8,
       EP_EEL, EP_QQ, EP_VE0, EP_VE1, EP_VE2, EP_VE4, EP_VE5, EP_VE8, EP_COUNT };

// minimum image of a cell-shifted displacement for boxes narrower than two
// list radii: the nearest lattice vector m = rint(H^-1 d) is subtracted only
// when it is not zero, so that d keeps its precision in the common case
template <class Box>
__device__ __forceinline__ void min_image(const Box &B, float &dx, float &dy, float &dz) {
  const float m0 = rintf(B.hiF[0] * dx + B.hiF[1] * dy + B.hiF[2] * dz);
  const float m1 = rintf(B.hiF[3] * dx + B.hiF[4] * dy + B.hiF[5] * dz);
  const float m2 = rintf(B.hiF[6] * dx + B.hiF[7] * dy + B.hiF[8] * dz);
  if (m0 != 0.f || m1 != 0.f || m2 != 0.f) {
    dx -= B.hF[0] * m0 + B.hF[1] * m1 + B.hF[2] * m2;
    dy -= B.hF[3] * m0 + B.hF[4] * m1 + B.hF[5] * m2;
    dz -= B.hF[6] * m0 + B.hF[7] * m1 + B.hF[8] * m2;
  }
}

// ------------------------------------------------------------------
// Windowed pair kernel: one system whose cell grid has at least 3 cells per
// axis (no on-the-fly minimum image).  A work item is one cell of i-atoms (or
// a part of one); its block stages the 27 cells around it -- the only cells
// its atoms' neighbours can be in -- into shared memory, each cell's atoms
// already moved by that cell's periodic shift into the frame of the i-cell's
// corner.  A list entry (j's sorted index u, shift code) then addresses the
// staged copy as u + delta[code]: with 3 or more cells per axis the shift code
// names the stencil cell, so no gather leaves the SM.  The list itself is
// streamed in 16-byte vectors, one vector ahead of use.
//
// Window capacity is fixed at launch; an item whose 27 cells hold more atoms
// reads its j-atoms from global memory instead (same arithmetic), so no
// occupancy ever writes past the staged arrays.
struct WinP {
  int ncx, ncy, ncz;         // cells per axis (all >= 3)
  int nitems, nsplit;        // items = cells x parts
  int cap;                   // staged atoms per window
};

// Sums of one i-atom over its lanes' pairs (registers after inlining).
struct WinAcc {
  float fx, fy, fz, sx, sy, sz;   // FP32 chunk sums
  double Fx, Fy, Fz, Sx, Sy, Sz, elj_hi;
  float e[EP_COUNT];
  int cnt;
  unsigned under;
};

// Where an i-atom's j-atoms come from.
//   SRC_WIN:    the staged window of its cell (periodic shift applied)
//   SRC_GLOBAL: global memory (shift from the entry's code): a work item
//               whose window did not fit
enum { SRC_WIN = 0, SRC_GLOBAL = 1 };
struct WinSrc {
  const float4 *wx;              // staged positions (shift applied) + charge
  const unsigned short *wt;      // staged types
  const int *delta;              // window index = sorted index + delta[code]
  unsigned wlast;                // staged atoms - 1
  const float4 *xq;              // global: cell-relative positions + charge
  const int *styp;
  const float4 *shift;           // global: 27 hi shifts; shift_lo: 27 lo
  const float4 *shift_lo;
};
// The tables of the atom's system.
struct PairTab {
  const float4 *tl, *te;         // LJ (3 float4 per knot) and erfc coefficients (ntable force
                                 // float4, then ntable energy float4)
  const float *fcut;             // 8 floats per interaction
  const int *map;                // ntypes^2 interaction indices
  int ntypes;
  float rc2_el, dx2c, offc;
};

__device__ __forceinline__ void win_flush(WinAcc &A, bool need_s) {
  A.Fx += A.fx; A.Fy += A.fy; A.Fz += A.fz;
  A.fx = A.fy = A.fz = 0.f;
  if (need_s) {
    A.Sx += A.sx; A.Sy += A.sy; A.Sz += A.sz;
    A.sx = A.sy = A.sz = 0.f;
  }
}

// One segment [lo, hi) of atom i's slot.  LJ: the front segment (pairs in an
// LJ list; their electrostatics too when HAS_EL); otherwise the back segment
// (electrostatics only) or an electrostatics-only pass over the front.  The
// arithmetic is branch-free: a pair that is not in range -- past the segment,
// beyond the cut-off, or without the list flag -- contributes exact zeros
// (its charge product and table weight are selected to 0), and every table
// and window index is clamped in bounds.
template <int TPA, bool NEED_S, bool HAS_EL, bool LJ, int SRC>
__device__ __forceinline__ void win_segment(const MixedP &P, const WinSrc &S, const PairTab &T,
                                            const uint32_t *__restrict__ nbr, long long lo, long long hi, int g,
                                            float4 xi, int ti, WinAcc &A) {
  const uint32_t fl_lj = P.iflg == 1 ? ENT_LJ : ENT_LJS;
  const uint32_t fl_el = P.iflg == 1 ? ENT_EL : ENT_ELS;
  const int ntm2 = P.ntable - 2;
  auto pair = [&](uint32_t en, bool valid) {
    en = valid ? en : (13u << ENT_CODE_SHIFT);      // sorted atom 0, zero shift, no list flag
    const int code = (en >> ENT_CODE_SHIFT) & 31;
    const int u = (int)(en & ENT_JMASK);
    float4 xj;
    int tj = 0;
    float dx, dy, dz;
    if (SRC == SRC_WIN) {
      unsigned jl = (unsigned)(u + S.delta[code]);
      jl = jl < S.wlast ? jl : S.wlast;
      xj = S.wx[jl];
      if (LJ) tj = S.wt[jl];
      dx = xi.x - xj.x;
      dy = xi.y - xj.y;
      dz = xi.z - xj.z;
    } else {
      xj = S.xq[u];
      if (LJ) tj = S.styp[u];
      const float4 sh = S.shift[code], shl = S.shift_lo[code];
      dx = ((xi.x - xj.x) + sh.x) + shl.x;
      dy = ((xi.y - xj.y) + sh.y) + shl.y;
      dz = ((xi.z - xj.z) + sh.z) + shl.z;
    }
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    float ftot = 0.f, fsh = 0.f;
    if (HAS_EL) {
      const bool ok = (en & fl_el) != 0 && r2 < T.rc2_el;
      const float p = fmaf(r2, T.dx2c, -T.offc);
      int kk = (int)p;
      A.under += (ok && kk < 1) ? 1u : 0u;
      // below the table: CM3D's clamp (kk = 1, p = 1: the first knot)
      const float fr = ok && kk >= 1 ? p - (float)kk : 0.f;
      kk = kk < 1 ? 1 : (kk > ntm2 ? ntm2 : kk);
      const float4 c0 = T.te[kk];
      const float qq = ok ? xi.w * xj.w : 0.f;
      const float fe = qq * poly(fr, c0.x, c0.y, c0.z);
      ftot = fe;
      if (P.iflg == 1) {
        const float4 c1 = T.te[P.ntable + kk];
        A.e[EP_EEL] = fmaf(qq, poly(fr, c0.w, c1.x, c1.y), A.e[EP_EEL]);
        A.e[EP_QQ] += qq;
        const float fdx = fe * dx, fdy = fe * dy, fdz = fe * dz;
        A.e[EP_VE0] = fmaf(fdx, dx, A.e[EP_VE0]);
        A.e[EP_VE1] = fmaf(fdx, dy, A.e[EP_VE1]);
        A.e[EP_VE2] = fmaf(fdx, dz, A.e[EP_VE2]);
        A.e[EP_VE4] = fmaf(fdy, dy, A.e[EP_VE4]);
        A.e[EP_VE5] = fmaf(fdy, dz, A.e[EP_VE5]);
        A.e[EP_VE8] = fmaf(fdz, dz, A.e[EP_VE8]);
        if (NEED_S) fsh = fe;                        // force_e's switch is never engaged
      }
    }
    if (LJ) {
      const bool isl = (en & fl_lj) != 0;
      int in = T.map[ti * T.ntypes + tj];
      in = in < 0 ? 0 : in;
      // {rmaxl_cut2, rmins_cut2 dx2tab, dx2tab, vt} {rminl_cut2, rmaxs_cut2, -, -}
      const float4 cA = reinterpret_cast<const float4 *>(T.fcut)[2 * in];
      const bool needB = P.iflg == 0 || NEED_S;
      const float4 cB = needB ? reinterpret_cast<const float4 *>(T.fcut)[2 * in + 1] : cA;
      const bool ok = isl && r2 < (P.iflg == 1 ? cA.x : cB.y);
      const float p = fmaf(r2, cA.z, -cA.y);
      int kk = (int)p;
      A.under += (ok && kk < 1) ? 1u : 0u;
      const float fr = ok && kk >= 1 ? p - (float)kk : 0.f;
      kk = kk < 1 ? 1 : (kk > ntm2 ? ntm2 : kk);
      const float4 *Tk = T.tl + 3 * ((size_t)in * P.ntable + kk);
      const float4 a0 = Tk[0], a1 = Tk[1], a2 = Tk[2];
      const float okf = ok ? 1.f : 0.f;
      const float f = okf * poly(fr, a0.x, a0.y, a0.z);
      const float swv = (needB && r2 > cB.x) ? poly(fr, a1.z, a1.w, a2.x) : 1.f;
      if (P.iflg == 1) {
        ftot += f;
        // V = v0 + p (vA + p vB) with v0 = hi (a0.w) + lo (a2.y): the hi
        // parts are summed in FP64, so that an LJ energy whose pair terms
        // cancel keeps FP64-like accuracy
        A.elj_hi += ok ? (double)a0.w : 0.0;
        const float vlo = okf * (a2.y + fr * fmaf(fr, a1.y, a1.x));
        A.e[EP_ELJ] += vlo;
        A.e[EP_ELJH] = fmaf(-okf, cA.w, A.e[EP_ELJH] + vlo);
        const float fdx = f * dx, fdy = f * dy, fdz = f * dz;
        A.e[EP_VL0] = fmaf(fdx, dx, A.e[EP_VL0]);
        A.e[EP_VL1] = fmaf(fdx, dy, A.e[EP_VL1]);
        A.e[EP_VL2] = fmaf(fdx, dz, A.e[EP_VL2]);
        A.e[EP_VL4] = fmaf(fdy, dy, A.e[EP_VL4]);
        A.e[EP_VL5] = fmaf(fdy, dz, A.e[EP_VL5]);
        A.e[EP_VL8] = fmaf(fdz, dz, A.e[EP_VL8]);
        if (NEED_S) fsh = fmaf(f, swv, fsh);
      } else {
        ftot = fmaf(f, swv, ftot);
      }
    }
    // F_i = -f d  (md_fnopol.c:227-229)
    A.fx = fmaf(-ftot, dx, A.fx);
    A.fy = fmaf(-ftot, dy, A.fy);
    A.fz = fmaf(-ftot, dz, A.fz);
    if (NEED_S) {
      A.sx = fmaf(-fsh, dx, A.sx);
      A.sy = fmaf(-fsh, dy, A.sy);
      A.sz = fmaf(-fsh, dz, A.sz);
    }
  };
  // lane g owns the 16-byte vectors at la + 4 g + 4 TPA m (la: lo rounded
  // down to a vector boundary; slots start on 128-byte boundaries since
  // stride is a multiple of 32).  A vector that starts below hi ends inside
  // the slot.  The next vector is loaded while the current one is used.
  constexpr int STEP = 4 * TPA;
  const long long la = lo & ~3LL;
  long long kb = la + 4 * g;
  uint4 nxt = make_uint4(0u, 0u, 0u, 0u);
  if (kb < hi) nxt = __ldg(reinterpret_cast<const uint4 *>(nbr + kb));
  for (; kb < hi; kb += STEP) {
    const uint4 cur = nxt;
    if (kb + STEP < hi) nxt = __ldg(reinterpret_cast<const uint4 *>(nbr + kb + STEP));
    pair(cur.x, kb >= lo && kb < hi);
    pair(cur.y, kb + 1 >= lo && kb + 1 < hi);
    pair(cur.z, kb + 2 >= lo && kb + 2 < hi);
    pair(cur.w, kb + 3 >= lo && kb + 3 < hi);
    if (++A.cnt == 4) {                              // 16 pairs per FP32 chunk
      win_flush(A, NEED_S);
      A.cnt = 0;
    }
  }
}

template <int TPA, bool NEED_S, bool HAS_EL, int SRC>
__device__ __forceinline__ void win_atom(const MixedP &P, const WinSrc &S, const PairTab &T,
                                         const uint32_t *__restrict__ nbr, long long k0, int stride, int na, int nb,
                                         int g, float4 xi, int ti, bool has_lj, bool has_el, WinAcc &A) {
  // the front segment's pairs may carry charges too (an electrostatics-only
  // call still walks it); a system without charges skips the electrostatic
  // arithmetic altogether
  const bool el = HAS_EL && has_el;
  if (has_lj) {
    if (el) win_segment<TPA, NEED_S, true, true, SRC>(P, S, T, nbr, k0, k0 + na, g, xi, ti, A);
    else win_segment<TPA, NEED_S, false, true, SRC>(P, S, T, nbr, k0, k0 + na, g, xi, ti, A);
  } else if (el) {
    win_segment<TPA, NEED_S, true, false, SRC>(P, S, T, nbr, k0, k0 + na, g, xi, ti, A);
  }
  if (el) win_segment<TPA, NEED_S, true, false, SRC>(P, S, T, nbr, k0 + stride - nb, k0 + stride, g, xi, ti, A);
  win_flush(A, NEED_S);
}

template <int TPA, bool NEED_S, bool HAS_EL>
__global__ void __launch_bounds__(512, 1) k_pair_win(
    MixedP P, WinP W, const float4 *__restrict__ xq, const int *__restrict__ styp, const int *__restrict__ sorig,
    const int *__restrict__ cell_start, const int *__restrict__ nlen, int stride, const uint32_t *__restrict__ nbr,
    const float4 *__restrict__ gshift, const int *__restrict__ gmap, const float *__restrict__ gfcut,
    const float4 *__restrict__ gtl, const float4 *__restrict__ gte, double *__restrict__ fout,
    double *__restrict__ fshort, float *__restrict__ epart, double *__restrict__ epart64,
    long long *__restrict__ stat, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  extern __shared__ float4 sm[];
  float4 *shift = sm;                                   // 27 hi + 27 lo
  float *fcut = reinterpret_cast<float *>(sm + 54);     // 8 * ninter
  const int nf4 = (8 * P.ninter + 3) / 4;
  int *map = reinterpret_cast<int *>(sm + 54 + nf4);    // ntypes^2
  const int nm4 = (P.ntypes * P.ntypes + 3) / 4;
  float4 *tl = sm + 54 + nf4 + nm4;                     // LJ tables (3 * ninter * ntable)
  const int nl = (P.mask & 1) ? 3 * P.ninter * P.ntable : 0;
  // erfc table (2 * ntable): the force coefficients of every knot, then the
  // energy coefficients -- two arrays at a 16-byte stride, so that random
  // knots spread over all bank groups (interleaved, each half would use half)
  float4 *te = tl + nl;
  const int ne = HAS_EL ? 2 * P.ntable : 0;
  float4 *wx = te + ne;                                 // staged window: cap float4
  unsigned short *wt = reinterpret_cast<unsigned short *>(wx + W.cap);   // cap types
  __shared__ int s_cs[27], s_cnt[27], s_off[27], s_delta[32], s_tot;

  for (int k = threadIdx.x; k < 54; k += blockDim.x) shift[k] = gshift[k];
  for (int k = threadIdx.x; k < 8 * P.ninter; k += blockDim.x) fcut[k] = gfcut[k];
  for (int k = threadIdx.x; k < P.ntypes * P.ntypes; k += blockDim.x) map[k] = gmap[k];
  for (int k = threadIdx.x; k < nl; k += blockDim.x) tl[k] = gtl[k];
  for (int k = threadIdx.x; k < ne; k += blockDim.x) te[(k & 1) * P.ntable + (k >> 1)] = gte[k];

  const int g = threadIdx.x % TPA;
  const int groups = blockDim.x / TPA;
  const bool has_lj = (P.mask & 1) != 0;
  unsigned under = 0;

  for (int item = blockIdx.x; item < W.nitems; item += gridDim.x) {
    const int c = item / W.nsplit, part = item - c * W.nsplit;
    const int cz = c % W.ncz, cy = (c / W.ncz) % W.ncy, cx = c / (W.ncz * W.ncy);
    __syncthreads();                                     // the previous window is no longer read
    if (threadIdx.x < 32) {
      // window cell w = shift code: j-cell = i-cell - k, k = (w/9-1, w/3%3-1, w%3-1)
      const int w = threadIdx.x;
      int cnt = 0, cs = 0;
      if (w < 27) {
        int jx = cx - (w / 9 - 1), jy = cy - ((w / 3) % 3 - 1), jz = cz - (w % 3 - 1);
        jx = jx < 0 ? jx + W.ncx : (jx >= W.ncx ? jx - W.ncx : jx);
        jy = jy < 0 ? jy + W.ncy : (jy >= W.ncy ? jy - W.ncy : jy);
        jz = jz < 0 ? jz + W.ncz : (jz >= W.ncz ? jz - W.ncz : jz);
        const int jc = (jx * W.ncy + jy) * W.ncz + jz;
        cs = cell_start[jc];
        cnt = cell_start[jc + 1] - cs;
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (w >= o) incl += v;
      }
      if (w < 27) {
        s_cs[w] = cs;
        s_cnt[w] = cnt;
        s_off[w] = incl - cnt;
      }
      s_delta[w] = w < 27 ? incl - cnt - cs : 0;       // codes 27..31 never occur
      if (w == 26) s_tot = incl;
    }
    __syncthreads();
    const int wtot = s_tot;
    const bool staged = wtot <= W.cap;
    if (staged) {
      for (int w = 0; w < 27; w++) {
        const int cs = s_cs[w], cnt = s_cnt[w], off = s_off[w];
        const float4 sh = shift[w], shl = shift[27 + w];
        for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
          const float4 x = xq[cs + k];
          wx[off + k] = make_float4((x.x - sh.x) - shl.x, (x.y - sh.y) - shl.y, (x.z - sh.z) - shl.z, x.w);
          if (has_lj) wt[off + k] = (unsigned short)styp[cs + k];
        }
      }
    }
    __syncthreads();
    WinSrc S;
    S.wx = wx;
    S.wt = wt;
    S.delta = s_delta;
    S.wlast = (unsigned)(wtot > 0 ? wtot - 1 : 0);
    S.xq = xq;
    S.styp = styp;
    S.shift = shift;
    S.shift_lo = shift + 27;
    PairTab T;
    T.tl = tl;
    T.te = te;
    T.fcut = fcut;
    T.map = map;
    T.ntypes = P.ntypes;
    T.rc2_el = P.rc2_el;
    T.dx2c = P.dx2c;
    T.offc = P.offc;
    const int ci0 = s_cs[13], cin = s_cnt[13], ioff = s_off[13];
    for (int r = part; r * groups < cin; r += W.nsplit) {
      const int a = r * groups + threadIdx.x / TPA;
      const bool active = a < cin;
      const int t = ci0 + (active ? a : 0);
      WinAcc A;
      A.fx = A.fy = A.fz = A.sx = A.sy = A.sz = 0.f;
      A.Fx = A.Fy = A.Fz = A.Sx = A.Sy = A.Sz = A.elj_hi = 0.0;
#pragma unroll
      for (int k = 0; k < EP_COUNT; k++) A.e[k] = 0.f;
      A.cnt = 0;
      A.under = 0;
      if (active) {
        // the centre cell's shift is zero: staged i and xq agree exactly
        const float4 xi = staged ? wx[ioff + a] : xq[t];
        const int ti = has_lj ? styp[t] : 0;
        const int na = nlen[t], nb = nlen[P.n + t];
        const long long k0 = (long long)t * stride;
        if (staged)
          win_atom<TPA, NEED_S, HAS_EL, SRC_WIN>(P, S, T, nbr, k0, stride, na, nb, g, xi, ti, has_lj, true, A);
        else
          win_atom<TPA, NEED_S, HAS_EL, SRC_GLOBAL>(P, S, T, nbr, k0, stride, na, nb, g, xi, ti, has_lj, true, A);
      }
      under += A.under;
#pragma unroll
      for (int o = TPA / 2; o > 0; o >>= 1) {
        A.Fx += __shfl_xor_sync(0xffffffffu, A.Fx, o);
        A.Fy += __shfl_xor_sync(0xffffffffu, A.Fy, o);
        A.Fz += __shfl_xor_sync(0xffffffffu, A.Fz, o);
        if (NEED_S) {
          A.Sx += __shfl_xor_sync(0xffffffffu, A.Sx, o);
          A.Sy += __shfl_xor_sync(0xffffffffu, A.Sy, o);
          A.Sz += __shfl_xor_sync(0xffffffffu, A.Sz, o);
        }
        if (P.iflg == 1) {
#pragma unroll
          for (int k = 0; k < EP_COUNT; k++) A.e[k] += __shfl_xor_sync(0xffffffffu, A.e[k], o);
          A.elj_hi += __shfl_xor_sync(0xffffffffu, A.elj_hi, o);
        }
      }
      if (active && g == 0) {
        const int i = sorig[t], n = P.n;
        fout[i] += A.Fx;
        fout[n + i] += A.Fy;
        fout[2 * n + i] += A.Fz;
        if (NEED_S && P.iflg == 1) {
          fshort[i] += A.Sx;
          fshort[n + i] += A.Sy;
          fshort[2 * n + i] += A.Sz;
        }
        if (P.iflg == 1) {
#pragma unroll
          for (int k = 0; k < EP_COUNT; k++) epart[(size_t)k * n + t] = A.e[k];
          epart64[t] = A.elj_hi;
        }
      }
    }
  }
  if (under) atomicAdd((unsigned long long *)(stat + ST_UNDERFLOW), (unsigned long long)under);
}

// Gather kernel: batches, and single systems whose cell grid is too coarse
// for the windowed kernel (or when that kernel is switched off).  Its lane
// groups read j-atoms from global memory (L1/L2: a batch's systems are
// small) and skip out-of-range pairs by branching, which suits short lists
// where a good share of the listed pairs lies beyond the cut-off.
//
// BATCH = false: one system, its parameters in P and its shifts, cut-offs,
// type map and (when they fit) tables staged in shared memory.  BATCH = true:
// several systems; each atom group reads its system's parameters, shifts and
// tables (global interaction / Coulomb-table indices) from sp[sys_of[t]].
//
// STAGE (batches, full force without the RESPA switch): the blocks walk work
// items -- a system, or a part of at most SYS_PART atoms of one -- instead of
// striding over all atoms, and first copy the item's system parameters into
// shared memory: its cell shifts, type map (local interaction indices),
// cut-offs, LJ force/energy coefficients (2 float4 per knot) and erfc table.
// Every per-pair parameter and table read is then a shared-memory load; the
// j-atoms still come from global memory through L1.  Items come largest
// system first (host-ordered), so the long ones start early.
constexpr int SYS_PART = 1024;

// TABLE2: the compact LJ table (2 float4 per knot), for the full force
// without the RESPA switch (iflg 1, no short-force copy).
template <int TPA, bool SMALLBOX, bool NEED_S, bool BATCH, bool STAGE = false, bool TABLE2 = false>
__global__ void __launch_bounds__(256, NEED_S ? 2 : 3) k_pair_mixed(
    MixedP P, const float4 *__restrict__ xq, const int *__restrict__ styp, const int *__restrict__ sorig,
    const int *__restrict__ nlen, int stride, const uint32_t *__restrict__ nbr, const float4 *__restrict__ gshift,
    const int *__restrict__ gmap, const float *__restrict__ gfcut, const float4 *__restrict__ gtl,
    const float4 *__restrict__ gte, const SysP *__restrict__ sp, const int *__restrict__ sys_of,
    double *__restrict__ fout, double *__restrict__ fshort, float *__restrict__ epart,
    double *__restrict__ epart64, long long *__restrict__ stat, const int *__restrict__ gs,
    const int4 *__restrict__ items = nullptr, int nitems = 0, const float4 *__restrict__ gtl2 = nullptr,
    int st_ntypes = 0, int st_ninter = 0, const int *__restrict__ gidx = nullptr, int ng = 0) {
  static_assert(!STAGE || BATCH, "staging is for batches");
  if (gated_off(gs, 0)) return;
  extern __shared__ float4 sm[];
  // STAGE: one system's parameters (layout sized for the largest system)
  float4 *st_shift = sm;                                                      // 54
  int *st_map = reinterpret_cast<int *>(sm + 54);                             // st_ntypes^2
  const int st_nm4 = (st_ntypes * st_ntypes + 3) / 4;
  float *st_fcut = reinterpret_cast<float *>(sm + 54 + st_nm4);               // 8 * st_ninter
  float4 *st_tl = sm + 54 + st_nm4 + 2 * st_ninter;                           // 2 * st_ninter * ntable
  float4 *st_te = st_tl + 2 * st_ninter * P.ntable;                           // 2 * ntable
  float4 *shift = sm;                                   // 27 hi + 27 lo
  float *fcut = reinterpret_cast<float *>(sm + 54);     // 8 * ninter
  int nf4 = (8 * P.ninter + 3) / 4;
  int *map = reinterpret_cast<int *>(sm + 54 + nf4);    // ntypes^2
  int nm4 = (P.ntypes * P.ntypes + 3) / 4;
  float4 *tl_s = sm + 54 + nf4 + nm4;
  const float4 *tl = gtl, *te = gte;
  if (!BATCH) {
    for (int k = threadIdx.x; k < 54; k += blockDim.x) shift[k] = gshift[k];
    for (int k = threadIdx.x; k < 8 * P.ninter; k += blockDim.x) fcut[k] = gfcut[k];
    for (int k = threadIdx.x; k < P.ntypes * P.ntypes; k += blockDim.x) map[k] = gmap[k];
  }
  if (!BATCH && P.tab_smem) {
    int nl = (P.mask & 1) ? 3 * P.ninter * P.ntable : 0;
    int ne = (P.mask & 2) ? 2 * P.ntable : 0;
    for (int k = threadIdx.x; k < nl; k += blockDim.x) tl_s[k] = gtl[k];
    float4 *te_s = tl_s + 3 * P.ninter * P.ntable;
    for (int k = threadIdx.x; k < ne; k += blockDim.x) te_s[k] = gte[k];
    tl = tl_s;
    te = te_s;
  }
  __syncthreads();

  const int g = threadIdx.x % TPA;
  const int groups = blockDim.x / TPA;
  const uint32_t fl_lj = P.iflg == 1 ? ENT_LJ : ENT_LJS;
  const uint32_t fl_el = P.iflg == 1 ? ENT_EL : ENT_ELS;
  unsigned under = 0;
  // one i-atom per lane group (every lane of the block calls it: it ends in
  // warp shuffles)
  auto do_atom = [&](const int t, const bool active) {
    double Fx = 0, Fy = 0, Fz = 0, Sx = 0, Sy = 0, Sz = 0, elj_hi = 0;
    float e[EP_COUNT];
#pragma unroll
    for (int k = 0; k < EP_COUNT; k++) e[k] = 0.f;
    if (active) {
      const float4 xi = xq[t];
      const int ti = styp[t];
      // the slot's two segments: LJ-list pairs at the front, pairs in the
      // electrostatic lists only at the back
      const long long k0 = (long long)t * stride;
      const long long seg[4] = {k0, k0 + nlen[t], k0 + stride - nlen[P.n + t], k0 + stride};
      float fx = 0, fy = 0, fz = 0, sx = 0, sy = 0, sz = 0;
      int cnt = 0;
      // this atom's system: shifts, type map, cut-offs and tables
      const SysP *Sp = BATCH ? sp + sys_of[t] : nullptr;
      const float4 *shp = STAGE ? st_shift : BATCH ? Sp->shift : shift;
      const float4 *shlp = STAGE ? st_shift + 27 : BATCH ? Sp->shift_lo : shift + 27;
      const int *mapp = STAGE ? st_map : BATCH ? gmap + Sp->map0 : map;
      const float *fcp = STAGE ? st_fcut : BATCH ? gfcut : fcut;
      const int ntyp = BATCH ? Sp->ntypes : P.ntypes;
      const bool has_el = (P.mask & 2) && (!BATCH || Sp->coul >= 0);
      const float4 *tep = STAGE ? st_te : BATCH ? gte + (size_t)2 * P.ntable * (Sp->coul > 0 ? Sp->coul : 0) : te;
      const float rc2_el = BATCH ? Sp->rc2_el : P.rc2_el;
      const float dx2c = BATCH ? Sp->dx2c : P.dx2c;
      const float offc = BATCH ? Sp->offc : P.offc;
      const bool sb = BATCH ? Sp->smallbox != 0 : SMALLBOX;
      // one pair; xj and tj (j's type, needed only by LJ pairs) come from the
      // batched loads below
      auto pair = [&](const uint32_t en, const float4 xj, const int tj) {
        const int code = (en >> ENT_CODE_SHIFT) & 31;
        const float4 sh = shp[code], shl = shlp[code];
        float dx = ((xi.x - xj.x) + sh.x) + shl.x;
        float dy = ((xi.y - xj.y) + sh.y) + shl.y;
        float dz = ((xi.z - xj.z) + sh.z) + shl.z;
        if (BATCH) {
          if (sb && (en & ENT_NEAR)) min_image(*Sp, dx, dy, dz);
        } else if (SMALLBOX) {
          if (en & ENT_NEAR) min_image(P, dx, dy, dz);
        }
        const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        float ftot = 0.f, fsh = 0.f;
        if ((en & fl_el) && has_el && r2 < rc2_el) {
          float p = fmaf(r2, dx2c, -offc);
          int kk = (int)p;
          if (kk < 1) {
            under++;
            kk = 1;
            p = 1.f;
          }
          p -= (float)kk;
          const float4 c0 = tep[2 * kk];
          const float qq = xi.w * xj.w;
          const float fe = qq * poly(p, c0.x, c0.y, c0.z);
          ftot += fe;
          if (P.iflg == 1) {
            const float4 c1 = tep[2 * kk + 1];
            e[EP_EEL] = fmaf(qq, poly(p, c0.w, c1.x, c1.y), e[EP_EEL]);
            e[EP_QQ] += qq;
            const float fdx = fe * dx, fdy = fe * dy, fdz = fe * dz;
            e[EP_VE0] = fmaf(fdx, dx, e[EP_VE0]);
            e[EP_VE1] = fmaf(fdx, dy, e[EP_VE1]);
            e[EP_VE2] = fmaf(fdx, dz, e[EP_VE2]);
            e[EP_VE4] = fmaf(fdy, dy, e[EP_VE4]);
            e[EP_VE5] = fmaf(fdy, dz, e[EP_VE5]);
            e[EP_VE8] = fmaf(fdz, dz, e[EP_VE8]);
            if (NEED_S) fsh += fe;           // force_e's switch is never engaged
          }
        }
        if ((en & fl_lj) && (P.mask & 1)) {
          const int in = mapp[ti * ntyp + tj];
          // {rmaxl_cut2, rmins_cut2 dx2tab, dx2tab, vt} {rminl_cut2, rmaxs_cut2, -, -}
          const float4 cA = reinterpret_cast<const float4 *>(fcp)[2 * in];
          const bool needB = P.iflg == 0 || NEED_S;
          const float4 cB = needB ? reinterpret_cast<const float4 *>(fcp)[2 * in + 1] : cA;
          const float rmax2 = P.iflg == 1 ? cA.x : cB.y;
          if (r2 < rmax2) {
            float p = fmaf(r2, cA.z, -cA.y);
            int kk = (int)p;
            if (kk < 1) {
              under++;
              kk = 1;
              p = 1.f;
            }
            p -= (float)kk;
            float4 a0, a1, a2;
            const int knot = in * P.ntable + kk;
            if (STAGE || TABLE2) {
              // {d0, dA, dB, v0 hi} {vA, vB, v0 lo, -}
              const float4 *T = (STAGE ? st_tl : gtl2) + 2 * knot;
              a0 = T[0];
              const float4 b = T[1];
              a1 = make_float4(b.x, b.y, 0.f, 0.f);
              a2 = make_float4(0.f, b.z, 0.f, 0.f);
            } else {
              const float4 *T = tl + 3 * knot;
              a0 = T[0];
              a1 = T[1];
              a2 = T[2];
            }
            const float f = poly(p, a0.x, a0.y, a0.z);
            float swv = 1.f;
            if (needB && r2 > cB.x) swv = poly(p, a1.z, a1.w, a2.x);
            if (P.iflg == 1) {
              ftot += f;
              // V = v0 + p (vA + p vB) with v0 = hi (a0.w) + lo (a2.y): the
              // hi parts are summed in FP64, so that an LJ energy whose pair
              // terms cancel keeps FP64-like accuracy
              elj_hi += (double)a0.w;
              const float vlo = a2.y + p * fmaf(p, a1.y, a1.x);
              e[EP_ELJ] += vlo;
              e[EP_ELJH] += vlo - cA.w;
              const float fdx = f * dx, fdy = f * dy, fdz = f * dz;
              e[EP_VL0] = fmaf(fdx, dx, e[EP_VL0]);
              e[EP_VL1] = fmaf(fdx, dy, e[EP_VL1]);
              e[EP_VL2] = fmaf(fdx, dz, e[EP_VL2]);
              e[EP_VL4] = fmaf(fdy, dy, e[EP_VL4]);
              e[EP_VL5] = fmaf(fdy, dz, e[EP_VL5]);
              e[EP_VL8] = fmaf(fdz, dz, e[EP_VL8]);
              if (NEED_S) fsh += f * swv;
            } else {
              ftot += f * swv;
            }
          }
        }
        // F_i = -f d  (md_fnopol.c:227-229)
        fx = fmaf(-ftot, dx, fx);
        fy = fmaf(-ftot, dy, fy);
        fz = fmaf(-ftot, dz, fz);
        if (NEED_S) {
          sx = fmaf(-fsh, dx, sx);
          sy = fmaf(-fsh, dy, sy);
          sz = fmaf(-fsh, dz, sz);
        }
      };
      // the lane's pairs k0+g, k0+g+TPA, ... in batches of PU: the batch's
      // list entries, then its coordinates and types, are loaded together so
      // that PU independent loads are in flight; FP32 sums go to FP64 every
      // 16 pairs.  Entry 0 marks the end (a real entry has a list flag set).
      constexpr int PU = 4;
      for (int sg = 0; sg < 2; sg++)
      for (long long kb = seg[2 * sg] + g, k1 = seg[2 * sg + 1]; kb < k1; kb += PU * TPA) {
        uint32_t en[PU];
        float4 xj[PU];
        int tj[PU];
#pragma unroll
        for (int u = 0; u < PU; u++) {
          const long long k = kb + (long long)u * TPA;
          en[u] = k < k1 ? __ldg(nbr + k) : 0u;
        }
#pragma unroll
        for (int u = 0; u < PU; u++) {
          const int j = en[u] & ENT_JMASK;
          xj[u] = xq[j];
          // (a one-type system's j is type 0: no load)
          tj[u] = (ntyp > 1 && (en[u] & fl_lj)) ? styp[j] : 0;
        }
#pragma unroll
        for (int u = 0; u < PU; u++)
          if (en[u] != 0u) pair(en[u], xj[u], tj[u]);
        cnt += PU;
        if (cnt == 16) {
          Fx += fx; Fy += fy; Fz += fz;
          fx = fy = fz = 0.f;
          if (NEED_S) {
            Sx += sx; Sy += sy; Sz += sz;
            sx = sy = sz = 0.f;
          }
          cnt = 0;
        }
      }
      Fx += fx; Fy += fy; Fz += fz;
      if (NEED_S) {
        Sx += sx; Sy += sy; Sz += sz;
      }
    }
    // reduce atom i's sums over its TPA lanes (aligned lane groups)
#pragma unroll
    for (int o = TPA / 2; o > 0; o >>= 1) {
      Fx += __shfl_xor_sync(0xffffffffu, Fx, o);
      Fy += __shfl_xor_sync(0xffffffffu, Fy, o);
      Fz += __shfl_xor_sync(0xffffffffu, Fz, o);
      if (NEED_S) {
        Sx += __shfl_xor_sync(0xffffffffu, Sx, o);
        Sy += __shfl_xor_sync(0xffffffffu, Sy, o);
        Sz += __shfl_xor_sync(0xffffffffu, Sz, o);
      }
      if (P.iflg == 1) {
#pragma unroll
        for (int k = 0; k < EP_COUNT; k++) e[k] += __shfl_xor_sync(0xffffffffu, e[k], o);
        elj_hi += __shfl_xor_sync(0xffffffffu, elj_hi, o);
      }
    }
    if (active && g == 0) {
      const int i = sorig[t], n = P.n;
      fout[i] += Fx;
      fout[n + i] += Fy;
      fout[2 * n + i] += Fz;
      if (NEED_S && P.iflg == 1) {
        fshort[i] += Sx;
        fshort[n + i] += Sy;
        fshort[2 * n + i] += Sz;
      }
      if (P.iflg == 1) {
#pragma unroll
        for (int k = 0; k < EP_COUNT; k++) epart[(size_t)k * n + t] = e[k];
        epart64[t] = elj_hi;
      }
    }
  };
  if (!STAGE) {
    // persistent: every lane group walks atoms blockIdx-strided (with gidx:
    // only the listed sorted atoms, the rest of a batch being in the
    // compact kernel)
    const int nloop = gidx ? ng : P.n;
    for (int tb = blockIdx.x * groups; tb < nloop; tb += gridDim.x * groups) {
      const int tt = tb + threadIdx.x / TPA;
      const int t = gidx ? (tt < ng ? gidx[tt] : 0) : tt;
      do_atom(t, tt < nloop);
    }
  } else {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
      const int4 item = items[it];                       // {system, first atom, end atom, -}
      const SysP &S = sp[item.x];
      __syncthreads();                                   // the previous system is no longer read
      for (int k = threadIdx.x; k < 27; k += blockDim.x) {
        st_shift[k] = S.shift[k];
        st_shift[27 + k] = S.shift_lo[k];
      }
      for (int k = threadIdx.x; k < S.ntypes * S.ntypes; k += blockDim.x) {
        const int in = gmap[S.map0 + k];
        st_map[k] = in >= 0 ? in - S.inter0 : -1;
      }
      for (int k = threadIdx.x; k < 8 * S.ninter; k += blockDim.x) st_fcut[k] = gfcut[8 * S.inter0 + k];
      if (P.mask & 1)
        for (int k = threadIdx.x; k < 2 * S.ninter * P.ntable; k += blockDim.x)
          st_tl[k] = gtl2[(size_t)2 * S.inter0 * P.ntable + k];
      if ((P.mask & 2) && S.coul >= 0)
        for (int k = threadIdx.x; k < 2 * P.ntable; k += blockDim.x)
          st_te[k] = gte[(size_t)2 * P.ntable * S.coul + k];
      __syncthreads();
      for (int tb = item.y; tb < item.z; tb += groups) {
        const int t = tb + threadIdx.x / TPA;
        do_atom(t, t < item.z);
      }
    }
  }
  if (under) atomicAdd((unsigned long long *)(stat + ST_UNDERFLOW), (unsigned long long)under);
}

// FP64 sums of the per-atom partials into CM3D's accumulators (one block per
// quantity and system, fixed order: deterministic).  Every pair was seen from
// both ends, hence the factor 1/2; CM3D's virials are -sum d_a d_b f.
//
// A system's atoms may be split over gridDim.z blocks (one large system): each
// block stores its partial sum, and the last block of a quantity to finish
// adds the partials in block order -- the result does not depend on which
// block finished last -- and re-arms the counter for the next launch.
__device__ __forceinline__ void ep_to_acc(int q, double s, double *acc, float tablast_e);

__global__ void k_ereduce(int n, int mask, const SysP *__restrict__ sp, const float *__restrict__ epart,
                          const double *__restrict__ epart64, double *__restrict__ accs,
                          double *__restrict__ part, unsigned *__restrict__ done, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  __shared__ double red[32];
  __shared__ bool last;
  const int q = blockIdx.x, sy = blockIdx.y, nz = gridDim.z;
  if (!((q < EP_EEL && (mask & 1)) || (q >= EP_EEL && (mask & 2)))) return;
  const int sa0 = sp[sy].a0, sn = sp[sy].n;
  const int chunk = (sn + nz - 1) / nz;
  const int a0 = sa0 + blockIdx.z * chunk, a1 = min(sa0 + sn, a0 + chunk);
  const float tablast_e = sp[sy].tablast_e;
  double *acc = accs + (size_t)sy * ACC_STRIDE;
  // the LJ energies add the FP64 sums of the table's hi parts
  const bool hi = q == EP_ELJ || q == EP_ELJH;
  double s = 0;
  for (int t = a0 + threadIdx.x; t < a1; t += blockDim.x)
    s += (double)epart[(size_t)q * n + t] + (hi ? epart64[t] : 0.0);
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    s = warp_sum(s);
  }
  if (nz > 1) {
    if (threadIdx.x == 0) {
      part[(size_t)q * nz + blockIdx.z] = s;
      __threadfence();
      last = atomicAdd(done + q, 1u) == (unsigned)(nz - 1);
    }
    __syncthreads();
    if (!last) return;
    if (threadIdx.x == 0) {
      __threadfence();
      const volatile double *pv = part + (size_t)q * nz;
      s = 0;
      for (int z = 0; z < nz; z++) s += pv[z];
      done[q] = 0;
    }
  }
  if (threadIdx.x != 0) return;
  ep_to_acc(q, 0.5 * s, acc, tablast_e);
}

// CM3D's accumulator update for one reduced quantity (sum already halved)
__device__ __forceinline__ void ep_to_acc(int q, double s, double *acc, float tablast_e) {
  switch (q) {
    case EP_ELJ: atomicAdd(acc + ACC_SPOTL, s); break;
    case EP_ELJH: atomicAdd(acc + ACC_SPOTHL, s); break;
    case EP_VL0: atomicAdd(acc + ACC_SPRSLT + 0, -s); atomicAdd(acc + ACC_SPRSL, -s); break;
    case EP_VL1: atomicAdd(acc + ACC_SPRSLT + 1, -s); break;
    case EP_VL2: atomicAdd(acc + ACC_SPRSLT + 2, -s); break;
    case EP_VL4: atomicAdd(acc + ACC_SPRSLT + 4, -s); atomicAdd(acc + ACC_SPRSL, -s); break;
    case EP_VL5: atomicAdd(acc + ACC_SPRSLT + 5, -s); break;
    case EP_VL8: atomicAdd(acc + ACC_SPRSLT + 8, -s); atomicAdd(acc + ACC_SPRSL, -s); break;
    case EP_EEL: atomicAdd(acc + ACC_SPOTE, s); atomicAdd(acc + ACC_SPOTHE, s); break;
    case EP_QQ: atomicAdd(acc + ACC_SPOTHE, -(double)tablast_e * s); break;
    case EP_VE0: atomicAdd(acc + ACC_SPRSET + 0, -s); atomicAdd(acc + ACC_SPRSE, -s); break;
    case EP_VE1: atomicAdd(acc + ACC_SPRSET + 1, -s); break;
    case EP_VE2: atomicAdd(acc + ACC_SPRSET + 2, -s); break;
    case EP_VE4: atomicAdd(acc + ACC_SPRSET + 4, -s); atomicAdd(acc + ACC_SPRSE, -s); break;
    case EP_VE5: atomicAdd(acc + ACC_SPRSET + 5, -s); break;
    case EP_VE8: atomicAdd(acc + ACC_SPRSET + 8, -s); atomicAdd(acc + ACC_SPRSE, -s); break;
  }
}

// A batch's energy sums: one block per system adds up all its quantities in
// one pass over its atoms (every quantity in a fixed order, as k_ereduce),
// instead of a block per (quantity, system).
constexpr int ERS_THREADS = 256;

__global__ void __launch_bounds__(ERS_THREADS) k_ereduce_sys(int n, int mask, const SysP *__restrict__ sp,
                                                              const float *__restrict__ epart,
                                                              const double *__restrict__ epart64,
                                                              double *__restrict__ accs, const int *__restrict__ gs,
                                                              const int *__restrict__ skip = nullptr) {
  if (gated_off(gs, 0)) return;
  if (skip && skip[blockIdx.x]) return;                  // a compact system: its own reduction
  __shared__ double red[EP_COUNT][ERS_THREADS / 32];
  const int sy = blockIdx.x;
  const int a0 = sp[sy].a0, a1 = a0 + sp[sy].n;
  const int q0 = (mask & 1) ? 0 : EP_EEL;
  const int q1 = (mask & 2) && sp[sy].coul >= 0 ? EP_COUNT : EP_EEL;
  double s[EP_COUNT];
#pragma unroll
  for (int q = 0; q < EP_COUNT; q++) s[q] = 0.0;
  // (two atoms' loads in flight per thread: a large system's block is the
  // longest)
#pragma unroll 2
  for (int t = a0 + threadIdx.x; t < a1; t += blockDim.x) {
    const double h = (mask & 1) ? epart64[t] : 0.0;
#pragma unroll
    for (int q = 0; q < EP_COUNT; q++)
      if (q >= q0 && q < q1) s[q] += (double)epart[(size_t)q * n + t] + ((q == EP_ELJ || q == EP_ELJH) ? h : 0.0);
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < EP_COUNT; q++) {
    const double v = warp_sum(s[q]);
    if (lane == 0) red[q][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < EP_COUNT) {
    const int q = threadIdx.x;
    if (q < q0 || q >= q1) return;
    double v = 0.0;
    for (int k = 0; k < ERS_THREADS / 32; k++) v += red[q][k];
    ep_to_acc(q, 0.5 * v, accs + (size_t)sy * ACC_STRIDE, sp[sy].tablast_e);
  }
}

// ------------------------------------------------------------------ host
constexpr int EREDUCE_MAX_Z = 64;   // blocks per quantity for one large system

// per-atom FP64 partials of the LJ energy's table hi parts, stored after the
// EP_COUNT FP32 rows of epart
static double *epart_hi(Ctx *c) { return reinterpret_cast<double *>(c->epart + (size_t)EP_COUNT * c->n); }

static size_t smem_bytes(Ctx *c, bool with_tables, int mask) {
  size_t nf4 = (8 * (size_t)c->ninter + 3) / 4, nm4 = ((size_t)c->ntypes * c->ntypes + 3) / 4;
  size_t b = (54 + nf4 + nm4) * sizeof(float4);
  if (with_tables) {
    b += (size_t)3 * c->ninter * c->ntable * sizeof(float4);
    if (mask & 2) b += (size_t)2 * c->ntable * sizeof(float4);
  }
  return b;
}

template <int TPA, bool SB, bool NS, bool BT, bool ST = false, bool T2 = false>
static void launch_t(Ctx *c, const MixedP &P, size_t smem, double *fout) {
  const int B = 256;
  auto kern = k_pair_mixed<TPA, SB, NS, BT, ST, T2>;
  // the shared-memory limit is a per-device attribute: set it for every
  // device this process launches on
  static unsigned long long attr_devs = 0;
  if (c->dev < 64 && !(attr_devs & (1ull << c->dev))) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_devs |= 1ull << c->dev;
  }
  // persistent grid: as many resident blocks as the SMs hold, no more than
  // the atoms need
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, B, smem);
  if (per_sm < 1) per_sm = 1;
  const long long nat = c->pair_gidx ? c->pair_ng : c->n;
  long long need = ST ? (long long)c->nsys_items : (nat * TPA + B - 1) / B;
  long long grid = (long long)c->num_sms * per_sm;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  kern<<<grid, B, smem, c->st>>>(P, c->xq, c->styp, c->cell_atoms, c->nlen, c->nbr_stride, c->nbr, c->shift,
                                 c->map, c->fcut, c->ftab_lj, c->ftab_el, c->sp, c->sys_of, fout, c->fxs, c->epart,
                                 epart_hi(c), c->stat, c->gate, c->sys_items, c->nsys_items, c->ftab_lj2,
                                 c->stage_ntypes, c->stage_ninter, c->pair_gidx, c->pair_ng);
}

template <bool SB, bool NS, bool BT, bool ST = false, bool T2 = false>
static int launch_tpa(Ctx *c, const MixedP &P, size_t smem, double *fout) {
  switch (c->tpa) {
    case 4: launch_t<4, SB, NS, BT, ST, T2>(c, P, smem, fout); break;
    case 8: launch_t<8, SB, NS, BT, ST, T2>(c, P, smem, fout); break;
    case 16: launch_t<16, SB, NS, BT, ST, T2>(c, P, smem, fout); break;
    case 32: launch_t<32, SB, NS, BT, ST, T2>(c, P, smem, fout); break;
    default: launch_t<8, SB, NS, BT, ST, T2>(c, P, smem, fout); break;
  }
  return CM3D_NB_OK;
}

// shared memory of the staged batch kernel: one system's parameters, sized
// for the largest system
static size_t stage_bytes(Ctx *c) {
  const size_t nm4 = ((size_t)c->stage_ntypes * c->stage_ntypes + 3) / 4;
  return (54 + nm4 + 2 * (size_t)c->stage_ninter + 2 * (size_t)c->stage_ninter * c->ntable + 2 * (size_t)c->ntable) *
         sizeof(float4);
}

// whether a batch's pair launch can stage each system's parameters: the full
// force level without the RESPA switch (the compact LJ knots hold no switch)
static bool stage_applies(Ctx *c, int iflg, bool ns) {
  return c->nsys > 1 && c->sys_items != nullptr && iflg == 1 && !ns;
}

// Windowed kernel for one system with >= 3 cells per axis: returns false
// (nothing launched) when it does not apply and the list-gather kernel runs.
// The window capacity is what shared memory leaves after the tables; an item
// whose 27 cells hold more atoms falls back to global loads inside the kernel.
constexpr size_t WIN_STATIC_SMEM = 1024;   // >= k_pair_win's static shared arrays (448 bytes)

template <int TPA, bool NS, bool EL>
static void launch_win_t(Ctx *c, const MixedP &P, const WinP &W, size_t smem, double *fout) {
  auto kern = k_pair_win<TPA, NS, EL>;
  // dynamic + static shared memory must fit the opt-in limit: the window
  // budget keeps WIN_STATIC_SMEM bytes for the kernel's static arrays
  static unsigned long long attr_devs = 0;
  if (c->dev < 64 && !(attr_devs & (1ull << c->dev))) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(c->smem_optin - WIN_STATIC_SMEM));
    attr_devs |= 1ull << c->dev;
  }
  int grid = W.nitems < c->num_sms ? W.nitems : c->num_sms;
  kern<<<grid, 512, smem, c->st>>>(P, W, c->xq, c->styp, c->cell_atoms, c->cell_start, c->nlen, c->nbr_stride,
                                   c->nbr, c->shift, c->map, c->fcut, c->ftab_lj, c->ftab_el, fout, c->fxs, c->epart,
                                   epart_hi(c), c->stat, c->gate);
}

template <int TPA>
static void launch_win_tpa(Ctx *c, const MixedP &P, const WinP &W, size_t smem, double *fout, bool ns, bool el) {
  if (ns) {
    if (el) launch_win_t<TPA, true, true>(c, P, W, smem, fout);
    else launch_win_t<TPA, true, false>(c, P, W, smem, fout);
  } else {
    if (el) launch_win_t<TPA, false, true>(c, P, W, smem, fout);
    else launch_win_t<TPA, false, false>(c, P, W, smem, fout);
  }
}

// whether the windowed kernel can run this context (shape only)
bool win_applies(Ctx *c) {
  return c->mode == CM3D_NB_MIXED && c->nsys == 1 && c->nc[0] >= 3 && c->nc[1] >= 3 && c->nc[2] >= 3 &&
         c->ntypes <= 65535;
}

static bool launch_win(Ctx *c, const MixedP &P, bool ns, double *fout) {
  if (!c->win_ok || !win_applies(c)) return false;
  const int mask = P.mask;
  size_t nf4 = (8 * (size_t)c->ninter + 3) / 4, nm4 = ((size_t)c->ntypes * c->ntypes + 3) / 4;
  size_t fixed = (54 + nf4 + nm4) * sizeof(float4);
  if (mask & 1) fixed += (size_t)3 * c->ninter * c->ntable * sizeof(float4);
  if (mask & 2) fixed += (size_t)2 * c->ntable * sizeof(float4);
  const size_t budget = c->smem_optin > WIN_STATIC_SMEM ? c->smem_optin - WIN_STATIC_SMEM : 0;
  if (budget <= fixed) return false;
  long long cap = (long long)((budget - fixed) / (sizeof(float4) + sizeof(unsigned short))) / 8 * 8;
  const double mean_window = 27.0 * (double)c->n / (double)c->ncells;
  if ((double)cap < 1.25 * mean_window) return false;
  if (cap > 65536) cap = 65536;
  WinP W;
  W.ncx = c->nc[0];
  W.ncy = c->nc[1];
  W.ncz = c->nc[2];
  W.cap = (int)cap;
  const int groups = 512 / c->tpa;
  const double per_cell = (double)c->n / (double)c->ncells;
  int rounds = (int)ceil(per_cell / groups);
  if (rounds < 1) rounds = 1;
  // about four items per block where the cells allow it (parts of one cell
  // restage its window, so no more than needed)
  int want = (4 * c->num_sms + c->ncells - 1) / c->ncells;
  W.nsplit = want < rounds ? want : rounds;
  if (W.nsplit < 1) W.nsplit = 1;
  W.nitems = c->ncells * W.nsplit;
  const size_t smem = fixed + (size_t)cap * (sizeof(float4) + sizeof(unsigned short));
  const bool el = (mask & 2) != 0;
  switch (c->tpa) {
    case 4: launch_win_tpa<4>(c, P, W, smem, fout, ns, el); break;
    case 16: launch_win_tpa<16>(c, P, W, smem, fout, ns, el); break;
    case 32: launch_win_tpa<32>(c, P, W, smem, fout, ns, el); break;
    default: launch_win_tpa<8>(c, P, W, smem, fout, ns, el); break;
  }
  return true;
}

// mixed mode: which bit0 LJ, bit1 charges; iflg 1 -> fxl (+fxs), 0 -> fxs
int mixed_pairs(Ctx *c, int iflg, int mask) {
  if (c->ncharge == 0) mask &= 1;
  if (c->ninter == 0) mask &= 2;
  if (!mask || !c->lists_built) return CM3D_NB_OK;
  MixedP P;
  P.n = c->n;
  P.ntypes = c->ntypes;
  P.ninter = c->ninter;
  P.ntable = c->ntable;
  P.iflg = iflg;
  P.mask = mask;
  P.rc2_el = (float)c->rmaxl_coul2;
  P.dx2c = (float)c->dx2coul;
  P.offc = (float)(c->rmins_coul2 * c->dx2coul);
  P.tablast_e = (float)c->tablast_e;
  for (int k = 0; k < 9; k++) {
    P.hF[k] = (float)c->hmat[k];
    P.hiF[k] = (float)c->hmati[k];
  }
  size_t full = smem_bytes(c, true, mask);
  P.tab_smem = full <= 160 * 1024;
  size_t smem = smem_bytes(c, P.tab_smem, mask);
  bool ns = iflg == 1 && (c->need_short || c->nres_lrf > 1);
  // boxes narrower than two list radii need the on-the-fly minimum image
  bool sb = false;
  for (int d = 0; d < 3; d++) {
    double w = 1.0 / sqrt(c->hmati[3 * d] * c->hmati[3 * d] + c->hmati[3 * d + 1] * c->hmati[3 * d + 1] +
                          c->hmati[3 * d + 2] * c->hmati[3 * d + 2]);
    if (w < 2.0 * c->rlist_max) sb = true;
  }
  double *fout = iflg == 1 ? c->fxl : c->fxs;
  const int B = 256;
  k_xq_update<<<grid_for(c->n, B), B, 0, c->st>>>(c->n, c->cell_atoms, c->pos, c->corner, c->q, c->xq,
                                                  c->gate);
  cudaEvent_t e0;
  tbegin(c, 0, &e0);
  if (cw_applies(c, iflg, ns)) {
    // one system with >= 3 cells per axis, full force level: the compact
    // window list (nb_cwin.cu) and its own energy sums
    c->pair_used = c->cw_batch && c->cw_row == CM3D_CS_LPA ? CM3D_NB_PAIR_COMPACT8 : CM3D_NB_PAIR_COMPACT;
    c->launches++;                                   // k_xq_update
    int rc = cw_pairs(c, mask, fout);
    if (rc) return rc;
    if (c->cw_batch && c->cw_ng > 0) {
      // a batch: the other systems' atoms in the gather kernel
      P.tab_smem = 0;
      c->pair_gidx = c->cw_gidx;
      c->pair_ng = c->cw_ng;
      launch_tpa<false, false, true, false, true>(c, P, 0, fout);
      c->pair_gidx = nullptr;
      c->pair_ng = 0;
      c->launches++;
      k_ereduce_sys<<<c->nsys, ERS_THREADS, 0, c->st>>>(c->n, mask, c->sp, c->epart, epart_hi(c), c->acc, c->gate,
                                                         c->cw_sys);
      c->launches++;
    }
    tend(c, 0, e0);
    CKL(c);
    return cw_ereduce(c, mask);
  }
  // one system with >= 3 cells per axis: staged 27-cell windows; anything
  // else (batches, coarse cell grids): the gather kernel
  c->pair_used = CM3D_NB_PAIR_WINDOW;
  if (launch_win(c, P, ns, fout)) {
  } else if (c->win_ok && stage_applies(c, iflg, ns)) {
    // several systems: a block copies the parameters and tables of the
    // system it works on into shared memory
    c->pair_used = CM3D_NB_PAIR_SYSTEM;
    P.tab_smem = 0;
    launch_tpa<false, false, true, true>(c, P, stage_bytes(c), fout);
  } else if ((c->pair_used = CM3D_NB_PAIR_GATHER), c->nsys > 1) {
    // several systems: per-system parameters and tables from global memory;
    // the full force without the switch reads the compact LJ table
    P.tab_smem = 0;
    if (ns) launch_tpa<false, true, true>(c, P, 0, fout);
    else if (iflg == 1) launch_tpa<false, false, true, false, true>(c, P, 0, fout);
    else launch_tpa<false, false, true>(c, P, 0, fout);
  } else if (sb) {
    if (ns) launch_tpa<true, true, false>(c, P, smem, fout);
    else launch_tpa<true, false, false>(c, P, smem, fout);
  } else {
    if (ns) launch_tpa<false, true, false>(c, P, smem, fout);
    else launch_tpa<false, false, false>(c, P, smem, fout);
  }
  tend(c, 0, e0);
  c->launches += 2;
  if (iflg == 1) {
    if (c->nsys > 1) {
      // a batch: one block per system, every quantity in one pass
      k_ereduce_sys<<<c->nsys, ERS_THREADS, 0, c->st>>>(c->n, mask, c->sp, c->epart, epart_hi(c), c->acc, c->gate);
    } else {
      // one large system: its atoms over several blocks per quantity
      const int nz = std::max(1, std::min(EREDUCE_MAX_Z, c->n / 8192));
      k_ereduce<<<dim3(EP_COUNT, 1, nz), 512, 0, c->st>>>(c->n, mask, c->sp, c->epart, epart_hi(c), c->acc,
                                                           c->ered, c->ered_done, c->gate);
    }
    c->launches++;
  }
  CKL(c);
  return CM3D_NB_OK;
}

// FP32 interpolation coefficients and the 27 cell shifts (mixed mode)
int pair_setup(Ctx *c) {
  if (c->mode != CM3D_NB_MIXED) return CM3D_NB_OK;
  const int nt = c->ntable, ni = c->ninter;
  std::vector<double> vt((size_t)ni * nt), dv((size_t)ni * nt), sw((size_t)ni * nt), cut(8 * (size_t)ni);
  if (ni > 0) {
    CK(cudaMemcpy(vt.data(), c->vtab, sizeof(double) * vt.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dv.data(), c->dvtab, sizeof(double) * dv.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(sw.data(), c->switchs, sizeof(double) * sw.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(cut.data(), c->icut, sizeof(double) * cut.size(), cudaMemcpyDeviceToHost));
  }
  auto coef = [](const double *t, int k, double &f0, double &a, double &b) {
    if (k < 1) k = 1;
    f0 = t[k];
    a = 0.5 * (t[k + 1] - t[k - 1]);
    b = 0.5 * (t[k - 1] - 2.0 * t[k] + t[k + 1]);
  };
  const int ncoul = c->ncoul > 0 ? c->ncoul : 1;
  std::vector<float4> tl((size_t)3 * ni * nt), te((size_t)2 * nt * ncoul);
  for (int in = 0; in < ni; in++) {
    for (int k = 0; k < nt; k++) {
      double d0 = 0, da = 0, db = 0, v0 = 0, va = 0, vb = 0, s0 = 0, sa = 0, sb = 0;
      if (k >= 1 && k <= nt - 2) {
        coef(&dv[(size_t)in * nt], k, d0, da, db);
        coef(&vt[(size_t)in * nt], k, v0, va, vb);
        coef(&sw[(size_t)in * nt], k, s0, sa, sb);
      }
      size_t b = 3 * ((size_t)in * nt + k);
      tl[b] = make_float4((float)d0, (float)da, (float)db, (float)v0);
      tl[b + 1] = make_float4((float)va, (float)vb, (float)s0, (float)sa);
      // v0 as hi + lo: the kernel sums the hi parts of the LJ energy in FP64
      tl[b + 2] = make_float4((float)sb, (float)(v0 - (double)(float)v0), 0.f, 0.f);
    }
  }
  if (c->ncharge > 0) {
    // one erfc table per charged system (back to back, ntable each)
    std::vector<double> ct((size_t)nt * c->ncoul), dct((size_t)nt * c->ncoul);
    CK(cudaMemcpy(ct.data(), c->coultab, sizeof(double) * ct.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dct.data(), c->dcoultab, sizeof(double) * dct.size(), cudaMemcpyDeviceToHost));
    for (int tb = 0; tb < c->ncoul; tb++)
      for (int k = 0; k < nt; k++) {
        double d0 = 0, da = 0, db = 0, v0 = 0, va = 0, vb = 0;
        if (k >= 1 && k <= nt - 2) {
          coef(dct.data() + (size_t)tb * nt, k, d0, da, db);
          coef(ct.data() + (size_t)tb * nt, k, v0, va, vb);
        }
        te[(size_t)2 * nt * tb + 2 * k] = make_float4((float)d0, (float)da, (float)db, (float)v0);
        te[(size_t)2 * nt * tb + 2 * k + 1] = make_float4((float)va, (float)vb, 0.f, 0.f);
      }
  }
  // per interaction, two float4: {rmaxl_cut2, rmins_cut2*dx2tab, dx2tab,
  // vtab[ntable-4]} {rminl_cut2, rmaxs_cut2, -, -}
  std::vector<float> fc(8 * (size_t)(ni > 0 ? ni : 1), 0.f);
  for (int in = 0; in < ni; in++) {
    const double *q = &cut[8 * (size_t)in];
    fc[8 * in + 0] = (float)q[2];
    fc[8 * in + 1] = (float)(q[1] * q[6]);
    fc[8 * in + 2] = (float)q[6];
    fc[8 * in + 3] = (float)q[7];
    fc[8 * in + 4] = (float)q[3];
    fc[8 * in + 5] = (float)q[0];
  }
  CK(cudaMalloc(&c->ftab_lj, sizeof(float4) * (tl.size() > 0 ? tl.size() : 1)));
  CK(cudaMalloc(&c->ftab_el, sizeof(float4) * te.size()));
  CK(cudaMalloc(&c->fcut, sizeof(float) * fc.size()));
  if (!tl.empty()) CK(cudaMemcpy(c->ftab_lj, tl.data(), sizeof(float4) * tl.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->ftab_el, te.data(), sizeof(float4) * te.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->fcut, fc.data(), sizeof(float) * fc.size(), cudaMemcpyHostToDevice));
  // (the 27 cell shifts H k / nc are set up with the cell grid, list_setup)
  CK(cudaMalloc(&c->epart, (sizeof(float) * EP_COUNT + sizeof(double)) * (size_t)c->n));
  CK(cudaMalloc(&c->ered, sizeof(double) * EP_COUNT * EREDUCE_MAX_Z));
  CK(cudaMalloc(&c->ered_done, sizeof(unsigned) * EP_COUNT));
  CK(cudaMemset(c->ered_done, 0, sizeof(unsigned) * EP_COUNT));
  if (c->nsys > 1) {
    // work items of the staged batch kernel: every system in parts of at most
    // SYS_PART atoms, largest system first; staging applies while the largest
    // system fits in shared memory next to two more blocks on the SM
    int mt = 0, mi = 0;
    for (int sy = 0; sy < c->nsys; sy++) {
      mt = std::max(mt, c->h_sp[sy].ntypes);
      mi = std::max(mi, c->h_sp[sy].ninter);
    }
    c->stage_ntypes = mt;
    c->stage_ninter = mi;
    if (stage_bytes(c) <= c->smem_optin / 2 - 1024) {
      std::vector<int> order(c->nsys);
      for (int sy = 0; sy < c->nsys; sy++) order[sy] = sy;
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return c->h_sp[a].n > c->h_sp[b].n; });
      std::vector<int4> items;
      for (int sy : order) {
        const SysP &S = c->h_sp[sy];
        for (int a = 0; a < S.n; a += SYS_PART)
          items.push_back(make_int4(sy, S.a0 + a, S.a0 + std::min(S.n, a + SYS_PART), 0));
      }
      CK(cudaMalloc(&c->sys_items, sizeof(int4) * items.size()));
      CK(cudaMemcpy(c->sys_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice));
      c->nsys_items = (int)items.size();
    }
    // compact LJ coefficients for a batch's full force without the switch:
    // {d0, dA, dB, v0 hi} {vA, vB, v0 lo, 0}
    std::vector<float4> tl2((size_t)2 * (ni > 0 ? ni : 1) * nt, make_float4(0.f, 0.f, 0.f, 0.f));
    for (size_t k = 0; k < (size_t)ni * nt; k++) {
      tl2[2 * k] = tl[3 * k];
      tl2[2 * k + 1] = make_float4(tl[3 * k + 1].x, tl[3 * k + 1].y, tl[3 * k + 2].y, 0.f);
    }
    CK(cudaMalloc(&c->ftab_lj2, sizeof(float4) * tl2.size()));
    CK(cudaMemcpy(c->ftab_lj2, tl2.data(), sizeof(float4) * tl2.size(), cudaMemcpyHostToDevice));
  }
  if (c->tpa == 0) {
    // 8 lanes per atom: a group reads a full 32-byte sector of the list; more
    // lanes only for systems too small to fill the GPU
    long long want = (long long)c->num_sms * 1024;
    int tpa = 8;
    while (tpa < 32 && (long long)c->n * tpa < want) tpa *= 2;
    c->tpa = tpa;
  }
  return CM3D_NB_OK;
}

int pair_forces(Ctx *c, int iflg, int which) {
  if (c->mode == CM3D_NB_PLAIN_FP64) {
    if (which & 1) {
      int rc = plain_pairs(c, iflg, 0);
      if (rc) return rc;
    }
    if (which & 2) return plain_pairs(c, iflg, 1);
    return CM3D_NB_OK;
  }
  return mixed_pairs(c, iflg, which);
}

}  // namespace cm3d
