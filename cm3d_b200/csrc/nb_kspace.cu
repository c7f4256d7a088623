// nb_kspace.cu -- Ewald reciprocal space: fk_ewald (energy/inter/md_ewald.c:185-361)
// and its getvewald totals (md_ewald.c:336-348, 364-380).
//
// CM3D's k set (ewald_setup, md_ewald.c:93-114) comes in rows of constant
// (ka, kb) with consecutive kc; fk_ewald seeds cos/sin(k.r) at the start of
// every row and advances along kc by a complex multiply with
// exp(i 2 pi s_c) (md_ewald.c:239-280).  Both engines keep that structure:
//
//   k_sfac_*   structure factors: a block owns a tile of charged atoms and a
//              chunk of rows; every thread carries A atoms' phases through the
//              row, the per-k sums are reduced across the warp and then across
//              the block in FP64 and written as per-tile partials
//   k_sred     sums the tiles in FP64 (fixed order: deterministic), forms
//              preg, prep, the energy and the virial tensor of every k and the
//              force coefficients A(k) = 2 preg S(k)
//   k_kforce_* per atom, the sum over all k of k (Re A sin - Im A cos),
//              accumulated per row in FP32 (mixed) and across rows in FP64
//
// Mixed mode forms every phase from fixed-point fractional coordinates:
// s = H^-1 r is taken in FP64, its fractional part stored as a 32-bit
// integer, and ka*u0 + kb*u1 + kc*u2 evaluated in wrapping 32-bit integer
// arithmetic -- an exact phase modulo 2 pi whatever the size of k.r -- so
// the only FP32 error is that of the sin/cos of a number in [-pi, pi) and of
// the recurrence along one row.  The plain mode does everything in FP64 with
// CM3D's expressions (rk = x aka + y akb + z akc, md_ewald.c:264).
#include <math.h>

#include <mutex>

#include "nb_common.cuh"

namespace cm3d {

constexpr int KS_THREADS = 256;
constexpr int KS_A = 8;            // atoms per thread, structure factors
constexpr int KF_A = 2;            // atoms per thread, forces
constexpr int MAX_ROWLEN = 128;    // 2 kmax + 1 <= 128
// A batch whose every system has at most KS_SMALL charges (small molecules
// with a large k set) runs the structure factors and forces with one warp
// per block and one atom per thread: the 256 x 8 atom tiles would leave all
// but a few lanes idle.  For such systems both tilings hold each atom in the
// same lane of warp 0 and add only exact zeros besides, so the results are
// bit for bit the same.
constexpr int KS_SMALL = 32;

// ------------------------------------------------------------ mixed mode
// BATCH = true (every kernel below): the context holds several systems and
// each tile / k / atom takes its box, rows and tiles from its system's SysP;
// BATCH = false: one system described by the scalar arguments.
template <bool BATCH>
__global__ void k_kprep(int nq, const int *__restrict__ icharge, int n, const double *__restrict__ pos,
                        const double *__restrict__ q, const double *__restrict__ hmati_one,
                        const SysP *__restrict__ sp, const int *__restrict__ sys_of, uint4 *__restrict__ kfrac,
                        double4 *__restrict__ kposd, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  int jq = blockIdx.x * blockDim.x + threadIdx.x;
  if (jq >= nq) return;
  int i = icharge[jq];
  const double *hmati = BATCH ? sp[sys_of[i]].hi : hmati_one;
  double x = pos[i], y = pos[n + i], z = pos[2 * n + i];
  const double fact = sqrt(4.0 * M_PI);   // md_ewald.c:202
  double tq = q[i] * fact;
  unsigned u[3];
  for (int d = 0; d < 3; d++) {
    double s = x * hmati[3 * d] + y * hmati[3 * d + 1] + z * hmati[3 * d + 2];
    double f = s - floor(s);
    unsigned long long w = (unsigned long long)(f * 4294967296.0);
    u[d] = (unsigned)(w & 0xffffffffull);
  }
  if (kfrac) kfrac[jq] = make_uint4(u[0], u[1], u[2], __float_as_uint((float)tq));
  if (kposd) kposd[jq] = make_double4(x, y, z, tq);
}

// One step of the phase recursion along kc for two atoms at once, in packed
// FP32 (sm_100's two-wide FMA and multiply): per element the same roundings
// as the scalar c' = fma(c, cs, -(s sn)), s' = fma(s, cs, c sn), so a
// system's phases do not depend on which form ran (nsn = -sn, exact).
__device__ __forceinline__ void rot2(float2 &c, float2 &s, float2 cs, float2 sn, float2 nsn) {
  const float2 cn = __ffma2_rn(c, cs, __fmul2_rn(s, nsn));
  const float2 snn = __ffma2_rn(s, cs, __fmul2_rn(c, sn));
  c = cn;
  s = snn;
}

__device__ __forceinline__ float phase_rad(unsigned phi) {
  // (int)phi / 2^32 of a turn, in [-pi, pi)
  return (float)(int)phi * 1.4629180792671596e-09f;   // 2 pi / 2^32
}

template <bool BATCH, int A = KS_A>
__global__ void __launch_bounds__(KS_THREADS, 2) k_sfac_mixed(int nq, const uint4 *__restrict__ kfrac, int nrows,
                                                           const int4 *__restrict__ rows,
                                                           const int *__restrict__ row_k0, int rows_per_block,
                                                           int ktot, double2 *__restrict__ spart,
                                                           const SysP *__restrict__ sp,
                                                           const int *__restrict__ tile_sys,
                                                           const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  __shared__ float2 red[KS_THREADS / 32][MAX_ROWLEN];
  // this block's atoms [abase, aend), rows [rbeg, rend) and partial-S(k) base
  int abase = blockIdx.x * (blockDim.x * A), aend = nq, rbeg = 0, rend = nrows;
  long long sbase = (long long)blockIdx.x * ktot;
  if (BATCH) {
    const SysP &S = sp[tile_sys[blockIdx.x]];
    const int lt = blockIdx.x - S.ktile0;
    abase = S.q0 + lt * (blockDim.x * A);
    aend = S.q0 + S.nq;
    rbeg = S.krow0;
    rend = S.krow0 + S.nrows;
    sbase = S.spart0 + (long long)lt * S.ktot - S.kk0;
  }
  const int r0 = rbeg + blockIdx.y * rows_per_block;
  const int r1 = min(rend, r0 + rows_per_block);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned u0[A], u1[A], u2[A];
  float tq[A], cs[A], sn[A];
#pragma unroll
  for (int m = 0; m < A; m++) {
    int a = abase + m * blockDim.x + threadIdx.x;
    if (a < aend) {
      uint4 v = kfrac[a];
      u0[m] = v.x; u1[m] = v.y; u2[m] = v.z;
      tq[m] = __uint_as_float(v.w);
      // step exp(i 2 pi s_c), accurately (it is applied up to 2 kmax times)
      sincospif((float)(int)v.z * 4.656612873077393e-10f, &sn[m], &cs[m]);
    } else {
      u0[m] = u1[m] = u2[m] = 0;
      tq[m] = 0.f; cs[m] = 1.f; sn[m] = 0.f;
    }
  }
  // atoms in pairs for the packed phase recursion (A even)
  constexpr int H = A / 2 > 0 ? A / 2 : 1;
  float2 cs2[H], sn2[H], nsn2[H];
  if constexpr (A % 2 == 0) {
#pragma unroll
    for (int j = 0; j < A / 2; j++) {
      cs2[j] = make_float2(cs[2 * j], cs[2 * j + 1]);
      sn2[j] = make_float2(sn[2 * j], sn[2 * j + 1]);
      nsn2[j] = make_float2(-sn[2 * j], -sn[2 * j + 1]);
    }
  }
  for (int r = r0; r < r1; r++) {
    const int4 row = rows[r];
    const int len = row.w;
    float c[A], s[A];
#pragma unroll
    for (int m = 0; m < A; m++) {
      unsigned phi = (unsigned)row.x * u0[m] + (unsigned)row.y * u1[m] + (unsigned)row.z * u2[m];
      __sincosf(phase_rad(phi), &s[m], &c[m]);
    }
    float2 c2[H], s2[H];
    if constexpr (A % 2 == 0) {
#pragma unroll
      for (int j = 0; j < A / 2; j++) {
        c2[j] = make_float2(c[2 * j], c[2 * j + 1]);
        s2[j] = make_float2(s[2 * j], s[2 * j + 1]);
      }
    }
    if constexpr (A % 2 == 0) {
      // k in groups of KG: each thread's KG (sr, si) pairs, then one
      // transposing warp reduction -- lane l ends with value l (k = l / 2,
      // component l % 2) after the same additions, in the same tree, as a
      // butterfly sum of each value (warp_sum): the same bits, a sixteenth
      // of the shuffles
      constexpr int KG = 16;
      float *redf = reinterpret_cast<float *>(red[w]);
      for (int kb = 0; kb < len; kb += KG) {
        float v[2 * KG];
#pragma unroll
        for (int q = 0; q < KG; q++) {
          float sr = 0.f, si = 0.f;
          if (kb + q < len) {
            // the sums in atom order; the recursion two atoms at a time
#pragma unroll
            for (int j = 0; j < A / 2; j++) {
              sr = fmaf(tq[2 * j], c2[j].x, sr);
              si = fmaf(tq[2 * j], s2[j].x, si);
              sr = fmaf(tq[2 * j + 1], c2[j].y, sr);
              si = fmaf(tq[2 * j + 1], s2[j].y, si);
              rot2(c2[j], s2[j], cs2[j], sn2[j], nsn2[j]);
            }
          }
          v[2 * q] = sr;
          v[2 * q + 1] = si;
        }
#pragma unroll
        for (int h = KG, o = 16; h >= 1; h >>= 1, o >>= 1) {
          const bool hi = (lane & o) != 0;
#pragma unroll
          for (int i = 0; i < h; i++) {
            const float snd = hi ? v[i] : v[i + h];
            const float kp = hi ? v[i + h] : v[i];
            v[i] = kp + __shfl_xor_sync(0xffffffffu, snd, o);
          }
        }
        if (kb + (lane >> 1) < len) redf[2 * kb + lane] = v[0];
      }
    } else {
    for (int kk = 0; kk < len; kk++) {
      float sr = 0.f, si = 0.f;
      {
#pragma unroll
        for (int m = 0; m < A; m++) {
          sr = fmaf(tq[m], c[m], sr);
          si = fmaf(tq[m], s[m], si);
          // explicit roundings: every instantiation (tile shape) rotates
          // the phase with the same operations, so a system's sums do not
          // depend on the tiling the compiler saw
          float cn = fmaf(c[m], cs[m], -__fmul_rn(s[m], sn[m]));
          float snn = fmaf(s[m], cs[m], __fmul_rn(c[m], sn[m]));
          c[m] = cn;
          s[m] = snn;
        }
      }
      sr = warp_sum(sr);
      si = warp_sum(si);
      if (lane == 0) red[w][kk] = make_float2(sr, si);
    }
    }
    __syncthreads();
    const int k0 = row_k0[r];
    for (int kk = threadIdx.x; kk < len; kk += blockDim.x) {
      double ar = 0, ai = 0;
#pragma unroll
      for (int q2 = 0; q2 < (int)(blockDim.x >> 5); q2++) {
        ar += red[q2][kk].x;
        ai += red[q2][kk].y;
      }
      spart[sbase + k0 + kk] = make_double2(ar, ai);
    }
    __syncthreads();
  }
}

// per-k totals; every k of CM3D's list is one thread (md_ewald.c:247-305).
// BATCH: exactly one k per thread (ktot = all systems' k-vectors), so that
// each thread's sums belong to one system.
template <bool BATCH>
__global__ void k_sred(int ktot, int ntiles, const double2 *__restrict__ spart, const int *__restrict__ ka,
                       const int *__restrict__ kb, const int *__restrict__ kc, const double *__restrict__ hmati_one,
                       double rvol_one, double falp2_one, double2 *__restrict__ sk, float2 *__restrict__ akf,
                       double2 *__restrict__ akd, double *__restrict__ acc, const SysP *__restrict__ sp,
                       const int *__restrict__ k_sys, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  double v[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double TPI = 2.0 * M_PI;
  int sys = -1;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ktot; k += gridDim.x * blockDim.x) {
    const double *hmati = hmati_one;
    double rvol = rvol_one, falp2 = falp2_one;
    int nt = ntiles, kstride = ktot;
    long long sb = k;
    if (BATCH) {
      sys = k_sys[k];
      const SysP &S = sp[sys];
      hmati = S.hi;
      rvol = S.rvol;
      falp2 = S.falp2;
      nt = S.ktiles;
      kstride = S.ktot;
      sb = S.spart0 + (k - S.kk0);
    }
    double sr = 0, si = 0;
    for (int t = 0; t < nt; t++) {
      double2 p = spart[sb + (long long)t * kstride];
      sr += p.x;
      si += p.y;
    }
    double six = TPI * ka[k], siy = TPI * kb[k], siz = TPI * kc[k];
    double aka = (six * hmati[0] + siy * hmati[3] + siz * hmati[6]);
    double akb = (six * hmati[1] + siy * hmati[4] + siz * hmati[7]);
    double akc = (six * hmati[2] + siy * hmati[5] + siz * hmati[8]);
    double g2 = aka * aka + akb * akb + akc * akc;
    double preg = exp(-g2 * falp2) * rvol / g2;
    double prep = -2. * preg * (g2 * falp2 + 1.) / g2;
    double smag = sr * sr + si * si;
    v[0] += preg * smag;
    v[1] += prep * smag * g2;
    double ps = prep * smag;
    v[2] += ps * aka * aka; v[3] += ps * akb * aka; v[4] += ps * akc * aka;
    v[5] += ps * aka * akb; v[6] += ps * akb * akb; v[7] += ps * akc * akb;
    v[8] += ps * aka * akc; v[9] += ps * akb * akc; v[10] += ps * akc * akc;
    sk[k] = make_double2(sr, si);
    if (akf) akf[k] = make_float2((float)(2. * preg * sr), (float)(2. * preg * si));
    if (akd) akd[k] = make_double2(2. * preg * sr, 2. * preg * si);
  }
  const int slots[11] = {ACC_VK, ACC_VP, ACC_VPT + 0, ACC_VPT + 1, ACC_VPT + 2, ACC_VPT + 3,
                         ACC_VPT + 4, ACC_VPT + 5, ACC_VPT + 6, ACC_VPT + 7, ACC_VPT + 8};
  if (BATCH) sys_acc<11>(v, sys, acc, slots);
  else block_acc<11>(v, acc, slots);
}

template <bool BATCH, int A = KF_A>
__global__ void __launch_bounds__(KS_THREADS) k_kforce_mixed(int nq, const uint4 *__restrict__ kfrac,
                                                             const int *__restrict__ icharge, int n, int nrows,
                                                             const int4 *__restrict__ rows,
                                                             const int *__restrict__ row_k0, int rows_per_split,
                                                             const float2 *__restrict__ akf, int ktot,
                                                             const double *__restrict__ hmati_one, int atomic,
                                                             double *__restrict__ fxl, double *__restrict__ part,
                                                             const SysP *__restrict__ sp,
                                                             const int *__restrict__ tile_sys,
                                                             const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  extern __shared__ float2 ak_s[];
  // this block's charged atoms [abase, aend), rows [r0, r1) and k range
  int r0, r1, kend, abase, aend;
  const double *hmati = hmati_one;
  if (BATCH) {
    const SysP &S = sp[tile_sys[blockIdx.x]];
    const int rps = (S.nrows + gridDim.y - 1) / gridDim.y;
    const int rend = S.krow0 + S.nrows;
    r0 = S.krow0 + blockIdx.y * rps;
    r1 = min(rend, r0 + rps);
    kend = r1 < rend ? (r1 > r0 ? row_k0[r1] : 0) : S.kk0 + S.ktot;
    abase = S.q0 + (blockIdx.x - S.ftile0) * (blockDim.x * A);
    aend = S.q0 + S.nq;
    hmati = S.hi;
  } else {
    r0 = blockIdx.y * rows_per_split;
    r1 = min(nrows, r0 + rows_per_split);
    kend = (r1 < nrows) ? row_k0[r1] : ktot;
    abase = blockIdx.x * (blockDim.x * A);
    aend = nq;
  }
  if (r0 >= r1) {
    // no rows for this split: its share of the partial forces is zero
    if (part)
      for (int m = 0; m < A; m++) {
        const int jq = abase + m * blockDim.x + threadIdx.x;
        if (jq < aend) {
          const size_t o = ((size_t)blockIdx.y * nq + jq) * 3;
          part[o] = part[o + 1] = part[o + 2] = 0.0;
        }
      }
    return;
  }
  const int kbase = row_k0[r0];
  for (int k = threadIdx.x; k < kend - kbase; k += blockDim.x) ak_s[k] = akf[kbase + k];
  __syncthreads();
  unsigned u0[A], u1[A], u2[A];
  float cs[A], sn[A], tq[A];
  double U0[A], U1[A], U2[A];
  int jq[A];
#pragma unroll
  for (int m = 0; m < A; m++) {
    jq[m] = abase + m * blockDim.x + threadIdx.x;
    U0[m] = U1[m] = U2[m] = 0.0;
    if (jq[m] < aend) {
      uint4 v = kfrac[jq[m]];
      u0[m] = v.x; u1[m] = v.y; u2[m] = v.z;
      tq[m] = __uint_as_float(v.w);
      sincospif((float)(int)v.z * 4.656612873077393e-10f, &sn[m], &cs[m]);
    } else {
      u0[m] = u1[m] = u2[m] = 0;
      tq[m] = 0.f; cs[m] = 1.f; sn[m] = 0.f;
    }
  }
  constexpr int H = A / 2 > 0 ? A / 2 : 1;
  float2 cs2[H], sn2[H], nsn2[H];
  if constexpr (A % 2 == 0) {
#pragma unroll
    for (int j = 0; j < A / 2; j++) {
      cs2[j] = make_float2(cs[2 * j], cs[2 * j + 1]);
      sn2[j] = make_float2(sn[2 * j], sn[2 * j + 1]);
      nsn2[j] = make_float2(-sn[2 * j], -sn[2 * j + 1]);
    }
  }
  for (int r = r0; r < r1; r++) {
    const int4 row = rows[r];
    const int len = row.w;
    const int kb0 = row_k0[r] - kbase;
    float c[A], s[A], W0[A], W1[A];
#pragma unroll
    for (int m = 0; m < A; m++) {
      unsigned phi = (unsigned)row.x * u0[m] + (unsigned)row.y * u1[m] + (unsigned)row.z * u2[m];
      __sincosf(phase_rad(phi), &s[m], &c[m]);
      W0[m] = W1[m] = 0.f;
    }
    float kcf = (float)row.z;
    if constexpr (A % 2 == 0) {
      // two atoms per packed operation; per element the roundings of the
      // scalar form below (wv = fma(a.x, s, -(a.y c)), W0 += wv, W1 += kc wv)
      float2 c2[A / 2], s2[A / 2], w02[A / 2], w12[A / 2];
#pragma unroll
      for (int j = 0; j < A / 2; j++) {
        c2[j] = make_float2(c[2 * j], c[2 * j + 1]);
        s2[j] = make_float2(s[2 * j], s[2 * j + 1]);
        w02[j] = make_float2(0.f, 0.f);
        w12[j] = make_float2(0.f, 0.f);
      }
      float2 kc2 = make_float2(kcf, kcf);
      const float2 one2 = make_float2(1.f, 1.f);
      for (int kk = 0; kk < len; kk++) {
        const float2 a = ak_s[kb0 + kk];
        const float2 ax2 = make_float2(a.x, a.x), nay2 = make_float2(-a.y, -a.y);
#pragma unroll
        for (int j = 0; j < A / 2; j++) {
          const float2 wv = __ffma2_rn(ax2, s2[j], __fmul2_rn(nay2, c2[j]));
          w02[j] = __fadd2_rn(w02[j], wv);
          w12[j] = __ffma2_rn(kc2, wv, w12[j]);
          rot2(c2[j], s2[j], cs2[j], sn2[j], nsn2[j]);
        }
        kc2 = __fadd2_rn(kc2, one2);
      }
#pragma unroll
      for (int j = 0; j < A / 2; j++) {
        W0[2 * j] = w02[j].x;
        W0[2 * j + 1] = w02[j].y;
        W1[2 * j] = w12[j].x;
        W1[2 * j + 1] = w12[j].y;
      }
    } else {
      for (int kk = 0; kk < len; kk++) {
        const float2 a = ak_s[kb0 + kk];
#pragma unroll
        for (int m = 0; m < A; m++) {
          float wv = fmaf(a.x, s[m], -__fmul_rn(a.y, c[m]));
          W0[m] = __fadd_rn(W0[m], wv);
          W1[m] = fmaf(kcf, wv, W1[m]);
          // explicit roundings: every instantiation (tile shape) rotates
          // the phase with the same operations, so a system's sums do not
          // depend on the tiling the compiler saw
          float cn = fmaf(c[m], cs[m], -__fmul_rn(s[m], sn[m]));
          float snn = fmaf(s[m], cs[m], __fmul_rn(c[m], sn[m]));
          c[m] = cn;
          s[m] = snn;
        }
        kcf += 1.f;
      }
    }
#pragma unroll
    for (int m = 0; m < A; m++) {
      U0[m] = fma((double)row.x, (double)W0[m], U0[m]);
      U1[m] = fma((double)row.y, (double)W0[m], U1[m]);
      U2[m] = __dadd_rn(U2[m], (double)W1[m]);
    }
  }
  const double TPI = 2.0 * M_PI;
#pragma unroll
  for (int m = 0; m < A; m++) {
    if (jq[m] >= aend) continue;
    int i = icharge[jq[m]];
    double t = TPI * (double)tq[m];
    // F = tq 2 pi H^-T U  (k = 2 pi H^-T n, md_ewald.c:248-251)
    double fx = __dmul_rn(t, fma(hmati[6], U2[m], fma(hmati[3], U1[m], __dmul_rn(hmati[0], U0[m]))));
    double fy = __dmul_rn(t, fma(hmati[7], U2[m], fma(hmati[4], U1[m], __dmul_rn(hmati[1], U0[m]))));
    double fz = __dmul_rn(t, fma(hmati[8], U2[m], fma(hmati[5], U1[m], __dmul_rn(hmati[2], U0[m]))));
    if (part) {
      // one partial per row split, summed in a fixed order by k_kforce_sum
      const size_t o = ((size_t)blockIdx.y * nq + jq[m]) * 3;
      part[o] = fx;
      part[o + 1] = fy;
      part[o + 2] = fz;
    } else if (atomic) {
      atomicAdd(fxl + i, fx);
      atomicAdd(fxl + n + i, fy);
      atomicAdd(fxl + 2 * n + i, fz);
    } else {
      fxl[i] += fx;
      fxl[n + i] += fy;
      fxl[2 * n + i] += fz;
    }
  }
}

// the row splits' partial reciprocal forces of every charged atom, summed in
// split order (deterministic: the same result whatever else the device runs)
__global__ void k_kforce_sum(int nq, int nsplit, const double *__restrict__ part, const int *__restrict__ icharge,
                             int n, double *__restrict__ fxl, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  const int jq = blockIdx.x * blockDim.x + threadIdx.x;
  if (jq >= nq) return;
  double fx = 0, fy = 0, fz = 0;
  for (int y = 0; y < nsplit; y++) {
    const size_t o = ((size_t)y * nq + jq) * 3;
    fx += part[o];
    fy += part[o + 1];
    fz += part[o + 2];
  }
  const int i = icharge[jq];
  fxl[i] += fx;
  fxl[n + i] += fy;
  fxl[2 * n + i] += fz;
}

// ------------------------------------------------------------ plain FP64
__global__ void __launch_bounds__(KS_THREADS) k_sfac_plain(int nq, const double4 *__restrict__ kp, int nrows,
                                                           const int4 *__restrict__ rows,
                                                           const int *__restrict__ row_k0, int rows_per_block,
                                                           int ktot, const double *__restrict__ hmati,
                                                           double2 *__restrict__ spart,
                                                           const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  __shared__ double2 red[KS_THREADS / 32][MAX_ROWLEN];
  const int tile = blockIdx.x;
  const int r0 = blockIdx.y * rows_per_block;
  const int r1 = min(nrows, r0 + rows_per_block);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const double TPI = 2.0 * M_PI;
  const int a = tile * KS_THREADS + threadIdx.x;
  double4 p = a < nq ? kp[a] : make_double4(0, 0, 0, 0);
  double akc0 = (p.x * hmati[6] + p.y * hmati[7] + p.z * hmati[8]) * TPI;   // md_ewald.c:240
  double cs = cos(akc0), sn = sin(akc0);
  for (int r = r0; r < r1; r++) {
    const int4 row = rows[r];
    double six = TPI * row.x, siy = TPI * row.y, siz = TPI * row.z;
    double aka = (six * hmati[0] + siy * hmati[3] + siz * hmati[6]);
    double akb = (six * hmati[1] + siy * hmati[4] + siz * hmati[7]);
    double akc = (six * hmati[2] + siy * hmati[5] + siz * hmati[8]);
    double rk = (p.x * aka + p.y * akb + p.z * akc);
    double c = cos(rk), s = sin(rk);
    for (int kk = 0; kk < row.w; kk++) {
      double sr = warp_sum(p.w * c), si = warp_sum(p.w * s);
      if (lane == 0) red[w][kk] = make_double2(sr, si);
      double cn = c * cs - s * sn;
      double snn = s * cs + c * sn;
      c = cn;
      s = snn;
    }
    __syncthreads();
    const int k0 = row_k0[r];
    for (int kk = threadIdx.x; kk < row.w; kk += blockDim.x) {
      double ar = 0, ai = 0;
      for (int q2 = 0; q2 < KS_THREADS / 32; q2++) {
        ar += red[q2][kk].x;
        ai += red[q2][kk].y;
      }
      spart[(size_t)tile * ktot + k0 + kk] = make_double2(ar, ai);
    }
    __syncthreads();
  }
}

__global__ void k_kforce_plain(int nq, const double4 *__restrict__ kp, const int *__restrict__ icharge, int n,
                               int nrows, const int4 *__restrict__ rows, const int *__restrict__ row_k0,
                               int rows_per_split, const double2 *__restrict__ akd, int ktot,
                               const double *__restrict__ hmati, int atomic, double *__restrict__ fxl,
                               const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  const int jq = blockIdx.x * blockDim.x + threadIdx.x;
  const int r0 = blockIdx.y * rows_per_split;
  const int r1 = min(nrows, r0 + rows_per_split);
  if (jq >= nq || r0 >= r1) return;
  const double TPI = 2.0 * M_PI;
  const double4 p = kp[jq];
  const double akc0 = (p.x * hmati[6] + p.y * hmati[7] + p.z * hmati[8]) * TPI;   // md_ewald.c:240
  const double cs = cos(akc0), sn = sin(akc0);
  double fx = 0, fy = 0, fz = 0;
  for (int r = r0; r < r1; r++) {
    const int4 row = rows[r];
    const double six = TPI * row.x, siy = TPI * row.y;
    double c = 1.0, s = 0.0;
    for (int kk = 0; kk < row.w; kk++) {
      const double siz = TPI * (row.z + kk);
      const double aka = (six * hmati[0] + siy * hmati[3] + siz * hmati[6]);
      const double akb = (six * hmati[1] + siy * hmati[4] + siz * hmati[7]);
      const double akc = (six * hmati[2] + siy * hmati[5] + siz * hmati[8]);
      if (kk == 0) {
        // seed at the start of every row (md_ewald.c:261-267)
        const double rk = (p.x * aka + p.y * akb + p.z * akc);
        c = cos(rk);
        s = sin(rk);
      } else {
        // cos(a+b), sin(a+b) recursion along kc (md_ewald.c:273-278)
        const double cn = c * cs - s * sn, snn = s * cs + c * sn;
        c = cn;
        s = snn;
      }
      const double2 a = akd[row_k0[r] + kk];
      const double wv = a.x * s - a.y * c;
      fx += aka * wv;
      fy += akb * wv;
      fz += akc * wv;
    }
  }
  const int i = icharge[jq];
  fx *= p.w;
  fy *= p.w;
  fz *= p.w;
  if (atomic) {
    atomicAdd(fxl + i, fx);
    atomicAdd(fxl + n + i, fy);
    atomicAdd(fxl + 2 * n + i, fz);
  } else {
    fxl[i] += fx;
    fxl[n + i] += fy;
    fxl[2 * n + i] += fz;
  }
}

// ------------------------------------------------------------------ host
// k rows, tiles and partial-S(k) layout of every system (SysP fields q0 ..
// spart0), all systems' rows / k-vectors concatenated
int kspace_setup(Ctx *c) {
  std::vector<int4> rows;
  std::vector<int> k0, ka, kb, kc, k_sys, ktile_sys, ftile_sys;
  const bool mixed = c->mode == CM3D_NB_MIXED;
  bool small = mixed && c->nsys > 1;
  for (int sy = 0; sy < c->nsys && small; sy++) small = c->hs[sy].ncharge <= KS_SMALL;
  c->ks_small = small;
  const int per_tile = small ? KS_SMALL : mixed ? KS_THREADS * KS_A : KS_THREADS;
  const int per_ftile = small ? KS_SMALL : mixed ? KS_THREADS * KF_A : KS_THREADS;
  int qoff = 0, nrows_max = 0;
  long long spart_tot = 0;
  for (int sy = 0; sy < c->nsys; sy++) {
    SysP &P = c->h_sp[sy];
    const SysH &H = c->hs[sy];
    P.q0 = qoff;
    P.nq = H.ncharge;
    qoff += H.ncharge;
    P.krow0 = (int)rows.size();
    P.kk0 = (int)ka.size();
    P.ktot = H.ncharge > 0 ? H.ktot : 0;
    // CM3D's k set (ewald_setup, md_ewald.c:93-114) as rows of constant
    // (ka, kb) and consecutive kc
    for (int k = 0; k < P.ktot;) {
      int e = k + 1;
      while (e < P.ktot && H.ka[e] == H.ka[k] && H.kb[e] == H.kb[k] && H.kc[e] == H.kc[e - 1] + 1 &&
             e - k < MAX_ROWLEN)
        e++;
      rows.push_back(make_int4(H.ka[k], H.kb[k], H.kc[k], e - k));
      k0.push_back(P.kk0 + k);
      k = e;
    }
    for (int k = 0; k < P.ktot; k++) {
      ka.push_back(H.ka[k]);
      kb.push_back(H.kb[k]);
      kc.push_back(H.kc[k]);
      k_sys.push_back(sy);
    }
    P.nrows = (int)rows.size() - P.krow0;
    nrows_max = std::max(nrows_max, P.nrows);
    P.ktile0 = (int)ktile_sys.size();
    P.ktiles = P.ktot > 0 ? (P.nq + per_tile - 1) / per_tile : 0;
    for (int t = 0; t < P.ktiles; t++) ktile_sys.push_back(sy);
    P.ftile0 = (int)ftile_sys.size();
    P.ftiles = P.ktot > 0 ? (P.nq + per_ftile - 1) / per_ftile : 0;
    for (int t = 0; t < P.ftiles; t++) ftile_sys.push_back(sy);
    P.spart0 = spart_tot;
    spart_tot += (long long)P.ktiles * P.ktot;
  }
  c->ktot = (int)ka.size();
  c->nrows = (int)rows.size();
  c->nrows_max = nrows_max;
  c->ktiles_tot = (int)ktile_sys.size();
  c->ftiles_tot = (int)ftile_sys.size();
  if (c->ncharge == 0 || c->ktot == 0) return CM3D_NB_OK;
  c->ks_tiles = c->h_sp[0].ktiles;
  c->ks_tile_atoms = per_tile;
  auto up = [&](int **dst, const std::vector<int> &v) -> int {
    CK(cudaMalloc(dst, sizeof(int) * (v.empty() ? 1 : v.size())));
    if (!v.empty()) CK(cudaMemcpy(*dst, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice));
    return CM3D_NB_OK;
  };
  int rc;
  CK(cudaMalloc(&c->rows, sizeof(int4) * rows.size()));
  CK(cudaMemcpy(c->rows, rows.data(), sizeof(int4) * rows.size(), cudaMemcpyHostToDevice));
  if ((rc = up(&c->row_k0, k0)) || (rc = up(&c->ka_d, ka)) || (rc = up(&c->kb_d, kb)) || (rc = up(&c->kc_d, kc)) ||
      (rc = up(&c->k_sys, k_sys)) || (rc = up(&c->ktile_sys, ktile_sys)) || (rc = up(&c->ftile_sys, ftile_sys)))
    return rc;
  CK(cudaMalloc(&c->spart, sizeof(double2) * (size_t)(spart_tot > 0 ? spart_tot : 1)));
  CK(cudaMalloc(&c->sk, sizeof(double2) * (size_t)c->ktot));
  if (mixed) {
    CK(cudaMalloc(&c->akf, sizeof(float2) * (size_t)c->ktot));
    CK(cudaMalloc(&c->kfrac, sizeof(uint4) * (size_t)c->ncharge));
  } else {
    CK(cudaMalloc(&c->akd, sizeof(double2) * (size_t)c->ktot));
  }
  CK(cudaMalloc(&c->kposd, sizeof(double4) * (size_t)c->ncharge));
  // split the rows over enough blocks to fill the machine in the force pass
  int split = 1;
  while ((long long)c->ftiles_tot * split < (long long)c->num_sms * 4 && split < nrows_max) split *= 2;
  // every split's A(k) must fit in shared memory -- in 48 KB, so that four
  // or more blocks share an SM and hide each other's latency (a single split
  // of a large k set would leave one block per SM)
  for (;;) {
    size_t mx = 0;
    for (int sy = 0; sy < c->nsys; sy++) {
      const SysP &P = c->h_sp[sy];
      if (P.nrows == 0) continue;
      const int rps = (P.nrows + split - 1) / split;
      for (int r0 = 0; r0 < P.nrows; r0 += rps) {
        const int r1 = r0 + rps < P.nrows ? r0 + rps : P.nrows;
        const int kb1 = r1 < P.nrows ? k0[P.krow0 + r1] : P.kk0 + P.ktot;
        const size_t nk = (size_t)(kb1 - k0[P.krow0 + r0]);
        if (nk > mx) mx = nk;
      }
    }
    c->kf_smem = mx * sizeof(float2);
    if (c->kf_smem <= 48 * 1024 || split >= nrows_max) break;
    split *= 2;
  }
  if (split > nrows_max) split = nrows_max;
  c->kf_split = split;
  if (mixed) {
    // (also with one split: the forked k-space of a step writes partials)
    // zeroed once: the charged atoms of systems without k-vectors keep zero partials
    CK(cudaMalloc(&c->kf_part, sizeof(double) * 3 * (size_t)split * c->ncharge));
    CK(cudaMemset(c->kf_part, 0, sizeof(double) * 3 * (size_t)split * c->ncharge));
  }
  return CM3D_NB_OK;
}

// the force kernels' shared-memory limit, once per device
static void kforce_attr(int dev) {
  static unsigned long long done = 0;
  if (dev < 64 && (done & (1ull << dev))) return;
  cudaFuncSetAttribute(k_kforce_mixed<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_kforce_mixed<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_kforce_mixed<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (dev < 64) done |= 1ull << dev;
}

// several systems (mixed mode): every system's structure factors, totals
// and forces in one launch per stage
static int kspace_forces_batch(Ctx *c, cudaStream_t st, bool defer) {
  cudaEvent_t e0;
  tbegin(c, 1, &e0);
  k_kprep<true><<<grid_for(c->ncharge, 256), 256, 0, st>>>(c->ncharge, c->icharge, c->n, c->pos, c->q, nullptr,
                                                               c->sp, c->sys_of, c->kfrac, nullptr, c->gate);
  // enough row chunks per tile to fill the machine (one-warp blocks: 32
  // blocks per SM)
  const long long target = (long long)c->num_sms * (c->ks_small ? 32 : 4);
  int ych = 1;
  while ((long long)c->ktiles_tot * ych < target && ych < c->nrows_max) ych *= 2;
  const int rpb = (c->nrows_max + ych - 1) / ych;
  dim3 gsf(c->ktiles_tot, (c->nrows_max + rpb - 1) / rpb);
  if (c->ks_small)
    k_sfac_mixed<true, 1><<<gsf, KS_SMALL, 0, st>>>(c->ncharge, c->kfrac, 0, c->rows, c->row_k0, rpb, 0,
                                                       c->spart, c->sp, c->ktile_sys, c->gate);
  else
    k_sfac_mixed<true><<<gsf, KS_THREADS, 0, st>>>(c->ncharge, c->kfrac, 0, c->rows, c->row_k0, rpb, 0,
                                                      c->spart, c->sp, c->ktile_sys, c->gate);
  k_sred<true><<<grid_for(c->ktot, 256), 256, 0, st>>>(c->ktot, 0, c->spart, c->ka_d, c->kb_d, c->kc_d, nullptr,
                                                           0.0, 0.0, c->sk, c->akf, nullptr, c->acc, c->sp,
                                                           c->k_sys, c->gate);
  kforce_attr(c->dev);
  dim3 gf(c->ftiles_tot, c->kf_split);
  double *part = c->kf_split > 1 || defer ? c->kf_part : nullptr;
  if (c->ks_small)
    k_kforce_mixed<true, 1><<<gf, KS_SMALL, c->kf_smem, st>>>(c->ncharge, c->kfrac, c->icharge, c->n, 0,
                                                                 c->rows, c->row_k0, 0, c->akf, 0, nullptr, 0,
                                                                 c->fxl, part, c->sp, c->ftile_sys, c->gate);
  else
    k_kforce_mixed<true><<<gf, KS_THREADS, c->kf_smem, st>>>(c->ncharge, c->kfrac, c->icharge, c->n, 0,
                                                                 c->rows, c->row_k0, 0, c->akf, 0, nullptr, 0,
                                                                 c->fxl, part, c->sp, c->ftile_sys, c->gate);
  c->launches += 4;
  if (part && !defer) {
    k_kforce_sum<<<grid_for(c->ncharge, 256), 256, 0, st>>>(c->ncharge, c->kf_split, part, c->icharge, c->n,
                                                                c->fxl, c->gate);
    c->launches++;
  }
  tend(c, 1, e0);
  CKL(c);
  return CM3D_NB_OK;
}

// k-space of force(1) on stream `st`; with `defer` (mixed mode) the forces
// stay in the per-split partials and kspace_sum adds them to fxl later
static int kspace_run(Ctx *c, cudaStream_t st, bool defer) {
  if (c->ncharge == 0 || c->ktot == 0) return CM3D_NB_OK;
  if (c->nsys > 1) return kspace_forces_batch(c, st, defer);
  const double *dhmati = c->acc + ACC_COUNT;
  double vol = c->hmat[0] * (c->hmat[4] * c->hmat[8] - c->hmat[5] * c->hmat[7]) +
               c->hmat[1] * (c->hmat[5] * c->hmat[6] - c->hmat[3] * c->hmat[8]) +
               c->hmat[2] * (c->hmat[3] * c->hmat[7] - c->hmat[4] * c->hmat[6]);
  cudaEvent_t e0;
  tbegin(c, 1, &e0);
  const bool mixed = c->mode == CM3D_NB_MIXED;
  k_kprep<false><<<grid_for(c->ncharge, 256), 256, 0, st>>>(c->ncharge, c->icharge, c->n, c->pos, c->q, dhmati,
                                                                nullptr, nullptr, mixed ? c->kfrac : nullptr,
                                                                c->kposd, c->gate);
  // structure factors: enough row chunks per tile to fill the machine
  int rpb = c->nrows;
  while (rpb > 1 && (long long)c->ks_tiles * ((c->nrows + rpb - 1) / rpb) < (long long)c->num_sms * 4)
    rpb = (rpb + 1) / 2;
  dim3 gsf(c->ks_tiles, (c->nrows + rpb - 1) / rpb);
  if (mixed)
    k_sfac_mixed<false><<<gsf, KS_THREADS, 0, st>>>(c->ncharge, c->kfrac, c->nrows, c->rows, c->row_k0, rpb,
                                                       c->ktot, c->spart, nullptr, nullptr, c->gate);
  else
    k_sfac_plain<<<gsf, KS_THREADS, 0, st>>>(c->ncharge, c->kposd, c->nrows, c->rows, c->row_k0, rpb, c->ktot,
                                                dhmati, c->spart, c->gate);
  int ib = 256, gb = grid_for(c->ktot, ib);
  if (gb > c->num_sms * 4) gb = c->num_sms * 4;
  k_sred<false><<<gb, ib, 0, st>>>(c->ktot, c->ks_tiles, c->spart, c->ka_d, c->kb_d, c->kc_d, dhmati, 1.0 / vol,
                                      c->falp2, c->sk, mixed ? c->akf : nullptr, mixed ? nullptr : c->akd, c->acc,
                                      nullptr, nullptr, c->gate);
  int split = c->kf_split;
  int rps = (c->nrows + split - 1) / split;
  if (mixed) {
    int per = KS_THREADS * KF_A;
    dim3 gf((c->ncharge + per - 1) / per, split);
    // shared memory: the A(k) of one split's rows
    size_t smem = c->kf_smem;
    kforce_attr(c->dev);
    k_kforce_mixed<false><<<gf, KS_THREADS, smem, st>>>(c->ncharge, c->kfrac, c->icharge, c->n, c->nrows,
                                                            c->rows, c->row_k0, rps, c->akf, c->ktot, dhmati,
                                                            0, c->fxl, split > 1 || defer ? c->kf_part : nullptr,
                                                            nullptr, nullptr, c->gate);
    if (split > 1 && !defer) {
      k_kforce_sum<<<grid_for(c->ncharge, 256), 256, 0, st>>>(c->ncharge, split, c->kf_part, c->icharge,
                                                                  c->n, c->fxl, c->gate);
      c->launches++;
    }
  } else {
    dim3 gf((c->ncharge + 255) / 256, split);
    k_kforce_plain<<<gf, 256, 0, st>>>(c->ncharge, c->kposd, c->icharge, c->n, c->nrows, c->rows, c->row_k0,
                                          rps, c->akd, c->ktot, dhmati, split > 1, c->fxl, c->gate);
  }
  c->launches += 4;
  tend(c, 1, e0);
  CKL(c);
  return CM3D_NB_OK;
}

int kspace_forces(Ctx *c) { return kspace_run(c, c->st, false); }

// Whether force(1)'s k-space can run beside the list build and the pair
// kernels: mixed mode (its forces go through the per-split partials, which
// nothing else writes), charges with k-vectors, no per-class kernel timing
// (whose events live on the main stream).
bool kspace_async_ok(const Ctx *c) {
  return c->mode == CM3D_NB_MIXED && c->ncharge > 0 && c->ktot > 0 && c->kf_part && c->st2 && !c->timing.on;
}

// Fork: the k-space kernels of force(1) on the side stream, after what the
// main stream has enqueued so far (positions final, accumulators zeroed).
// They read positions and charges and write the k-space accumulators and
// the partial forces only -- none of which the list build, group_init or
// the pair kernels touch.
int kspace_fork(Ctx *c) {
  CK(cudaEventRecord(c->ev_fork, c->st));
  CK(cudaStreamWaitEvent(c->st2, c->ev_fork, 0));
  int rc = kspace_run(c, c->st2, true);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev_join, c->st2));
  return CM3D_NB_OK;
}

// Join: the main stream waits for the forked k-space and adds its partial
// forces to fxl in split order (after the pair forces, as without the fork)
int kspace_join(Ctx *c) {
  CK(cudaStreamWaitEvent(c->st, c->ev_join, 0));
  k_kforce_sum<<<grid_for(c->ncharge, 256), 256, 0, c->st>>>(c->ncharge, c->kf_split, c->kf_part, c->icharge, c->n,
                                                              c->fxl, c->gate);
  c->launches++;
  CKL(c);
  return CM3D_NB_OK;
}

// ------------------------------------------------- no-allocation variant
// cm3d_nb_fk_ewald_noalloc runs the mixed-mode kernels above on one fixed
// scratch area in the library's static device memory instead of the buffers
// of an engine context, so a call allocates nothing.  Its size is set by the
// limits below (about 2.9 MiB in all).
constexpr int NA_MAX_CHARGES = CM3D_NB_NOALLOC_MAX_CHARGES;
constexpr int NA_MAX_KMAX = CM3D_NB_NOALLOC_MAX_KMAX;
constexpr int NA_MAX_K = 7073;                   // k-vectors of ewald_setup at kmax 15
constexpr int NA_MAX_ROWS = (NA_MAX_KMAX + 1) * (2 * NA_MAX_KMAX + 1);
constexpr int NA_MAX_TILES = (NA_MAX_CHARGES + KS_THREADS * KS_A - 1) / (KS_THREADS * KS_A);
constexpr int NA_MAX_DEVICES = 64;
static_assert(2 * NA_MAX_KMAX + 1 <= MAX_ROWLEN, "a k row must fit the structure-factor kernel");

constexpr size_t na_align(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t NA_OFF_KFRAC = 0;
constexpr size_t NA_OFF_SPART = NA_OFF_KFRAC + na_align(sizeof(uint4) * NA_MAX_CHARGES);
constexpr size_t NA_OFF_SK = NA_OFF_SPART + na_align(sizeof(double2) * NA_MAX_TILES * NA_MAX_K);
constexpr size_t NA_OFF_AKF = NA_OFF_SK + na_align(sizeof(double2) * NA_MAX_K);
constexpr size_t NA_OFF_KABC = NA_OFF_AKF + na_align(sizeof(float2) * NA_MAX_K);
constexpr size_t NA_OFF_ROWS = NA_OFF_KABC + na_align(sizeof(int) * 3 * NA_MAX_K);
constexpr size_t NA_OFF_ROWK0 = NA_OFF_ROWS + na_align(sizeof(int4) * NA_MAX_ROWS);
constexpr size_t NA_OFF_ACC = NA_OFF_ROWK0 + na_align(sizeof(int) * NA_MAX_ROWS);
constexpr size_t NA_BYTES = NA_OFF_ACC + na_align(sizeof(double) * (ACC_COUNT + 9));

// the scratch area: per-atom fixed-point phases, per-tile partial S(k), S(k),
// A(k), the k-vectors and rows of ewald_setup's set, and the accumulators
// (+ H^-1 at ACC_COUNT, where the k-space kernels read it)
static __device__ __align__(256) unsigned char g_na_scratch[NA_BYTES];

struct Mat9 {
  double m[9];
};

__host__ __device__ inline int na_isqrt(int r) {
  int m = (int)sqrt((double)r);
  while (m * m > r) m--;
  while ((m + 1) * (m + 1) <= r) m++;
  return m;
}

// ewald_setup's loops (md_ewald.c:93-114) as rows: candidate c is the pair
// (i, j) = (c / (2 kmax + 1), c % (2 kmax + 1) - kmax) of the two outer
// loops; its k's are the consecutive kc with i^2 + j^2 + kc^2 <= kmax^2
// (kc >= 1 when i = j = 0).  Returns the row length, 0 for an empty row.
__host__ __device__ inline int na_row(int kmax, int c, int *i, int *j, int *kc0) {
  const int w = 2 * kmax + 1;
  *i = c / w;
  *j = c % w - kmax;
  *kc0 = 0;
  if (*i == 0 && *j < 0) return 0;
  const int r2 = kmax * kmax - *i * *i - *j * *j;
  if (r2 < 0) return 0;
  const int m = na_isqrt(r2);
  if (*i == 0 && *j == 0) {
    *kc0 = 1;
    return m;
  }
  *kc0 = -m;
  return 2 * m + 1;
}

// one block: the rows, row offsets and per-k (ka, kb, kc) of the k set in
// CM3D's order (a block-wide scan over the candidates), H^-1, and zeroed
// reciprocal-space accumulators
constexpr int NA_SETUP_THREADS = 512;
__global__ void __launch_bounds__(NA_SETUP_THREADS) k_na_setup(int kmax, Mat9 hmati, int4 *__restrict__ rows,
                                                               int *__restrict__ row_k0, int *__restrict__ ka,
                                                               int *__restrict__ kb, int *__restrict__ kc,
                                                               double *__restrict__ acc) {
  __shared__ int wsum[2][NA_SETUP_THREADS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ncand = (kmax + 1) * (2 * kmax + 1);
  int rbase = 0, kbase = 0;
  for (int base = 0; base < ncand; base += NA_SETUP_THREADS) {
    const int c = base + threadIdx.x;
    int i = 0, j = 0, kc0 = 0, len = 0;
    if (c < ncand) len = na_row(kmax, c, &i, &j, &kc0);
    int fr = len > 0 ? 1 : 0, fk = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int a = __shfl_up_sync(0xffffffffu, fr, o), b = __shfl_up_sync(0xffffffffu, fk, o);
      if (lane >= o) {
        fr += a;
        fk += b;
      }
    }
    if (lane == 31) {
      wsum[0][w] = fr;
      wsum[1][w] = fk;
    }
    __syncthreads();
    int pr = 0, pk = 0, tr = 0, tk = 0;
    for (int q2 = 0; q2 < NA_SETUP_THREADS / 32; q2++) {
      if (q2 < w) {
        pr += wsum[0][q2];
        pk += wsum[1][q2];
      }
      tr += wsum[0][q2];
      tk += wsum[1][q2];
    }
    if (len > 0) {
      const int r = rbase + pr + fr - 1;
      const int k0 = kbase + pk + fk - len;
      rows[r] = make_int4(i, j, kc0, len);
      row_k0[r] = k0;
      for (int t = 0; t < len; t++) {
        ka[k0 + t] = i;
        kb[k0 + t] = j;
        kc[k0 + t] = kc0 + t;
      }
    }
    rbase += tr;
    kbase += tk;
    __syncthreads();
  }
  if (threadIdx.x < 9) acc[ACC_COUNT + threadIdx.x] = hmati.m[threadIdx.x];
  if (threadIdx.x < 11) acc[ACC_VK + threadIdx.x] = 0.0;
}

// fk_ewald's totals (md_ewald.c:336-348) into the caller's 11 doubles
__global__ void k_na_finish(const double *__restrict__ acc, double six, double self, double *__restrict__ out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const double vk = acc[ACC_VK], vp = acc[ACC_VP];
  out[0] = vk + six + self;
  out[1] = vp + 3. * (vk + six);
  for (int k = 0; k < 9; k++) out[2 + k] = acc[ACC_VPT + k] + (k % 4 == 0 ? vk + six : 0.0);
}

// per-device set-up, once: the scratch area's address (cudaGetSymbolAddress
// with the device current) and the force kernel's shared-memory limit
// per-device set-up, done by the first call on a device that succeeds: a
// failed set-up (say, a first call made during a stream capture) is not
// remembered, the next call tries again
static std::mutex g_na_mu;
static bool g_na_ready[NA_MAX_DEVICES];
static unsigned char *g_na_ptr[NA_MAX_DEVICES];
static int g_na_sms[NA_MAX_DEVICES];

static cudaError_t na_device_setup(int dev, const char **what) {
  void *p = nullptr;
  *what = "cudaGetSymbolAddress(scratch)";
  cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
  if (e != cudaSuccess) return e;
  // the same limit kspace_forces sets, so that neither caller lowers it
  *what = "cudaFuncSetAttribute(k_kforce_mixed)";
  e = cudaFuncSetAttribute(k_kforce_mixed<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e != cudaSuccess) return e;
  int sms = 0;
  *what = "cudaDeviceGetAttribute(multiProcessorCount)";
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  g_na_ptr[dev] = (unsigned char *)p;
  g_na_sms[dev] = sms > 0 ? sms : 1;
  g_na_ready[dev] = true;
  return cudaSuccess;
}

struct NaDeviceGuard {
  int prev = -1;
  bool switched = false;
  ~NaDeviceGuard() {
    if (switched) cudaSetDevice(prev);
  }
};

static int fk_ewald_noalloc(int device, cudaStream_t st, int natoms, const double *pos, const double *q,
                            int ncharge, const int *icharge, const double *hmat, int kmax, double falp2,
                            double ewald_self, double ewald_bkg, double *fxl, double *out) {
  if (!hmat || !out || (ncharge > 0 && (!pos || !q || !icharge || !fxl))) {
    set_error("fk_ewald_noalloc: null argument");
    return CM3D_NB_ERR_ARG;
  }
  if (natoms < 1 || natoms > (1 << 28) || ncharge < 0 || ncharge > natoms) {
    set_error("fk_ewald_noalloc: natoms = %d, ncharge = %d", natoms, ncharge);
    return CM3D_NB_ERR_ARG;
  }
  if (ncharge > NA_MAX_CHARGES) {
    set_error("fk_ewald_noalloc: %d charged atoms exceed the fixed scratch limit of %d "
              "(CM3D_NB_NOALLOC_MAX_CHARGES); use cm3d_nb_fk_ewald",
              ncharge, NA_MAX_CHARGES);
    return CM3D_NB_ERR_ARG;
  }
  if (kmax < 0 || kmax > NA_MAX_KMAX) {
    set_error("fk_ewald_noalloc: kmax = %d is outside the fixed scratch limit 0..%d "
              "(CM3D_NB_NOALLOC_MAX_KMAX); use cm3d_nb_fk_ewald",
              kmax, NA_MAX_KMAX);
    return CM3D_NB_ERR_ARG;
  }
  const double *h = hmat;
  const double vol = h[0] * (h[4] * h[8] - h[5] * h[7]) + h[1] * (h[5] * h[6] - h[3] * h[8]) +
                     h[2] * (h[3] * h[7] - h[4] * h[6]);
  if (!(vol != 0.0) || !isfinite(vol)) {
    set_error("fk_ewald_noalloc: singular cell matrix (det = %g)", vol);
    return CM3D_NB_ERR_ARG;
  }
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev || device >= NA_MAX_DEVICES) {
    set_error("fk_ewald_noalloc: device %d (the process sees %d)", device, ndev);
    return CM3D_NB_ERR_ARG;
  }
  NaDeviceGuard guard;
  CK(cudaGetDevice(&guard.prev));
  if (guard.prev != device) {
    CK(cudaSetDevice(device));
    guard.switched = true;
  }
  {
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (!g_na_ready[device]) {
      const char *what = "";
      const cudaError_t e = na_device_setup(device, &what);
      if (e != cudaSuccess) return cuda_fail(e, what);
    }
  }
  unsigned char *base = g_na_ptr[device];
  const int nsm = g_na_sms[device];
  uint4 *kfrac = (uint4 *)(base + NA_OFF_KFRAC);
  double2 *spart = (double2 *)(base + NA_OFF_SPART);
  double2 *sk = (double2 *)(base + NA_OFF_SK);
  float2 *akf = (float2 *)(base + NA_OFF_AKF);
  int *ka = (int *)(base + NA_OFF_KABC);
  int *kb = ka + NA_MAX_K, *kc = ka + 2 * NA_MAX_K;
  int4 *rows = (int4 *)(base + NA_OFF_ROWS);
  int *row_k0 = (int *)(base + NA_OFF_ROWK0);
  double *acc = (double *)(base + NA_OFF_ACC);
  const double *dhmati = acc + ACC_COUNT;

  // H^-1 as cm3d_nb_create forms it
  const double rvol = 1. / vol;
  Mat9 hi;
  hi.m[0] = (h[4] * h[8] - h[5] * h[7]) * rvol;
  hi.m[1] = (h[2] * h[7] - h[1] * h[8]) * rvol;
  hi.m[2] = (h[1] * h[5] - h[2] * h[4]) * rvol;
  hi.m[3] = (h[5] * h[6] - h[3] * h[8]) * rvol;
  hi.m[4] = (h[0] * h[8] - h[2] * h[6]) * rvol;
  hi.m[5] = (h[2] * h[3] - h[0] * h[5]) * rvol;
  hi.m[6] = (h[3] * h[7] - h[4] * h[6]) * rvol;
  hi.m[7] = (h[1] * h[6] - h[0] * h[7]) * rvol;
  hi.m[8] = (h[0] * h[4] - h[1] * h[3]) * rvol;
  // the same rows on the host (sizes and the force kernel's shared memory)
  int hk0[NA_MAX_ROWS + 1];
  int nrows = 0, ktot = 0;
  for (int c = 0; c < (kmax + 1) * (2 * kmax + 1); c++) {
    int i, j, kc0;
    const int len = na_row(kmax, c, &i, &j, &kc0);
    if (len == 0) continue;
    hk0[nrows++] = ktot;
    ktot += len;
  }
  hk0[nrows] = ktot;
  if (ktot > NA_MAX_K || nrows > NA_MAX_ROWS) {
    set_error("fk_ewald_noalloc: internal size check failed (ktot %d, rows %d)", ktot, nrows);
    return CM3D_NB_ERR_ARG;
  }

  k_na_setup<<<1, NA_SETUP_THREADS, 0, st>>>(kmax, hi, rows, row_k0, ka, kb, kc, acc);
  if (ncharge > 0 && ktot > 0) {
    k_kprep<false><<<grid_for(ncharge, 256), 256, 0, st>>>(ncharge, icharge, natoms, pos, q, dhmati, nullptr,
                                                           nullptr, kfrac, nullptr, nullptr);
    // grids chosen as kspace_setup/kspace_forces choose them
    const int ks_tiles = (ncharge + KS_THREADS * KS_A - 1) / (KS_THREADS * KS_A);
    int rpb = nrows;
    while (rpb > 1 && (long long)ks_tiles * ((nrows + rpb - 1) / rpb) < nsm * 4) rpb = (rpb + 1) / 2;
    dim3 gsf(ks_tiles, (nrows + rpb - 1) / rpb);
    k_sfac_mixed<false><<<gsf, KS_THREADS, 0, st>>>(ncharge, kfrac, nrows, rows, row_k0, rpb, ktot, spart, nullptr,
                                                    nullptr, nullptr);
    int gb = grid_for(ktot, 256);
    if (gb > nsm * 4) gb = nsm * 4;
    k_sred<false><<<gb, 256, 0, st>>>(ktot, ks_tiles, spart, ka, kb, kc, dhmati, rvol, falp2, sk, akf, nullptr, acc,
                                      nullptr, nullptr, nullptr);
    const int per_block = KS_THREADS * KF_A;
    const int tiles = (ncharge + per_block - 1) / per_block;
    int split = 1;
    while (tiles * split < nsm * 4 && split < nrows) split *= 2;
    if (split > nrows) split = nrows;
    const int rps = (nrows + split - 1) / split;
    size_t smem = 0;
    for (int r0 = 0; r0 < nrows; r0 += rps) {
      const int r1 = r0 + rps < nrows ? r0 + rps : nrows;
      const size_t nk = (size_t)(hk0[r1] - hk0[r0]) * sizeof(float2);
      if (nk > smem) smem = nk;
    }
    dim3 gf(tiles, split);
    k_kforce_mixed<false><<<gf, KS_THREADS, smem, st>>>(ncharge, kfrac, icharge, natoms, nrows, rows, row_k0, rps,
                                                        akf, ktot, dhmati, split > 1, fxl, nullptr, nullptr, nullptr,
                                                        nullptr);
  }
  const double six = ncharge > 0 ? ewald_bkg / vol : 0.0;
  k_na_finish<<<1, 32, 0, st>>>(acc, six, ncharge > 0 ? ewald_self : 0.0, out);
  CK(cudaPeekAtLastError());
  return CM3D_NB_OK;
}

}  // namespace cm3d

extern "C" int cm3d_nb_fk_ewald_noalloc(int device, void *stream, int natoms, const double *pos,
                                        const double *q, int ncharge, const int *icharge, const double hmat[9],
                                        int kmax, double falp2, double ewald_self, double ewald_bkg,
                                        double *fxl, double *out) {
  return cm3d::fk_ewald_noalloc(device, (cudaStream_t)stream, natoms, pos, q, ncharge, icharge, hmat, kmax,
                                falp2, ewald_self, ewald_bkg, fxl, out);
}
