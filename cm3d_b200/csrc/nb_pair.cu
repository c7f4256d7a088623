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

// BATCH = false: one system, its parameters in P and its shifts, cut-offs,
// type map and (when they fit) tables staged in shared memory.  BATCH = true:
// several systems; each atom group reads its system's parameters, shifts and
// tables (global interaction / Coulomb-table indices) from sp[sys_of[t]].
template <int TPA, bool SMALLBOX, bool NEED_S, bool BATCH>
__global__ void __launch_bounds__(256, NEED_S ? 2 : 3) k_pair_mixed(
    MixedP P, const float4 *__restrict__ xq, const int *__restrict__ styp, const int *__restrict__ sorig,
    const int *__restrict__ nlen, int stride, const uint32_t *__restrict__ nbr, const float4 *__restrict__ gshift,
    const int *__restrict__ gmap, const float *__restrict__ gfcut, const float4 *__restrict__ gtl,
    const float4 *__restrict__ gte, const SysP *__restrict__ sp, const int *__restrict__ sys_of,
    double *__restrict__ fout, double *__restrict__ fshort, float *__restrict__ epart,
    double *__restrict__ epart64, long long *__restrict__ stat, const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  extern __shared__ float4 sm[];
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
  // persistent: every lane group walks atoms blockIdx-strided
  for (int tb = blockIdx.x * groups; tb < P.n; tb += gridDim.x * groups) {
    const int t = tb + threadIdx.x / TPA;
    const bool active = t < P.n;
    double Fx = 0, Fy = 0, Fz = 0, Sx = 0, Sy = 0, Sz = 0, elj_hi = 0;
    float e[EP_COUNT];
#pragma unroll
    for (int k = 0; k < EP_COUNT; k++) e[k] = 0.f;
    if (active) {
      const float4 xi = xq[t];
      const int ti = styp[t];
      const long long k0 = (long long)t * stride, k1 = k0 + nlen[t];
      float fx = 0, fy = 0, fz = 0, sx = 0, sy = 0, sz = 0;
      int cnt = 0;
      // this atom's system: shifts, type map, cut-offs and tables
      const SysP *Sp = BATCH ? sp + sys_of[t] : nullptr;
      const float4 *shp = BATCH ? Sp->shift : shift;
      const float4 *shlp = BATCH ? Sp->shift_lo : shift + 27;
      const int *mapp = BATCH ? gmap + Sp->map0 : map;
      const float *fcp = BATCH ? gfcut : fcut;
      const int ntyp = BATCH ? Sp->ntypes : P.ntypes;
      const bool has_el = (P.mask & 2) && (!BATCH || Sp->coul >= 0);
      const float4 *tep = BATCH ? gte + (size_t)2 * P.ntable * (Sp->coul > 0 ? Sp->coul : 0) : te;
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
            const float4 *T = tl + 3 * ((size_t)in * P.ntable + kk);
            const float4 a0 = T[0], a1 = T[1], a2 = T[2];
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
      for (long long kb = k0 + g; kb < k1; kb += PU * TPA) {
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
          tj[u] = (en[u] & fl_lj) ? styp[j] : 0;
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
  }
  if (under) atomicAdd((unsigned long long *)(stat + ST_UNDERFLOW), (unsigned long long)under);
}

// FP64 sums of the per-atom partials into CM3D's accumulators (one block per
// quantity and system, fixed order: deterministic).  Every pair was seen from
// both ends, hence the factor 1/2; CM3D's virials are -sum d_a d_b f.
__global__ void k_ereduce(int n, int mask, const SysP *__restrict__ sp, const float *__restrict__ epart,
                          const double *__restrict__ epart64, double *__restrict__ accs,
                          const int *__restrict__ gs) {
  if (gated_off(gs, 0)) return;
  __shared__ double red[32];
  const int q = blockIdx.x, sy = blockIdx.y;
  if (!((q < EP_EEL && (mask & 1)) || (q >= EP_EEL && (mask & 2)))) return;
  const int a0 = sp[sy].a0, a1 = a0 + sp[sy].n;
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
  if (threadIdx.x >= 32) return;
  s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
  s = warp_sum(s);
  if (threadIdx.x != 0) return;
  s *= 0.5;
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

// ------------------------------------------------------------------ host
static size_t smem_bytes(Ctx *c, bool with_tables, int mask) {
  size_t nf4 = (8 * (size_t)c->ninter + 3) / 4, nm4 = ((size_t)c->ntypes * c->ntypes + 3) / 4;
  size_t b = (54 + nf4 + nm4) * sizeof(float4);
  if (with_tables) {
    b += (size_t)3 * c->ninter * c->ntable * sizeof(float4);
    if (mask & 2) b += (size_t)2 * c->ntable * sizeof(float4);
  }
  return b;
}

// per-atom FP64 partials of the LJ energy's table hi parts, stored after the
// EP_COUNT FP32 rows of epart
static double *epart_hi(Ctx *c) { return reinterpret_cast<double *>(c->epart + (size_t)EP_COUNT * c->n); }

template <int TPA, bool SB, bool NS, bool BT>
static void launch_t(Ctx *c, const MixedP &P, size_t smem, double *fout) {
  const int B = 256;
  auto kern = k_pair_mixed<TPA, SB, NS, BT>;
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
  long long need = ((long long)c->n * TPA + B - 1) / B;
  long long grid = (long long)c->num_sms * per_sm;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  kern<<<grid, B, smem, c->st>>>(P, c->xq, c->styp, c->cell_atoms, c->nlen, c->nbr_stride, c->nbr, c->shift,
                                 c->map, c->fcut, c->ftab_lj, c->ftab_el, c->sp, c->sys_of, fout, c->fxs, c->epart,
                                 epart_hi(c), c->stat, c->gate);
}

template <bool SB, bool NS, bool BT>
static int launch_tpa(Ctx *c, const MixedP &P, size_t smem, double *fout) {
  switch (c->tpa) {
    case 4: launch_t<4, SB, NS, BT>(c, P, smem, fout); break;
    case 8: launch_t<8, SB, NS, BT>(c, P, smem, fout); break;
    case 16: launch_t<16, SB, NS, BT>(c, P, smem, fout); break;
    case 32: launch_t<32, SB, NS, BT>(c, P, smem, fout); break;
    default: launch_t<8, SB, NS, BT>(c, P, smem, fout); break;
  }
  return CM3D_NB_OK;
}

bool g_smallbox_warned = false;

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
  if (c->nsys > 1) {
    // several systems: per-system parameters and tables from global memory
    P.tab_smem = 0;
    if (ns) launch_tpa<false, true, true>(c, P, 0, fout);
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
    k_ereduce<<<dim3(EP_COUNT, c->nsys), c->nsys > 1 ? 256 : 1024, 0, c->st>>>(c->n, mask, c->sp, c->epart,
                                                                                 epart_hi(c), c->acc, c->gate);
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
